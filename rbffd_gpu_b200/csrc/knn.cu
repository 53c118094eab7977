// n-nearest-neighbour stencils on the device: the stencil generation of
// Grid::generateStencilsKDTree (src/grids/grid_interface.cpp:688-725) with the
// k-d tree of external/kdtree/KDTree.h:407-433, bit-identical to the host
// search rbffd_stencils_knn (host_inputs.cpp).
//
// A stencil is the n smallest (squared distance, index) pairs, closest first,
// with the squared distance summed as ((0 + dx^2) + dy^2) + dz^2 in FP64
// without contraction (the k-d tree's distance_squared, KDTree.h:45-51); a
// duplicate point at distance 0 sorted ahead of the centre swaps with it.
// That definition fixes the result whatever order candidates are visited in,
// so the device search only has to see every point that can be among them.
//
// Layout: the host bins the points into the same uniform cell grid as the
// host search and uploads the points in cell order (x, y, z, index).  One
// warp per query point (queries taken in cell order, so neighbouring warps
// read neighbouring cells): it appends the points of the cells within
// Chebyshev distance R of the query's cell to a shared-memory buffer of
// KNN_CAP (distance, index) pairs; when the buffer fills it is sorted
// (bitonic, by distance then index) and cut to the best n + 1.  Once at least
// n candidates are in, the n-th distance is compared with the searched reach
// (R times the smallest cell edge): as in the host search, a smaller n-th
// distance proves no unvisited point can enter; otherwise the next shell is
// added.
//
// The same search serves the reference's default brute-force generator
// (Grid::generateStencilsBruteForce, grid_interface.cpp:637-686): there equal
// distances fall in decreasing index (DESC), with no centre swap; both cut a
// list at the first node not closer than max_st_radius.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "internal.h"

namespace {

constexpr int KNN_CAP = 512;        // candidate buffer per warp (power of two)
constexpr int KNN_WARPS = 4;        // queries per block
constexpr int KNN_MAX_N = KNN_CAP / 2 - 1;

struct CellGrid {
    double lo[3], hc[3], minh;
    int dims[3];
};

__device__ __forceinline__ int cell_coord(const CellGrid& G, double p, int a)
{
    int c = (int)floor((p - G.lo[a]) / G.hc[a]);
    return max(0, min(G.dims[a] - 1, c));
}

template <bool DESC>
__device__ __forceinline__ bool pair_less(double da, int ia, double db, int ib)
{
    return da < db || (da == db && (DESC ? ia > ib : ia < ib));
}

// Sort the first cnt (<= KNN_CAP) entries of (d, id) ascending by distance,
// then index (descending with DESC): a bitonic network over the next power of
// two, the slots beyond cnt padded with +inf distances.  One warp.
template <bool DESC>
__device__ void warp_bitonic_sort(double* d, int* id, int cnt, int lane)
{
    int S = 32;
    while (S < cnt) S <<= 1;
    for (int t = cnt + lane; t < S; t += 32) {
        d[t] = __longlong_as_double(0x7ff0000000000000ll);
        id[t] = 0x7fffffff;
    }
    __syncwarp();
    for (int k = 2; k <= S; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int t = lane; t < S; t += 32) {
                const int p = t ^ j;
                if (p > t) {
                    const bool up = (t & k) == 0;
                    const bool sw = up ? pair_less<DESC>(d[p], id[p], d[t], id[t])
                                       : pair_less<DESC>(d[t], id[t], d[p], id[p]);
                    if (sw) {
                        const double td = d[t];
                        d[t] = d[p];
                        d[p] = td;
                        const int ti = id[t];
                        id[t] = id[p];
                        id[p] = ti;
                    }
                }
            }
            __syncwarp();
        }
}

template <bool DESC>
__global__ void __launch_bounds__(32 * KNN_WARPS)
k_knn(const double4* __restrict__ pts, const int* __restrict__ start, CellGrid G, int N, int n, double max_radius,
      int* __restrict__ st, int* __restrict__ st_len, int* __restrict__ tie)
{
    __shared__ double sd[KNN_WARPS][KNN_CAP];
    __shared__ int si[KNN_WARPS][KNN_CAP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qs = blockIdx.x * KNN_WARPS + w;  // query slot in cell order
    if (qs >= N) return;
    double* d = sd[w];
    int* id = si[w];
    const double4 q = pts[qs];
    const int qi = (int)q.w;
    const int cc[3] = {cell_coord(G, q.x, 0), cell_coord(G, q.y, 1), cell_coord(G, q.z, 2)};
    const int maxr = max(G.dims[0], max(G.dims[1], G.dims[2]));
    int cnt = 0;
    for (int R = 0; R <= maxr; R++) {
        // the shell of cells at Chebyshev distance R, in the host's a, b, c order
        for (int a = cc[0] - R; a <= cc[0] + R; a++) {
            if (a < 0 || a >= G.dims[0]) continue;
            for (int b = cc[1] - R; b <= cc[1] + R; b++) {
                if (b < 0 || b >= G.dims[1]) continue;
                for (int c = cc[2] - R; c <= cc[2] + R; c++) {
                    if (c < 0 || c >= G.dims[2]) continue;
                    const int ring = max(abs(a - cc[0]), max(abs(b - cc[1]), abs(c - cc[2])));
                    if (ring != R) continue;
                    const size_t cell = ((size_t)a * G.dims[1] + b) * G.dims[2] + c;
                    const int t0 = start[cell], t1 = start[cell + 1];
                    for (int t = t0; t < t1; t += 32) {
                        if (cnt + 32 > KNN_CAP) {  // full: keep the best n + 1
                            warp_bitonic_sort<DESC>(d, id, cnt, lane);
                            cnt = n + 1;
                        }
                        const bool have = t + lane < t1;
                        if (have) {
                            const double4 p = pts[t + lane];
                            const double dx = __dsub_rn(q.x, p.x), dy = __dsub_rn(q.y, p.y), dz = __dsub_rn(q.z, p.z);
                            double s = __dmul_rn(dx, dx);
                            s = __dadd_rn(s, __dmul_rn(dy, dy));
                            s = __dadd_rn(s, __dmul_rn(dz, dz));
                            d[cnt + lane] = s;
                            id[cnt + lane] = (int)p.w;
                        }
                        __syncwarp();
                        cnt += min(32, t1 - t);
                    }
                }
            }
        }
        if (cnt >= n) {
            warp_bitonic_sort<DESC>(d, id, cnt, lane);
            cnt = min(cnt, n + 1);
            const double reach = R * G.minh;  // every unvisited point is farther than this
            if (d[n - 1] < reach * reach || R == maxr) break;
        }
    }
    // d/id hold the sorted best min(cnt, n + 1) candidates; the list stops at
    // the first one not closer than max_radius (the rest: the centre)
    int len = n;
    if (lane == 0)
        for (int k = 0; k < n; k++)
            if (!(sqrt(d[k]) < max_radius)) {
                len = k;
                break;
            }
    len = __shfl_sync(0xffffffffu, len, 0);
    int* out = st + (size_t)qi * n;
    for (int k = lane; k < n; k += 32) out[k] = k < len ? id[k] : qi;
    __syncwarp();
    if (lane == 0) {
        int first = -1;  // the centre's slot (the lowest if listed twice)
        for (int k = 0; k < len && first < 0; k++)
            if (id[k] == qi) first = k;
        if (!DESC && first > 0) {  // k-d tree lists: a duplicate at distance 0 sorted ahead of the centre
            out[first] = out[0];
            out[0] = qi;
        }
        if (st_len) st_len[qi] = len;
        int t = 0;
        for (int k = 0; k + 1 < cnt && k < n; k++)
            if (d[k] == d[k + 1]) {
                t = 1;
                break;
            }
        tie[qi] = t;
    }
}

}  // namespace

static int stencils_gpu(rbffd_ctx* ctx, const double* xyz, int N, int n, int method, double max_radius, int* st,
                        int* st_len, int* ties)
{
    if (!ctx || !xyz || !st || N <= 0 || n <= 0 || n > N) return RBFFD_ERR_INVALID;
    if (method != RBFFD_ST_KDTREE && method != RBFFD_ST_BRUTE_FORCE) return RBFFD_ERR_INVALID;
    if (!(max_radius > 0.0)) return RBFFD_ERR_INVALID;
    if (n > KNN_MAX_N) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "stencil size %d above %d", n, KNN_MAX_N);
    cudaSetDevice(ctx->device);
    // the host search's cell grid (host_inputs.cpp)
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < N; i++)
        for (int a = 0; a < 3; a++) {
            lo[a] = std::min(lo[a], xyz[3 * (size_t)i + a]);
            hi[a] = std::max(hi[a], xyz[3 * (size_t)i + a]);
        }
    const double rk = std::sqrt(4.0 * n / (double)N);
    const double h = std::max(rk * 0.5, 1e-12);
    CellGrid G;
    for (int a = 0; a < 3; a++) {
        G.lo[a] = lo[a];
        G.dims[a] = std::max(1, std::min(400, (int)std::ceil((hi[a] - lo[a]) / h) + 1));
        G.hc[a] = std::max((hi[a] - lo[a]) / G.dims[a], 1e-300) * (1.0 + 1e-12);
    }
    G.minh = std::min(G.hc[0], std::min(G.hc[1], G.hc[2]));
    const size_t ncell = (size_t)G.dims[0] * G.dims[1] * G.dims[2];
    auto coord = [&](double p, int a) {
        int c = (int)std::floor((p - G.lo[a]) / G.hc[a]);
        return std::max(0, std::min(G.dims[a] - 1, c));
    };
    std::vector<int> cell_of(N), start(ncell + 1, 0);
    for (int i = 0; i < N; i++) {
        const double* p = xyz + 3 * (size_t)i;
        const size_t c = ((size_t)coord(p[0], 0) * G.dims[1] + coord(p[1], 1)) * G.dims[2] + coord(p[2], 2);
        cell_of[i] = (int)c;
        start[c + 1]++;
    }
    for (size_t c = 0; c < ncell; c++) start[c + 1] += start[c];
    std::vector<double4> pts(N);
    {
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (int i = 0; i < N; i++) {
            const double* p = xyz + 3 * (size_t)i;
            pts[fill[cell_of[i]]++] = make_double4(p[0], p[1], p[2], (double)i);
        }
    }
    double4* d_pts = nullptr;
    int *d_start = nullptr, *d_st = nullptr, *d_tie = nullptr, *d_len = nullptr;
    const size_t b_pts = (size_t)N * sizeof(double4), b_start = (ncell + 1) * sizeof(int),
                 b_st = (size_t)N * n * sizeof(int), b_tie = (size_t)N * sizeof(int);
    int rc;
    if ((rc = dev_alloc(ctx, (void**)&d_pts, b_pts)) || (rc = dev_alloc(ctx, (void**)&d_start, b_start)) ||
        (rc = dev_alloc(ctx, (void**)&d_st, b_st)) || (rc = dev_alloc(ctx, (void**)&d_tie, b_tie)) ||
        (st_len && (rc = dev_alloc(ctx, (void**)&d_len, b_tie)))) {
        dev_free(ctx, d_pts, b_pts);
        dev_free(ctx, d_start, b_start);
        dev_free(ctx, d_st, b_st);
        dev_free(ctx, d_tie, b_tie);
        return rc;
    }
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(d_pts, pts.data(), b_pts, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_start, start.data(), b_start, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        const unsigned nb = (unsigned)((N + KNN_WARPS - 1) / KNN_WARPS);
        if (method == RBFFD_ST_BRUTE_FORCE)
            k_knn<true><<<nb, 32 * KNN_WARPS, 0, s>>>(d_pts, d_start, G, N, n, max_radius, d_st, d_len, d_tie);
        else
            k_knn<false><<<nb, 32 * KNN_WARPS, 0, s>>>(d_pts, d_start, G, N, n, max_radius, d_st, d_len, d_tie);
        e = cudaGetLastError();
    }
    std::vector<int> tie(N);
    if (e == cudaSuccess) e = cudaMemcpyAsync(st, d_st, b_st, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tie.data(), d_tie, b_tie, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && st_len) e = cudaMemcpyAsync(st_len, d_len, b_tie, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    dev_free(ctx, d_pts, b_pts);
    dev_free(ctx, d_start, b_start);
    dev_free(ctx, d_st, b_st);
    dev_free(ctx, d_tie, b_tie);
    dev_free(ctx, d_len, b_tie);
    if (e != cudaSuccess) return cuda_error(ctx, e, "stencils on the device");
    if (ties) {
        long long t = 0;
        for (int i = 0; i < N; i++) t += tie[i];
        *ties = (int)t;
    }
    return RBFFD_OK;
}

extern "C" int rbffd_stencils_knn_gpu(rbffd_ctx* ctx, const double* xyz, int N, int n, int* st, int* ties)
{
    return stencils_gpu(ctx, xyz, N, n, RBFFD_ST_KDTREE, DBL_MAX, st, nullptr, ties);
}

extern "C" int rbffd_stencils_generate_gpu(rbffd_ctx* ctx, const double* xyz, int N, int n, int method,
                                           double max_radius, int* st, int* st_len, int* ties)
{
    return stencils_gpu(ctx, xyz, N, n, method, max_radius, st, st_len, ties);
}
