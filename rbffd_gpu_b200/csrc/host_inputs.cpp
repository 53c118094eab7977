// Host-side input builders for the RBF-FD path: synthetic sphere nodes,
// k-nearest-neighbour stencils and the exact solutions used as initial
// conditions.  These produce the inputs the reference's Grid and ExactSolution
// classes produce; nothing here runs on the GPU.
//
//   rbffd_nodes_fibonacci  -- stands in for the reference's maximum-determinant
//                             node files (GridReader, src/grids/grid_reader.*),
//                             which are not distributed with the reference.
//   rbffd_stencils_knn     -- Grid::generateStencilsKDTree
//                             (src/grids/grid_interface.cpp:688-725): the n nearest
//                             nodes, closest first, centre at [0].
//   rbffd_exact_cosine_bell -- ExactAdvection::operator()
//                             (tests/experiments/cosine_bell_on_sphere/exact_advection.h:37-53)
//   rbffd_exact_sph_heat   -- heat on the unit sphere: sum c_lm e^{-l(l+1)t} Y_lm.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/rbffd_sm100.h"

namespace {

uint64_t splitmix64(uint64_t& s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

double uniform01(uint64_t& s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

int default_threads(int nthreads)
{
    if (nthreads > 0) return nthreads;
    unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}

template <class F>
void parallel_for(int n, int nthreads, F&& f)
{
    nthreads = std::max(1, std::min(default_threads(nthreads), n));
    if (nthreads == 1) {
        for (int i = 0; i < n; i++) f(i);
        return;
    }
    std::atomic<int> next(0);
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; t++)
        pool.emplace_back([&]() {
            for (;;) {
                int b = next.fetch_add(256);
                if (b >= n) break;
                int e = std::min(n, b + 256);
                for (int i = b; i < e; i++) f(i);
            }
        });
    for (auto& th : pool) th.join();
}

}  // namespace

extern "C" int rbffd_nodes_fibonacci(int N, uint64_t seed, double* xyz)
{
    if (N <= 0 || !xyz) return RBFFD_ERR_INVALID;
    // Uniform random rotation from three uniforms (Shoemake's quaternion method).
    uint64_t s = seed;
    double u1 = uniform01(s), u2 = uniform01(s), u3 = uniform01(s);
    const double two_pi = 6.283185307179586476925286766559;
    double q0 = std::sqrt(1.0 - u1) * std::sin(two_pi * u2), q1 = std::sqrt(1.0 - u1) * std::cos(two_pi * u2);
    double q2 = std::sqrt(u1) * std::sin(two_pi * u3), q3 = std::sqrt(u1) * std::cos(two_pi * u3);
    // rotation matrix of the unit quaternion (w=q3, x=q0, y=q1, z=q2)
    double w = q3, x = q0, y = q1, z = q2;
    double R[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)},
                      {2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)},
                      {2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)}};
    const double golden = 3.14159265358979323846264338327950288 * (3.0 - std::sqrt(5.0));
    for (int i = 0; i < N; i++) {
        double zz = 1.0 - (2.0 * i + 1.0) / N;
        double r = std::sqrt(std::max(0.0, 1.0 - zz * zz));
        double ph = golden * (double)i;
        double p[3] = {r * std::cos(ph), r * std::sin(ph), zz};
        double q[3];
        for (int a = 0; a < 3; a++) q[a] = R[a][0] * p[0] + R[a][1] * p[1] + R[a][2] * p[2];
        double nrm = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
        for (int a = 0; a < 3; a++) xyz[3 * (size_t)i + a] = q[a] / nrm;
    }
    return RBFFD_OK;
}

// Squared distance with the summation order of the reference k-d tree's
// distance_squared (external/kdtree/KDTree.h:45-51): ((0 + dx^2) + dy^2) + dz^2.
static inline double dist2(const double* a, const double* b)
{
    double d = 0;
    for (int i = 0; i < 3; i++) d += (a[i] - b[i]) * (a[i] - b[i]);
    return d;
}

// Exact n-nearest search over a uniform cell grid, shared by the k-d tree and
// brute-force generators (method RBFFD_ST_KDTREE / RBFFD_ST_BRUTE_FORCE).
// Shells of cells are added until the n-th squared distance is below the
// searched reach, so every node tied with the n-th is a candidate.  Order:
// k-d tree (squared distance, index), the centre first if a duplicate point
// sorted ahead of it; brute force (squared distance, decreasing index), as
// the reference's std::set with a `<=` comparator leaves equal keys
// (grid_interface.h:442-461).  Each list is cut at the first entry whose
// distance sqrt(d2) is not below max_radius (grid_interface.cpp:676, 716);
// the rest is padding (the centre).
static int stencils_cell_search(const double* xyz, int N, int n, int method, double max_radius, int* st,
                                int* st_len, int* ties, int nthreads)
{
    if (!xyz || !st || N <= 0 || n <= 0 || n > N) return RBFFD_ERR_INVALID;
    if (method != RBFFD_ST_KDTREE && method != RBFFD_ST_BRUTE_FORCE) return RBFFD_ERR_INVALID;
    if (!(max_radius > 0.0)) return RBFFD_ERR_INVALID;  // every stencil would be empty
    // Uniform cell grid over the bounding box; cell edge ~ half the radius
    // expected to hold n points on the unit sphere.
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < N; i++)
        for (int a = 0; a < 3; a++) {
            lo[a] = std::min(lo[a], xyz[3 * (size_t)i + a]);
            hi[a] = std::max(hi[a], xyz[3 * (size_t)i + a]);
        }
    double rk = std::sqrt(4.0 * n / (double)N);
    double h = std::max(rk * 0.5, 1e-12);
    int dims[3];
    for (int a = 0; a < 3; a++) {
        double ext = hi[a] - lo[a];
        dims[a] = std::max(1, std::min(400, (int)std::ceil(ext / h) + 1));
    }
    double hc[3];
    for (int a = 0; a < 3; a++) hc[a] = std::max((hi[a] - lo[a]) / dims[a], 1e-300) * (1.0 + 1e-12);
    size_t ncell = (size_t)dims[0] * dims[1] * dims[2];
    std::vector<int> cell_of(N), start(ncell + 1, 0), order(N);
    auto cell_coord = [&](const double* p, int a) {
        int c = (int)std::floor((p[a] - lo[a]) / hc[a]);
        return std::max(0, std::min(dims[a] - 1, c));
    };
    for (int i = 0; i < N; i++) {
        const double* p = xyz + 3 * (size_t)i;
        size_t c = ((size_t)cell_coord(p, 0) * dims[1] + cell_coord(p, 1)) * dims[2] + cell_coord(p, 2);
        cell_of[i] = (int)c;
        start[c + 1]++;
    }
    for (size_t c = 0; c < ncell; c++) start[c + 1] += start[c];
    {
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (int i = 0; i < N; i++) order[fill[cell_of[i]]++] = i;
    }
    double minh = std::min(hc[0], std::min(hc[1], hc[2]));
    std::atomic<int> tie_count(0);
    std::atomic<int> failed(0);
    parallel_for(N, nthreads, [&](int i) {
        const double* q = xyz + 3 * (size_t)i;
        int cc[3] = {cell_coord(q, 0), cell_coord(q, 1), cell_coord(q, 2)};
        std::vector<std::pair<double, int>> cand;
        cand.reserve(4 * n);
        int maxr = std::max(dims[0], std::max(dims[1], dims[2]));
        for (int R = 0; R <= maxr; R++) {
            // add the shell of cells at Chebyshev distance R
            for (int a = cc[0] - R; a <= cc[0] + R; a++) {
                if (a < 0 || a >= dims[0]) continue;
                for (int b = cc[1] - R; b <= cc[1] + R; b++) {
                    if (b < 0 || b >= dims[1]) continue;
                    for (int c = cc[2] - R; c <= cc[2] + R; c++) {
                        if (c < 0 || c >= dims[2]) continue;
                        int ring = std::max(std::abs(a - cc[0]), std::max(std::abs(b - cc[1]), std::abs(c - cc[2])));
                        if (ring != R) continue;
                        size_t cell = ((size_t)a * dims[1] + b) * dims[2] + c;
                        for (int t = start[cell]; t < start[cell + 1]; t++) {
                            int j = order[t];
                            cand.emplace_back(dist2(q, xyz + 3 * (size_t)j), j);
                        }
                    }
                }
            }
            if ((int)cand.size() >= n) {
                std::nth_element(cand.begin(), cand.begin() + (n - 1), cand.end());
                double kth = cand[n - 1].first;
                double reach = R * minh;  // every unsearched node is farther than this
                if (kth < reach * reach || R == maxr) break;
            }
        }
        if ((int)cand.size() < n) {
            failed.store(1);
            return;
        }
        if (method == RBFFD_ST_KDTREE)
            std::sort(cand.begin(), cand.end());  // (distance, index): closest first
        else
            std::sort(cand.begin(), cand.end(), [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
                return a.first < b.first || (a.first == b.first && a.second > b.second);
            });
        int* out = st + (size_t)i * n;
        int len = n;
        for (int k = 0; k < n; k++) {
            out[k] = cand[k].second;
            if (len == n && !(std::sqrt(cand[k].first) < max_radius)) len = k;
        }
        if (method == RBFFD_ST_KDTREE && out[0] != i) {
            // duplicate point at distance 0 sorted ahead of the centre: put the centre first
            for (int k = 1; k < n; k++)
                if (out[k] == i) { std::swap(out[0], out[k]); break; }
        }
        for (int k = len; k < n; k++) out[k] = i;
        if (st_len) st_len[i] = len;
        for (int k = 0; k + 1 < (int)cand.size() && k < n; k++)
            if (cand[k].first == cand[k + 1].first) { tie_count.fetch_add(1); break; }
    });
    if (ties) *ties = tie_count.load();
    return failed.load() ? RBFFD_ERR_INVALID : RBFFD_OK;
}

extern "C" int rbffd_stencils_knn(const double* xyz, int N, int n, int* st, int* ties, int nthreads)
{
    return stencils_cell_search(xyz, N, n, RBFFD_ST_KDTREE, DBL_MAX, st, nullptr, ties, nthreads);
}

extern "C" int rbffd_stencils_generate(const double* xyz, int N, int n, int method, double max_radius, int* st,
                                       int* st_len, int* ties, int nthreads)
{
    return stencils_cell_search(xyz, N, n, method, max_radius, st, st_len, ties, nthreads);
}

extern "C" int rbffd_exact_cosine_bell(int N, const double* xyz, double a, double* h)
{
    if (N < 0 || !xyz || !h) return RBFFD_ERR_INVALID;
    const double PI = 3.14159265358979323846264338327950288;
    const double h0 = 1.0, R = a / 3.0, lambda_c = (3. * PI) / 2., theta_c = 0.;
    for (int i = 0; i < N; i++) {
        double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1], z = xyz[3 * (size_t)i + 2];
        double LI = std::atan2(y, x), TI = std::atan2(z, std::sqrt(x * x + y * y));
        double r = a * std::acos(std::sin(theta_c) * std::sin(TI) + std::cos(theta_c) * std::cos(TI) * std::cos(LI - lambda_c));
        double v = (h0 / 2.) * (1. + std::cos(PI * (r / R)));
        h[i] = (r >= R) ? 0.0 : v;
    }
    return RBFFD_OK;
}

// Real, orthonormal spherical harmonics Y_lm on the unit sphere, l <= lmax,
// coefficient order (l, m = -l..l).  u(x, t) = sum c_lm exp(-kappa l(l+1) t) Y_lm(x):
// the exact solution of u_t = kappa * Laplace-Beltrami(u).
extern "C" int rbffd_exact_sph_heat(int N, const double* xyz, int lmax, const double* coeffs, double kappa, double t,
                                    double* u)
{
    if (N < 0 || !xyz || !coeffs || !u || lmax < 0 || lmax > 200) return RBFFD_ERR_INVALID;
    const double PI = 3.14159265358979323846264338327950288;
    std::vector<double> decay(lmax + 1);
    for (int l = 0; l <= lmax; l++) decay[l] = std::exp(-kappa * l * (l + 1.0) * t);
    parallel_for(N, 0, [&](int i) {
        double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1], z = xyz[3 * (size_t)i + 2];
        double rho = std::sqrt(x * x + y * y);
        double ct = z, st = rho;  // cos/sin of colatitude
        double lam = std::atan2(y, x);
        std::vector<double> P((size_t)(lmax + 1) * (lmax + 1));
        auto idx = [&](int l, int m) { return (size_t)l * (lmax + 1) + m; };
        // fully normalised associated Legendre functions (4pi-normalised / 4pi)
        P[idx(0, 0)] = std::sqrt(1.0 / (4.0 * PI));
        for (int m = 1; m <= lmax; m++) P[idx(m, m)] = -std::sqrt((2.0 * m + 1.0) / (2.0 * m)) * st * P[idx(m - 1, m - 1)];
        for (int m = 0; m < lmax; m++) P[idx(m + 1, m)] = std::sqrt(2.0 * m + 3.0) * ct * P[idx(m, m)];
        for (int m = 0; m <= lmax; m++)
            for (int l = m + 2; l <= lmax; l++) {
                double a = std::sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
                double b = std::sqrt(((l - 1.0) * (l - 1.0) - (double)m * m) / (4.0 * (l - 1.0) * (l - 1.0) - 1.0));
                P[idx(l, m)] = a * (ct * P[idx(l - 1, m)] - b * P[idx(l - 2, m)]);
            }
        double s = 0.0;
        size_t k = 0;
        for (int l = 0; l <= lmax; l++) {
            double acc = 0.0;
            for (int m = -l; m <= l; m++, k++) {
                int am = m < 0 ? -m : m;
                double Y = P[idx(l, am)];
                if (m > 0) Y *= std::sqrt(2.0) * std::cos(am * lam);
                if (m < 0) Y *= std::sqrt(2.0) * std::sin(am * lam);
                acc += coeffs[k] * Y;
            }
            s += decay[l] * acc;
        }
        u[i] = s;
    });
    return RBFFD_OK;
}

// ---------------------------------------------------------------------------
// Node orders.  A grid stores its rows and nodes in an internal order so that
// rows handled together gather from nearby nodes (the reordering step before
// the SpMV, tests/util/cuthill_mckee/{main.cpp,reorder.h} in the reference).
// order[k] is the node placed at position k, as the reference's `order`
// vector (reorder.h: inv_order[order[i]] = i).
//
//   RBFFD_ORDER_MORTON -- nodes along a 3-D Morton curve: coordinates scaled
//     to 21-bit integers over the bounding box, bits interleaved x, y, z from
//     the top, ties by index.  The order every grid uses by default.
//   RBFFD_ORDER_RCM -- reverse Cuthill-McKee on the stencil graph, the order
//     the reference's utility computes with Boost's cuthill_mckee_ordering
//     (reorder.h:50-60; Boost is not part of the reference tree and its version
//     is not pinned).  Restated from the published algorithm (George & Liu):
//     the undirected graph joins every stencil's centre to its other nodes;
//     components are taken in order of their smallest node; each starts from a
//     pseudo-peripheral node found as Boost's find_starting_node does (from a
//     node r, x = the first node of least degree, in breadth-first order, on
//     the last level of r's level structure; repeat from x while its
//     eccentricity grows); a breadth-first search numbers each node's
//     unnumbered neighbours by increasing degree (ties by index); the whole
//     sequence is reversed.  Neighbour lists are sorted by index here, while
//     Boost keeps insertion order, so ties may break differently.
namespace {

void morton_order(int N, const double* xyz, int* order)
{
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < N; i++)
        for (int a = 0; a < 3; a++) {
            lo[a] = std::min(lo[a], xyz[3 * (size_t)i + a]);
            hi[a] = std::max(hi[a], xyz[3 * (size_t)i + a]);
        }
    std::vector<std::pair<uint64_t, int>> key(N);
    for (int i = 0; i < N; i++) {
        uint64_t code = 0;
        uint32_t q[3];
        for (int a = 0; a < 3; a++) {
            const double ext = hi[a] - lo[a];
            const double f = ext > 0 ? (xyz[3 * (size_t)i + a] - lo[a]) / ext : 0.0;
            q[a] = (uint32_t)std::min(2097151.0, std::max(0.0, f * 2097151.0));
        }
        for (int b = 20; b >= 0; b--)
            for (int a = 0; a < 3; a++) code = (code << 1) | ((q[a] >> b) & 1u);
        key[i] = {code, i};
    }
    std::sort(key.begin(), key.end());
    for (int i = 0; i < N; i++) order[i] = key[i].second;
}

struct StencilGraph {
    std::vector<int> ptr, adj;  // CSR, neighbours sorted by index, no self loops
    int deg(int v) const { return ptr[v + 1] - ptr[v]; }
};

StencilGraph stencil_graph(int N, int n_pad, const int* st, const int* st_len)
{
    std::vector<std::vector<int>> nb(N);
    for (int i = 0; i < N; i++) {
        const int L = st_len ? st_len[i] : n_pad;
        for (int s = 0; s < L; s++) {
            const int j = st[(size_t)i * n_pad + s];
            if (j == i) continue;
            nb[i].push_back(j);
            nb[j].push_back(i);
        }
    }
    StencilGraph G;
    G.ptr.assign(N + 1, 0);
    for (int v = 0; v < N; v++) {
        std::sort(nb[v].begin(), nb[v].end());
        nb[v].erase(std::unique(nb[v].begin(), nb[v].end()), nb[v].end());
        G.ptr[v + 1] = G.ptr[v] + (int)nb[v].size();
    }
    G.adj.reserve(G.ptr[N]);
    for (int v = 0; v < N; v++) G.adj.insert(G.adj.end(), nb[v].begin(), nb[v].end());
    return G;
}

// Breadth-first level structure from r over the nodes not yet numbered:
// returns the first node of least degree on the last level and sets ecc to
// r's eccentricity.
int last_level_min_degree(const StencilGraph& G, int r, const std::vector<char>& numbered, std::vector<int>& mark,
                          int stamp, int* ecc)
{
    std::vector<int> level{r}, next;
    mark[r] = stamp;
    int e = 0;
    for (;;) {
        next.clear();
        for (int v : level)
            for (int k = G.ptr[v]; k < G.ptr[v + 1]; k++) {
                const int w = G.adj[k];
                if (!numbered[w] && mark[w] != stamp) {
                    mark[w] = stamp;
                    next.push_back(w);
                }
            }
        if (next.empty()) break;
        level.swap(next);
        e++;
    }
    *ecc = e;
    int best = level[0];
    for (int v : level)
        if (G.deg(v) < G.deg(best)) best = v;
    return best;
}

void rcm_order(int N, int n_pad, const int* st, const int* st_len, int* order)
{
    const StencilGraph G = stencil_graph(N, n_pad, st, st_len);
    std::vector<char> numbered(N, 0);
    std::vector<int> mark(N, -1), cm;
    cm.reserve(N);
    int stamp = 0;
    for (int v0 = 0; v0 < N; v0++) {
        if (numbered[v0]) continue;
        // starting node of v0's component (Boost's find_starting_node)
        int r = v0, ecc_r = 0, ecc_x = 0;
        int x = last_level_min_degree(G, r, numbered, mark, stamp++, &ecc_r);
        int y = last_level_min_degree(G, x, numbered, mark, stamp++, &ecc_x);
        while (ecc_x > ecc_r) {
            r = x;
            ecc_r = ecc_x;
            x = y;
            y = last_level_min_degree(G, x, numbered, mark, stamp++, &ecc_x);
        }
        // Cuthill-McKee from x: unnumbered neighbours by increasing degree, ties by index
        const size_t head0 = cm.size();
        numbered[x] = 1;
        cm.push_back(x);
        std::vector<int> fresh;
        for (size_t h = head0; h < cm.size(); h++) {
            const int v = cm[h];
            fresh.clear();
            for (int k = G.ptr[v]; k < G.ptr[v + 1]; k++)
                if (!numbered[G.adj[k]]) {
                    numbered[G.adj[k]] = 1;
                    fresh.push_back(G.adj[k]);
                }
            std::sort(fresh.begin(), fresh.end(), [&](int a, int b) {
                return G.deg(a) != G.deg(b) ? G.deg(a) < G.deg(b) : a < b;
            });
            cm.insert(cm.end(), fresh.begin(), fresh.end());
        }
    }
    for (int k = 0; k < N; k++) order[k] = cm[N - 1 - k];  // reversed
}

}  // namespace

extern "C" int rbffd_node_order(int N, const double* xyz, int n_pad, const int* st, const int* st_len, int method,
                                int* order)
{
    if (N <= 0 || !order) return RBFFD_ERR_INVALID;
    if (method == RBFFD_ORDER_MORTON) {
        if (!xyz) return RBFFD_ERR_INVALID;
        morton_order(N, xyz, order);
        return RBFFD_OK;
    }
    if (method == RBFFD_ORDER_GIVEN) {
        for (int i = 0; i < N; i++) order[i] = i;
        return RBFFD_OK;
    }
    if (method != RBFFD_ORDER_RCM) return RBFFD_ERR_INVALID;
    if (!st || n_pad <= 0) return RBFFD_ERR_INVALID;
    for (int i = 0; i < N; i++) {
        const int L = st_len ? st_len[i] : n_pad;
        if (L < 1 || L > n_pad) return RBFFD_ERR_INVALID;
        for (int s = 0; s < L; s++)
            if (st[(size_t)i * n_pad + s] < 0 || st[(size_t)i * n_pad + s] >= N) return RBFFD_ERR_INVALID;
    }
    rcm_order(N, n_pad, st, st_len, order);
    return RBFFD_OK;
}

// ---------------------------------------------------------------------------
// Hash-grid stencils: Grid::generateStencilsHash
// (src/grids/grid_interface.cpp:733-966), the generator the reference's
// cosine-bell experiment uses (tests/experiments/cosine_bell_on_sphere/main.cpp:197-200).
// Not an exact nearest-neighbour search: candidates come from the cells around
// a node's cell, so a closer node just outside them can be missed.  Restated
// step by step so that the stencils and the node order are the reference's:
//  * extents: given, or the Grid defaults [0,1] x [0,1] x [0,0] widened by the
//    nodes (refreshExtents, grid_interface.h:376-398, as GridReader sets them);
//  * each node's cell (floor of (p - min) / cell size, the top cell closed);
//  * the node list re-sorted by cell id (nodes of a cell in index order): the
//    reference renumbers the grid, and order[k] is the node placed at k;
//  * per node, the cells within Chebyshev level 0, 1, 2, ... joined until they
//    hold at least n nodes and the level has passed 1; the z index is bounded
//    by the y cell count, as in the reference (grid_interface.cpp:894);
//  * candidates by distance sqrt(dx*dx + dy*dy + dz*dz) (Vec3d::magnitude), ties
//    in decreasing node number (the order the reference's std::set with a
//    `<=` comparator leaves them in, grid_interface.h:465-471), the first n
//    below max_radius kept (shorter stencils are trimmed).
// Where the reference would loop forever (fewer reachable nodes than n) or
// index out of range (a node outside given extents, a cell id past the last
// cell), this returns RBFFD_ERR_INVALID instead.
extern "C" int rbffd_stencils_hash(const double* xyz, int N, int n, int nbx, int nby, int nbz, const double* extents,
                                   double max_radius, int* order, int* st, int* st_len)
{
    if (!xyz || N <= 0 || n < 1 || n > N || nbx < 1 || nby < 1 || nbz < 1 || !order || !st || !st_len)
        return RBFFD_ERR_INVALID;
    const unsigned hnx = nbx, hny = nby, hnz = nbz;
    const size_t ncell = (size_t)hnx * hny * hnz;
    double lo[3], hi[3];
    if (extents) {
        lo[0] = extents[0], hi[0] = extents[1], lo[1] = extents[2], hi[1] = extents[3], lo[2] = extents[4],
        hi[2] = extents[5];
    } else {
        lo[0] = 0., hi[0] = 1., lo[1] = 0., hi[1] = 1., lo[2] = 0., hi[2] = 0.;
        for (int i = 0; i < N; i++)
            for (int a = 0; a < 3; a++) {
                const double v = xyz[3 * (size_t)i + a];
                if (v < lo[a]) lo[a] = v;
                if (v > hi[a]) hi[a] = v;
            }
    }
    const double cd[3] = {(hi[0] - lo[0]) / hnx, (hi[1] - lo[1]) / hny, (hi[2] - lo[2]) / hnz};
    if (!(cd[0] > 0 && cd[1] > 0 && cd[2] > 0)) return RBFFD_ERR_INVALID;  // a flat extent
    const unsigned hn[3] = {hnx, hny, hnz};
    std::vector<unsigned> cc(3 * (size_t)N);  // cell coordinates of each node
    for (int i = 0; i < N; i++)
        for (int a = 0; a < 3; a++) {
            const double f = std::floor((xyz[3 * (size_t)i + a] - lo[a]) / cd[a]);
            if (!(f >= 0.0 && f <= (double)hn[a])) return RBFFD_ERR_INVALID;  // outside the extents
            unsigned c = (unsigned)f;
            if (c == hn[a]) c--;
            cc[3 * (size_t)i + a] = c;
        }
    auto cell_of = [&](int i) {
        return ((size_t)cc[3 * (size_t)i] * hny + cc[3 * (size_t)i + 1]) * hnz + cc[3 * (size_t)i + 2];
    };
    // re-sort the nodes by cell: new number k holds old node order[k]
    std::vector<size_t> start(ncell + 1, 0);
    for (int i = 0; i < N; i++) start[cell_of(i) + 1]++;
    for (size_t c = 0; c < ncell; c++) start[c + 1] += start[c];
    {
        std::vector<size_t> fill(start.begin(), start.end() - 1);
        for (int i = 0; i < N; i++) order[fill[cell_of(i)]++] = i;
    }
    // node k (new numbering) lies in cell cell_of(order[k]); cell c holds new numbers start[c] .. start[c+1]-1
    std::atomic<int> failed(0);
    parallel_for(N, 0, [&](int p) {
        const int op = order[p];
        const int xc = (int)cc[3 * (size_t)op], yc = (int)cc[3 * (size_t)op + 1], zc = (int)cc[3 * (size_t)op + 2];
        static thread_local std::vector<char> in;  // the reference's std::set of non-empty neighbour cells
        if (in.size() < ncell) in.assign(ncell, 0);
        std::vector<size_t> cells;
        struct Clear {  // leave the flags cleared for this thread's next node
            std::vector<char>& f;
            std::vector<size_t>& c;
            ~Clear()
            {
                for (size_t k : c) f[k] = 0;
            }
        } clear{in, cells};
        size_t count = 0;
        const int maxlevel = (int)std::max(hnx, std::max(hny, hnz)) + 1;
        for (int level = 0; count < (size_t)n || level < 2; level++) {
            if (level > maxlevel) {  // every reachable cell is in: the reference would not stop
                failed = 1;
                return;
            }
            const int xl = level, yl = hny > 1 ? level : 0, zl = hnz > 1 ? level : 0;
            for (int dx = -xl; dx <= xl; dx++)
                for (int dy = -yl; dy <= yl; dy++)
                    for (int dz = -zl; dz <= zl; dz++) {
                        const int xo = xc + dx, yo = yc + dy, zo = zc + dz;
                        if (xo < 0 || xo >= (int)hnx || yo < 0 || yo >= (int)hny || zo < 0 || zo >= (int)hny)
                            continue;
                        const size_t cid = ((size_t)xo * hny + yo) * hnz + zo;
                        if (cid >= ncell) continue;  // past the last cell: undefined in the reference
                        if (!in[cid] && start[cid + 1] > start[cid]) {
                            in[cid] = 1;
                            cells.push_back(cid);
                            count += start[cid + 1] - start[cid];
                        }
                    }
        }
        const double* P = xyz + 3 * (size_t)op;
        std::vector<std::pair<double, int>> cand;
        cand.reserve(count);
        for (size_t cid : cells)
            for (size_t k = start[cid]; k < start[cid + 1]; k++) {
                const double* Q = xyz + 3 * (size_t)order[k];
                const double a = P[0] - Q[0], b = P[1] - Q[1], c = P[2] - Q[2];
                double s = a * a;
                s = s + b * b;
                s = s + c * c;
                cand.push_back({std::sqrt(s), (int)k});
            }
        auto less = [](const std::pair<double, int>& u, const std::pair<double, int>& v) {
            return u.first < v.first || (u.first == v.first && u.second > v.second);
        };
        std::nth_element(cand.begin(), cand.begin() + (n - 1), cand.end(), less);
        std::sort(cand.begin(), cand.begin() + n, less);
        int L = 0;
        while (L < n && cand[L].first < max_radius) {
            st[(size_t)p * n + L] = cand[L].second;
            L++;
        }
        for (int j = L; j < n; j++) st[(size_t)p * n + j] = p;  // padding: the centre
        st_len[p] = L;
    });
    return failed ? RBFFD_ERR_INVALID : RBFFD_OK;
}

// ---------------------------------------------------------------------------
// Vortex roll-up and solution norms.

namespace {

// The angular velocity of VortexRollup::solve / ExactRollup at one node, with
// the reference's operations: latitude from cart2sph, sech = 1 / cosh.
double rollup_w(double x, double y, double z, double* rho_out)
{
    const double theta_p = std::atan2(z, std::sqrt(x * x + y * y));
    const double rho_p = 3. * std::cos(theta_p);
    const double sech = 1. / std::cosh(rho_p);
    const double Vt = (3. * std::sqrt(3.) / 2.) * (sech * sech) * std::tanh(rho_p);
    if (rho_out) *rho_out = rho_p;
    return (std::fabs(rho_p) < 4. * 2.220446049250313080847e-16) ? 0. : Vt / rho_p;
}

}  // namespace

extern "C" int rbffd_vortex_rollup_coefficients(int N, const double* xyz, double* w)
{
    if (N < 0 || !xyz || !w) return RBFFD_ERR_INVALID;
    for (int i = 0; i < N; i++) w[i] = rollup_w(xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2], nullptr);
    return RBFFD_OK;
}

extern "C" int rbffd_exact_vortex_rollup(int N, const double* xyz, double t, double* h)
{
    if (N < 0 || !xyz || !h) return RBFFD_ERR_INVALID;
    const double gamma = 5.;
    for (int i = 0; i < N; i++) {
        const double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1], z = xyz[3 * (size_t)i + 2];
        double rho_p;
        const double w = rollup_w(x, y, z, &rho_p);
        const double phi_p = std::atan2(y, x);
        h[i] = 1. - std::tanh((rho_p / gamma) * std::sin(phi_p - w * t));
    }
    return RBFFD_OK;
}

extern "C" int rbffd_sol_norms(const double* sol, const double* exact, int n, double* out)
{
    if (n < 0 || !out || (n > 0 && (!sol || !exact))) return RBFFD_ERR_INVALID;
    double l1 = 0., l1d = 0., l2 = 0., l2d = 0., li = 0., lid = 0.;
    for (int i = 0; i < n; i++) {  // norms.cpp: l1norm, l2norm, linfnorm, in index order
        const double err = std::fabs(sol[i] - exact[i]);
        l1 += err;
        l2 += err * err;
        li = (li < err) ? err : li;
        l1d += std::fabs(exact[i]);
        l2d += exact[i] * exact[i];
        lid = (lid < std::fabs(exact[i])) ? std::fabs(exact[i]) : lid;
    }
    l2 = std::sqrt(l2);
    l2d = std::sqrt(l2d);
    auto rel = [](double a, double d) { return d > 1e-10 ? a / d : (a + 1.) / (d + 1.); };  // pde.cpp:470-480
    out[0] = l1;
    out[1] = rel(l1, l1d);
    out[2] = l2;
    out[3] = rel(l2, l2d);
    out[4] = li;
    out[5] = rel(li, lid);
    return RBFFD_OK;
}

// RBFFD::setVariableEpsilon (src/rbffd/rbffd.cpp:1378-1420, its
// VARIABLE_EPS_TYPE 1, Sarler 2006): eps at each stencil's centre =
// 1 / (alpha * r_max), r_max the distance from the centre to the stencil's
// last node (Grid::computeStencilRadii, grid_interface.cpp:556-557), as
// Vec3d::magnitude of the difference: sqrt(dx*dx + dy*dy + dz*dz).
extern "C" int rbffd_variable_epsilon(int N, const double* xyz, int n_pad, const int* st, const int* st_len,
                                      double alpha, double* eps)
{
    if (N <= 0 || !xyz || n_pad <= 0 || !st || !eps || alpha == 0.0) return RBFFD_ERR_INVALID;
    for (int i = 0; i < N; i++) {
        const int len = st_len ? st_len[i] : n_pad;
        if (len < 1 || len > n_pad) return RBFFD_ERR_INVALID;
        const int c = st[(size_t)i * n_pad], last = st[(size_t)i * n_pad + len - 1];
        if (c < 0 || c >= N || last < 0 || last >= N) return RBFFD_ERR_INVALID;
        const double dx = xyz[3 * (size_t)last] - xyz[3 * (size_t)c];
        const double dy = xyz[3 * (size_t)last + 1] - xyz[3 * (size_t)c + 1];
        const double dz = xyz[3 * (size_t)last + 2] - xyz[3 * (size_t)c + 2];
        eps[c] = 1. / (alpha * std::sqrt(dx * dx + dy * dy + dz * dz));
    }
    return RBFFD_OK;
}
