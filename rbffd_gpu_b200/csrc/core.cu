// Context, grid and derivative application (K2: ELL SpMV) of librbffd_sm100.
//
// Device layout of a grid: the sliced ELL arrays of ell.cuh (32-row slices,
// 4-slot chunks), n4 = n_pad rounded up to 4 slots per row, rows in the
// grid's internal (Morton) order.  A lane reads four consecutive slots of its
// row with one 16-byte index load and one 16-byte (FP32) or two 16-byte
// (FP64) weight loads.  Padding slots (s >= len[i]) hold the centre index and
// weight 0, as RBFFD_CL's ELL packing does (src/rbffd/rbffd_cl.cpp:238-242,
// 349-353), so every row runs n4 slots without a length check and the extra
// terms add exactly zero.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cstring>
#include <functional>
#include <iterator>
#include <new>
#include <thread>

#include "ell.cuh"
#include "internal.h"

// ---------------------------------------------------------------------------
// errors and accounting

int set_error(rbffd_ctx* ctx, int status, const char* fmt, ...)
{
    if (ctx) {
        char buf[1024];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        std::lock_guard<std::mutex> lk(ctx->err_mu);
        ctx->last_error = buf;
    }
    return status;
}

int cuda_error(rbffd_ctx* ctx, cudaError_t e, const char* what)
{
    int st = (e == cudaErrorMemoryAllocation) ? RBFFD_ERR_OOM : RBFFD_ERR_CUDA;
    cudaGetLastError();  // clear a sticky non-fatal error so the context stays usable
    return set_error(ctx, st, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

int dev_alloc(rbffd_ctx* ctx, void** p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) return RBFFD_OK;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return cuda_error(ctx, e, "cudaMalloc");
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->held += bytes;
    return RBFFD_OK;
}

void dev_free(rbffd_ctx* ctx, void* p, size_t bytes)
{
    if (!p) return;
    cudaFree(p);
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->held -= std::min(ctx->held, bytes);
}

extern "C" const char* rbffd_version(void) { return RBFFD_VERSION_STRING; }

extern "C" const char* rbffd_status_string(int s)
{
    switch (s) {
    case RBFFD_OK: return "ok";
    case RBFFD_ERR_INVALID: return "invalid argument";
    case RBFFD_ERR_OOM: return "out of memory";
    case RBFFD_ERR_CUDA: return "CUDA error";
    case RBFFD_ERR_TIMEOUT: return "timeout";
    case RBFFD_ERR_UNSUPPORTED: return "unsupported";
    case RBFFD_ERR_STATE: return "invalid state";
    case RBFFD_ERR_SINGULAR: return "singular stencil system";
    case RBFFD_ERR_BUDGET: return "over device memory budget";
    case RBFFD_ERR_NO_DEVICE: return "no CUDA device";
    case RBFFD_ERR_CANCELLED: return "request cancelled";
    }
    return "unknown status";
}

extern "C" int rbffd_device_count(int* count)
{
    if (!count) return RBFFD_ERR_INVALID;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *count = 0;
        return RBFFD_ERR_NO_DEVICE;
    }
    *count = n;
    return RBFFD_OK;
}

// ---------------------------------------------------------------------------
// context

extern "C" int rbffd_ctx_create(int device, rbffd_ctx** out)
{
    if (!out) return RBFFD_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return RBFFD_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) return RBFFD_ERR_INVALID;
    rbffd_ctx* c = new (std::nothrow) rbffd_ctx();
    if (!c) return RBFFD_ERR_OOM;
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return RBFFD_ERR_CUDA;
    }
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (cudaMalloc((void**)&c->d_status, sizeof(int)) != cudaSuccess ||
        cudaMemset(c->d_status, 0, sizeof(int)) != cudaSuccess || noalloc_preload() != RBFFD_OK) {
        cudaGetLastError();
        if (c->d_status) cudaFree(c->d_status);
        cudaStreamDestroy(c->stream);
        delete c;
        return RBFFD_ERR_CUDA;
    }
    *out = c;
    return RBFFD_OK;
}

int ctx_check_device_status(rbffd_ctx* ctx)
{
    int st = 0;
    RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (st == DEV_STATUS_OK) return RBFFD_OK;
    RBFFD_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return set_error(ctx, RBFFD_ERR_TIMEOUT, "a stage kernel gave up waiting for its bulk copies (device status %d)", st);
}

extern "C" int rbffd_ctx_destroy(rbffd_ctx* ctx)
{
    if (!ctx) return RBFFD_ERR_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    if (ctx->d_status) cudaFree(ctx->d_status);
    delete ctx;
    return RBFFD_OK;
}

extern "C" const char* rbffd_ctx_last_error(const rbffd_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

extern "C" int rbffd_ctx_synchronize(rbffd_ctx* ctx)
{
    if (!ctx) return RBFFD_ERR_INVALID;
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RBFFD_OK;
}

extern "C" int rbffd_ctx_mem_info(rbffd_ctx* ctx, size_t* held, size_t* free_bytes, size_t* total_bytes)
{
    if (!ctx) return RBFFD_ERR_INVALID;
    cudaSetDevice(ctx->device);
    size_t f = 0, t = 0;
    RBFFD_CUDA_TRY(ctx, cudaMemGetInfo(&f, &t));
    if (held) {
        std::lock_guard<std::mutex> lk(ctx->mu);
        *held = ctx->held;
    }
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return RBFFD_OK;
}

extern "C" int rbffd_ctx_stream(rbffd_ctx* ctx, void** stream)
{
    if (!ctx || !stream) return RBFFD_ERR_INVALID;
    *stream = (void*)ctx->stream;
    return RBFFD_OK;
}

// ---------------------------------------------------------------------------
// grid

// Host stencils [N][n_pad] (valid prefix len[i]) -> sliced ELL with centre padding.
__global__ void k_pack_stencils(const int* __restrict__ st_rm, const int* __restrict__ len, int N, int n_pad, int n4,
                                int nc, int* __restrict__ idx)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int L = len[i];
    for (int s = 0; s < n4; s++) idx[sell_elem(i, s, nc)] = (s < L) ? st_rm[(size_t)i * n_pad + s] : i;
}

__global__ void k_xyz4(const double* __restrict__ xyz, int N, double4* __restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    out[i] = make_double4(xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2], 0.0);
}

extern "C" int rbffd_grid_create(rbffd_ctx* ctx, int N, const double* xyz, int n_pad, const int* st, const int* st_len,
                                 rbffd_grid** out)
{
    return rbffd_grid_create_ordered(ctx, N, xyz, n_pad, st, st_len, RBFFD_ORDER_MORTON, out);
}

extern "C" int rbffd_grid_create_ordered(rbffd_ctx* ctx, int N, const double* xyz, int n_pad, const int* st,
                                         const int* st_len, int order_method, rbffd_grid** out)
{
    if (!ctx || !out || !xyz || !st || N <= 0 || n_pad <= 0 || n_pad > 1024) return RBFFD_ERR_INVALID;
    *out = nullptr;
    // Host-side validation: every index in range, centre first, lengths in [1, n_pad].
    std::vector<int> len(N);
    for (int i = 0; i < N; i++) {
        int L = st_len ? st_len[i] : n_pad;
        if (L < 1 || L > n_pad)
            return set_error(ctx, RBFFD_ERR_INVALID, "stencil %d: length %d outside [1, %d]", i, L, n_pad);
        const int* row = st + (size_t)i * n_pad;
        if (row[0] != i)
            return set_error(ctx, RBFFD_ERR_INVALID,
                             "stencil %d: centre must be the first entry (found %d; rbffd.cpp:916-928)", i, row[0]);
        for (int s = 0; s < L; s++)
            if (row[s] < 0 || row[s] >= N)
                return set_error(ctx, RBFFD_ERR_INVALID, "stencil %d slot %d: node index %d outside [0, %d)", i, s,
                                 row[s], N);
        len[i] = L;
    }
    cudaSetDevice(ctx->device);
    rbffd_grid* g = new (std::nothrow) rbffd_grid();
    if (!g) return RBFFD_ERR_OOM;
    g->ctx = ctx;
    g->N = N;
    g->n_pad = n_pad;
    g->n4 = round_up(n_pad, 4);
    g->nc = g->n4 / 4;
    g->N32 = round_up(N, 32);
    // Internal order (rbffd_node_order): by default nodes along a 3-D Morton
    // curve, so consecutive rows are spatial neighbours and share most of the
    // nodes their stencils gather.
    g->h_perm.resize(N);
    g->h_iperm.resize(N);
    {
        const int rc = rbffd_node_order(N, xyz, n_pad, st, st_len, order_method, g->h_perm.data());
        if (rc) {
            delete g;
            return set_error(ctx, rc, "node order %d", order_method);
        }
        for (int i = 0; i < N; i++) g->h_iperm[g->h_perm[i]] = i;
    }
    std::vector<int> st_int((size_t)N * n_pad, 0);
    std::vector<double> xyz_int((size_t)N * 3);
    g->h_len.resize(N);
    for (int i = 0; i < N; i++) {
        const int o = g->h_perm[i];
        g->h_len[i] = len[o];
        for (int s = 0; s < len[o]; s++) st_int[(size_t)i * n_pad + s] = g->h_iperm[st[(size_t)o * n_pad + s]];
        for (int a = 0; a < 3; a++) xyz_int[3 * (size_t)i + a] = xyz[3 * (size_t)o + a];
    }
    size_t b_idx = (size_t)g->N32 * g->n4 * sizeof(int), b_len = (size_t)N * sizeof(int),
           b_xyz = (size_t)N * sizeof(double4);
    int rc;
    int* d_st = nullptr;
    double* d_x3 = nullptr;
    if ((rc = dev_alloc(ctx, (void**)&g->d_idx, b_idx)) || (rc = dev_alloc(ctx, (void**)&g->d_len, b_len)) ||
        (rc = dev_alloc(ctx, (void**)&g->d_xyz, b_xyz)) || (rc = dev_alloc(ctx, (void**)&g->d_perm, b_len)) ||
        (rc = dev_alloc(ctx, (void**)&d_st, (size_t)N * n_pad * sizeof(int))) ||
        (rc = dev_alloc(ctx, (void**)&d_x3, (size_t)N * 3 * sizeof(double)))) {
        dev_free(ctx, d_st, (size_t)N * n_pad * sizeof(int));
        dev_free(ctx, d_x3, (size_t)N * 3 * sizeof(double));
        rbffd_grid_destroy(g);
        return rc;
    }
    g->bytes = b_idx + 2 * b_len + b_xyz;
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMemsetAsync(g->d_idx, 0, b_idx, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_st, st_int.data(), (size_t)N * n_pad * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g->d_len, g->h_len.data(), b_len, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g->d_perm, g->h_perm.data(), b_len, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_x3, xyz_int.data(), (size_t)N * 3 * sizeof(double), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        int B = 256, G = (N + B - 1) / B;
        k_pack_stencils<<<G, B, 0, s>>>(d_st, g->d_len, N, n_pad, g->n4, g->nc, g->d_idx);
        k_xyz4<<<G, B, 0, s>>>(d_x3, N, g->d_xyz);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    dev_free(ctx, d_st, (size_t)N * n_pad * sizeof(int));
    dev_free(ctx, d_x3, (size_t)N * 3 * sizeof(double));
    if (e != cudaSuccess) {
        rbffd_grid_destroy(g);
        return cuda_error(ctx, e, "rbffd_grid_create");
    }
    *out = g;
    return RBFFD_OK;
}

extern "C" int rbffd_grid_destroy(rbffd_grid* g)
{
    if (!g) return RBFFD_ERR_INVALID;
    rbffd_ctx* ctx = g->ctx;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    weights_work_free(g);
    size_t wsz = (size_t)g->N32 * g->n4;
    for (int t = 0; t < 16; t++) {
        dev_free(ctx, g->d_w64[t], wsz * sizeof(double));
        dev_free(ctx, g->d_w32[t], wsz * sizeof(float));
        dev_free(ctx, g->d_w32s[t], wsz * sizeof(float));
    }
    dev_free(ctx, g->d_idx, wsz * sizeof(int));
    dev_free(ctx, g->d_len, (size_t)g->N * sizeof(int));
    dev_free(ctx, g->d_perm, (size_t)g->N * sizeof(int));
    dev_free(ctx, g->d_xyz, (size_t)g->N * sizeof(double4));
    resident_free(g);
    for (auto& kv : g->halos) {
        Halo* h = kv.second;
        dev_free(ctx, h->d_ptr, (size_t)(h->nblocks + 1) * sizeof(int));
        dev_free(ctx, h->d_rows, (size_t)(h->nblocks + 1) * sizeof(int));
        dev_free(ctx, h->d_nodes, h->b_nodes);
        dev_free(ctx, h->d_lidx, h->b_lidx);
        for (int k = 0; k < 4; k++) {
            dev_free(ctx, h->d_lidx_s[k], h->b_lidx);
            dev_free(ctx, h->d_slot_s[k], h->b_lidx);
        }
        delete h;
    }
    delete g;
    return RBFFD_OK;
}

// Row blocks and their halos (see struct Halo).  Built on the host from the
// device's stencil array the first time a block size is used.
// Weights in a slot schedule: element e of the sliced ELL array (row i,
// scheduled slot t) takes row i's weight at its original slot slot[e], or 0
// for a padding entry.
__global__ void k_schedule_f32(const float* __restrict__ w, const unsigned short* __restrict__ slot, size_t n, int nc,
                               float* __restrict__ ws)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const size_t q = e >> 2;                      // (slice, chunk, lane) of the element
    const int i = (int)((q / 32) / nc) * 32 + (int)(q % 32);
    const unsigned short s = slot[e];
    ws[e] = s == SLOT_FREE ? 0.0f : w[sell_elem(i, s, nc)];
}

static void parallel_for(int count, const std::function<void(int)>& f)
{
    std::atomic<int> next(0);
    unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < hw; t++)
        pool.emplace_back([&]() {
            for (int k; (k = next.fetch_add(1)) < count;) f(k);
        });
    for (auto& t : pool) t.join();
}

// Slot schedule of one wavefront group (rows q0 .. q1-1, at most P) of a
// block whose halo has hn positions.  A row's reads of one step are 16-byte
// vectors of a 128/P-byte node record; the group's rows read in one
// shared-memory wavefront when their positions are different mod P (the bank
// group).  Each step is a maximum matching of rows to bank groups (Kuhn's
// augmenting paths): a row may take a remaining slot of that group
// (preferring the group it has most slots left in) or, while it has padding
// entries to spend, a padding entry placed in any free group.  Rows that stay
// unmatched take a remaining slot anyway (a conflict).
static void schedule_group(const rbffd_grid* g, const std::vector<unsigned short>& lidx, int q0, int q1, int hn,
                           int P, std::vector<unsigned short>& lidx_s, std::vector<unsigned short>& slot_s)
{
    const int nc = g->nc, n4 = g->n4, G = q1 - q0;
    std::vector<int> by[8][8];  // by[row][group]: remaining slots, the lowest last
    int realrem[8] = {}, freerem[8] = {};
    for (int r = 0; r < G; r++) {
        const int len = g->h_len[q0 + r];
        for (int s = len - 1; s >= 0; s--) by[r][lidx[sell_elem(q0 + r, s, nc)] & (P - 1)].push_back(s);
        realrem[r] = len;
        freerem[r] = n4 - len;
    }
    for (int t = 0; t < n4; t++) {
        int pref[8][8], npref[8] = {};
        for (int r = 0; r < G; r++) {
            int cs[8], k = 0;
            for (int c = 0; c < P; c++)
                if (!by[r][c].empty()) cs[k++] = c;
            std::sort(cs, cs + k, [&](int a, int b) { return by[r][a].size() > by[r][b].size(); });
            for (int j = 0; j < k; j++) pref[r][npref[r]++] = cs[j];
            if (freerem[r] > 0)
                for (int c = 0; c < P; c++)
                    if (by[r][c].empty()) pref[r][npref[r]++] = c;
        }
        int order[8];
        for (int r = 0; r < G; r++) order[r] = r;
        std::sort(order, order + G, [&](int a, int b) {
            if ((freerem[a] == 0) != (freerem[b] == 0)) return freerem[a] == 0;
            return npref[a] < npref[b];
        });
        int owner[8];
        for (int c = 0; c < P; c++) owner[c] = -1;
        std::function<bool(int, unsigned&)> augment = [&](int r, unsigned& seen) {
            for (int j = 0; j < npref[r]; j++) {
                const int c = pref[r][j];
                if (seen & (1u << c)) continue;
                seen |= 1u << c;
                if (owner[c] < 0 || augment(owner[c], seen)) {
                    owner[c] = r;
                    return true;
                }
            }
            return false;
        };
        for (int j = 0; j < G; j++) {
            unsigned seen = 0;
            augment(order[j], seen);
        }
        int colour[8];
        for (int r = 0; r < G; r++) colour[r] = -1;
        for (int c = 0; c < P; c++)
            if (owner[c] >= 0) colour[owner[c]] = c;
        for (int r = 0; r < G; r++) {
            const size_t e = sell_elem(q0 + r, t, nc);
            int c = colour[r];
            if (c < 0 || (by[r][c].empty() && freerem[r] == 0)) {  // unmatched: a conflicting slot
                c = -1;
                for (int k = 0; k < P; k++)
                    if (!by[r][k].empty() && (c < 0 || by[r][k].size() > by[r][c].size())) c = k;
            }
            if (c >= 0 && !by[r][c].empty()) {
                const int s = by[r][c].back();
                by[r][c].pop_back();
                realrem[r]--;
                slot_s[e] = (unsigned short)s;
                lidx_s[e] = lidx[sell_elem(q0 + r, s, nc)];
            } else {  // a padding entry, placed in group c (or 0)
                freerem[r]--;
                const int p = c < 0 ? 0 : c;
                slot_s[e] = SLOT_FREE;
                lidx_s[e] = (unsigned short)(p < hn ? p : p % std::max(hn, 1));
            }
        }
    }
}

int grid_halo_schedule(rbffd_grid* g, int R, int P, const Halo** out)
{
    rbffd_ctx* ctx = g->ctx;
    const int k = P == 2 ? 1 : (P == 4 ? 2 : (P == 8 ? 3 : -1));
    if (k < 0) return set_error(ctx, RBFFD_ERR_INVALID, "slot schedule for %d rows per wavefront", P);
    const Halo* hc = nullptr;
    int rc = grid_halo(g, R, &hc);
    if (rc) return rc;
    Halo* h = const_cast<Halo*>(hc);
    if (h->d_lidx_s[k]) {
        *out = h;
        return RBFFD_OK;
    }
    const size_t nidx = (size_t)g->N32 * g->n4;
    std::vector<unsigned short> lidx(nidx), lidx_s(nidx, 0), slot_s(nidx, SLOT_FREE);
    std::vector<int> rows(h->nblocks + 1), ptr(h->nblocks + 1);
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    RBFFD_CUDA_TRY(ctx, cudaMemcpy(lidx.data(), h->d_lidx, nidx * sizeof(unsigned short), cudaMemcpyDeviceToHost));
    RBFFD_CUDA_TRY(ctx, cudaMemcpy(rows.data(), h->d_rows, rows.size() * sizeof(int), cudaMemcpyDeviceToHost));
    RBFFD_CUDA_TRY(ctx, cudaMemcpy(ptr.data(), h->d_ptr, ptr.size() * sizeof(int), cudaMemcpyDeviceToHost));
    parallel_for(h->nblocks, [&](int b) {
        const int hn = ptr[b + 1] - ptr[b];
        for (int q0 = rows[b]; q0 < rows[b + 1]; q0 += P)
            schedule_group(g, lidx, q0, std::min(rows[b + 1], q0 + P), hn, P, lidx_s, slot_s);
    });
    const size_t bytes = nidx * sizeof(unsigned short);
    if ((rc = dev_alloc(ctx, (void**)&h->d_lidx_s[k], bytes))) return rc;
    if ((rc = dev_alloc(ctx, (void**)&h->d_slot_s[k], bytes))) {
        dev_free(ctx, h->d_lidx_s[k], bytes);
        h->d_lidx_s[k] = nullptr;
        return rc;
    }
    cudaError_t e = cudaMemcpy(h->d_lidx_s[k], lidx_s.data(), bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_slot_s[k], slot_s.data(), bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        dev_free(ctx, h->d_lidx_s[k], bytes);
        dev_free(ctx, h->d_slot_s[k], bytes);
        h->d_lidx_s[k] = h->d_slot_s[k] = nullptr;
        return cuda_error(ctx, e, "slot schedule upload");
    }
    g->bytes += 2 * bytes;
    *out = h;
    return RBFFD_OK;
}

int grid_halo(rbffd_grid* g, int R, const Halo** out)
{
    auto it = g->halos.find(R);
    if (it != g->halos.end()) {
        *out = it->second;
        return RBFFD_OK;
    }
    rbffd_ctx* ctx = g->ctx;
    if (R < 32 || R % 32) return set_error(ctx, RBFFD_ERR_INVALID, "rows per block %d must be a multiple of 32", R);
    const int N = g->N, nc = g->nc, n4 = g->n4;
    const size_t nidx = (size_t)g->N32 * n4;
    std::vector<int> idx(nidx);
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    RBFFD_CUDA_TRY(ctx, cudaMemcpy(idx.data(), g->d_idx, nidx * sizeof(int), cudaMemcpyDeviceToHost));
    // Per-slice (32 rows) sorted unique node lists.
    const int nsl = (N + 31) / 32;
    std::vector<std::vector<int>> snodes(nsl);
    auto run = [&](int count, const std::function<void(int)>& f) {
        std::atomic<int> next(0);
        unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < hw; t++)
            pool.emplace_back([&]() {
                for (int k; (k = next.fetch_add(1)) < count;) f(k);
            });
        for (auto& t : pool) t.join();
    };
    run(nsl, [&](int q) {
        std::vector<int>& v = snodes[q];
        for (int r = 32 * q; r < std::min(N, 32 * q + 32); r++)
            for (int s = 0; s < n4; s++) v.push_back(idx[sell_elem(r, s, nc)]);
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
    });
    auto merge = [](const std::vector<int>& x, const std::vector<int>& y) {
        std::vector<int> m;
        m.reserve(x.size() + y.size());
        std::set_union(x.begin(), x.end(), y.begin(), y.end(), std::back_inserter(m));
        return m;
    };
    // Cap on a block's halo: the 90th percentile of fixed R-row blocks' halos
    // (shared memory is sized by the largest halo, so outliers are split).
    const int spb = R / 32, nfixed = (nsl + spb - 1) / spb;
    std::vector<int> fsize(nfixed);
    run(nfixed, [&](int b) {
        std::vector<int> u;
        for (int q = b * spb; q < std::min(nsl, (b + 1) * spb); q++) u = merge(u, snodes[q]);
        fsize[b] = (int)u.size();
    });
    std::vector<int> sorted_f(fsize);
    std::sort(sorted_f.begin(), sorted_f.end());
    size_t cap = (size_t)sorted_f[(size_t)(0.9 * (sorted_f.size() - 1))];
    for (int q = 0; q < nsl; q++) cap = std::max(cap, snodes[q].size());
    if (cap > 65535) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "a block halo exceeds 65535 nodes");
    // Greedy partition: grow each block slice by slice while the halo stays under the cap.
    std::vector<int> bstart;
    std::vector<std::vector<int>> nodes;
    for (int q = 0; q < nsl;) {
        bstart.push_back(q);
        std::vector<int> cur = snodes[q++];
        while (q < nsl && q - bstart.back() < spb) {
            std::vector<int> m = merge(cur, snodes[q]);
            if (m.size() > cap) break;
            cur.swap(m);
            q++;
        }
        nodes.push_back(std::move(cur));
    }
    const int nblocks = (int)bstart.size();
    bstart.push_back(nsl);
    std::vector<int> rows(nblocks + 1);
    for (int b = 0; b <= nblocks; b++) rows[b] = std::min(N, 32 * bstart[b]);
    // Placement of each block's halo nodes in shared memory.  A block's kernel
    // reads, per stencil slot, one value (or 16-byte vector) per row; the 8
    // rows of a quarter-warp are served in one shared-memory wavefront only if
    // their nodes sit in different 16-byte bank groups (position mod 8).  A
    // greedy colouring gives the nodes read together different positions mod 8
    // where it can: position = 8 * rank + colour, padding slots repeat a node
    // of the block (staging stays branch-free).  Only positions change: the
    // arithmetic of every row is the same.
    std::vector<unsigned short> lidx(nidx, 0);
    std::vector<std::vector<int>> layout(nblocks);
    run(nblocks, [&](int b) {
        const std::vector<int>& v = nodes[b];
        const int K = (int)v.size(), r0 = rows[b], r1 = rows[b + 1];
        std::vector<int> kidx((size_t)(r1 - r0) * n4);  // sorted-halo index of each (row, slot)
        for (int r = r0; r < r1; r++)
            for (int s = 0; s < n4; s++)
                kidx[(size_t)(r - r0) * n4 + s] =
                    (int)(std::lower_bound(v.begin(), v.end(), idx[sell_elem(r, s, nc)]) - v.begin());
        // groups: the distinct nodes that 8 consecutive rows read at one slot
        std::vector<std::vector<int>> groups;
        std::vector<std::vector<int>> of_node(K);
        for (int q0 = r0; q0 < r1; q0 += 8)
            for (int s = 0; s < n4; s++) {
                std::vector<int> gset;
                for (int r = q0; r < std::min(r1, q0 + 8); r++) gset.push_back(kidx[(size_t)(r - r0) * n4 + s]);
                std::sort(gset.begin(), gset.end());
                gset.erase(std::unique(gset.begin(), gset.end()), gset.end());
                if (gset.size() < 2) continue;
                for (int k : gset) of_node[k].push_back((int)groups.size());
                groups.push_back(std::move(gset));
            }
        std::vector<int> order(K), colour(K, -1), used(8, 0);
        std::vector<std::array<int, 8>> cnt(groups.size());
        for (auto& c : cnt) c.fill(0);
        for (int k = 0; k < K; k++) order[k] = k;
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int c) { return of_node[a].size() > of_node[c].size(); });
        const int cap = (K + 7) / 8 + 1;
        for (int k : order) {
            int best = -1;
            long best_cost = 0;
            for (int c = 0; c < 8; c++) {
                if (used[c] >= cap) continue;
                long cost = 0;
                for (int g : of_node[k]) cost += cnt[g][c];
                if (best < 0 || cost < best_cost || (cost == best_cost && used[c] < used[best])) {
                    best = c;
                    best_cost = cost;
                }
            }
            colour[k] = best;
            used[best]++;
            for (int g : of_node[k]) cnt[g][best]++;
        }
        std::vector<int> pos(K), rank(8, 0);
        for (int k = 0; k < K; k++) pos[k] = 8 * rank[colour[k]]++ + colour[k];
        int hn = 0;
        for (int k = 0; k < K; k++) hn = std::max(hn, pos[k] + 1);
        std::vector<int>& lay = layout[b];
        lay.assign(hn, v[0]);
        for (int k = 0; k < K; k++) lay[pos[k]] = v[k];
        for (int r = r0; r < r1; r++)
            for (int s = 0; s < n4; s++)
                lidx[sell_elem(r, s, nc)] = (unsigned short)pos[kidx[(size_t)(r - r0) * n4 + s]];
    });
    std::vector<int> ptr(nblocks + 1, 0), flat;
    int max_halo = 0;
    for (int b = 0; b < nblocks; b++) {
        if (layout[b].size() > 65535) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "a block halo exceeds 65535 slots");
        ptr[b + 1] = ptr[b] + (int)layout[b].size();
        max_halo = std::max(max_halo, (int)layout[b].size());
    }
    flat.reserve(ptr[nblocks]);
    for (int b = 0; b < nblocks; b++) flat.insert(flat.end(), layout[b].begin(), layout[b].end());
    Halo* h = new (std::nothrow) Halo();
    if (!h) return RBFFD_ERR_OOM;
    h->R = R;
    h->nblocks = nblocks;
    h->max_halo = max_halo;
    const size_t b_ptr = ptr.size() * sizeof(int), b_nodes = flat.size() * sizeof(int),
                 b_lidx = nidx * sizeof(unsigned short);
    int rc;
    if ((rc = dev_alloc(ctx, (void**)&h->d_ptr, b_ptr)) || (rc = dev_alloc(ctx, (void**)&h->d_nodes, b_nodes)) ||
        (rc = dev_alloc(ctx, (void**)&h->d_lidx, b_lidx)) || (rc = dev_alloc(ctx, (void**)&h->d_rows, b_ptr))) {
        dev_free(ctx, h->d_ptr, b_ptr);
        dev_free(ctx, h->d_nodes, b_nodes);
        dev_free(ctx, h->d_lidx, b_lidx);
        delete h;
        return rc;
    }
    cudaError_t e = cudaMemcpy(h->d_ptr, ptr.data(), b_ptr, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_rows, rows.data(), b_ptr, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_nodes, flat.data(), b_nodes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_lidx, lidx.data(), b_lidx, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        dev_free(ctx, h->d_ptr, b_ptr);
        dev_free(ctx, h->d_nodes, b_nodes);
        dev_free(ctx, h->d_lidx, b_lidx);
        dev_free(ctx, h->d_rows, b_ptr);
        delete h;
        return cuda_error(ctx, e, "grid_halo upload");
    }
    h->b_nodes = b_nodes;
    h->b_lidx = b_lidx;
    g->bytes += 2 * b_ptr + b_nodes + b_lidx;
    g->halos[R] = h;
    *out = h;
    return RBFFD_OK;
}

// ---------------------------------------------------------------------------
// caller order <-> internal order

template <typename E>
__global__ void k_permute(const E* __restrict__ src, E* __restrict__ dst, const int* __restrict__ perm, int N, int T,
                          int to_internal)
{
    size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)N * T) return;
    int i = (int)(e / T), t = (int)(e % T);
    size_t o = (size_t)perm[i] * T + t;
    if (to_internal)
        dst[e] = src[o];
    else
        dst[o] = src[e];
}

static int grid_permute(rbffd_grid* g, const void* src, void* dst, int T, int elem_bytes, cudaStream_t s, int to_int)
{
    size_t n = (size_t)g->N * T;
    int nb = (int)((n + 255) / 256);
    if (elem_bytes == 8)
        k_permute<unsigned long long><<<nb, 256, 0, s>>>((const unsigned long long*)src, (unsigned long long*)dst,
                                                         g->d_perm, g->N, T, to_int);
    else if (elem_bytes == 4)
        k_permute<unsigned int><<<nb, 256, 0, s>>>((const unsigned int*)src, (unsigned int*)dst, g->d_perm, g->N, T,
                                                   to_int);
    else
        return set_error(g->ctx, RBFFD_ERR_INVALID, "element size %d", elem_bytes);
    RBFFD_CUDA_TRY(g->ctx, cudaGetLastError());
    return RBFFD_OK;
}

int grid_to_internal(rbffd_grid* g, const void* src, void* dst, int T, int elem_bytes, cudaStream_t s)
{
    return grid_permute(g, src, dst, T, elem_bytes, s, 1);
}

int grid_to_caller(rbffd_grid* g, const void* src, void* dst, int T, int elem_bytes, cudaStream_t s)
{
    return grid_permute(g, src, dst, T, elem_bytes, s, 0);
}

int grid_permute_preload()
{
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, k_permute<unsigned long long>) != cudaSuccess ||
        cudaFuncGetAttributes(&a, k_permute<unsigned int>) != cudaSuccess)
        return RBFFD_ERR_CUDA;
    return RBFFD_OK;
}

extern "C" int rbffd_grid_nbytes(const rbffd_grid* g, size_t* bytes)
{
    if (!g || !bytes) return RBFFD_ERR_INVALID;
    *bytes = g->bytes;
    return RBFFD_OK;
}

// ---------------------------------------------------------------------------
// weights in and out

// host layout [N][n_pad] in the caller's order -> sliced ELL in internal
// order (internal row i is the caller's row perm[i]), zero beyond the stencil length
__global__ void k_pad_rows(const double* __restrict__ w_rm, const int* __restrict__ len, const int* __restrict__ perm,
                           int N, int n_pad, int n4, int nc, double* __restrict__ w)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int L = len[i];
    const double* src = w_rm + (size_t)perm[i] * n_pad;
    for (int s = 0; s < n4; s++) w[sell_elem(i, s, nc)] = (s < L) ? src[s] : 0.0;
}

__global__ void k_unpad_rows(const double* __restrict__ w, const int* __restrict__ perm, int N, int n_pad, int nc,
                             double* __restrict__ w_rm)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double* dst = w_rm + (size_t)perm[i] * n_pad;
    for (int s = 0; s < n_pad; s++) dst[s] = w[sell_elem(i, s, nc)];
}

__global__ void k_cast_f32(const double* __restrict__ a, float* __restrict__ b, size_t n)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t stride = (size_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) b[i] = __double2float_rn(a[i]);
}

int grid_make_f32(rbffd_grid* g, int op)
{
    rbffd_ctx* ctx = g->ctx;
    size_t n = (size_t)g->N32 * g->n4;
    if (!g->d_w32[op]) {
        int rc = dev_alloc(ctx, (void**)&g->d_w32[op], n * sizeof(float));
        if (rc) return rc;
        g->bytes += n * sizeof(float);
    }
    k_cast_f32<<<std::max(1, std::min<int>((int)((n + 255) / 256), ctx->sm_count * 16)), 256, 0, ctx->stream>>>(
        g->d_w64[op], g->d_w32[op], n);
    RBFFD_CUDA_TRY(ctx, cudaGetLastError());
    g->w32_ver[op]++;
    if (g->d_w32s[op]) {  // keep the scheduled copy in step
        const Halo* h = g->halos.at(g->sched_R);
        k_schedule_f32<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(g->d_w32[op], h->d_slot_s[3], n, g->nc,
                                                                          g->d_w32s[op]);
        RBFFD_CUDA_TRY(ctx, cudaGetLastError());
    }
    return RBFFD_OK;
}

int grid_schedule_weights(rbffd_grid* g, const float* src, const unsigned short* slot, float* dst, cudaStream_t s)
{
    const size_t n = (size_t)g->N32 * g->n4;
    k_schedule_f32<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, slot, n, g->nc, dst);
    RBFFD_CUDA_TRY(g->ctx, cudaGetLastError());
    return RBFFD_OK;
}

int grid_f32_scheduled(rbffd_grid* g, int R, int op, const float** out)
{
    rbffd_ctx* ctx = g->ctx;
    // the grid's scheduled copies (d_w32s) all follow the 8-row schedule of one halo
    if (g->sched_R != 0 && g->sched_R != R)
        return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "a grid keeps its scheduled FP32 weights for one block size");
    const Halo* hs = nullptr;
    int rc = grid_halo_schedule(g, R, 8, &hs);
    if (rc) return rc;
    g->sched_R = R;
    if (!g->d_w32[op] && (rc = grid_make_f32(g, op))) return rc;
    if (!g->d_w32s[op]) {
        const size_t n = (size_t)g->N32 * g->n4;
        if ((rc = dev_alloc(ctx, (void**)&g->d_w32s[op], n * sizeof(float)))) return rc;
        g->bytes += n * sizeof(float);
        const Halo* h = g->halos.at(g->sched_R);
        k_schedule_f32<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(g->d_w32[op], h->d_slot_s[3], n, g->nc,
                                                                          g->d_w32s[op]);
        RBFFD_CUDA_TRY(ctx, cudaGetLastError());
    }
    *out = g->d_w32s[op];
    return RBFFD_OK;
}

// Allocate (once) the FP64 array of operator `op`.
int grid_alloc_w64(rbffd_grid* g, int op)
{
    if (g->d_w64[op]) return RBFFD_OK;
    size_t n = (size_t)g->N32 * g->n4;
    int rc = dev_alloc(g->ctx, (void**)&g->d_w64[op], n * sizeof(double));
    if (rc) return rc;
    g->bytes += n * sizeof(double);
    RBFFD_CUDA_TRY(g->ctx, cudaMemsetAsync(g->d_w64[op], 0, n * sizeof(double), g->ctx->stream));
    return RBFFD_OK;
}

extern "C" int rbffd_weights_set(rbffd_grid* g, unsigned der_type, const double* w)
{
    if (!g || !w) return RBFFD_ERR_INVALID;
    int op = der_index(der_type);
    if (op < 0) return set_error(g->ctx, RBFFD_ERR_INVALID, "der_type 0x%x is not a single operator", der_type);
    rbffd_ctx* ctx = g->ctx;
    cudaSetDevice(ctx->device);
    int rc = grid_alloc_w64(g, op);
    if (rc) return rc;
    size_t bytes = (size_t)g->N * g->n_pad * sizeof(double);
    double* tmp = nullptr;
    if ((rc = dev_alloc(ctx, (void**)&tmp, bytes))) return rc;
    cudaError_t e = cudaMemcpyAsync(tmp, w, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        k_pad_rows<<<(g->N + 255) / 256, 256, 0, ctx->stream>>>(tmp, g->d_len, g->d_perm, g->N, g->n_pad, g->n4,
                                                                 g->nc, g->d_w64[op]);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    dev_free(ctx, tmp, bytes);
    if (e != cudaSuccess) return cuda_error(ctx, e, "rbffd_weights_set");
    if ((rc = grid_make_f32(g, op))) return rc;
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RBFFD_OK;
}

extern "C" int rbffd_weights_get(rbffd_grid* g, unsigned der_type, double* w)
{
    if (!g || !w) return RBFFD_ERR_INVALID;
    int op = der_index(der_type);
    if (op < 0) return set_error(g->ctx, RBFFD_ERR_INVALID, "der_type 0x%x is not a single operator", der_type);
    if (!g->d_w64[op]) return set_error(g->ctx, RBFFD_ERR_STATE, "weights for der_type 0x%x not computed", der_type);
    rbffd_ctx* ctx = g->ctx;
    cudaSetDevice(ctx->device);
    size_t bytes = (size_t)g->N * g->n_pad * sizeof(double);
    double* tmp = nullptr;
    int rc = dev_alloc(ctx, (void**)&tmp, bytes);
    if (rc) return rc;
    k_unpad_rows<<<(g->N + 255) / 256, 256, 0, ctx->stream>>>(g->d_w64[op], g->d_perm, g->N, g->n_pad, g->nc, tmp);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(w, tmp, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    dev_free(ctx, tmp, bytes);
    if (e != cudaSuccess) return cuda_error(ctx, e, "rbffd_weights_get");
    return RBFFD_OK;
}

// ---------------------------------------------------------------------------
// K2: ELL apply.  G lanes per (row, tracer); lane g handles the 4-slot chunks
// g, g+G, ...; partial sums combined by xor-shuffle.  With G == 1 the
// accumulation order is the reference's (s = 0 .. n-1, rbffd.cpp:680-684) and
// FP64 results equal those of a fused-multiply-add CPU loop.

// PLAIN: each multiply-add rounded twice, product then sum (madd, ell.cuh):
// the reference's own build, whose x86-64 flags have no FMA.
template <typename T, int G, bool PLAIN = false>
__global__ void __launch_bounds__(256) k_ell_apply(const int* __restrict__ idx, const T* __restrict__ w, int nc,
                                                   const T* __restrict__ u, T* __restrict__ out, int start, int count,
                                                   int T_tr)
{
    int gt = blockIdx.x * blockDim.x + threadIdx.x;
    int r = gt / G, lane = gt % G;
    int rows = count * T_tr;
    bool active = r < rows;
    int i = start + (active ? r / T_tr : 0), t = active ? r % T_tr : 0;
    T acc = T(0);
    if (active) {
        for (int c = lane; c < nc; c += G) {
            const size_t o = sell_off(i, c, nc);
            int4 j = ld_idx4(idx + o);
            T wv[4];
            ld_w4(w + o, wv);
            acc = madd<T, PLAIN>(wv[0], __ldg(u + (size_t)j.x * T_tr + t), acc);
            acc = madd<T, PLAIN>(wv[1], __ldg(u + (size_t)j.y * T_tr + t), acc);
            acc = madd<T, PLAIN>(wv[2], __ldg(u + (size_t)j.z * T_tr + t), acc);
            acc = madd<T, PLAIN>(wv[3], __ldg(u + (size_t)j.w * T_tr + t), acc);
        }
    }
    acc = group_sum<G>(acc);
    if (active && lane == 0) out[(size_t)i * T_tr + t] = acc;
}

template <typename T>
static void launch_apply(rbffd_grid* g, const T* w, const T* u, T* out, int start, int count, int T_tr, int G,
                         cudaStream_t s)
{
    long long threads = (long long)count * T_tr * G;
    int B = 256, nb = (int)((threads + B - 1) / B);
    switch (G) {
    case 1: k_ell_apply<T, 1><<<nb, B, 0, s>>>(g->d_idx, w, g->nc, u, out, start, count, T_tr); break;
    case 2: k_ell_apply<T, 2><<<nb, B, 0, s>>>(g->d_idx, w, g->nc, u, out, start, count, T_tr); break;
    case 4: k_ell_apply<T, 4><<<nb, B, 0, s>>>(g->d_idx, w, g->nc, u, out, start, count, T_tr); break;
    default: k_ell_apply<T, 8><<<nb, B, 0, s>>>(g->d_idx, w, g->nc, u, out, start, count, T_tr); break;
    }
}

// Used by the unfused RK4 path as well (rk4.cu).
int grid_apply_dev(rbffd_grid* g, int op, int dtype, int T_tr, const void* u, void* out, int start, int count, int G,
                   cudaStream_t s)
{
    if (dtype == RBFFD_F64) {
        if (!g->d_w64[op]) return set_error(g->ctx, RBFFD_ERR_STATE, "weights of operator bit %d not computed", op);
        launch_apply<double>(g, g->d_w64[op], (const double*)u, (double*)out, start, count, T_tr, G, s);
    } else {
        if (!g->d_w32[op]) return set_error(g->ctx, RBFFD_ERR_STATE, "weights of operator bit %d not computed", op);
        launch_apply<float>(g, g->d_w32[op], (const float*)u, (float*)out, start, count, T_tr, G, s);
    }
    RBFFD_CUDA_TRY(g->ctx, cudaGetLastError());
    return RBFFD_OK;
}

int grid_apply_dev_plain(rbffd_grid* g, int op, int T_tr, const double* u, double* out, int start, int count,
                         cudaStream_t s)
{
    if (!g->d_w64[op]) return set_error(g->ctx, RBFFD_ERR_STATE, "weights of operator bit %d not computed", op);
    long long threads = (long long)count * T_tr;
    int nb = (int)((threads + 255) / 256);
    k_ell_apply<double, 1, true><<<nb, 256, 0, s>>>(g->d_idx, g->d_w64[op], g->nc, u, out, start, count, T_tr);
    RBFFD_CUDA_TRY(g->ctx, cudaGetLastError());
    return RBFFD_OK;
}

extern "C" int rbffd_ctx_set_arithmetic(rbffd_ctx* ctx, int arith)
{
    if (!ctx) return RBFFD_ERR_INVALID;
    if (arith != RBFFD_ARITH_FUSED && arith != RBFFD_ARITH_UNFUSED)
        return set_error(ctx, RBFFD_ERR_INVALID, "unknown arithmetic %d", arith);
    ctx->arith = arith;
    return RBFFD_OK;
}

extern "C" int rbffd_ctx_get_arithmetic(rbffd_ctx* ctx, int* arith)
{
    if (!ctx || !arith) return RBFFD_ERR_INVALID;
    *arith = ctx->arith;
    return RBFFD_OK;
}

__global__ void k_d2f(const double* __restrict__ a, float* __restrict__ b, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __double2float_rn(a[i]);
}
__global__ void k_f2d(const float* __restrict__ a, double* __restrict__ b, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
}

extern "C" int rbffd_apply(rbffd_grid* g, unsigned der_type, int dtype, unsigned start, unsigned count, const double* u,
                           double* deriv)
{
    if (!g || !u || !deriv) return RBFFD_ERR_INVALID;
    if (dtype != RBFFD_F32 && dtype != RBFFD_F64) return set_error(g->ctx, RBFFD_ERR_INVALID, "bad dtype %d", dtype);
    if ((size_t)start + count > (size_t)g->N) return set_error(g->ctx, RBFFD_ERR_INVALID, "range outside the grid");
    int op = der_index(der_type);
    if (op < 0) return set_error(g->ctx, RBFFD_ERR_INVALID, "der_type 0x%x is not a single operator", der_type);
    if (count == 0) return RBFFD_OK;
    rbffd_ctx* ctx = g->ctx;
    cudaSetDevice(ctx->device);
    int N = g->N;
    size_t b64 = (size_t)N * sizeof(double);
    double *du = nullptr, *dd = nullptr;
    float *fu = nullptr, *fd = nullptr;
    int rc = RBFFD_OK;
    if ((rc = dev_alloc(ctx, (void**)&du, b64)) || (rc = dev_alloc(ctx, (void**)&dd, b64)) ||
        (dtype == RBFFD_F32 && ((rc = dev_alloc(ctx, (void**)&fu, N * sizeof(float))) ||
                                (rc = dev_alloc(ctx, (void**)&fd, N * sizeof(float)))))) {
        dev_free(ctx, du, b64);
        dev_free(ctx, dd, b64);
        dev_free(ctx, fu, N * sizeof(float));
        return rc;
    }
    cudaStream_t s = ctx->stream;
    // du: caller order -> dd: internal order -> apply (all rows) -> du -> dd: caller order
    cudaError_t e = cudaMemcpyAsync(du, u, b64, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) rc = grid_to_internal(g, du, dd, 1, 8, s);
    if (e == cudaSuccess && rc == RBFFD_OK) {
        if (dtype == RBFFD_F64) {
            rc = ctx->arith == RBFFD_ARITH_UNFUSED ? grid_apply_dev_plain(g, op, 1, dd, du, 0, N, s)
                                                   : grid_apply_dev(g, op, dtype, 1, dd, du, 0, N, 1, s);
        } else {
            k_d2f<<<(N + 255) / 256, 256, 0, s>>>(dd, fu, N);
            rc = grid_apply_dev(g, op, dtype, 1, fu, fd, 0, N, 1, s);
            if (rc == RBFFD_OK) k_f2d<<<(N + 255) / 256, 256, 0, s>>>(fd, du, N);
        }
        if (rc == RBFFD_OK) rc = grid_to_caller(g, du, dd, 1, 8, s);
        e = cudaGetLastError();
    }
    if (rc == RBFFD_OK && e == cudaSuccess)
        e = cudaMemcpyAsync(deriv + start, dd + start, (size_t)count * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    dev_free(ctx, du, b64);
    dev_free(ctx, dd, b64);
    dev_free(ctx, fu, N * sizeof(float));
    dev_free(ctx, fd, N * sizeof(float));
    if (rc != RBFFD_OK) return rc;
    if (e != cudaSuccess) return cuda_error(ctx, e, "rbffd_apply");
    return RBFFD_OK;
}

extern "C" int rbffd_apply_dev(rbffd_grid* g, unsigned der_type, int dtype, int ntracers, const void* u_dev,
                               void* deriv_dev)
{
    if (!g || !u_dev || !deriv_dev || ntracers < 1) return RBFFD_ERR_INVALID;
    if (dtype != RBFFD_F32 && dtype != RBFFD_F64) return set_error(g->ctx, RBFFD_ERR_INVALID, "bad dtype %d", dtype);
    int op = der_index(der_type);
    if (op < 0) return set_error(g->ctx, RBFFD_ERR_INVALID, "der_type 0x%x is not a single operator", der_type);
    rbffd_ctx* ctx = g->ctx;
    cudaSetDevice(ctx->device);
    const int es = dtype == RBFFD_F64 ? 8 : 4;
    const size_t bytes = (size_t)g->N * ntracers * es;
    void *tin = nullptr, *tout = nullptr;
    int rc;
    if ((rc = dev_alloc(ctx, &tin, bytes)) || (rc = dev_alloc(ctx, &tout, bytes))) {
        dev_free(ctx, tin, bytes);
        return rc;
    }
    cudaStream_t s = ctx->stream;
    rc = grid_to_internal(g, u_dev, tin, ntracers, es, s);
    if (rc == RBFFD_OK)
        rc = dtype == RBFFD_F64 && ctx->arith == RBFFD_ARITH_UNFUSED
                 ? grid_apply_dev_plain(g, op, ntracers, (const double*)tin, (double*)tout, 0, g->N, s)
                 : grid_apply_dev(g, op, dtype, ntracers, tin, tout, 0, g->N, 1, s);
    if (rc == RBFFD_OK) rc = grid_to_caller(g, tout, deriv_dev, ntracers, es, s);
    cudaError_t e = cudaStreamSynchronize(s);
    dev_free(ctx, tin, bytes);
    dev_free(ctx, tout, bytes);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_error(ctx, e, "rbffd_apply_dev");
    return RBFFD_OK;
}
