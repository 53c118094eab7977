// Context, grid and derivative application (K2: ELL SpMV) of librbffd_sm100.
//
// Device layout of a grid (row-major ELL): for row i and stencil slot s,
//   idx[i * n4 + s], w[i * n4 + s],   n4 = n_pad rounded up to 4,
// so a lane reads four consecutive slots of its row with one 16-byte index
// load and one 16-byte (FP32) or two 16-byte (FP64) weight loads, and the G
// lanes that share a row read its contiguous run together.  Padding slots
// (s >= len[i]) hold the centre index and weight 0, as RBFFD_CL's ELL packing
// does (src/rbffd/rbffd_cl.cpp:238-242, 349-353), so every row runs n4 slots
// without a length check and the extra terms add exactly zero.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>

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
    *out = c;
    return RBFFD_OK;
}

extern "C" int rbffd_ctx_destroy(rbffd_ctx* ctx)
{
    if (!ctx) return RBFFD_ERR_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
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
    g->h_len = len;
    size_t b_idx = (size_t)g->N32 * g->n4 * sizeof(int), b_len = (size_t)N * sizeof(int),
           b_xyz = (size_t)N * sizeof(double4);
    int rc;
    int* d_st = nullptr;
    double* d_x3 = nullptr;
    if ((rc = dev_alloc(ctx, (void**)&g->d_idx, b_idx)) || (rc = dev_alloc(ctx, (void**)&g->d_len, b_len)) ||
        (rc = dev_alloc(ctx, (void**)&g->d_xyz, b_xyz)) ||
        (rc = dev_alloc(ctx, (void**)&d_st, (size_t)N * n_pad * sizeof(int))) ||
        (rc = dev_alloc(ctx, (void**)&d_x3, (size_t)N * 3 * sizeof(double)))) {
        dev_free(ctx, d_st, (size_t)N * n_pad * sizeof(int));
        dev_free(ctx, d_x3, (size_t)N * 3 * sizeof(double));
        rbffd_grid_destroy(g);
        return rc;
    }
    g->bytes = b_idx + b_len + b_xyz;
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMemsetAsync(g->d_idx, 0, b_idx, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_st, st, (size_t)N * n_pad * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g->d_len, len.data(), b_len, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_x3, xyz, (size_t)N * 3 * sizeof(double), cudaMemcpyHostToDevice, s);
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
    size_t wsz = (size_t)g->N32 * g->n4;
    for (int t = 0; t < 16; t++) {
        dev_free(ctx, g->d_w64[t], wsz * sizeof(double));
        dev_free(ctx, g->d_w32[t], wsz * sizeof(float));
    }
    dev_free(ctx, g->d_idx, wsz * sizeof(int));
    dev_free(ctx, g->d_len, (size_t)g->N * sizeof(int));
    dev_free(ctx, g->d_xyz, (size_t)g->N * sizeof(double4));
    delete g;
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

// host layout [N][n_pad] -> sliced ELL, zero beyond the stencil length
__global__ void k_pad_rows(const double* __restrict__ w_rm, const int* __restrict__ len, int N, int n_pad, int n4, int nc,
                           double* __restrict__ w)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int L = len[i];
    for (int s = 0; s < n4; s++) w[sell_elem(i, s, nc)] = (s < L) ? w_rm[(size_t)i * n_pad + s] : 0.0;
}

__global__ void k_unpad_rows(const double* __restrict__ w, int N, int n_pad, int nc, double* __restrict__ w_rm)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    for (int s = 0; s < n_pad; s++) w_rm[(size_t)i * n_pad + s] = w[sell_elem(i, s, nc)];
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
        k_pad_rows<<<(g->N + 255) / 256, 256, 0, ctx->stream>>>(tmp, g->d_len, g->N, g->n_pad, g->n4, g->nc,
                                                                 g->d_w64[op]);
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
    k_unpad_rows<<<(g->N + 255) / 256, 256, 0, ctx->stream>>>(g->d_w64[op], g->N, g->n_pad, g->nc, tmp);
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

template <typename T, int G>
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
            acc = fma_rn<T>(wv[0], __ldg(u + (size_t)j.x * T_tr + t), acc);
            acc = fma_rn<T>(wv[1], __ldg(u + (size_t)j.y * T_tr + t), acc);
            acc = fma_rn<T>(wv[2], __ldg(u + (size_t)j.z * T_tr + t), acc);
            acc = fma_rn<T>(wv[3], __ldg(u + (size_t)j.w * T_tr + t), acc);
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
    cudaError_t e = cudaMemcpyAsync(du, u, b64, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        if (dtype == RBFFD_F64) {
            rc = grid_apply_dev(g, op, dtype, 1, du, dd, (int)start, (int)count, 1, s);
        } else {
            k_d2f<<<(N + 255) / 256, 256, 0, s>>>(du, fu, N);
            rc = grid_apply_dev(g, op, dtype, 1, fu, fd, (int)start, (int)count, 1, s);
            if (rc == RBFFD_OK) k_f2d<<<(N + 255) / 256, 256, 0, s>>>(fd, dd, N);
        }
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
    cudaSetDevice(g->ctx->device);
    return grid_apply_dev(g, op, dtype, ntracers, u_dev, deriv_dev, 0, g->N, 1, g->ctx->stream);
}
