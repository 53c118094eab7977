// Eigenvalue stability check of an assembled operator: RBFFD::computeEigenvalues
// (src/rbffd/rbffd.cpp:703-873).  The reference copies the weights of one
// operator (plus the hyperviscosity weights when it uses them,
// rbffd.cpp:737-749) into a dense N x N matrix, computes every eigenvalue with
// Armadillo's eig_gen (LAPACK dgeev) and classifies the real parts
// (rbffd.cpp:781-858).  Here the dense matrix is assembled on the device from
// the grid's FP64 sliced-ELL weights by a scatter kernel and handed to
// cuSOLVER's dense nonsymmetric eigensolver (cusolverDnXgeev, the geev of the
// same LAPACK family), resolved with dlopen at first use so the library does
// not depend on cuSOLVER unless this check runs.  Grids on the sphere have no
// boundary nodes, so the reference's identity rows for them are absent.
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <dlfcn.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "ell.cuh"
#include "internal.h"

namespace {

// A[col][row] (column-major, caller's order) = w[row][slot] (+ hv[row][slot])
// for every used slot of every row; the padding slots are skipped, so their
// zero weights do not overwrite the centre's entry.
__global__ void k_dense_operator(const int* __restrict__ idx, const double* __restrict__ w,
                                 const double* __restrict__ hv, const int* __restrict__ len,
                                 const int* __restrict__ perm, int N, int n4, int nc, double* __restrict__ A)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)N * n4) return;
    const int r = (int)(t / n4), s = (int)(t % n4);
    if (s >= len[r]) return;
    const size_t o = sell_elem(r, s, nc);
    const int row = perm[r], col = perm[idx[o]];
    A[(size_t)col * N + row] = hv ? w[o] + hv[o] : w[o];
}

// Real column-major matrix to complex (imaginary parts zero).
__global__ void k_to_complex(const double* __restrict__ A, double2* __restrict__ Z, size_t n)
{
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) Z[t] = make_double2(A[t], 0.0);
}

// cuSOLVER entry points, resolved once.
struct Solver {
    bool tried = false, ok = false;
    std::string why;
    decltype(&cusolverDnCreate) create = nullptr;
    decltype(&cusolverDnDestroy) destroy = nullptr;
    decltype(&cusolverDnSetStream) set_stream = nullptr;
    decltype(&cusolverDnCreateParams) create_params = nullptr;
    decltype(&cusolverDnDestroyParams) destroy_params = nullptr;
    decltype(&cusolverDnXgeev_bufferSize) geev_size = nullptr;
    decltype(&cusolverDnXgeev) geev = nullptr;
};

std::mutex solver_mu;
Solver solver;

const Solver& load_solver()
{
    std::lock_guard<std::mutex> lk(solver_mu);
    if (solver.tried) return solver;
    solver.tried = true;
    void* h = nullptr;
    for (const char* name : {"libcusolver.so.11", "libcusolver.so"})
        if ((h = dlopen(name, RTLD_NOW | RTLD_LOCAL))) break;
    if (!h) {
        const char* e = dlerror();
        solver.why = std::string("cuSOLVER not loadable: ") + (e ? e : "unknown");
        return solver;
    }
    auto sym = [&](auto& fp, const char* name) {
        fp = reinterpret_cast<std::remove_reference_t<decltype(fp)>>(dlsym(h, name));
        return fp != nullptr;
    };
    solver.ok = sym(solver.create, "cusolverDnCreate") && sym(solver.destroy, "cusolverDnDestroy") &&
                sym(solver.set_stream, "cusolverDnSetStream") &&
                sym(solver.create_params, "cusolverDnCreateParams") &&
                sym(solver.destroy_params, "cusolverDnDestroyParams") &&
                sym(solver.geev_size, "cusolverDnXgeev_bufferSize") && sym(solver.geev, "cusolverDnXgeev");
    if (!solver.ok) solver.why = "cuSOLVER lacks cusolverDnXgeev";
    return solver;
}

}  // namespace

extern "C" int rbffd_eig_classify(const double* re, int n, double zero_tol, rbffd_eig_output* out,
                                  double* max_neg_eig)
{
    if (!re || n <= 0 || !(zero_tol >= 0.0)) return RBFFD_ERR_INVALID;
    rbffd_eig_output o;
    // every extreme starts at |re[0]|, as in the reference (rbffd.cpp:771-776)
    const double e0 = std::fabs(re[0]);
    o.max_pos_eig = o.min_pos_eig = o.max_neg_eig = o.min_neg_eig = e0;
    o.nb_positive = o.nb_negative = o.nb_zero = 0;
    for (int i = 0; i < n; i++) {
        const double e = re[i], a = std::fabs(e);
        if (e > zero_tol) {
            o.nb_positive++;
            if (a > o.max_pos_eig) o.max_pos_eig = a;
            if (a < o.min_pos_eig) o.min_pos_eig = a;
        } else if (e < -zero_tol) {
            o.nb_negative++;
            if (a > o.max_neg_eig) o.max_neg_eig = a;
            if (a < o.min_neg_eig) o.min_neg_eig = a;
        } else {
            o.nb_zero++;
        }
    }
    if (out) *out = o;
    if (max_neg_eig) *max_neg_eig = o.max_neg_eig;
    return RBFFD_OK;
}

extern "C" int rbffd_eigenvalues(rbffd_grid* g, unsigned der_type, int use_hv, double* eig_re, double* eig_im,
                                 rbffd_eig_output* out, double* max_neg_eig)
{
    if (!g) return RBFFD_ERR_INVALID;
    rbffd_ctx* ctx = g->ctx;
    const int op = der_index(der_type);
    if (op < 0) return set_error(ctx, RBFFD_ERR_INVALID, "der_type 0x%x is not a single operator", der_type);
    const int N = g->N;
    if (N > RBFFD_EIG_MAX_N)
        return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "dense eigenvalues of N = %d above %d", N, RBFFD_EIG_MAX_N);
    const int hv_op = der_index(RBFFD_HV);
    if (!g->d_w64[op]) return set_error(ctx, RBFFD_ERR_STATE, "weights for der_type 0x%x not computed", der_type);
    if (use_hv && !g->d_w64[hv_op]) return set_error(ctx, RBFFD_ERR_STATE, "hyperviscosity weights not computed");
    const Solver& S = load_solver();
    if (!S.ok) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "%s", S.why.c_str());
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;

    const size_t nn = (size_t)N * N;
    double* A = nullptr;
    double2* Z = nullptr;  // complex copy, only if the solver refuses a real matrix
    double2* W = nullptr;
    int* info = nullptr;
    void* dwork = nullptr;
    size_t b_dwork = 0;
    std::vector<char> hwork;
    cusolverDnHandle_t handle = nullptr;
    cusolverDnParams_t params = nullptr;
    int rc = RBFFD_OK;
    cudaError_t e = cudaSuccess;
    cusolverStatus_t cs = CUSOLVER_STATUS_SUCCESS;
    cudaDataType typeA = CUDA_R_64F;
    void* Ain = nullptr;
    size_t b_host = 0;

    if ((rc = dev_alloc(ctx, (void**)&A, nn * sizeof(double))) ||
        (rc = dev_alloc(ctx, (void**)&W, (size_t)N * sizeof(double2))) ||
        (rc = dev_alloc(ctx, (void**)&info, sizeof(int))))
        goto done;
    e = cudaMemsetAsync(A, 0, nn * sizeof(double), s);
    if (e == cudaSuccess) {
        const long long threads = (long long)N * g->n4;
        k_dense_operator<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(
            g->d_idx, g->d_w64[op], use_hv ? g->d_w64[hv_op] : nullptr, g->d_len, g->d_perm, N, g->n4, g->nc, A);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        rc = cuda_error(ctx, e, "dense operator");
        goto done;
    }
    if ((cs = S.create(&handle)) != CUSOLVER_STATUS_SUCCESS || (cs = S.set_stream(handle, s)) ||
        (cs = S.create_params(&params))) {
        rc = set_error(ctx, RBFFD_ERR_CUDA, "cuSOLVER setup failed (status %d)", (int)cs);
        goto done;
    }
    // eigenvalues only (no eigenvectors) of the real matrix; if this solver
    // build takes only complex matrices, of its complex copy
    Ain = A;
    cs = S.geev_size(handle, params, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_NOVECTOR, N, CUDA_R_64F, A, N,
                     CUDA_C_64F, W, CUDA_R_64F, nullptr, 1, CUDA_R_64F, nullptr, 1, CUDA_R_64F, &b_dwork, &b_host);
    if (cs != CUSOLVER_STATUS_SUCCESS) {
        typeA = CUDA_C_64F;
        if ((rc = dev_alloc(ctx, (void**)&Z, nn * sizeof(double2)))) goto done;
        k_to_complex<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(A, Z, nn);
        if ((e = cudaGetLastError()) != cudaSuccess) {
            rc = cuda_error(ctx, e, "complex copy");
            goto done;
        }
        Ain = Z;
        cs = S.geev_size(handle, params, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_NOVECTOR, N, CUDA_C_64F, Z,
                         N, CUDA_C_64F, W, CUDA_C_64F, nullptr, 1, CUDA_C_64F, nullptr, 1, CUDA_C_64F, &b_dwork,
                         &b_host);
        if (cs != CUSOLVER_STATUS_SUCCESS) {
            rc = set_error(ctx, RBFFD_ERR_UNSUPPORTED, "cusolverDnXgeev_bufferSize failed (status %d)", (int)cs);
            goto done;
        }
    }
    if ((rc = dev_alloc(ctx, &dwork, b_dwork))) goto done;
    hwork.resize(b_host > 0 ? b_host : 1);
    cs = S.geev(handle, params, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_NOVECTOR, N, typeA, Ain, N, CUDA_C_64F,
                W, typeA, nullptr, 1, typeA, nullptr, 1, typeA, dwork, b_dwork, hwork.data(), b_host, info);
    if (cs != CUSOLVER_STATUS_SUCCESS) {
        rc = set_error(ctx, RBFFD_ERR_CUDA, "cusolverDnXgeev failed (status %d)", (int)cs);
        goto done;
    }
    {
        std::vector<double2> w(N);
        int h_info = 0;
        e = cudaMemcpyAsync(w.data(), W, (size_t)N * sizeof(double2), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            rc = cuda_error(ctx, e, "rbffd_eigenvalues");
            goto done;
        }
        if (h_info != 0) {
            rc = set_error(ctx, RBFFD_ERR_SINGULAR, "geev did not converge (info %d)", h_info);
            goto done;
        }
        std::vector<double> re(N);
        for (int i = 0; i < N; i++) {
            re[i] = w[i].x;
            if (eig_re) eig_re[i] = w[i].x;
            if (eig_im) eig_im[i] = w[i].y;
        }
        rc = rbffd_eig_classify(re.data(), N, 1e-8, out, max_neg_eig);  // tolerance of rbffd.cpp:794-802
    }
done:
    if (params) S.destroy_params(params);
    if (handle) S.destroy(handle);
    cudaStreamSynchronize(s);
    dev_free(ctx, dwork, b_dwork);
    dev_free(ctx, Z, nn * sizeof(double2));
    dev_free(ctx, info, sizeof(int));
    dev_free(ctx, W, (size_t)N * sizeof(double2));
    dev_free(ctx, A, nn * sizeof(double));
    return rc;
}
