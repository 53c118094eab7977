// Rightmost eigenvalues of an assembled operator on large grids: the
// stability question of RBFFD::computeEigenvalues (src/rbffd/rbffd.cpp:703-873)
// -- does the derivative operator (plus hyperviscosity) have eigenvalues with
// positive real part? -- answered without the dense N x N matrix.
//
// Implicitly restarted Arnoldi (Sorensen's method, the one ARPACK implements)
// for the eigenvalues of largest real part:
//   * the Krylov basis V (N x (ncv + 1), FP64, column-major) lives on the
//     device; a step applies the operator with the grid's FP64 sliced-ELL
//     kernel (K2), then orthogonalises twice against the basis (classical
//     Gram-Schmidt with one reorthogonalisation, CGS2), with deterministic
//     block-partial dot products;
//   * the small Hessenberg matrix H (ncv x ncv) stays on the host: its
//     eigenvalues come from the shifted QR algorithm in complex arithmetic
//     (Wilkinson shifts, Givens rotations, deflation on negligible
//     subdiagonals), the Ritz estimates |h_{m+1,m}| |e_m^T y| from inverse
//     iteration on H - theta I;
//   * a restart keeps the nev wanted Ritz values (never splitting a complex
//     pair) and filters the rest with exact shifts: H <- Q^T H Q with Q from
//     the QR factorisation of H - mu I (real mu) or of
//     H^2 - 2 Re(mu) H + |mu|^2 I (a complex pair, in real arithmetic), so the
//     basis stays real; V_k <- V_m Q[:, :k] and the new residual vector follow.
// Grids keep their internal node order throughout (eigenvalues do not depend
// on the numbering).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <vector>

#include "ell.cuh"
#include "internal.h"

int grid_apply_dev(rbffd_grid* g, int op, int dtype, int T_tr, const void* u, void* out, int start, int count, int G,
                   cudaStream_t s);

namespace {

using cd = std::complex<double>;

// ---------------------------------------------------------------------------
// small dense routines (host; row-major n x n)

// Eigenvalues of a real upper Hessenberg matrix by the shifted QR algorithm
// in complex arithmetic: Wilkinson shift from the trailing 2 x 2 block of the
// active window, one QR step by Givens rotations, deflation where a
// subdiagonal entry is negligible against its diagonal neighbours; an ad hoc
// shift every 11th iteration without deflation.  Returns false when a window
// does not converge in 100 iterations per eigenvalue.
bool hess_eigs(int n, const double* H, std::vector<cd>& ev)
{
    std::vector<cd> a((size_t)n * n);
    for (int i = 0; i < n * n; i++) a[i] = H[i];
    auto A = [&](int i, int j) -> cd& { return a[(size_t)i * n + j]; };
    ev.assign(n, cd(0.0));
    const double eps = 2.220446049250313e-16;
    int hi = n - 1, its = 0, total = 0;
    while (hi >= 0) {
        if (hi == 0) {
            ev[0] = A(0, 0);
            break;
        }
        int lo = hi;
        while (lo > 0) {
            const double s = std::abs(A(lo, lo)) + std::abs(A(lo - 1, lo - 1));
            if (std::abs(A(lo, lo - 1)) <= eps * (s > 0 ? s : 1.0)) {
                A(lo, lo - 1) = 0.0;
                break;
            }
            lo--;
        }
        if (lo == hi) {  // one eigenvalue deflated
            ev[hi] = A(hi, hi);
            hi--;
            its = 0;
            continue;
        }
        if (++its > 100 || ++total > 100 * n) return false;
        // shift: the eigenvalue of the trailing 2 x 2 block nearer its last diagonal entry
        cd mu;
        if (its % 11 == 0) {
            mu = A(hi, hi) + cd(std::abs(A(hi, hi - 1)) * 0.75, 0.0);
        } else {
            const cd p = A(hi - 1, hi - 1), q = A(hi - 1, hi), r = A(hi, hi - 1), d = A(hi, hi);
            const cd tr = p + d, det = p * d - q * r;
            const cd disc = std::sqrt(tr * tr * 0.25 - det);
            const cd l1 = tr * 0.5 + disc, l2 = tr * 0.5 - disc;
            mu = std::abs(l1 - d) < std::abs(l2 - d) ? l1 : l2;
        }
        // QR step on rows/columns lo..hi of A - mu I, then add mu back
        for (int i = lo; i <= hi; i++) A(i, i) -= mu;
        std::vector<cd> cs(hi - lo), sn(hi - lo);
        for (int k = lo; k < hi; k++) {
            const cd x = A(k, k), y = A(k + 1, k);
            const double r = std::sqrt(std::norm(x) + std::norm(y));
            cd c = 1.0, s = 0.0;
            if (r > 0) {
                c = x / r;
                s = y / r;
            }
            cs[k - lo] = c;
            sn[k - lo] = s;
            for (int j = k; j < n; j++) {  // rows k, k+1 <- G^H [rows]
                const cd u = A(k, j), v = A(k + 1, j);
                A(k, j) = std::conj(c) * u + std::conj(s) * v;
                A(k + 1, j) = -s * u + c * v;
            }
        }
        for (int k = lo; k < hi; k++) {  // columns k, k+1 <- [columns] G
            const cd c = cs[k - lo], s = sn[k - lo];
            const int top = std::min(hi, k + 2);
            for (int i = 0; i <= top; i++) {
                const cd u = A(i, k), v = A(i, k + 1);
                A(i, k) = u * c + v * s;
                A(i, k + 1) = -u * std::conj(s) + v * std::conj(c);
            }
        }
        for (int i = lo; i <= hi; i++) A(i, i) += mu;
    }
    return true;
}

// |e_{n-1}^T y| for the unit eigenvector y of H belonging to theta: two
// steps of inverse iteration with H - (theta + tiny) I, Gaussian elimination
// with partial pivoting in complex arithmetic.
double last_component(int n, const double* H, cd theta, double scale)
{
    std::vector<cd> y(n, cd(1.0)), a((size_t)n * n);
    const cd sh = theta + cd(1e-13 * scale, 0.0);
    for (int it = 0; it < 2; it++) {
        for (int i = 0; i < n * n; i++) a[i] = H[i];
        for (int i = 0; i < n; i++) a[(size_t)i * n + i] -= sh;
        std::vector<cd> b = y;
        for (int k = 0; k < n; k++) {
            int p = k;
            for (int i = k + 1; i < n; i++)
                if (std::abs(a[(size_t)i * n + k]) > std::abs(a[(size_t)p * n + k])) p = i;
            if (p != k) {
                for (int j = 0; j < n; j++) std::swap(a[(size_t)k * n + j], a[(size_t)p * n + j]);
                std::swap(b[k], b[p]);
            }
            cd piv = a[(size_t)k * n + k];
            if (std::abs(piv) == 0.0) piv = cd(1e-300, 0.0);
            for (int i = k + 1; i < n; i++) {
                const cd l = a[(size_t)i * n + k] / piv;
                if (l == cd(0.0)) continue;
                for (int j = k; j < n; j++) a[(size_t)i * n + j] -= l * a[(size_t)k * n + j];
                b[i] -= l * b[k];
            }
            a[(size_t)k * n + k] = piv;
        }
        for (int k = n - 1; k >= 0; k--) {
            cd s = b[k];
            for (int j = k + 1; j < n; j++) s -= a[(size_t)k * n + j] * y[j];
            y[k] = s / a[(size_t)k * n + k];
        }
        double nrm = 0.0;
        for (int i = 0; i < n; i++) nrm += std::norm(y[i]);
        nrm = std::sqrt(nrm);
        if (!(nrm > 0.0) || !std::isfinite(nrm)) return 1.0;
        for (int i = 0; i < n; i++) y[i] /= nrm;
    }
    return std::abs(y[n - 1]);
}

// Q of the Householder QR factorisation of the real n x n matrix M (row-major).
void householder_q(int n, std::vector<double> M, std::vector<double>& Q)
{
    Q.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) Q[(size_t)i * n + i] = 1.0;
    std::vector<double> v(n);
    for (int k = 0; k < n - 1; k++) {
        double alpha = 0.0;
        for (int i = k; i < n; i++) alpha += M[(size_t)i * n + k] * M[(size_t)i * n + k];
        alpha = std::sqrt(alpha);
        if (alpha == 0.0) continue;
        if (M[(size_t)k * n + k] > 0) alpha = -alpha;
        double vn = 0.0;
        for (int i = 0; i < n; i++) v[i] = i < k ? 0.0 : M[(size_t)i * n + k];
        v[k] -= alpha;
        for (int i = k; i < n; i++) vn += v[i] * v[i];
        if (vn == 0.0) continue;
        // M <- (I - 2 v v^T / vn) M ; Q <- Q (I - 2 v v^T / vn)
        for (int j = 0; j < n; j++) {
            double s = 0.0;
            for (int i = k; i < n; i++) s += v[i] * M[(size_t)i * n + j];
            s *= 2.0 / vn;
            for (int i = k; i < n; i++) M[(size_t)i * n + j] -= s * v[i];
        }
        for (int i = 0; i < n; i++) {
            double s = 0.0;
            for (int j = k; j < n; j++) s += Q[(size_t)i * n + j] * v[j];
            s *= 2.0 / vn;
            for (int j = k; j < n; j++) Q[(size_t)i * n + j] -= s * v[j];
        }
    }
}

// ---------------------------------------------------------------------------
// device kernels (vectors of N doubles; basis columns at stride N)

constexpr int AR_THREADS = 256;

// partial[b * nc + c] = sum over this block's rows of V[c][i] * w[i]
__global__ void __launch_bounds__(AR_THREADS) k_partial_dots(const double* __restrict__ V, const double* __restrict__ w,
                                                             int N, int nc, double* __restrict__ partial)
{
    __shared__ double red[AR_THREADS / 32];
    const int rows_per_block = (N + gridDim.x - 1) / gridDim.x;
    const int r0 = blockIdx.x * rows_per_block, r1 = min(N, r0 + rows_per_block);
    for (int c = 0; c < nc; c++) {
        double s = 0.0;
        const double* v = V + (size_t)c * N;
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) s = fma(v[i], w[i], s);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int k = 0; k < AR_THREADS / 32; k++) t += red[k];
            partial[(size_t)blockIdx.x * nc + c] = t;
        }
        __syncthreads();
    }
}

// out[c] = sum over blocks, in block order
__global__ void k_sum_partials(const double* __restrict__ partial, int nblocks, int nc, double* __restrict__ out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    double t = 0.0;
    for (int b = 0; b < nblocks; b++) t += partial[(size_t)b * nc + c];
    out[c] = t;
}

// w[i] -= sum_c V[c][i] * h[c]
__global__ void k_sub_combination(const double* __restrict__ V, const double* __restrict__ h, int N, int nc,
                                  double* __restrict__ w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double s = 0.0;
    for (int c = 0; c < nc; c++) s = fma(V[(size_t)c * N + i], h[c], s);
    w[i] -= s;
}

__global__ void k_scale_to(const double* __restrict__ w, double a, int N, double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) out[i] = w[i] * a;
}

__global__ void k_add_to(const double* __restrict__ a, int N, double* __restrict__ b)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) b[i] += a[i];
}

// out[c][i] = sum_r V[r][i] * Q[r][c] for c < kk (Q row-major m x m), and
// f[i] = beta * sum_r V[r][i] * Q[r][kk] + sigma * vres[i]
__global__ void k_restart_basis(const double* __restrict__ V, const double* __restrict__ Q, int N, int m, int kk,
                                double beta, double sigma, const double* __restrict__ vres, double* __restrict__ out,
                                double* __restrict__ f)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    for (int c = 0; c <= kk; c++) {
        double s = 0.0;
        for (int r = 0; r < m; r++) s = fma(V[(size_t)r * N + i], Q[(size_t)r * m + c], s);
        if (c < kk)
            out[(size_t)c * N + i] = s;
        else
            f[i] = beta * s + sigma * vres[i];
    }
}

struct DevBuf {
    rbffd_ctx* ctx;
    void* p = nullptr;
    size_t n = 0;
    explicit DevBuf(rbffd_ctx* c) : ctx(c) {}
    int alloc(size_t bytes)
    {
        n = bytes;
        return dev_alloc(ctx, &p, bytes);
    }
    ~DevBuf() { dev_free(ctx, p, n); }
    double* d() const { return (double*)p; }
};

}  // namespace

extern "C" int rbffd_hessenberg_eigenvalues(int n, const double* H, double* re, double* im)
{
    if (n < 1 || n > 4096 || !H || !re || !im) return RBFFD_ERR_INVALID;
    std::vector<cd> ev;
    if (!hess_eigs(n, H, ev)) return RBFFD_ERR_UNSUPPORTED;
    for (int i = 0; i < n; i++) {
        re[i] = ev[i].real();
        im[i] = ev[i].imag();
    }
    return RBFFD_OK;
}

extern "C" int rbffd_eigen_rightmost(rbffd_grid* g, unsigned der_type, int use_hv, int nev, int ncv, double tol,
                                     int max_restarts, unsigned long long seed, double* re, double* im,
                                     double* ritz_resid, int* nconv, int* restarts, int* matvecs)
{
    if (!g || !re || !im || nev < 1 || ncv < nev + 2 || ncv > 256 || !(tol > 0) || max_restarts < 1)
        return RBFFD_ERR_INVALID;
    rbffd_ctx* ctx = g->ctx;
    const int op = der_index(der_type), hv = use_hv ? der_index(RBFFD_HV) : -1;
    if (op < 0) return set_error(ctx, RBFFD_ERR_INVALID, "der_type 0x%x is not a single operator", der_type);
    if (!g->d_w64[op] || (use_hv && !g->d_w64[hv]))
        return set_error(ctx, RBFFD_ERR_STATE, "the operator's FP64 weights are not on the device");
    const int N = g->N, m = ncv;
    if (m >= N) return set_error(ctx, RBFFD_ERR_INVALID, "ncv %d must be below N %d", m, N);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const int nb_dot = std::min(4 * ctx->sm_count, (N + AR_THREADS - 1) / AR_THREADS);
    DevBuf V(ctx), W(ctx), T(ctx), part(ctx), small(ctx), Vn(ctx), F(ctx), Qd(ctx);
    int rc;
    if ((rc = V.alloc((size_t)(m + 1) * N * 8)) || (rc = W.alloc((size_t)N * 8)) || (rc = T.alloc((size_t)N * 8)) ||
        (rc = part.alloc((size_t)nb_dot * (m + 1) * 8)) || (rc = small.alloc((size_t)(m + 1) * 8)) ||
        (rc = Vn.alloc((size_t)m * N * 8)) || (rc = F.alloc((size_t)N * 8)) || (rc = Qd.alloc((size_t)m * m * 8)))
        return rc;
    const int nbN = (N + AR_THREADS - 1) / AR_THREADS;
    // w = A x (+ H x)
    auto apply = [&](const double* x, double* y) -> int {
        int r = grid_apply_dev(g, op, RBFFD_F64, 1, x, y, 0, N, 1, s);
        if (r == RBFFD_OK && use_hv) {
            r = grid_apply_dev(g, hv, RBFFD_F64, 1, x, T.d(), 0, N, 1, s);
            if (r == RBFFD_OK) k_add_to<<<nbN, AR_THREADS, 0, s>>>(T.d(), N, y);
        }
        return r;
    };
    // h = V[:, :nc]^T w (host)
    std::vector<double> hbuf(m + 1);
    auto dots = [&](int nc, const double* w, double* h) -> int {
        k_partial_dots<<<nb_dot, AR_THREADS, 0, s>>>(V.d(), w, N, nc, part.d());
        k_sum_partials<<<(nc + 127) / 128, 128, 0, s>>>(part.d(), nb_dot, nc, small.d());
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(h, small.d(), nc * 8, cudaMemcpyDeviceToHost, s));
        RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
        return RBFFD_OK;
    };
    auto norm2 = [&](const double* w, double* out) -> int {
        k_partial_dots<<<nb_dot, AR_THREADS, 0, s>>>(w, w, N, 1, part.d());
        k_sum_partials<<<1, 128, 0, s>>>(part.d(), nb_dot, 1, small.d());
        double v = 0;
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(&v, small.d(), 8, cudaMemcpyDeviceToHost, s));
        RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
        *out = std::sqrt(v);
        return RBFFD_OK;
    };
    // seeded start vector (splitmix64 uniforms in [-1, 1))
    {
        std::vector<double> v0(N);
        uint64_t st = seed ? seed : 0x5EEDull;
        for (int i = 0; i < N; i++) {
            uint64_t z = (st += 0x9E3779B97F4A7C15ull);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z ^= z >> 31;
            v0[i] = (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
        }
        double nv = 0;
        for (double x : v0) nv += x * x;
        nv = std::sqrt(nv);
        for (double& x : v0) x /= nv;
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(V.d(), v0.data(), (size_t)N * 8, cudaMemcpyHostToDevice, s));
        RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    }
    std::vector<double> H((size_t)(m + 1) * m, 0.0);  // row-major (m + 1) x m
    auto Hm = [&](int i, int j) -> double& { return H[(size_t)i * m + j]; };
    int j0 = 0, nmv = 0, kk = nev, it = 0;
    std::vector<cd> th;
    std::vector<double> est;
    double scale = 0.0;  // largest |Ritz value|: the spectral scale of the convergence test
    bool converged = false;
    for (it = 0; it < max_restarts; it++) {
        // extend the factorisation from j0 to m columns
        for (int j = j0; j < m; j++) {
            double* vj = V.d() + (size_t)j * N;
            if ((rc = apply(vj, W.d()))) return rc;
            nmv++;
            std::vector<double> h(j + 1, 0.0);
            for (int pass = 0; pass < 2; pass++) {  // CGS2
                if ((rc = dots(j + 1, W.d(), hbuf.data()))) return rc;  // also left in small.d()
                k_sub_combination<<<nbN, AR_THREADS, 0, s>>>(V.d(), small.d(), N, j + 1, W.d());
                for (int c = 0; c <= j; c++) h[c] += hbuf[c];
            }
            double beta;
            if ((rc = norm2(W.d(), &beta))) return rc;
            for (int c = 0; c <= j; c++) Hm(c, j) = h[c];
            Hm(j + 1, j) = beta;
            if (!(beta > 0.0)) beta = 1e-300;  // an invariant subspace: continue with a zero vector
            k_scale_to<<<nbN, AR_THREADS, 0, s>>>(W.d(), 1.0 / beta, N, V.d() + (size_t)(j + 1) * N);
        }
        RBFFD_CUDA_TRY(ctx, cudaGetLastError());
        // Ritz values, rightmost first
        std::vector<double> Hsq((size_t)m * m);
        for (int i = 0; i < m; i++)
            for (int j = 0; j < m; j++) Hsq[(size_t)i * m + j] = Hm(i, j);
        if (!hess_eigs(m, Hsq.data(), th))
            return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "the projected eigenproblem did not converge");
        std::stable_sort(th.begin(), th.end(), [](const cd& a, const cd& b) { return a.real() > b.real(); });
        scale = 0.0;
        for (const cd& t : th) scale = std::max(scale, std::abs(t));
        kk = nev;
        // keep a complex pair together
        if (kk < m && std::abs(th[kk - 1].imag()) > 1e-12 * scale && std::abs(th[kk].real() - th[kk - 1].real()) <=
                                                                        1e-10 * scale)
            kk++;
        if (kk > m - 2) kk = m - 2;
        est.assign(kk, 0.0);
        converged = true;
        for (int i = 0; i < kk; i++) {
            est[i] = std::abs(Hm(m, m - 1)) * last_component(m, Hsq.data(), th[i], scale);
            if (est[i] > tol * std::max(std::abs(th[i]), 1e-3 * scale)) converged = false;
        }
        if (converged) break;
        // exact shifts: the unwanted Ritz values, a complex pair as one real double shift
        std::vector<double> Hk = Hsq, Q((size_t)m * m, 0.0), Qi, M((size_t)m * m);
        for (int i = 0; i < m; i++) Q[(size_t)i * m + i] = 1.0;
        for (size_t q = kk; q < th.size();) {
            const cd mu = th[q];
            const bool pair = std::abs(mu.imag()) > 1e-12 * scale && q + 1 < th.size();
            for (int i = 0; i < m; i++)
                for (int j = 0; j < m; j++) {
                    double v = 0.0;
                    if (pair) {
                        for (int l = 0; l < m; l++) v += Hk[(size_t)i * m + l] * Hk[(size_t)l * m + j];
                        v -= 2.0 * mu.real() * Hk[(size_t)i * m + j];
                        if (i == j) v += std::norm(mu);
                    } else {
                        v = Hk[(size_t)i * m + j] - (i == j ? mu.real() : 0.0);
                    }
                    M[(size_t)i * m + j] = v;
                }
            householder_q(m, M, Qi);
            std::vector<double> Tm((size_t)m * m, 0.0), Hn((size_t)m * m, 0.0);
            for (int i = 0; i < m; i++)  // Tm = Hk Qi
                for (int l = 0; l < m; l++) {
                    const double a = Hk[(size_t)i * m + l];
                    if (a == 0.0) continue;
                    for (int j = 0; j < m; j++) Tm[(size_t)i * m + j] += a * Qi[(size_t)l * m + j];
                }
            for (int l = 0; l < m; l++)  // Hn = Qi^T Tm
                for (int i = 0; i < m; i++) {
                    const double a = Qi[(size_t)l * m + i];
                    if (a == 0.0) continue;
                    for (int j = 0; j < m; j++) Hn[(size_t)i * m + j] += a * Tm[(size_t)l * m + j];
                }
            for (int i = 0; i < m; i++)
                for (int j = 0; j < i - 1; j++) Hn[(size_t)i * m + j] = 0.0;  // Hessenberg again
            Hk = Hn;
            std::vector<double> Qn((size_t)m * m, 0.0);
            for (int i = 0; i < m; i++)
                for (int l = 0; l < m; l++) {
                    const double a = Q[(size_t)i * m + l];
                    if (a == 0.0) continue;
                    for (int j = 0; j < m; j++) Qn[(size_t)i * m + j] += a * Qi[(size_t)l * m + j];
                }
            Q = Qn;
            q += pair ? 2 : 1;
        }
        // restart: V_k <- V_m Q[:, :k]; f <- V_m Q[:, k] Hk[k][k-1] + h_{m+1,m} Q[m-1][k-1] v_{m+1}
        const double beta = Hk[(size_t)kk * m + kk - 1], sigma = Hm(m, m - 1) * Q[(size_t)(m - 1) * m + kk - 1];
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(Qd.d(), Q.data(), (size_t)m * m * 8, cudaMemcpyHostToDevice, s));
        k_restart_basis<<<nbN, AR_THREADS, 0, s>>>(V.d(), Qd.d(), N, m, kk, beta, sigma, V.d() + (size_t)m * N,
                                                    Vn.d(), F.d());
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(V.d(), Vn.d(), (size_t)kk * N * 8, cudaMemcpyDeviceToDevice, s));
        double fn;
        if ((rc = norm2(F.d(), &fn))) return rc;
        std::fill(H.begin(), H.end(), 0.0);
        for (int i = 0; i < kk; i++)
            for (int j = 0; j < kk; j++) Hm(i, j) = Hk[(size_t)i * m + j];
        Hm(kk, kk - 1) = fn;
        if (!(fn > 0.0)) fn = 1e-300;
        k_scale_to<<<nbN, AR_THREADS, 0, s>>>(F.d(), 1.0 / fn, N, V.d() + (size_t)kk * N);
        j0 = kk;
    }
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    const int nout = std::min(nev, (int)th.size());
    for (int i = 0; i < nout; i++) {
        re[i] = th[i].real();
        im[i] = th[i].imag();
        if (ritz_resid) ritz_resid[i] = i < (int)est.size() ? est[i] : 0.0;
    }
    int nc = 0;  // the loop's own test
    for (int i = 0; i < nout && i < (int)est.size(); i++)
        if (est[i] <= tol * std::max(std::abs(th[i]), 1e-3 * scale)) nc++;
    if (nconv) *nconv = nc;
    if (restarts) *restarts = it;
    if (matvecs) *matvecs = nmv;
    return RBFFD_OK;
}
