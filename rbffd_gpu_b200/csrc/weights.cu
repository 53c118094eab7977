// K1: batched FP64 RBF-FD weight computation.
//
// Per stencil (RBFFD::computeAllWeightsForStencil_Direct, src/rbffd/rbffd.cpp:225-352):
//   assemble  A = [Phi P; P^T 0] (distanceMatrix rbffd.cpp:888-969, getStencilLHS :129-191)
//   assemble  B = one column per selected operator (getStencilRHS :356-537)
//   solve     A W = B  (arma::solve -> LAPACK dgesv, :259)
//   store     weights[type][stencil][j] = W(j, col) * scale (HV: getHVScalar, :285-306)
// all fused in one kernel: a "team" of TW threads owns one system at a time,
// holds the augmented matrix [A | B] (m x (m+K), FP64) in shared memory and
// runs Gaussian elimination with partial pivoting (first maximal |pivot|,
// multipliers by division, fused updates) and a column-oriented back
// substitution -- the arithmetic of dgetf2 + dgetrs, so given the same
// assembled matrix the solution equals the CPU restatement bit for bit.
// Teams loop over the systems of one size bucket (persistent, grid-stride);
// buckets group stencils by system size m = n + np so shared memory is sized
// per bucket, and a small autotuner picks the team width per bucket.
//
// Polynomial augmentation: poly_deg 0 is the reference build (constant
// column, RHS row 0 for every operator, rbffd.cpp:1,150-155,506-508);
// poly_deg 1 is {1,x,y,z} (rbffd.cpp:150-172) with the operator applied
// exactly to each function (the reference does this for X/Y/Z/LAPL only and
// zeroes the other rows with a warning, rbffd.cpp:510-531).  Beyond the
// reference, poly_deg 2..4 use polynomials of total degree <= d in scaled
// tangent-plane coordinates of the centre c,
//   xi = (x - c).e_lambda / s,  eta = (x - c).e_theta / s,  s = max_j |x_j - c|,
// (d+1)(d+2)/2 terms; 3-D monomials restricted to a small cap are nearly
// dependent and would make the border block singular to working precision.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <map>
#include <vector>

#include "ell.cuh"
#include "internal.h"

int grid_alloc_w64(rbffd_grid* g, int op);

namespace {

constexpr int MAX_K = 8;       // operators per solve
constexpr int MAX_WARPS = 8;   // per team
constexpr int MAX_M = 160;     // largest system (stencil + polynomial terms)
constexpr int ELIM_CHUNKS = (MAX_M + MAX_K + 31) / 32;  // 32-column chunks of a row

constexpr int MAX_CLASSES = 24;  // system sizes in one persistent launch

// One system size in the persistent launch: its rows are rows[rows_off ..
// rows_off + nrows), solved `teams` at a time per CTA by teams of `team`
// threads, each holding its system at row stride lda in `stride` doubles of
// shared memory; its work units are numbered from unit0.
struct WClass {
    int m, lda, team, teams, stride, blocked, rows_off, nrows, unit0;
};

struct WParams {
    const double4* xyz;
    const int* idx;
    const int* len;
    const double* eps;
    const int* deg;
    const int* rows;
    double* w[MAX_K];
    int* status;  // min(row) + 1 over rows with a zero pivot, INT_MAX if none
    int* work;    // next work unit (the persistent launch's counter, zeroed before it)
    double eps_uniform, hv_scale;
    int n4, n_pad, deg_uniform, nrows, K, m, dim, hv_k, team_stride;  // n4: row stride; team_stride: doubles per team
    int opbit[MAX_K];
    int nclasses, nunits;
    WClass cls[MAX_CLASSES];
};

struct Team {
    int tid, size, id;  // thread index in team, team width, team index in CTA
    __device__ __forceinline__ void sync() const
    {
        if (size == 32)
            __syncwarp();
        else
            asm volatile("bar.sync %0, %1;" ::"r"(id + 1), "r"(size) : "memory");
    }
    __device__ __forceinline__ int warp() const { return tid >> 5; }
    __device__ __forceinline__ int lane() const { return tid & 31; }
    __device__ __forceinline__ int nwarps() const { return size >> 5; }
};

__device__ __forceinline__ double ipow(double x, int a)
{
    double r = 1.0;
    for (int i = 0; i < a; i++) r *= x;
    return r;
}

// exponent of basis function q (ordering documented above)
__device__ void basis_exp(int q, int& a, int& b, int& c)
{
    int t = 0;
    while ((t + 1) * (t + 1) <= q) t++;  // first index of degree t is t^2
    int r = q - t * t;
    if (r <= t) {
        a = t - r; b = r; c = 0;
    } else {
        r -= t + 1;
        a = t - 1 - r; b = r; c = 1;
    }
}

// d^(da,db,dc) of x^a y^b z^c at (x,y,z)
__device__ double mono_d(int a, int b, int c, int da, int db, int dc, double x, double y, double z)
{
    if (da > a || db > b || dc > c) return 0.0;
    double k = 1.0;
    for (int i = 0; i < da; i++) k *= (a - i);
    for (int i = 0; i < db; i++) k *= (b - i);
    for (int i = 0; i < dc; i++) k *= (c - i);
    return k * ipow(x, a - da) * ipow(y, b - db) * ipow(z, c - dc);
}

__device__ double lapl_dim(int a, int b, int c, int dim, double x, double y, double z)
{
    double s = mono_d(a, b, c, 2, 0, 0, x, y, z);
    if (dim > 1) s += mono_d(a, b, c, 0, 2, 0, x, y, z);
    if (dim > 2) s += mono_d(a, b, c, 0, 0, 2, x, y, z);
    return s;
}

// Operator `bit` applied to basis function q at the centre c.
__device__ double poly_row(unsigned bit, int q, const double* c, int dim, int hv_k, double lam, double th)
{
    int a, b, cc;
    basis_exp(q, a, b, cc);
    double x = c[0], y = c[1], z = c[2];
    double gx = mono_d(a, b, cc, 1, 0, 0, x, y, z), gy = mono_d(a, b, cc, 0, 1, 0, x, y, z),
           gz = mono_d(a, b, cc, 0, 0, 1, x, y, z);
    double cg = x * gx + y * gy + z * gz;
    switch (bit) {
    case RBFFD_X: return gx;
    case RBFFD_Y: return gy;
    case RBFFD_Z: return gz;
    case RBFFD_LAPL: return lapl_dim(a, b, cc, dim, x, y, z);
    case RBFFD_INTERP: return mono_d(a, b, cc, 0, 0, 0, x, y, z);
    case RBFFD_LAMBDA: return -sin(lam) * gx + cos(lam) * gy;
    case RBFFD_THETA: return -sin(th) * cos(lam) * gx - sin(th) * sin(lam) * gy + cos(th) * gz;
    case RBFFD_LSFC: {
        double H[3][3];
        const int e[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                H[i][j] = mono_d(a, b, cc, e[i][0] + e[j][0], e[i][1] + e[j][1], e[i][2] + e[j][2], x, y, z);
        double tr = H[0][0] + H[1][1] + H[2][2], qf = 0.0;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) qf += c[i] * H[i][j] * c[j];
        return tr - qf - 2.0 * cg;
    }
    case RBFFD_XSFC: return gx - x * cg;
    case RBFFD_YSFC: return gy - y * cg;
    case RBFFD_ZSFC: return gz - z * cg;
    case RBFFD_HV: {
        if (hv_k == 0) return mono_d(a, b, cc, 0, 0, 0, x, y, z);
        if (hv_k == 1) return lapl_dim(a, b, cc, dim, x, y, z);
        if (hv_k == 2) {
            double s = 0.0;
            for (int i = 0; i < dim && i < 3; i++)
                for (int j = 0; j < dim && j < 3; j++) {
                    int d[3] = {0, 0, 0};
                    d[i] += 2;
                    d[j] += 2;
                    s += mono_d(a, b, cc, d[0], d[1], d[2], x, y, z);
                }
            return s;
        }
        return 0.0;  // degree <= 4 < 2k
    }
    default: return 0.0;  // R, ALT_*: no polynomial counterpart (rbffd.cpp:527-531)
    }
}

__host__ __device__ inline int poly_size(int deg)
{
    return deg < 0 ? 0 : (deg == 0 ? 1 : (deg == 1 ? 4 : (deg + 1) * (deg + 2) / 2));
}

// exponents (a, b) of tangent basis function q: total degree t, a = t..0
__device__ void tangent_exp(int q, int& a, int& b)
{
    int t = 0;
    while ((t + 1) * (t + 2) / 2 <= q) t++;
    int r = q - t * (t + 1) / 2;
    a = t - r;
    b = r;
}

__device__ double dfact(int a)
{
    double f = 1.0;
    for (int i = 2; i <= a; i++) f *= i;
    return f;
}

// Operator `bit` applied to xi^a eta^b at the centre (xi = eta = 0).
__device__ double tangent_row(unsigned bit, int a, int b, const double* e1, const double* e2, double s, int dim, int hv_k)
{
    const int t = a + b;
    switch (bit) {
    case RBFFD_INTERP: return t == 0 ? 1.0 : 0.0;
    case RBFFD_LAMBDA: return (a == 1 && b == 0) ? 1.0 / s : 0.0;
    case RBFFD_THETA: return (a == 0 && b == 1) ? 1.0 / s : 0.0;
    case RBFFD_X: case RBFFD_Y: case RBFFD_Z: case RBFFD_XSFC: case RBFFD_YSFC: case RBFFD_ZSFC: {
        int ax = (bit == RBFFD_X || bit == RBFFD_XSFC) ? 0 : ((bit == RBFFD_Y || bit == RBFFD_YSFC) ? 1 : 2);
        if (a == 1 && b == 0) return e1[ax] / s;
        if (a == 0 && b == 1) return e2[ax] / s;
        return 0.0;
    }
    case RBFFD_LSFC: return ((a == 2 && b == 0) || (a == 0 && b == 2)) ? 2.0 / (s * s) : 0.0;
    case RBFFD_LAPL: {
        double q = 0.0;
        for (int ax = 0; ax < dim && ax < 3; ax++) {
            if (a == 2 && b == 0) q += 2.0 * e1[ax] * e1[ax];
            if (a == 1 && b == 1) q += 2.0 * e1[ax] * e2[ax];
            if (a == 0 && b == 2) q += 2.0 * e2[ax] * e2[ax];
        }
        return q / (s * s);
    }
    case RBFFD_HV: {
        if (t != 2 * hv_k || (a & 1) || (b & 1)) return 0.0;
        double binom = dfact(hv_k) / (dfact(a / 2) * dfact(hv_k - a / 2));
        return binom * dfact(a) * dfact(b) / pow(s, 2 * hv_k);
    }
    default: return 0.0;
    }
}

// Gaussian RBF pieces (src/rbffd/rbfs/rbf_gaussian.h)
__device__ __forceinline__ double g_eval(double eps2, double r2) { return exp(-(r2 * eps2)); }

__device__ double hv_p_k(double eps2r2, int dim, int k)
{
    // iterative form of RBF_Gaussian::hv_p_k (rbf_gaussian.h:229-249), same arithmetic per level
    if (k == 0) return 1.0;
    double pm2 = 1.0, pm1 = 4. * eps2r2 - 2. * dim;
    for (int j = 2; j <= k; j++) {
        double p = 4. * (eps2r2 - 2. * (j - 1) - dim / 2.) * pm1 - 8. * (j - 1) * (2. * (j - 1) - 2. + dim) * pm2;
        pm2 = pm1;
        pm1 = p;
    }
    return pm1;
}

// RHS entry for node j (rbffd.cpp:375-503); dx, dy, dz = x0 - xj, r2 its
// squared length and phi = g_eval(eps2, r2) (one evaluation shared by the
// operators of a node); eps_2k = pow(eps, 2 hv_k) (per stencil).
__device__ double rhs_rbf(unsigned bit, const double* x0, const double* xj, double eps2, int dim, int hv_k,
                          double eps_2k, double lam_i, double th_i, double lam_j, double th_j, double dx, double dy,
                          double dz, double r2, double phi)
{
    double rdr = -2. * eps2 * phi;  // rderiv_over_r
    switch (bit) {
    case RBFFD_X: return -2. * (dx * eps2) * phi;
    case RBFFD_Y: return -2. * (dy * eps2) * phi;
    case RBFFD_Z: return -2. * (dz * eps2) * phi;
    case RBFFD_LAPL:
        if (dim == 1) return 2. * eps2 * (-1. + 2. * (dx * dx * eps2)) * phi;
        if (dim == 2) return 4. * eps2 * (-1. + dx * dx * eps2 + dy * dy * eps2) * phi;
        return (-6. * eps2 + 4. * (r2 * (eps2 * eps2))) * phi;
    case RBFFD_INTERP: return phi;
    case RBFFD_R: return -2. * (sqrt(r2) * eps2) * phi;
    case RBFFD_LAMBDA: {
        double d = cos(th_j) * sin(lam_i - lam_j);
        return fabs(d) > 0. ? d * rdr : 0.;
    }
    case RBFFD_THETA: {
        double d = cos(th_j) * sin(th_i) * cos(lam_i - lam_j) - sin(th_j) * cos(th_i);
        return fabs(d) > 0. ? d * rdr : 0.;
    }
    case RBFFD_LSFC: {
        double rd2 = rdr + 4. * (eps2 * eps2) * r2 * phi;  // rderiv2
        return (1. / 4.) * ((4. - r2) * rd2 + (4. - 3. * r2) * rdr);
    }
    case RBFFD_XSFC:
    case RBFFD_YSFC:
    case RBFFD_ZSFC: {
        double xTx = x0[0] * xj[0] + x0[1] * xj[1] + x0[2] * xj[2];
        int ax = bit == RBFFD_XSFC ? 0 : (bit == RBFFD_YSFC ? 1 : 2);
        return (x0[ax] * xTx - xj[ax]) * rdr;
    }
    case RBFFD_HV: return eps_2k * hv_p_k(eps2 * r2, dim, hv_k) * phi;
    default: return 0.;  // ALT_*: rbffd.cpp:490-494
    }
}

// ---------------------------------------------------------------------------
// Team elimination on the augmented row-major matrix a (m x ld, ld = m + K).
// cand_v / cand_r: one pivot candidate per warp.  Returns false on a zero pivot.

// Warp-wide first maximum: the largest v, ties to the smaller index i.
__device__ __forceinline__ void warp_argmax_index(double& v, int& i)
{
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, i, o);
        if (ov > v || (ov == v && oi < i)) {
            v = ov;
            i = oi;
        }
    }
}

__device__ void team_pivot_column0(const Team& T, const double* a, int m, int ld, double* cand_v, int* cand_r)
{
    // candidates for step 0: rows handled warp-strided, first maximum kept
    double bv = -1.0;
    int br = INT_MAX;
    for (int i = T.tid; i < m; i += T.size) {
        double v = fabs(a[i * ld]);
        if (v > bv) { bv = v; br = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
        double ov = __shfl_xor_sync(0xffffffffu, bv, o);
        int orr = __shfl_xor_sync(0xffffffffu, br, o);
        if (ov > bv || (ov == bv && orr < br)) { bv = ov; br = orr; }
    }
    if (T.lane() == 0) {
        cand_v[T.warp()] = bv;
        cand_r[T.warp()] = br;
    }
}

// Rows i = i0, i0 + stride, ... (< m) of a warp updated at step k against
// the pivot row's columns k+1 .. ld-1, held in registers as NCH 32-column
// chunks (column k+1+lane+32c in pr[c]; the last chunk may be partial):
// a_ij <- fma(-l_i, u_kj, a_ij) with l_i from mult(i) and the row's storage
// from row(i).  Two rows per pass, their loads issued before either row's
// stores.  Lane 0, whose first column is k+1, tracks the first maximum
// |a_i,k+1| over the rows in order (the next step's pivot candidates).
template <int NCH, typename RowF, typename MulF>
__device__ __forceinline__ void warp_rows_update(int k, int ld, int m, int i0, int stride, int lane, const double* pr,
                                                 RowF row, MulF mult, double& nbv, int& nbr)
{
    const int j0 = k + 1 + lane;
    bool in[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) in[c] = c < NCH - 1 || j0 + 32 * c < ld;
    for (int i = i0; i < m; i += 2 * stride) {
        const int i2 = i + stride;
        const bool two = i2 < m;
        double* a1 = row(i) + j0;
        double* a2 = two ? row(i2) + j0 : a1;
        const double l1 = mult(i);
        const double l2 = two ? mult(i2) : 0.0;
        double x1[NCH], x2[NCH];
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            x1[c] = in[c] ? a1[32 * c] : 0.0;
            x2[c] = in[c] && two ? a2[32 * c] : 0.0;
        }
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            x1[c] = __fma_rn(-l1, pr[c], x1[c]);
            x2[c] = __fma_rn(-l2, pr[c], x2[c]);
        }
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            if (in[c]) a1[32 * c] = x1[c];
            if (in[c] && two) a2[32 * c] = x2[c];
        }
        if (lane == 0) {
            const double v1 = fabs(x1[0]);
            if (v1 > nbv) { nbv = v1; nbr = i; }
            if (two) {
                const double v2 = fabs(x2[0]);
                if (v2 > nbv) { nbv = v2; nbr = i2; }
            }
        }
    }
}

// The pivot row's columns k+1 .. ld-1 (NCH chunks) into registers, then the
// warp's rows; NCH = number of 32-column chunks from column k+1 (at most
// ELIM_CHUNKS).
template <int NCH, typename RowF, typename MulF>
__device__ __forceinline__ void warp_step(int k, int ld, int m, int i0, int stride, int lane, const double* prow,
                                          RowF row, MulF mult, double& nbv, int& nbr)
{
    double pr[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        const int j = k + 1 + lane + 32 * c;
        pr[c] = j < ld ? prow[j] : 0.0;
    }
    warp_rows_update<NCH>(k, ld, m, i0, stride, lane, pr, row, mult, nbv, nbr);
}

template <typename RowF, typename MulF>
__device__ __forceinline__ void warp_step_any(int k, int ld, int m, int i0, int stride, int lane, const double* prow,
                                              RowF row, MulF mult, double& nbv, int& nbr)
{
    switch ((ld - k - 1 + 31) >> 5) {  // columns k+1 .. ld-1 (at least one: K >= 1)
    case 1: warp_step<1>(k, ld, m, i0, stride, lane, prow, row, mult, nbv, nbr); break;
    case 2: warp_step<2>(k, ld, m, i0, stride, lane, prow, row, mult, nbv, nbr); break;
    case 3: warp_step<3>(k, ld, m, i0, stride, lane, prow, row, mult, nbv, nbr); break;
    case 4: warp_step<4>(k, ld, m, i0, stride, lane, prow, row, mult, nbv, nbr); break;
    case 5: warp_step<5>(k, ld, m, i0, stride, lane, prow, row, mult, nbv, nbr); break;
    default: warp_step<ELIM_CHUNKS>(k, ld, m, i0, stride, lane, prow, row, mult, nbv, nbr); break;
    }
}

// Returns 0, or k + 1 when the pivot column at step k is exactly zero (dgetrf's INFO).
// a: m rows of ld = m + K columns at row stride lda (>= ld); lbuf: m doubles
// of scratch.  Two team barriers per step: after the barrier every thread
// reduces the warps' candidates (lanes in parallel) to the pivot row p, reads
// the pivot a_pk, exchanges rows k and p beyond column k and forms the
// multipliers into lbuf (row p's from the old a_kk, which the exchange would
// have moved there; column k itself is not written); after the next barrier
// the warps update their rows and publish the candidates of column k+1, and
// a_kk takes the pivot (the U diagonal the back substitution reads).  The
// same divisions, pivots and fma sequence as dgetf2.
__device__ int team_eliminate(const Team& T, double* a, int m, int K, int lda, double* cand_v, int* cand_r,
                              double* lbuf)
{
    const int ld = m + K;
    const int nw = T.nwarps(), w = T.warp(), lane = T.lane();
    team_pivot_column0(T, a, m, lda, cand_v, cand_r);
    T.sync();
    for (int k = 0; k < m; k++) {
        // the warps' candidates, first maximum (every warp, identical result)
        double bv = cand_v[0];
        int p = cand_r[0];
        if (nw > 1) {  // lanes 0 .. nw-1 (a power of two) combine by butterfly, lane 0's result broadcast
            bv = lane < nw ? cand_v[lane] : -1.0;
            p = lane < nw ? cand_r[lane] : INT_MAX;
            for (int o = 1; o < nw; o <<= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
                const int op = __shfl_xor_sync(0xffffffffu, p, o);
                if (ov > bv || (ov == bv && op < p)) {
                    bv = ov;
                    p = op;
                }
            }
            bv = __shfl_sync(0xffffffffu, bv, 0);
            p = __shfl_sync(0xffffffffu, p, 0);
        }
        if (!(bv > 0.0)) return k + 1;  // exactly zero (or NaN) pivot column
        const double piv = a[(size_t)p * lda + k];
        if (p != k)
            for (int j = k + 1 + T.tid; j < ld; j += T.size) {
                const double t = a[(size_t)k * lda + j];
                a[(size_t)k * lda + j] = a[(size_t)p * lda + j];
                a[(size_t)p * lda + j] = t;
            }
        for (int i = k + 1 + T.tid; i < m; i += T.size)
            lbuf[i] = (i == p ? a[(size_t)k * lda + k] : a[(size_t)i * lda + k]) / piv;
        T.sync();
        if (T.tid == 0) a[(size_t)k * lda + k] = piv;
        // rows split across warps, columns across lanes
        double nbv = -1.0;
        int nbr = INT_MAX;
        warp_step_any(
            k, ld, m, k + 1 + w, nw, lane, a + (size_t)k * lda, [&](int i) { return a + (size_t)i * lda; },
            [&](int i) { return lbuf[i]; }, nbv, nbr);
        if (lane == 0) {
            cand_v[w] = nbv;
            cand_r[w] = nbr;
        }
        T.sync();
    }
    return 0;
}

// The row-map elimination's update of a warp's rows at step k (NCH chunks
// of the pivot row from column k+1): the rows k+1+w, k+1+w+nw, ... in
// batches of 32, lane t finding the physical row of the batch's row t and
// dividing for its multiplier (the divisions side by side), then the rows
// two at a time with their row and multiplier broadcast, both rows' loads
// issued before their stores.  Lane 0 tracks the first maximum of column k+1.
template <int NCH>
__device__ __forceinline__ void perm_rows_update(double* a, int lda, int k, int ld, int m, int w, int nw, int lane,
                                                 int p, const int* P, const double* prow, double piv, double& nbv,
                                                 int& nbr)
{
    const int j0 = k + 1 + lane;
    double pr[NCH];
    bool in[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        in[c] = c < NCH - 1 || j0 + 32 * c < ld;
        pr[c] = in[c] ? prow[j0 + 32 * c] : 0.0;
    }
    for (int i0 = k + 1 + w; i0 < m; i0 += 32 * nw) {
        const int it = i0 + lane * nw;
        int phys = 0;
        double lt = 0.0;
        if (it < m) {
            phys = it == p ? P[k] : P[it];
            lt = a[(size_t)phys * lda + k] / piv;
        }
        const int cnt = min(32, (m - i0 + nw - 1) / nw);
        for (int t = 0; t < cnt; t += 2) {
            const bool two = t + 1 < cnt;
            const int r1 = __shfl_sync(0xffffffffu, phys, t), r2 = __shfl_sync(0xffffffffu, phys, t + 1);
            const double l1 = __shfl_sync(0xffffffffu, lt, t), l2 = __shfl_sync(0xffffffffu, lt, t + 1);
            double* a1 = a + (size_t)r1 * lda + j0;
            double* a2 = two ? a + (size_t)r2 * lda + j0 : a1;
            double x1[NCH], x2[NCH];
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                x1[c] = in[c] ? a1[32 * c] : 0.0;
                x2[c] = in[c] && two ? a2[32 * c] : 0.0;
            }
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                x1[c] = __fma_rn(-l1, pr[c], x1[c]);
                x2[c] = __fma_rn(-l2, pr[c], x2[c]);
            }
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                if (in[c]) a1[32 * c] = x1[c];
                if (in[c] && two) a2[32 * c] = x2[c];
            }
            if (lane == 0) {
                const double v1 = fabs(x1[0]);
                if (v1 > nbv) { nbv = v1; nbr = i0 + t * nw; }
                if (two) {
                    const double v2 = fabs(x2[0]);
                    if (v2 > nbv) { nbv = v2; nbr = i0 + (t + 1) * nw; }
                }
            }
        }
    }
}

// Unblocked elimination with one team barrier per step.  Rows are not
// swapped in memory: perm (2 m ints, two buffers) maps a logical row to its
// physical row, and step k writes the next map while it reads the current
// one; the pivot candidates are double-buffered the same way.  Each warp
// forms the multiplier of each of its rows itself (every lane divides) and
// updates the row against the pivot row held in registers.  The arithmetic --
// pivots, multipliers, the fma sequence of every element -- is
// team_eliminate's; only where a row lives changes.  On return the final map
// is perm + (m & 1) * m (logical row k at physical row map[k]).
__device__ int team_eliminate_perm(const Team& T, double* a, int m, int K, int lda, double* cand_v, int* cand_r,
                                   int* perm)
{
    const int ld = m + K;
    const int nw = T.nwarps(), w = T.warp(), lane = T.lane();
    for (int i = T.tid; i < m; i += T.size) perm[i] = i;
    team_pivot_column0(T, a, m, lda, cand_v, cand_r);  // candidates buffer 0
    T.sync();
    for (int k = 0; k < m; k++) {
        const int par = k & 1;
        const double* cv = cand_v + par * MAX_WARPS;
        const int* cr = cand_r + par * MAX_WARPS;
        double bv = cv[0];
        int p = cr[0];
        for (int q = 1; q < nw; q++) {
            const double v = cv[q];
            const int r = cr[q];
            if (v > bv || (v == bv && r < p)) { bv = v; p = r; }
        }
        if (!(bv > 0.0)) return k + 1;
        const int* P = perm + par * m;
        int* Q = perm + (par ^ 1) * m;
        for (int i = T.tid; i < m; i += T.size) Q[i] = i == k ? P[p] : (i == p ? P[k] : P[i]);
        const int prow = P[p];  // the pivot's physical row
        const double piv = a[prow * lda + k];
        double nbv = -1.0;
        int nbr = INT_MAX;
        switch ((ld - k - 1 + 31) >> 5) {
        case 1: perm_rows_update<1>(a, lda, k, ld, m, w, nw, lane, p, P, a + (size_t)prow * lda, piv, nbv, nbr); break;
        case 2: perm_rows_update<2>(a, lda, k, ld, m, w, nw, lane, p, P, a + (size_t)prow * lda, piv, nbv, nbr); break;
        case 3: perm_rows_update<3>(a, lda, k, ld, m, w, nw, lane, p, P, a + (size_t)prow * lda, piv, nbv, nbr); break;
        case 4: perm_rows_update<4>(a, lda, k, ld, m, w, nw, lane, p, P, a + (size_t)prow * lda, piv, nbv, nbr); break;
        case 5: perm_rows_update<5>(a, lda, k, ld, m, w, nw, lane, p, P, a + (size_t)prow * lda, piv, nbv, nbr); break;
        default:
            perm_rows_update<ELIM_CHUNKS>(a, lda, k, ld, m, w, nw, lane, p, P, a + (size_t)prow * lda, piv, nbv, nbr);
            break;
        }
        if (lane == 0) {
            cand_v[(par ^ 1) * MAX_WARPS + w] = nbv;
            cand_r[(par ^ 1) * MAX_WARPS + w] = nbr;
        }
        T.sync();
    }
    return 0;
}

// The panel of columns k0 .. k0+pw-1 (pw <= 8) over rows k0 .. m-1, factored
// by one warp in registers with dgetf2's steps: lane l holds rows
// k0 + l + 32 t (t < TS), the panel's 8 columns each.  Step k = k0 + s:
// first maximum |a_ik| over rows i >= k (smaller row on ties), the rows k and
// p exchanged across the panel's columns (the multipliers of earlier steps
// included, as dgetf2 swaps whole rows), multipliers a_ik / a_kk, then
// a_ij <- fma(-l_i, u_kj, a_ij) on the panel's later columns.  Pivot rows
// go to piv_rows[s].  Returns 0, or k + 1 at an exactly zero pivot column.
template <int TS>
__device__ int warp_panel(double* a, int lda, int m, int k0, int pw, int lane, int* piv_rows)
{
    double v[TS][8];
#pragma unroll
    for (int t = 0; t < TS; t++) {
        const int i = k0 + lane + 32 * t;
#pragma unroll
        for (int c = 0; c < 8; c++) v[t][c] = (i < m && c < pw) ? a[(size_t)i * lda + k0 + c] : 0.0;
    }
    int info = 0;
#pragma unroll
    for (int s = 0; s < 8; s++) {
        if (s >= pw) break;
        const int k = k0 + s;
        double bv = -1.0;
        int bi = INT_MAX;
#pragma unroll
        for (int t = 0; t < TS; t++) {
            const int i = k0 + lane + 32 * t;
            if (i >= k && i < m) {
                const double x = fabs(v[t][s]);
                if (x > bv) {
                    bv = x;
                    bi = i;
                }
            }
        }
        warp_argmax_index(bv, bi);
        if (!(bv > 0.0)) {
            info = k + 1;  // exactly zero (or NaN) pivot column
            break;
        }
        if (lane == 0) piv_rows[s] = bi;
        const int pl = (bi - k0) & 31, pt = (bi - k0) >> 5;
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const double xk = __shfl_sync(0xffffffffu, v[0][c], s);  // row k: lane s, slot 0
            double y = v[0][c];
#pragma unroll
            for (int t = 1; t < TS; t++)
                if (t == pt) y = v[t][c];
            const double xp = __shfl_sync(0xffffffffu, y, pl);  // row p
            if (lane == s) v[0][c] = xp;
#pragma unroll
            for (int t = 0; t < TS; t++)
                if (t == pt && lane == pl) v[t][c] = xk;
        }
        const double piv = __shfl_sync(0xffffffffu, v[0][s], s);
#pragma unroll
        for (int t = 0; t < TS; t++) {
            const int i = k0 + lane + 32 * t;
            if (i > k && i < m) v[t][s] = v[t][s] / piv;
        }
#pragma unroll
        for (int c = 0; c < 8; c++) {
            if (c > s && c < pw) {
                const double u = __shfl_sync(0xffffffffu, v[0][c], s);
#pragma unroll
                for (int t = 0; t < TS; t++) {
                    const int i = k0 + lane + 32 * t;
                    if (i > k && i < m) v[t][c] = __fma_rn(-v[t][s], u, v[t][c]);
                }
            }
        }
    }
#pragma unroll
    for (int t = 0; t < TS; t++) {
        const int i = k0 + lane + 32 * t;
        if (i < m)
#pragma unroll
            for (int c = 0; c < 8; c++)
                if (c < pw) a[(size_t)i * lda + k0 + c] = v[t][c];
    }
    return info;
}

__device__ int warp_panel_any(double* a, int lda, int m, int k0, int pw, int lane, int* piv_rows)
{
    switch ((m - k0 + 31) >> 5) {
    case 1: return warp_panel<1>(a, lda, m, k0, pw, lane, piv_rows);
    case 2: return warp_panel<2>(a, lda, m, k0, pw, lane, piv_rows);
    case 3: return warp_panel<3>(a, lda, m, k0, pw, lane, piv_rows);
    case 4: return warp_panel<4>(a, lda, m, k0, pw, lane, piv_rows);
    default: return warp_panel<(MAX_M + 31) / 32>(a, lda, m, k0, pw, lane, piv_rows);
    }
}

// Blocked elimination with delayed trailing updates, the same arithmetic as
// team_eliminate (and so as dgetf2): every element receives its updates
// a_ij <- fma(-l_ik, u_kj, a_ij) in ascending k, with the same multipliers
// (divisions by the same pivots) and the same first-maximum pivots; only the
// moment an update is applied changes.  Panels of 8 columns, as LAPACK's
// dgetrf blocks them: warp 0 factors the panel in registers (warp_panel, no
// team barrier inside); then every thread takes trailing columns, applies
// the panel's row exchanges to each in order (dlaswp) and solves the panel
// rows against the panel's unit lower triangle (dtrsm, steps in order); then
// the rows below take the panel's delayed updates at once as a
// register-tiled rank-8 product (each warp: 8 rows x 32 lanes x up to 4
// column groups held in registers, the L values broadcast, the U row read
// once per row tile).  Three team barriers per panel.
// cand_r: scratch of at least 9 ints (status, 8 pivot rows).
template <int PB>
__device__ int team_eliminate_blocked(const Team& T, double* a, int m, int K, int lda, double* cand_v, int* cand_r)
{
    static_assert(PB == 8, "warp_panel holds 8 columns");
    const int ncols = m + K;
    const int nw = T.nwarps(), w = T.warp(), lane = T.lane();
    int* piv_rows = cand_r + 1;
    for (int k0 = 0; k0 < m; k0 += PB) {
        const int kend = min(k0 + PB, m), pw = kend - k0;
        if (w == 0) {
            const int info = warp_panel_any(a, lda, m, k0, pw, lane, piv_rows);
            if (lane == 0) cand_r[0] = info;
        }
        T.sync();
        const int info = cand_r[0];
        if (info) return info;
        // trailing columns: the panel's row exchanges in order, then the panel rows (U), one column per thread
        for (int j = kend + T.tid; j < ncols; j += T.size) {
            for (int q = 0; q < pw; q++) {
                const int p = piv_rows[q];
                if (p != k0 + q) {
                    const double t = a[(size_t)(k0 + q) * lda + j];
                    a[(size_t)(k0 + q) * lda + j] = a[(size_t)p * lda + j];
                    a[(size_t)p * lda + j] = t;
                }
            }
            for (int r = k0 + 1; r < kend; r++) {
                double v = a[(size_t)r * lda + j];
                for (int pp = k0; pp < r; pp++) v = __fma_rn(-a[(size_t)r * lda + pp], a[(size_t)pp * lda + j], v);
                a[(size_t)r * lda + j] = v;
            }
        }
        T.sync();
        if (kend >= m) break;
        // delayed rank-(kend-k0) update of rows kend..m-1, columns kend..ncols-1
        const int nr = m - kend;
        const int ntiles = (nr + 7) >> 3;
        for (int cb = kend; cb < ncols; cb += 128) {
            for (int rt = w; rt < ntiles; rt += nw) {
                const int i0 = kend + rt * 8;
                double acc[8][4];
#pragma unroll
                for (int r = 0; r < 8; r++)
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        const int i = i0 + r, j = cb + lane + 32 * c;
                        acc[r][c] = (i < m && j < ncols) ? a[i * lda + j] : 0.0;
                    }
                for (int pp = k0; pp < kend; pp++) {
                    double u[4], l[8];
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        const int j = cb + lane + 32 * c;
                        u[c] = j < ncols ? a[pp * lda + j] : 0.0;
                    }
#pragma unroll
                    for (int r = 0; r < 8; r++) l[r] = (i0 + r < m) ? a[(i0 + r) * lda + pp] : 0.0;
#pragma unroll
                    for (int r = 0; r < 8; r++)
#pragma unroll
                        for (int c = 0; c < 4; c++) acc[r][c] = __fma_rn(-l[r], u[c], acc[r][c]);
                }
#pragma unroll
                for (int r = 0; r < 8; r++)
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        const int i = i0 + r, j = cb + lane + 32 * c;
                        if (i < m && j < ncols) a[i * lda + j] = acc[r][c];
                    }
            }
        }
        T.sync();
    }
    return 0;
}

// Column-oriented back substitution (dtrsm upper, non-unit), one warp per
// right-hand side: x_k = b_k / u_kk for k = m-1 .. 0, then b_i <- fma(-x_k,
// u_ik, b_i) for i < k.  Lane l keeps b_i of rows i = l + 32 q in registers
// (q < BS, m <= 32 BS); every lane divides row k's value by the diagonal and
// lane k mod 32's quotient is broadcast, so a step's critical path is one
// division, one shuffle and one fma.  Row storage from row(i) (the identity,
// or the row map of the row-map elimination).  The solution replaces the
// right-hand side.
template <int BS, typename RowF>
__device__ void back_substitute_bs(const Team& T, int m, int K, RowF row)
{
    const int lane = T.lane();
    for (int c = T.warp(); c < K; c += T.nwarps()) {
        const int col = m + c;
        double b[BS];
        double* ri[BS];
#pragma unroll
        for (int q = 0; q < BS; q++) {
            const int i = lane + 32 * q;
            ri[q] = row(i < m ? i : 0);
            b[q] = i < m ? ri[q][col] : 0.0;
        }
        for (int k = m - 1; k >= 0; k--) {
            const int qk = k >> 5, lk = k & 31;
            double bk = b[0];
#pragma unroll
            for (int q = 1; q < BS; q++)
                if (q == qk) bk = b[q];
            const double xk = __shfl_sync(0xffffffffu, bk / row(k)[k], lk);
#pragma unroll
            for (int q = 0; q < BS; q++) {
                const int i = lane + 32 * q;
                if (i < k) b[q] = __fma_rn(-xk, ri[q][k], b[q]);
                if (i == k) b[q] = xk;
            }
        }
#pragma unroll
        for (int q = 0; q < BS; q++)
            if (lane + 32 * q < m) ri[q][col] = b[q];
    }
}

template <typename RowF>
__device__ void team_back_substitute_rows(const Team& T, double* a, int m, int K, RowF row)
{
    switch ((m + 31) >> 5) {
    case 1: back_substitute_bs<1>(T, m, K, row); break;
    case 2: back_substitute_bs<2>(T, m, K, row); break;
    case 3: back_substitute_bs<3>(T, m, K, row); break;
    case 4: back_substitute_bs<4>(T, m, K, row); break;
    default: back_substitute_bs<(MAX_M + 31) / 32>(T, m, K, row); break;
    }
    T.sync();
}

// ---------------------------------------------------------------------------

// The per-stencil quantities of an assembly: sizes, shape parameter, centre,
// its angles, the tangent frame (e1 = fr[0..2], e2 = fr[3..5]) and scale s.
struct SysInputs {
    int n, deg, np, m;
    double eps, eps2, eps_2k, lam_i, th_i, s;
    double x0[3];
    bool angles;  // an operator needs the nodes' longitude and latitude
};

// Team step 1 of an assembly: the stencil's node coordinates into xs, the
// tangent frame and the largest squared distance from the centre into fr.
// Ends with a team barrier (xs and fr visible).
__device__ SysInputs team_inputs(const Team& T, const WParams& P, int r, double* xs, double* fr)
{
    SysInputs S;
    S.n = P.len[r];
    S.deg = P.deg ? P.deg[r] : P.deg_uniform;
    S.np = poly_size(S.deg);
    S.m = S.n + S.np;
    S.eps = P.eps ? P.eps[r] : P.eps_uniform;  // var_epsilon[stencil[0]]
    S.eps2 = S.eps * S.eps;
    const int n = S.n;
    for (int q = T.tid; q < n; q += T.size) {
        double4 v = P.xyz[P.idx[sell_elem(r, q, P.n4 >> 2)]];
        xs[3 * q] = v.x;
        xs[3 * q + 1] = v.y;
        xs[3 * q + 2] = v.z;
    }
    if (T.tid == 0) fr[7] = 0.0;  // max_j |x_j - c|^2, gathered below
    T.sync();
    const double* x0 = xs;
    S.x0[0] = x0[0];
    S.x0[1] = x0[1];
    S.x0[2] = x0[2];
    S.lam_i = atan2(x0[1], x0[0]);
    S.th_i = atan2(x0[2], sqrt(x0[0] * x0[0] + x0[1] * x0[1]));
    if (S.deg >= 2) {
        if (T.tid == 0) {
            fr[0] = -sin(S.lam_i); fr[1] = cos(S.lam_i); fr[2] = 0.0;
            fr[3] = -sin(S.th_i) * cos(S.lam_i); fr[4] = -sin(S.th_i) * sin(S.lam_i); fr[5] = cos(S.th_i);
        }
        // the largest squared distance from the centre: a maximum, so any
        // order of the comparisons gives the same value; non-negative doubles
        // order as their bit patterns, so the team combines with an integer max
        double s2 = 0.0;
        for (int j = T.tid; j < n; j += T.size) {
            double dx = xs[3 * j] - x0[0], dy = xs[3 * j + 1] - x0[1], dz = xs[3 * j + 2] - x0[2];
            double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            s2 = fmax(s2, r2);
        }
        for (int o = 16; o > 0; o >>= 1) s2 = fmax(s2, __shfl_xor_sync(0xffffffffu, s2, o));
        if (T.lane() == 0)
            atomicMax(reinterpret_cast<unsigned long long*>(fr + 7), (unsigned long long)__double_as_longlong(s2));
    }
    S.angles = false;
    for (int c = 0; c < P.K; c++) S.angles |= P.opbit[c] == RBFFD_LAMBDA || P.opbit[c] == RBFFD_THETA;
    S.eps_2k = pow(S.eps, 2 * P.hv_k);
    T.sync();  // frame and distance visible
    S.s = fr[7] > 0.0 ? sqrt(fr[7]) : 1.0;
    return S;
}

// Phi entry of nodes i >= j: phi(x_i - x_j)   (rbffd.cpp:943-966).
__device__ __forceinline__ double phi_pair(const double* xs, int i, int j, double eps2)
{
    double dx = xs[3 * i] - xs[3 * j], dy = xs[3 * i + 1] - xs[3 * j + 1], dz = xs[3 * i + 2] - xs[3 * j + 2];
    double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    return g_eval(eps2, r2);
}

// Polynomial border entry: basis function q at node i.
__device__ __forceinline__ double poly_entry(const SysInputs& S, const double* xs, const double* fr, int q, int i)
{
    if (S.deg >= 2) {
        const double* e1 = fr;
        const double* e2 = fr + 3;
        int pa, pb;
        tangent_exp(q, pa, pb);
        double dx = xs[3 * i] - S.x0[0], dy = xs[3 * i + 1] - S.x0[1], dz = xs[3 * i + 2] - S.x0[2];
        double u = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, e1[0]), __dmul_rn(dy, e1[1])), __dmul_rn(dz, e1[2])), S.s);
        double w = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, e2[0]), __dmul_rn(dy, e2[1])), __dmul_rn(dz, e2[2])), S.s);
        return ipow(u, pa) * ipow(w, pb);
    }
    int pa, pb, pc;
    basis_exp(q, pa, pb, pc);
    return ipow(xs[3 * i], pa) * ipow(xs[3 * i + 1], pb) * ipow(xs[3 * i + 2], pc);
}

// The node quantities a right-hand-side entry of node j < n needs: its
// angles (when an operator needs them), x0 - x_j, its squared length, phi.
struct NodeTerms {
    double lam_j, th_j, dx, dy, dz, r2, phi;
};

__device__ __forceinline__ NodeTerms node_terms(const SysInputs& S, const double* xj)
{
    NodeTerms t;
    t.lam_j = 0.0;
    t.th_j = 0.0;
    if (S.angles) {
        t.lam_j = atan2(xj[1], xj[0]);
        t.th_j = atan2(xj[2], sqrt(xj[0] * xj[0] + xj[1] * xj[1]));
    }
    t.dx = S.x0[0] - xj[0];
    t.dy = S.x0[1] - xj[1];
    t.dz = S.x0[2] - xj[2];
    t.r2 = __dadd_rn(__dadd_rn(__dmul_rn(t.dx, t.dx), __dmul_rn(t.dy, t.dy)), __dmul_rn(t.dz, t.dz));
    t.phi = g_eval(S.eps2, t.r2);
    return t;
}

// Right-hand-side entry of operator c at node j < n.
__device__ __forceinline__ double rhs_node(const WParams& P, const SysInputs& S, const double* xj, const NodeTerms& t,
                                           int c)
{
    return rhs_rbf(P.opbit[c], S.x0, xj, S.eps2, P.dim, P.hv_k, S.eps_2k, S.lam_i, S.th_i, t.lam_j, t.th_j, t.dx, t.dy,
                   t.dz, t.r2, t.phi);
}

// Right-hand-side entry of operator c at polynomial row j >= n.
__device__ __forceinline__ double rhs_poly(const WParams& P, const SysInputs& S, const double* fr, int j, int c)
{
    double v = 0.0;
    if (S.deg == 1) v = poly_row(P.opbit[c], j - S.n, S.x0, P.dim, P.hv_k, S.lam_i, S.th_i);
    if (S.deg >= 2) {
        int pa, pb;
        tangent_exp(j - S.n, pa, pb);
        v = tangent_row(P.opbit[c], pa, pb, fr, fr + 3, S.s, P.dim, P.hv_k);
    }
    return v;
}

// Team assembly of the augmented system [A | B] of stencil r into a (m rows of
// m + K columns at row stride ld).  xs: scratch for the stencil's coordinates;
// fr: 8 doubles of scratch (tangent frame, distance).  Returns m.  Ends with a
// team barrier.
__device__ int team_assemble(const Team& T, const WParams& P, int r, double* a, double* xs, double* fr, int& n_out,
                             int ld)
{
    const SysInputs S = team_inputs(T, P, r, xs, fr);
    const int n = S.n, np = S.np, m = S.m, K = P.K;
    // Phi block: symmetric to the last bit (x_j - x_i squares to the same
    // r^2), so each pair j <= i is evaluated once and written to both places:
    // n(n+1)/2 exponentials.
    for (int e = T.tid; e < n * (n + 1) / 2; e += T.size) {
        int i = (int)((sqrtf(8.0f * e + 1.0f) - 1.0f) * 0.5f);  // e = i(i+1)/2 + j, 0 <= j <= i (estimate, corrected below)
        while (i * (i + 1) / 2 > e) i--;
        while ((i + 1) * (i + 2) / 2 <= e) i++;
        const int j = e - i * (i + 1) / 2;
        const double v = phi_pair(xs, i, j, S.eps2);
        a[j * ld + i] = v;
        a[i * ld + j] = v;
    }
    // polynomial border and zero block
    for (int e = T.tid; e < np * n; e += T.size) {
        int q = e / n, i = e - q * n;
        const double v = poly_entry(S, xs, fr, q, i);
        a[(n + q) * ld + i] = v;
        a[i * ld + (n + q)] = v;
    }
    for (int e = T.tid; e < np * np; e += T.size) a[(n + e / np) * ld + n + e % np] = 0.0;
    // right-hand sides, one column per operator in bit order (rbffd.cpp:106-125);
    // a node's kernel value is evaluated once for all operators
    for (int j = T.tid; j < m; j += T.size) {
        if (j < n) {
            const double* xj = xs + 3 * j;
            const NodeTerms t = node_terms(S, xj);
            for (int c = 0; c < K; c++) a[j * ld + m + c] = rhs_node(P, S, xj, t, c);
        } else {
            for (int c = 0; c < K; c++) a[j * ld + m + c] = rhs_poly(P, S, fr, j, c);
        }
    }
    T.sync();
    n_out = n;
    return m;
}

// The elimination variants a size class can use (same arithmetic, same results).
enum { ELIM_UNBLOCKED = 0, ELIM_BLOCKED = 1, ELIM_PERM = 2, ELIM_REG = 3 };

// One system end to end by one team: assemble, eliminate, back-substitute,
// store the weights of row r.  a: the team's shared memory,
// [a: m rows at stride lda] [xs: 3 n_pad] [frame: 8] [cand_v: 2 MAX_WARPS]
// [cand_r: 2 MAX_WARPS ints] [perm: 2 m ints].
__device__ void team_solve(const Team& T, const WParams& P, int r, double* a, int m, int lda, int mode)
{
    double* xs = a + (size_t)m * lda;
    double* fr = xs + 3 * P.n_pad;
    double* cand_v = fr + 8;
    int* cand_r = (int*)(cand_v + 2 * MAX_WARPS);
    int* perm = cand_r + 2 * MAX_WARPS;
    const int K = P.K;
    int n;
    team_assemble(T, P, r, a, xs, fr, n, lda);
    const int st = mode == ELIM_BLOCKED ? team_eliminate_blocked<8>(T, a, m, K, lda, cand_v, cand_r)
                   : mode == ELIM_PERM  ? team_eliminate_perm(T, a, m, K, lda, cand_v, cand_r, perm)
                                        : team_eliminate(T, a, m, K, lda, cand_v, cand_r, (double*)perm);
    const bool ok = st == 0;
    const int* F = perm + (m & 1) * m;  // ELIM_PERM: where each logical row lives
    if (ok) {
        if (mode == ELIM_PERM)
            team_back_substitute_rows(T, a, m, K, [&](int i) { return a + (size_t)F[i] * lda; });
        else
            team_back_substitute_rows(T, a, m, K, [&](int i) { return a + (size_t)i * lda; });
    }
    if (!ok && T.tid == 0) atomicMin(P.status, r + 1);
    // store: weights[type][r][j] = W(j, col) * scale (rbffd.cpp:300-306), row r of the sliced ELL
    for (int e = T.tid; e < K * P.n4; e += T.size) {
        int c = e / P.n4, j = e - c * P.n4;
        double scale = P.opbit[c] == RBFFD_HV ? P.hv_scale : 1.0;
        const int rj = mode == ELIM_PERM && j < n ? F[j] : j;
        double v = (j < n) ? (ok ? a[rj * lda + m + c] * scale : __longlong_as_double(0x7ff8000000000000ll)) : 0.0;
        P.w[c][sell_elem(r, j, P.n4 >> 2)] = v;
    }
    T.sync();
}

// ---------------------------------------------------------------------------
// Register-resident elimination: one system per CTA of NW warps.  Warp w
// holds the physical rows w + NW q (q < R) in registers, lane l the columns
// l + 32 c (c < C), loaded from the system team_assemble stages in shared
// memory.  Rows never move:
// every row keeps its logical position (dgetf2's row order after its swaps)
// in lane q of its warp, so ties in the pivot search go to the smaller
// position as in dgetf2.  Step k, after the one block barrier:
//   every warp reduces the NW published candidates (first maximum |a_ik|,
//   smaller position on ties) and reads the winner's published row (the
//   pivot row, columns in its lanes); the pivot row takes position k and the
//   row at position k the pivot's; the pivot leaves the active set;
//   lane q divides its row's column-k value (gathered at the end of step k-1)
//   by the pivot, and the active rows take a_ij <- fma(-l_i, u_kj, a_ij);
//   lane q then gathers its row's column-(k+1) value, the warp finds its
//   candidate for step k+1 and publishes it with its row's values
//   (double-buffered by step parity).
// The multipliers, pivots and the fma sequence of every element are
// dgetf2's, so the result is team_eliminate's bit for bit.  The finished rows
// (U and the transformed right-hand sides) are written to shared memory in
// position order for the back substitution.  Valid for m <= NW R and
// m + K <= 32 C.
template <int NW, int R, int C>
struct RegElim {
    static constexpr int THREADS = NW * 32;
    // shared memory: U [m x lda] | xs [3 n_pad] | fr [8] | rows [2][NW][32 C] | cand_v [2][NW] |
    // cand_pos [2][NW] ints | cand_row [2][NW] ints
    static size_t smem_bytes(int m, int lda, int n_pad)
    {
        return ((size_t)m * lda + 3 * (size_t)n_pad + 8 + 2 * (size_t)NW * 32 * C + 2 * NW + 2 * NW) * sizeof(double);
    }
};

__device__ __forceinline__ void argmax_first(double& v, int& pos, int& who)
{
    // warp-wide maximum of v, ties to the smaller pos (then any who)
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int op = __shfl_xor_sync(0xffffffffu, pos, o);
        const int ow = __shfl_xor_sync(0xffffffffu, who, o);
        if (ov > v || (ov == v && op < pos)) {
            v = ov;
            pos = op;
            who = ow;
        }
    }
}

template <int NW, int R, int C>
__device__ __forceinline__ int reg_eliminate(double (&A)[R][C], int m, int ld, int w, int lane, int& mypos, double* rows,
                             double* cand_v, int* cand_p, int* cand_r)
{
    unsigned act = 0;
#pragma unroll
    for (int q = 0; q < R; q++)
        if (w + NW * q < m) act |= 1u << q;
    mypos = w + NW * lane;  // lane q: the position of row w + NW q (its own index to begin with)
    double num = 0.0;       // lane q: row q's value in the column of the current step
    // candidates of column 0, published in buffer 0
    {
#pragma unroll
        for (int q = 0; q < R; q++) {
            const double t = __shfl_sync(0xffffffffu, A[q][0], 0);
            if (lane == q) num = t;
        }
        const bool live = lane < R && ((act >> lane) & 1) && fabs(num) >= 0.0;  // NaN never a candidate
        double v = live ? fabs(num) : -1.0;
        int pos = live ? mypos : INT_MAX, who = lane;
        argmax_first(v, pos, who);
        if (lane == 0) {
            cand_v[w] = v;
            cand_p[w] = pos;
            cand_r[w] = w + NW * who;
        }
        if (v >= 0.0) {
#pragma unroll
            for (int q = 0; q < R; q++)
                if (q == who)
#pragma unroll
                    for (int c = 0; c < C; c++) rows[(size_t)w * 32 * C + lane + 32 * c] = A[q][c];
        }
    }
    __syncthreads();
    for (int k = 0; k < m; k++) {
        const int par = k & 1;
        // the pivot: first maximum over the warps' candidates
        double gv = lane < NW ? cand_v[par * NW + lane] : -1.0;
        int gpos = lane < NW ? cand_p[par * NW + lane] : INT_MAX, gw = lane;
        argmax_first(gv, gpos, gw);
        if (!(gv > 0.0)) return k + 1;  // exactly zero (or NaN) pivot column
        const int grow = cand_r[par * NW + gw];
        const double* prow = rows + ((size_t)par * NW + gw) * 32 * C;
        double pr[C];
#pragma unroll
        for (int c = 0; c < C; c++) pr[c] = prow[lane + 32 * c];
        const double piv = prow[k];
        // positions after dgetf2's swap of positions k and gpos; the pivot row leaves the active set
        if (lane < R) {
            if (w + NW * lane == grow)
                mypos = k;
            else if (mypos == k)
                mypos = gpos;
        }
        if (w == gw) act &= ~(1u << (grow / NW));
        // multipliers (lane q: row q), then the updates of the active rows
        const double lq = num / piv;
        const int c0 = (k + 1) >> 5;  // chunks below c0 hold only columns <= k
#pragma unroll
        for (int q = 0; q < R; q++) {
            if ((act >> q) & 1) {
                const double l = __shfl_sync(0xffffffffu, lq, q);
#pragma unroll
                for (int c = 0; c < C; c++)
                    if (c >= c0) A[q][c] = __fma_rn(-l, pr[c], A[q][c]);
            }
        }
        // candidates of column k + 1, published in the other buffer
        if (k + 1 < m) {
            const int kc = (k + 1) >> 5, kl = (k + 1) & 31;
#pragma unroll
            for (int q = 0; q < R; q++) {
                double x = A[q][0];
#pragma unroll
                for (int c = 1; c < C; c++)
                    if (kc == c) x = A[q][c];
                const double t = __shfl_sync(0xffffffffu, x, kl);
                if (lane == q) num = t;
            }
            const bool live = lane < R && ((act >> lane) & 1) && fabs(num) >= 0.0;  // NaN never a candidate
            double v = live ? fabs(num) : -1.0;
            int pos = live ? mypos : INT_MAX, who = lane;
            argmax_first(v, pos, who);
            const int nb = par ^ 1;
            if (lane == 0) {
                cand_v[nb * NW + w] = v;
                cand_p[nb * NW + w] = pos;
                cand_r[nb * NW + w] = w + NW * who;
            }
            if (v >= 0.0) {
                double* dst = rows + ((size_t)nb * NW + w) * 32 * C;
#pragma unroll
                for (int q = 0; q < R; q++)
                    if (q == who)
#pragma unroll
                        for (int c = 0; c < C; c++) dst[lane + 32 * c] = A[q][c];
            }
        }
        __syncthreads();
    }
    return 0;
}

// The register-resident solve of a class: per system, the inputs, the
// entries into registers, the elimination, the rows into shared memory in
// position order, the back substitution and the store of team_solve.
template <int NW, int R, int C>
__global__ void __launch_bounds__(NW * 32, NW == 16 ? 1 : 2) k_weights_reg(WParams P)
{
    extern __shared__ double smem[];
    __shared__ int s_unit;
    const WClass Cc = P.cls[0];
    const int m = Cc.m, lda = Cc.lda, K = P.K, ld = m + K;
    double* U = smem;
    double* xs = U + (size_t)m * lda;
    double* fr = xs + 3 * P.n_pad;
    double* rows = fr + 8;
    double* cand_v = rows + 2 * NW * 32 * C;
    int* cand_p = (int*)(cand_v + 2 * NW);
    int* cand_r = cand_p + 2 * NW;
    Team T;
    T.size = NW * 32;
    T.id = 0;
    T.tid = threadIdx.x;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (;;) {
        if (threadIdx.x == 0) s_unit = atomicAdd(P.work, 1);
        __syncthreads();
        const int u = s_unit;
        __syncthreads();
        if (u >= P.nunits) break;
        const int r = P.rows[Cc.rows_off + u];
        int n;
        team_assemble(T, P, r, U, xs, fr, n, lda);  // staged in shared memory, then into registers
        double A[R][C];
#pragma unroll
        for (int q = 0; q < R; q++)
#pragma unroll
            for (int c = 0; c < C; c++) {
                const int row = w + NW * q, col = lane + 32 * c;
                A[q][c] = (row < m && col < ld) ? U[(size_t)row * lda + col] : 0.0;
            }
        __syncthreads();  // every row read before the rows are written back in position order
        int mypos;
        const int st = reg_eliminate<NW, R, C>(A, m, ld, w, lane, mypos, rows, cand_v, cand_p, cand_r);
        const bool ok = st == 0;
        if (ok) {
#pragma unroll
            for (int q = 0; q < R; q++) {
                const int row = w + NW * q;
                const int pos = __shfl_sync(0xffffffffu, mypos, q);
                if (row < m)
#pragma unroll
                    for (int c = 0; c < C; c++)
                        if (lane + 32 * c < ld) U[(size_t)pos * lda + lane + 32 * c] = A[q][c];
            }
            __syncthreads();
            team_back_substitute_rows(T, U, m, K, [&](int i) { return U + (size_t)i * lda; });
        }
        if (!ok && threadIdx.x == 0) atomicMin(P.status, r + 1);
        for (int e = threadIdx.x; e < K * P.n4; e += T.size) {
            const int c = e / P.n4, j = e - c * P.n4;
            const double scale = P.opbit[c] == RBFFD_HV ? P.hv_scale : 1.0;
            const double v = (j < n) ? (ok ? U[(size_t)j * lda + m + c] * scale : __longlong_as_double(0x7ff8000000000000ll))
                                     : 0.0;
            P.w[c][sell_elem(r, j, P.n4 >> 2)] = v;
        }
        __syncthreads();
    }
}

// One size class in one persistent launch (the classes of a call run as a
// sequence of such launches, each with the shared memory and the resident
// CTAs its own systems allow).  A work unit is teams_per_cta systems of the
// class, one per team of the CTA; each CTA takes the next unit from the
// class's counter until none is left, splits itself into the class's teams
// and solves.  MODE is the class's elimination, so each variant is compiled
// with only its own registers (the unblocked and row-map eliminations fit
// four CTAs of 256 threads on an SM, the register-tiled blocked one two).
template <int MODE>
__global__ void __launch_bounds__(256, MODE == ELIM_BLOCKED ? 2 : 3) k_weights_class(WParams P)
{
    extern __shared__ double smem[];
    __shared__ int s_unit;
    const WClass C = P.cls[0];
    Team T;
    T.size = C.team;
    T.id = threadIdx.x / C.team;
    T.tid = threadIdx.x % C.team;
    for (;;) {
        if (threadIdx.x == 0) s_unit = atomicAdd(P.work, 1);
        __syncthreads();
        const int u = s_unit;
        __syncthreads();
        if (u >= P.nunits) break;
        const int t = u * C.teams + T.id;
        if (T.id < C.teams && t < C.nrows)
            team_solve(T, P, P.rows[C.rows_off + t], smem + (size_t)T.id * C.stride, C.m, C.lda, MODE);
        __syncthreads();  // every team done with the shared memory before the next unit
    }
}

// Assembled systems only (inspection): out[t] = [A | B] of row rows[t], m x (m+K) row-major.
__global__ void __launch_bounds__(512) k_assemble(WParams P, int team_size, double* out)
{
    extern __shared__ double smem[];
    Team T;
    T.size = team_size;
    T.id = threadIdx.x / team_size;
    T.tid = threadIdx.x % team_size;
    const int teams_per_cta = blockDim.x / team_size;
    double* a = smem + (size_t)T.id * P.team_stride;
    double* xs = a + (size_t)P.m * (P.m + P.K);
    double* fr = xs + 3 * P.n_pad;
    const size_t sz = (size_t)P.m * (P.m + P.K);
    for (int t = blockIdx.x * teams_per_cta + T.id; t < P.nrows; t += gridDim.x * teams_per_cta) {
        int n;
        team_assemble(T, P, P.rows[t], a, xs, fr, n, P.m + P.K);
        for (size_t e = T.tid; e < sz; e += T.size) out[(size_t)t * sz + e] = a[e];
        T.sync();
    }
}

// Plain batched solve: A [batch][m][m], B [batch][m][nrhs] row-major, X -> B.
__global__ void __launch_bounds__(512) k_gesv(double* A, double* B, int* info, int m, int K, int batch, int team_size,
                                              int team_stride, int blocked)
{
    extern __shared__ double smem[];
    Team T;
    T.size = team_size;
    T.id = threadIdx.x / team_size;
    T.tid = threadIdx.x % team_size;
    const int teams_per_cta = blockDim.x / team_size;
    const int ld = m + K;
    double* a = smem + (size_t)T.id * team_stride;
    double* cand_v = a + (size_t)m * ld;
    int* cand_r = (int*)(cand_v + 2 * MAX_WARPS);
    int* perm = cand_r + 2 * MAX_WARPS;
    const int* F = perm + (m & 1) * m;
    for (int b = blockIdx.x * teams_per_cta + T.id; b < batch; b += gridDim.x * teams_per_cta) {
        const double* Ab = A + (size_t)b * m * m;
        double* Bb = B + (size_t)b * m * K;
        for (int e = T.tid; e < m * m; e += T.size) a[(e / m) * ld + e % m] = Ab[e];
        for (int e = T.tid; e < m * K; e += T.size) a[(e / K) * ld + m + e % K] = Bb[e];
        T.sync();
        const int st = blocked == ELIM_BLOCKED ? team_eliminate_blocked<8>(T, a, m, K, ld, cand_v, cand_r)
                       : blocked == ELIM_PERM  ? team_eliminate_perm(T, a, m, K, ld, cand_v, cand_r, perm)
                                               : team_eliminate(T, a, m, K, ld, cand_v, cand_r, (double*)perm);
        if (st == 0) {
            if (blocked == ELIM_PERM)
                team_back_substitute_rows(T, a, m, K, [&](int i) { return a + (size_t)F[i] * ld; });
            else
                team_back_substitute_rows(T, a, m, K, [&](int i) { return a + (size_t)i * ld; });
        }
        if (T.tid == 0) info[b] = st;
        for (int e = T.tid; e < m * K; e += T.size) {
            const int row = e / K;
            Bb[e] = a[(blocked == ELIM_PERM ? F[row] : row) * ld + m + e % K];
        }
        T.sync();
    }
}

size_t team_bytes_w(int m, int K, int n_pad, int lda = 0)
{
    if (lda == 0) lda = m + K;
    // a, xs, frame, cand_v (2 MAX_WARPS), cand_r (2 MAX_WARPS ints), perm (2 m ints)
    return ((size_t)m * lda + 3 * (size_t)n_pad + 8 + 2 * MAX_WARPS + MAX_WARPS + (size_t)m) * sizeof(double);
}

int max_smem_optin(rbffd_ctx* ctx)
{
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
    return v;
}

constexpr int W_CTA = 256;  // threads per CTA of the persistent launch

// A class's team shape: team width (teams per CTA = W_CTA / team) and the elimination.
struct WShape {
    int team, blocked;
};

}  // namespace

// Row stride of a class's systems: m + K rounded up to odd, so a column walk
// (pivot search, multipliers) touches 32 different bank pairs.
static int class_lda(int m, int K) { return (m + K) | 1; }

static size_t class_stride_bytes(int m, int K, int n_pad)
{
    return (team_bytes_w(m, K, n_pad, class_lda(m, K)) + 127) / 128 * 128;
}

// Candidate shapes of a class: teams whose shared memory fits one CTA.
static std::vector<WShape> w_candidates(int m, int K, int n_pad, size_t stride_bytes, int smem_max)
{
    std::vector<WShape> out;
    const int teams[4] = {32, 64, 128, 256};
    for (int tw : teams) {
        if ((size_t)(W_CTA / tw) * stride_bytes > (size_t)smem_max) continue;
        if (m <= 40 && tw > 64) continue;   // small systems: narrow teams only
        if (m > 96 && tw < 128) continue;   // large systems: wide teams only
        out.push_back(WShape{tw, ELIM_UNBLOCKED});
        out.push_back(WShape{tw, ELIM_PERM});
        if (m >= 24) out.push_back(WShape{tw, ELIM_BLOCKED});
    }
    // register-resident elimination (one system per CTA of 256 or 512 threads), last: measured slower
    const int lda = class_lda(m, K);
    if (m <= 64 && m + K <= 64 && RegElim<8, 8, 2>::smem_bytes(m, lda, n_pad) <= (size_t)smem_max)
        out.push_back(WShape{RegElim<8, 8, 2>::THREADS, ELIM_REG});
    else if (m <= 128 && m + K <= 128 && RegElim<16, 8, 4>::smem_bytes(m, lda, n_pad) <= (size_t)smem_max)
        out.push_back(WShape{RegElim<16, 8, 4>::THREADS, ELIM_REG});
    return out;
}

// The per-grid device workspace of the weight solver, kept between calls so a
// captured launch can be replayed: row list, degrees, epsilons, status, counter.
struct WeightsWork {
    int* d_rows = nullptr;
    int* d_deg = nullptr;
    double* d_eps = nullptr;
    int* d_status = nullptr;  // [0] status, [1 + c] work counter of class c
    size_t bytes = 0;
    cudaGraphExec_t gexec = nullptr;
    WParams gparams;  // the parameters the graph was captured with (each class's launch follows from them)
};

void weights_work_free(rbffd_grid* g)
{
    WeightsWork* W = g->ww;
    if (!W) return;
    rbffd_ctx* ctx = g->ctx;
    if (W->gexec) cudaGraphExecDestroy(W->gexec);
    dev_free(ctx, W->d_rows, (size_t)g->N * sizeof(int));
    dev_free(ctx, W->d_deg, (size_t)g->N * sizeof(int));
    dev_free(ctx, W->d_eps, (size_t)g->N * sizeof(double));
    dev_free(ctx, W->d_status, (1 + MAX_CLASSES) * sizeof(int));
    delete W;
    g->ww = nullptr;
}

static int weights_work(rbffd_grid* g, WeightsWork** out)
{
    if (!g->ww) {
        rbffd_ctx* ctx = g->ctx;
        WeightsWork* W = new (std::nothrow) WeightsWork();
        if (!W) return set_error(ctx, RBFFD_ERR_OOM, "weights workspace");
        g->ww = W;
        int rc;
        if ((rc = dev_alloc(ctx, (void**)&W->d_rows, (size_t)g->N * sizeof(int))) ||
            (rc = dev_alloc(ctx, (void**)&W->d_deg, (size_t)g->N * sizeof(int))) ||
            (rc = dev_alloc(ctx, (void**)&W->d_eps, (size_t)g->N * sizeof(double))) ||
            (rc = dev_alloc(ctx, (void**)&W->d_status, (1 + MAX_CLASSES) * sizeof(int)))) {
            weights_work_free(g);
            return rc;
        }
    }
    *out = g->ww;
    return RBFFD_OK;
}

// The kernel of a shared-memory elimination mode.
static void (*class_kernel(int mode))(WParams)
{
    return mode == ELIM_BLOCKED ? k_weights_class<ELIM_BLOCKED>
           : mode == ELIM_PERM  ? k_weights_class<ELIM_PERM>
                                : k_weights_class<ELIM_UNBLOCKED>;
}

// Register-resident shapes: 16 warps x 8 rows x 4 column chunks (m <= 128,
// m + K <= 128) and 8 warps x 8 rows x 2 chunks (m <= 64, m + K <= 64).
using RegL = RegElim<16, 8, 4>;
using RegS = RegElim<8, 8, 2>;
static bool reg_small(int m, int K) { return m <= 64 && m + K <= 64; }

// Kernel, threads per CTA and dynamic shared memory of a one-class P's launch.
struct ClassLaunch {
    void (*kern)(WParams);
    int threads;
    size_t smem;
};

static ClassLaunch class_launch(const WParams& P)
{
    const WClass& C = P.cls[0];
    if (C.blocked == ELIM_REG) {
        if (reg_small(C.m, P.K)) return {k_weights_reg<8, 8, 2>, RegS::THREADS, RegS::smem_bytes(C.m, C.lda, P.n_pad)};
        return {k_weights_reg<16, 8, 4>, RegL::THREADS, RegL::smem_bytes(C.m, C.lda, P.n_pad)};
    }
    return {class_kernel(C.blocked), W_CTA, (size_t)C.teams * C.stride * sizeof(double)};
}

// Shared memory and grid of the persistent launch of a one-class P (cls[0]):
// as many CTAs as fit on the device at once, at most one per work unit.
static int persistent_geometry(rbffd_ctx* ctx, const WParams& P, size_t* smem, int* grid)
{
    const ClassLaunch L = class_launch(P);
    RBFFD_CUDA_TRY(ctx, cudaFuncSetAttribute(L.kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem));
    int per_sm = 0;
    RBFFD_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, L.kern, L.threads, L.smem));
    if (per_sm < 1) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "weight kernel shape does not fit an SM");
    *smem = L.smem;
    *grid = std::max(1, std::min(P.nunits, per_sm * ctx->sm_count));
    return RBFFD_OK;
}

// Each kernel allowed the largest dynamic shared memory of the classes that
// use it (the attribute is per kernel, and a captured or replayed launch
// needs it to cover its own size).
static int class_smem_attributes(rbffd_ctx* ctx, const WParams* Q, const size_t* smem, int n)
{
    for (int c = 0; c < n; c++) {
        const auto kern = class_launch(Q[c]).kern;
        size_t mx = 0;
        for (int d = 0; d < n; d++)
            if (class_launch(Q[d]).kern == kern) mx = std::max(mx, smem[d]);
        RBFFD_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx));
    }
    return RBFFD_OK;
}

// Zero the class's counter and launch (what the graph holds, class by class).
static void enqueue_persistent(const WParams& P, size_t smem, int grid, cudaStream_t s)
{
    const ClassLaunch L = class_launch(P);
    cudaMemsetAsync(P.work, 0, sizeof(int), s);
    L.kern<<<grid, L.threads, smem, s>>>(P);
}

// Shape a one-class P: its teams per CTA and work units (cls[0].team/blocked set).
static void number_units(WParams& P)
{
    WClass& C = P.cls[0];
    C.teams = C.blocked == ELIM_REG ? 1 : W_CTA / C.team;  // register-resident: one system per CTA
    C.unit0 = 0;
    P.nunits = (C.nrows + C.teams - 1) / C.teams;
}

// The one-class parameters of class c of P, counting on counter c.
static WParams class_params(const WParams& P, int c, int* counters)
{
    WParams Q = P;
    Q.nclasses = 1;
    Q.cls[0] = P.cls[c];
    Q.work = counters + c;
    number_units(Q);
    return Q;
}

constexpr unsigned ALT_BITS = RBFFD_ALT_XSFC | RBFFD_ALT_YSFC | RBFFD_ALT_ZSFC;

// ALT_XSFC, ALT_YSFC, ALT_ZSFC: the X, Y, Z weights projected on the tangent
// plane at the stencil centre (x, y, z), (I - x x^T) [wX; wY; wZ], the
// reference's loop (rbffd.cpp:337-347) with its left-to-right sums and no
// fused multiply-adds.  Padding rows and slots stay 0.
__global__ void k_alt_sfc(const double* __restrict__ wx, const double* __restrict__ wy,
                          const double* __restrict__ wz, const double4* __restrict__ xyz, int N, int rows, int nc,
                          double* __restrict__ ax, double* __restrict__ ay, double* __restrict__ az)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    double x = 0, y = 0, z = 0;
    if (i < N) {
        const double4 c = xyz[i];
        x = c.x, y = c.y, z = c.z;
    }
    const double axx = __dsub_rn(1.0, __dmul_rn(x, x)), ayy = __dsub_rn(1.0, __dmul_rn(y, y)),
                 azz = __dsub_rn(1.0, __dmul_rn(z, z));
    const double axy = __dmul_rn(-x, y), axz = __dmul_rn(-x, z), ayz = __dmul_rn(-y, z);
    for (int s = 0; s < 4 * nc; s++) {
        const size_t o = sell_elem(i, s, nc);
        const double a = wx[o], b = wy[o], c = wz[o];
        ax[o] = __dadd_rn(__dadd_rn(__dmul_rn(axx, a), __dmul_rn(axy, b)), __dmul_rn(axz, c));
        ay[o] = __dadd_rn(__dadd_rn(__dmul_rn(axy, a), __dmul_rn(ayy, b)), __dmul_rn(ayz, c));
        az[o] = __dadd_rn(__dadd_rn(__dmul_rn(axz, a), __dmul_rn(ayz, b)), __dmul_rn(azz, c));
    }
}

extern "C" int rbffd_weights_compute(rbffd_grid* g, const rbffd_weight_params* prm, const double* eps, double eps_uniform,
                                     const int* deg_per_row)
{
    if (!g || !prm) return RBFFD_ERR_INVALID;
    rbffd_ctx* ctx = g->ctx;
    unsigned types = prm->der_types & 0xFFFFu;
    if (!types) return set_error(ctx, RBFFD_ERR_INVALID, "no operator selected");
    // ALT_*SFC are formed from the X, Y and Z weights; asking for one computes
    // all three and X, Y, Z (RBFFD::adjustForSFCTypes, rbffd.h:507-522)
    const bool alt = (types & ALT_BITS) != 0;
    if (alt) types = (types & ~ALT_BITS) | RBFFD_X | RBFFD_Y | RBFFD_Z;
    if (prm->poly_deg < -1 || prm->poly_deg > 4) return set_error(ctx, RBFFD_ERR_INVALID, "poly_deg %d outside [-1, 4]", prm->poly_deg);
    if (prm->dim < 1 || prm->dim > 3) return set_error(ctx, RBFFD_ERR_INVALID, "dim %d outside [1, 3]", prm->dim);
    if (prm->hv_k < 0 || prm->hv_k > 16) return set_error(ctx, RBFFD_ERR_INVALID, "hv_k %d outside [0, 16]", prm->hv_k);
    if (!eps && !(eps_uniform > 0.0) && eps_uniform != 0.0) return set_error(ctx, RBFFD_ERR_INVALID, "bad epsilon");
    WParams P;
    memset(&P, 0, sizeof P);
    int K = 0;
    for (int b = 0; b < 16; b++)
        if (types & (1u << b)) {
            if (K == MAX_K) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "more than %d operators in one solve", MAX_K);
            P.opbit[K++] = 1u << b;
        }
    P.K = K;
    int N = g->N;
    std::vector<int> deg(N, prm->poly_deg);
    if (deg_per_row)
        for (int i = 0; i < N; i++) {
            if (deg_per_row[i] < -1 || deg_per_row[i] > 4)
                return set_error(ctx, RBFFD_ERR_INVALID, "deg_per_row[%d] = %d outside [-1, 4]", i, deg_per_row[i]);
            deg[g->h_iperm[i]] = deg_per_row[i];  // internal row order
        }
    // classes by system size m, largest first
    std::map<int, std::vector<int>, std::greater<int>> buckets;
    for (int i = 0; i < N; i++) {
        int np = poly_size(deg[i]);
        buckets[g->h_len[i] + np].push_back(i);
    }
    if ((int)buckets.size() > MAX_CLASSES)
        return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "%d different system sizes (at most %d)", (int)buckets.size(),
                         MAX_CLASSES);
    int smem_max = max_smem_optin(ctx);
    for (auto& kv : buckets)
        if (kv.first > MAX_M)
            return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "system size %d (stencil + polynomial terms) exceeds %d",
                             kv.first, MAX_M);
    for (auto& kv : buckets)
        if (class_stride_bytes(kv.first, K, g->n_pad) > (size_t)smem_max)
            return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "system size %d with %d operators exceeds shared memory", kv.first, K);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    int rc;
    for (int c = 0; c < K; c++) {
        int op = der_index(P.opbit[c]);
        if ((rc = grid_alloc_w64(g, op))) return rc;
        P.w[c] = g->d_w64[op];
    }
    WeightsWork* W = nullptr;
    if ((rc = weights_work(g, &W))) return rc;
    std::vector<int> rows;
    rows.reserve(N);
    for (auto& kv : buckets) rows.insert(rows.end(), kv.second.begin(), kv.second.end());
    const int status0[2] = {INT_MAX, 0};
    cudaError_t e = cudaMemcpyAsync(W->d_rows, rows.data(), (size_t)N * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(W->d_deg, deg.data(), (size_t)N * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(W->d_status, status0, 2 * sizeof(int), cudaMemcpyHostToDevice, s);
    std::vector<double> eps_int;
    if (eps) {
        eps_int.resize(N);
        for (int i = 0; i < N; i++) eps_int[i] = eps[g->h_perm[i]];  // internal row order
    }
    if (e == cudaSuccess && eps)
        e = cudaMemcpyAsync(W->d_eps, eps_int.data(), (size_t)N * sizeof(double), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // host vectors above go out of scope after this block
    if (e != cudaSuccess) return cuda_error(ctx, e, "rbffd_weights_compute upload");
    P.xyz = g->d_xyz;
    P.idx = g->d_idx;
    P.len = g->d_len;
    P.eps = eps ? W->d_eps : nullptr;
    P.eps_uniform = eps_uniform;
    P.deg = W->d_deg;
    P.deg_uniform = prm->poly_deg;
    P.rows = W->d_rows;
    P.nrows = N;
    P.status = W->d_status;
    P.work = W->d_status + 1;
    P.n4 = g->n4;
    P.n_pad = g->n_pad;
    P.dim = prm->dim;
    P.hv_k = prm->hv_k;
    double hvN = prm->hv_nodes > 0 ? prm->hv_nodes : (double)N;
    P.hv_scale = -prm->hv_gamma * pow(hvN, -(double)prm->hv_k);
    // classes, each with its tuned team shape
    int off = 0;
    P.nclasses = 0;
    for (auto& kv : buckets) {
        WClass& C = P.cls[P.nclasses++];
        C.m = kv.first;
        C.lda = class_lda(C.m, K);
        const size_t sb = class_stride_bytes(C.m, K, g->n_pad);
        C.stride = (int)(sb / sizeof(double));
        C.rows_off = off;
        C.nrows = (int)kv.second.size();
        off += C.nrows;
        // a forced elimination (rbffd_weights_set_elimination) narrows the candidates to its own shapes
        const int forced = ctx->weights_elim == RBFFD_ELIM_UNBLOCKED ? ELIM_UNBLOCKED
                           : ctx->weights_elim == RBFFD_ELIM_BLOCKED ? ELIM_BLOCKED
                           : ctx->weights_elim == RBFFD_ELIM_ROW_MAP ? ELIM_PERM
                           : ctx->weights_elim == RBFFD_ELIM_REGISTERS ? ELIM_REG
                                                                      : -1;
        TuneKey key{200 + K, C.m, g->n_pad, forced + 1, 0};
        WShape best{0, 0};
        {
            std::lock_guard<std::mutex> lk(ctx->mu);
            auto it = ctx->tuned.find(key);
            if (it != ctx->tuned.end()) best = WShape{it->second.lanes, it->second.block};
        }
        if (best.team == 0) {
            std::vector<WShape> cands = w_candidates(C.m, K, g->n_pad, sb, smem_max);
            if (forced >= 0) {  // the forced elimination where it applies to this size, else all shapes
                std::vector<WShape> f;
                for (const WShape& cs : cands)
                    if (cs.blocked == forced) f.push_back(cs);
                if (!f.empty()) cands = f;
            }
            if (cands.empty()) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "no kernel shape fits system size %d", C.m);
            best = cands[0];
            if (cands.size() > 1 && C.nrows >= 2048) {
                // time each shape on a prefix of the class (outputs are rewritten by the full launch)
                cudaEvent_t e0, e1;
                cudaEventCreate(&e0);
                cudaEventCreate(&e1);
                float best_ms = 1e30f;
                for (const WShape& cs : cands) {
                    WParams Q = P;
                    Q.nclasses = 1;
                    Q.cls[0] = C;
                    Q.cls[0].team = cs.team;
                    Q.cls[0].blocked = cs.blocked;
                    Q.cls[0].nrows =
                        std::min(C.nrows, 16 * ctx->sm_count * (cs.blocked == ELIM_REG ? 1 : W_CTA / cs.team));
                    Q.work = W->d_status + 1;
                    number_units(Q);
                    size_t smem;
                    int grid;
                    if (persistent_geometry(ctx, Q, &smem, &grid) != RBFFD_OK) {
                        cudaGetLastError();
                        continue;
                    }
                    cudaEventRecord(e0, s);
                    enqueue_persistent(Q, smem, grid, s);
                    cudaEventRecord(e1, s);
                    if (cudaEventSynchronize(e1) != cudaSuccess) {
                        cudaGetLastError();
                        continue;
                    }
                    float ms = 0;
                    cudaEventElapsedTime(&ms, e0, e1);
                    ms /= (float)Q.cls[0].nrows;
                    if (ms < best_ms) {
                        best_ms = ms;
                        best = cs;
                    }
                }
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
            }
            std::lock_guard<std::mutex> lk(ctx->mu);
            ctx->tuned[key] = Shape{best.team, best.blocked};
        }
        C.team = best.team;
        C.blocked = best.blocked;
    }
    // the whole batch: one persistent launch per class, largest systems first,
    // captured in a CUDA graph and replayed while the parameters stay the same
    WParams Qc[MAX_CLASSES];
    size_t smem_c[MAX_CLASSES];
    int grid_c[MAX_CLASSES];
    for (int c = 0; c < P.nclasses; c++) {
        Qc[c] = class_params(P, c, W->d_status + 1);
        if ((rc = persistent_geometry(ctx, Qc[c], &smem_c[c], &grid_c[c]))) return rc;
    }
    if ((rc = class_smem_attributes(ctx, Qc, smem_c, P.nclasses))) return rc;
    if (!W->gexec || memcmp(&W->gparams, &P, sizeof P) != 0) {
        if (W->gexec) {
            cudaGraphExecDestroy(W->gexec);
            W->gexec = nullptr;
        }
        cudaGraph_t graph;
        RBFFD_CUDA_TRY(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        for (int c = 0; c < P.nclasses; c++) enqueue_persistent(Qc[c], smem_c[c], grid_c[c], s);
        e = cudaStreamEndCapture(s, &graph);
        if (e != cudaSuccess) return cuda_error(ctx, e, "weights graph capture");
        e = cudaGraphInstantiate(&W->gexec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            W->gexec = nullptr;
            return cuda_error(ctx, e, "weights graph instantiate");
        }
        W->gparams = P;
    }
    e = cudaMemcpyAsync(W->d_status, status0, 2 * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaGraphLaunch(W->gexec, s);
    if (e != cudaSuccess) return cuda_error(ctx, e, "rbffd_weights_compute launch");
    int* d_status = W->d_status;
    int status = INT_MAX;
    e = cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(ctx, e, "rbffd_weights_compute");
    if (status != INT_MAX)
        return set_error(ctx, RBFFD_ERR_SINGULAR, "stencil %d: zero pivot in the weight system",
                         g->h_perm[status - 1]);
    for (int c = 0; c < K; c++)
        if ((rc = grid_make_f32(g, der_index(P.opbit[c])))) return rc;
    if (alt) {
        const int ox = der_index(RBFFD_X), oy = der_index(RBFFD_Y), oz = der_index(RBFFD_Z);
        const int oa[3] = {der_index(RBFFD_ALT_XSFC), der_index(RBFFD_ALT_YSFC), der_index(RBFFD_ALT_ZSFC)};
        for (int k = 0; k < 3; k++)
            if ((rc = grid_alloc_w64(g, oa[k]))) return rc;
        k_alt_sfc<<<(g->N32 + 127) / 128, 128, 0, s>>>(g->d_w64[ox], g->d_w64[oy], g->d_w64[oz], g->d_xyz, g->N,
                                                       g->N32, g->nc, g->d_w64[oa[0]], g->d_w64[oa[1]],
                                                       g->d_w64[oa[2]]);
        RBFFD_CUDA_TRY(ctx, cudaGetLastError());
        for (int k = 0; k < 3; k++)
            if ((rc = grid_make_f32(g, oa[k]))) return rc;
    }
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    return RBFFD_OK;
}

extern "C" int rbffd_weights_set_elimination(rbffd_ctx* ctx, int method)
{
    if (!ctx) return RBFFD_ERR_INVALID;
    if (method < RBFFD_ELIM_AUTO || method > RBFFD_ELIM_REGISTERS)
        return set_error(ctx, RBFFD_ERR_INVALID, "unknown elimination %d", method);
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->weights_elim = method;
    return RBFFD_OK;
}

extern "C" int rbffd_weights_get_elimination(rbffd_ctx* ctx, int* method)
{
    if (!ctx || !method) return RBFFD_ERR_INVALID;
    *method = ctx->weights_elim;
    return RBFFD_OK;
}

extern "C" int rbffd_batched_gesv_dev(rbffd_ctx* ctx, int m, int nrhs, int batch, void* A, void* B, void* info)
{
    if (!ctx || !A || !B || !info || m < 1 || m > 160 || nrhs < 1 || nrhs > 16 || batch < 0) return RBFFD_ERR_INVALID;
    if (batch == 0) return RBFFD_OK;
    cudaSetDevice(ctx->device);
    size_t tb = ((size_t)m * (m + nrhs) + 2 * MAX_WARPS + MAX_WARPS + m) * sizeof(double);  // a, candidates, map
    tb = (tb + 127) / 128 * 128;
    int smem_max = max_smem_optin(ctx);
    if (tb > (size_t)smem_max) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "system %d x %d exceeds shared memory", m, m);
    int team = m <= 48 ? 32 : (m <= 96 ? 64 : 128);
    int teams = std::max(1, std::min(8, (int)(smem_max / tb)));
    while (teams > 1 && team * teams > 512) teams--;
    int block = team * teams;
    size_t smem = tb * teams;
    RBFFD_CUDA_TRY(ctx, cudaFuncSetAttribute(k_gesv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    RBFFD_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gesv, block, smem));
    int grid = std::max(1, std::min((batch + teams - 1) / teams, std::max(1, per_sm) * ctx->sm_count));
    // the three eliminations (the same arithmetic): row swaps up to 40 unknowns, a row map from 41 to 96,
    // blocked above
    k_gesv<<<grid, block, smem, ctx->stream>>>((double*)A, (double*)B, (int*)info, m, nrhs, batch, team,
                                                (int)(tb / sizeof(double)),
                                                m <= 40 ? ELIM_UNBLOCKED : (m <= 96 ? ELIM_PERM : ELIM_BLOCKED));
    RBFFD_CUDA_TRY(ctx, cudaGetLastError());
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RBFFD_OK;
}

extern "C" int rbffd_weights_assemble(rbffd_grid* g, const rbffd_weight_params* prm, const double* eps,
                                      double eps_uniform, const int* deg_per_row, const int* rows, int count,
                                      double* out)
{
    if (!g || !prm || !rows || !out || count < 0) return RBFFD_ERR_INVALID;
    rbffd_ctx* ctx = g->ctx;
    if (count == 0) return RBFFD_OK;
    unsigned types = prm->der_types & 0xFFFFu;
    if (!types || (types & 0x7000u)) return set_error(ctx, RBFFD_ERR_INVALID, "bad operator set 0x%x", types);
    if (prm->poly_deg < -1 || prm->poly_deg > 4 || prm->dim < 1 || prm->dim > 3)
        return set_error(ctx, RBFFD_ERR_INVALID, "bad poly_deg or dim");
    WParams P;
    memset(&P, 0, sizeof P);
    int K = 0;
    for (int b = 0; b < 16; b++)
        if (types & (1u << b)) {
            if (K == MAX_K) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "more than %d operators", MAX_K);
            P.opbit[K++] = 1u << b;
        }
    int N = g->N, m = -1;
    // internal row order for degrees, epsilons and the requested rows
    std::vector<int> deg(N, prm->poly_deg), rows_int(count);
    std::vector<double> eps_int;
    if (deg_per_row)
        for (int i = 0; i < N; i++) deg[g->h_iperm[i]] = deg_per_row[i];
    if (eps) {
        eps_int.resize(N);
        for (int i = 0; i < N; i++) eps_int[i] = eps[g->h_perm[i]];
    }
    for (int t = 0; t < count; t++) {
        if (rows[t] < 0 || rows[t] >= N) return set_error(ctx, RBFFD_ERR_INVALID, "row %d out of range", rows[t]);
        rows_int[t] = g->h_iperm[rows[t]];
        int mt = g->h_len[rows_int[t]] + poly_size(deg[rows_int[t]]);
        if (m >= 0 && mt != m) return set_error(ctx, RBFFD_ERR_INVALID, "rows of one call must share the system size");
        m = mt;
    }
    size_t tb = (team_bytes_w(m, K, g->n_pad) + 127) / 128 * 128;
    if (tb > (size_t)max_smem_optin(ctx)) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "system too large");
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    int *d_rows = nullptr, *d_deg = nullptr;
    double *d_eps = nullptr, *d_out = nullptr;
    size_t osz = (size_t)count * m * (m + K) * sizeof(double);
    int rc;
    auto cleanup = [&]() {
        dev_free(ctx, d_rows, count * sizeof(int));
        dev_free(ctx, d_deg, (size_t)N * sizeof(int));
        dev_free(ctx, d_eps, (size_t)N * sizeof(double));
        dev_free(ctx, d_out, osz);
    };
    if ((rc = dev_alloc(ctx, (void**)&d_rows, count * sizeof(int))) ||
        (rc = dev_alloc(ctx, (void**)&d_deg, (size_t)N * sizeof(int))) ||
        (eps && (rc = dev_alloc(ctx, (void**)&d_eps, (size_t)N * sizeof(double)))) ||
        (rc = dev_alloc(ctx, (void**)&d_out, osz))) {
        cleanup();
        return rc;
    }
    cudaError_t e = cudaMemcpyAsync(d_rows, rows_int.data(), count * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_deg, deg.data(), (size_t)N * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && eps)
        e = cudaMemcpyAsync(d_eps, eps_int.data(), (size_t)N * sizeof(double), cudaMemcpyHostToDevice, s);
    P.xyz = g->d_xyz;
    P.idx = g->d_idx;
    P.len = g->d_len;
    P.eps = d_eps;
    P.eps_uniform = eps_uniform;
    P.deg = d_deg;
    P.deg_uniform = prm->poly_deg;
    P.rows = d_rows;
    P.nrows = count;
    P.K = K;
    P.m = m;
    P.n4 = g->n4;
    P.n_pad = g->n_pad;
    P.dim = prm->dim;
    P.hv_k = prm->hv_k;
    P.team_stride = (int)(tb / sizeof(double));
    if (e == cudaSuccess) {
        const int team = 64;
        RBFFD_CUDA_TRY(ctx, cudaFuncSetAttribute(k_assemble, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tb));
        k_assemble<<<std::min(count, 4 * ctx->sm_count), team, tb, s>>>(P, team, d_out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, osz, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cleanup();
    if (e != cudaSuccess) return cuda_error(ctx, e, "rbffd_weights_assemble");
    return RBFFD_OK;
}
