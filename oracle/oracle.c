/*
 * oracle.c -- CPU restatement of the reference RBF-FD hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is called by
 * tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg.
 * The product (rbffd_gpu_b200, librbffd_sm100.so) never links, loads or
 * calls anything here.
 *
 * It restates, in plain C and FP64, the reference functions on the path:
 *   - RBF_Gaussian evaluations        src/rbffd/rbfs/rbf_gaussian.h:40-249
 *   - cart2sph                        src/utils/geom/cart2sph.cpp:3-11
 *   - RBFFD::distanceMatrix           src/rbffd/rbffd.cpp:888-969
 *   - RBFFD::getStencilLHS            src/rbffd/rbffd.cpp:129-191
 *   - RBFFD::getStencilRHS            src/rbffd/rbffd.cpp:356-537
 *   - RBFFD::computeAllWeightsForStencil_Direct  src/rbffd/rbffd.cpp:225-352
 *       (arma::solve == LAPACK dgesv: LU with partial pivoting, dgetrs)
 *   - RBFFD::applyWeightsForDeriv     src/rbffd/rbffd.cpp:669-688
 *   - CosineBell::solve               src/pdes/hyperbolic/cosine_bell.cpp:23-70
 *   - TimeDependentPDE::advanceRungeKutta4  src/pdes/time_dependent_pde.cpp:172-304
 *
 * Floating-point model.  Compiled with -ffp-contract=off so every expression
 * is evaluated exactly as written.  Two models of the multiply-adds on the
 * time-stepping path (the SpMV accumulation, the RK4 axpys, the advection
 * right-hand side), selected by orc_set_fused():
 *   fused (default) -- each such multiply-add is one fma(), the arithmetic of
 *     the device kernels' FP64 path (one rounding per multiply-add);
 *   plain (orc_set_fused(0)) -- a rounded product, then a rounded sum, in the
 *     reference's source order: the arithmetic of the reference as its own
 *     build compiles it (CMakeLists.txt:130-140: g++ -O3 -ftree-vectorize for
 *     x86-64 without -march, which has no FMA instruction), checked bit for
 *     bit against the reference's RBFFD, TimeDependentPDE and CosineBell
 *     compiled from their sources (oracle/ref_rbffd.cpp, tests/test_ref_core.py).
 * The LU updates are always fused (the shim's arma::solve is the same code).
 * The RBF kernel evaluations are written without fma, operand order as in
 * rbf_gaussian.h (checked against the header itself, compiled from the
 * reference sources, by tests/test_oracle_pins.py).
 *
 * Polynomial augmentation.  poly_deg = 0 is the reference build
 * (ONE_MONOMIAL, np = 1, rbffd.cpp:1,230-234; constant row of the RHS is 0
 * for every operator, rbffd.cpp:506-508).  poly_deg = 1 uses {1,x,y,z} as the
 * reference does when ONE_MONOMIAL is 0 with dim 3 (rbffd.cpp:150-172); its
 * X/Y/Z/LAPL rows equal the reference's (rbffd.cpp:510-526); for the other
 * operators the rows hold the operator applied exactly to 1,x,y,z (the
 * reference prints a warning and leaves them 0, rbffd.cpp:527-531).
 * Beyond the reference, poly_deg 2..4 use polynomials of total degree <= d in
 * scaled tangent-plane coordinates of the stencil centre c:
 *   xi = (x - c).e_lambda / s,  eta = (x - c).e_theta / s,  s = max_j |x_j - c|,
 * basis xi^a eta^b ordered by total degree t (a = t..0), (d+1)(d+2)/2 terms.
 * (3-D monomials restricted to a small cap are nearly dependent; this basis
 * keeps the border block well conditioned.)  Operator rows at xi = eta = 0:
 * LAMBDA = d/dxi / s, THETA = d/deta / s, X/Y/Z and *SFC = components of
 * (p_xi e_lambda + p_eta e_theta) / s, LSFC = (p_xixi + p_etaeta) / s^2,
 * LAPL = sum_{a<dim} (p_xixi e1a^2 + 2 p_xieta e1a e2a + p_etaeta e2a^2) / s^2,
 * HV = (d_xixi + d_etaeta)^k / s^2k, INTERP = p(0).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* DerType bit values: src/rbffd/rbffd.h:43-60 */
enum {
    D_X = 0x1, D_Y = 0x2, D_Z = 0x4, D_LAPL = 0x8, D_R = 0x10, D_HV = 0x20,
    D_LAMBDA = 0x40, D_THETA = 0x80, D_LSFC = 0x100, D_XSFC = 0x200,
    D_YSFC = 0x400, D_ZSFC = 0x800, D_ALT_XSFC = 0x1000, D_ALT_YSFC = 0x2000,
    D_ALT_ZSFC = 0x4000, D_INTERP = 0x8000
};

/* ------------------------------------------------------------------ */
/* cart2sph (src/utils/geom/cart2sph.cpp:3-11): theta = longitude,     */
/* phi = latitude (the names are swapped on purpose, rbffd.cpp:402-412) */
static void cart2sph(double x, double y, double z, double* theta, double* phi)
{
    *theta = atan2(y, x);
    *phi = atan2(z, sqrt(x * x + y * y));
}

/* ------------------------------------------------------------------ */
/* Gaussian RBF, rbf_gaussian.h.  r2 = diff.square() = (dx*dx+dy*dy)+dz*dz */
static double g_eval(double eps2, double r2) { return exp(-(r2 * eps2)); }
static double g_rderiv_over_r(double eps2, double r2) { return -2. * eps2 * g_eval(eps2, r2); }
static double g_rderiv2(double eps2, double r2)
{
    return g_rderiv_over_r(eps2, r2) + 4. * (eps2 * eps2) * r2 * exp(-(eps2 * r2));
}
/* hv_p_k: rbf_gaussian.h:229-249 (recursive, dim/2. in floating point) */
static double g_hv_p_k(double eps2, int dim, double r2, int k)
{
    double eps2r2 = eps2 * r2;
    if (k == 0) return 1.;
    if (k == 1) return 4. * (eps2r2)-2. * dim;
    return 4. * (eps2r2 - 2. * (k - 1) - dim / 2.) * g_hv_p_k(eps2, dim, r2, k - 1)
        - 8. * (k - 1) * (2. * (k - 1) - 2. + dim) * g_hv_p_k(eps2, dim, r2, k - 2);
}

/* which: 0 eval, 1 x, 2 y, 3 z, 4 r, 5 rderiv_over_r, 6 rderiv2, 7 lapl(dim), 8 hyperviscosity(k) */
double orc_rbf(int which, double eps, int dim, double dx, double dy, double dz, int hv_k)
{
    double eps2 = eps * eps;
    double r2 = dx * dx + dy * dy + dz * dz;
    switch (which) {
    case 0: return g_eval(eps2, r2);
    case 1: { double xe = dx * eps2; return -2. * xe * g_eval(eps2, r2); }
    case 2: { double ye = dy * eps2; return -2. * ye * g_eval(eps2, r2); }
    case 3: { double ze = dz * eps2; return -2. * ze * g_eval(eps2, r2); }
    case 4: { double reps = sqrt(r2) * eps2; return -2. * reps * g_eval(eps2, r2); }
    case 5: return g_rderiv_over_r(eps2, r2);
    case 6: return g_rderiv2(eps2, r2);
    case 7:
        if (dim == 1) { double x2e = dx * dx * eps2; return 2. * eps2 * (-1. + 2. * x2e) * g_eval(eps2, r2); }
        if (dim == 2) {
            double x2e = dx * dx * eps2, y2e = dy * dy * eps2;
            return 4. * eps2 * (-1. + x2e + y2e) * g_eval(eps2, r2);
        }
        { double r2e4 = r2 * (eps2 * eps2); return (-6. * eps2 + 4. * r2e4) * g_eval(eps2, r2); }
    case 8: return pow(eps, 2 * hv_k) * g_hv_p_k(eps2, dim, r2, hv_k) * g_eval(eps2, r2);
    }
    return NAN;
}

/* ------------------------------------------------------------------ */
/* Polynomials in x,y,z of degree <= 4 as dense coefficient cubes.     */
#define PD 5
typedef struct { double c[PD][PD][PD]; } poly_t;

static void p_zero(poly_t* p) { memset(p, 0, sizeof(*p)); }
static void p_mono(poly_t* p, int a, int b, int c) { p_zero(p); p->c[a][b][c] = 1.0; }
static void p_d(const poly_t* p, int axis, poly_t* out)
{
    p_zero(out);
    for (int a = 0; a < PD; a++)
        for (int b = 0; b < PD; b++)
            for (int c = 0; c < PD; c++) {
                double v = p->c[a][b][c];
                if (v == 0.) continue;
                if (axis == 0 && a > 0) out->c[a - 1][b][c] += v * a;
                if (axis == 1 && b > 0) out->c[a][b - 1][c] += v * b;
                if (axis == 2 && c > 0) out->c[a][b][c - 1] += v * c;
            }
}
static double p_eval(const poly_t* p, double x, double y, double z)
{
    double s = 0.;
    for (int a = 0; a < PD; a++)
        for (int b = 0; b < PD; b++)
            for (int c = 0; c < PD; c++) {
                double v = p->c[a][b][c];
                if (v != 0.) s += v * pow(x, a) * pow(y, b) * pow(z, c);
            }
    return s;
}
static void p_lapl(const poly_t* p, int dim, poly_t* out)
{
    poly_t t1, t2;
    p_zero(out);
    for (int ax = 0; ax < dim && ax < 3; ax++) {
        p_d(p, ax, &t1);
        p_d(&t1, ax, &t2);
        for (int a = 0; a < PD; a++)
            for (int b = 0; b < PD; b++)
                for (int c = 0; c < PD; c++) out->c[a][b][c] += t2.c[a][b][c];
    }
}

/* Basis of degree d: for t = 0..d: x^a y^(t-a) (a = t..0), then x^a y^(t-1-a) z (a = t-1..0).
 * d = 1 gives {1, x, y, z}, the reference order (rbffd.cpp:150-172). */
int orc_poly_size(int deg) { return deg < 0 ? 0 : (deg == 0 ? 1 : (deg == 1 ? 4 : (deg + 1) * (deg + 2) / 2)); }
static int poly_exponents(int deg, int (*e)[3])
{
    int k = 0;
    for (int t = 0; t <= deg; t++) {
        for (int a = t; a >= 0; a--) { e[k][0] = a; e[k][1] = t - a; e[k][2] = 0; k++; }
        for (int a = t - 1; a >= 0; a--) { e[k][0] = a; e[k][1] = t - 1 - a; e[k][2] = 1; k++; }
    }
    return k;
}

/* Operator `which` applied to monomial x^a y^b z^c, evaluated at centre (x0,y0,z0). */
static double poly_op(unsigned which, const int* e, double x0, double y0, double z0, int dim, int hv_k)
{
    poly_t p, dx, dy, dz, t;
    p_mono(&p, e[0], e[1], e[2]);
    p_d(&p, 0, &dx); p_d(&p, 1, &dy); p_d(&p, 2, &dz);
    double gx = p_eval(&dx, x0, y0, z0), gy = p_eval(&dy, x0, y0, z0), gz = p_eval(&dz, x0, y0, z0);
    double lam, th;
    cart2sph(x0, y0, z0, &lam, &th);
    double cdotg = x0 * gx + y0 * gy + z0 * gz;
    switch (which) {
    case D_X: return gx;
    case D_Y: return gy;
    case D_Z: return gz;
    case D_LAPL: p_lapl(&p, dim, &t); return p_eval(&t, x0, y0, z0);
    case D_INTERP: return p_eval(&p, x0, y0, z0);
    case D_LAMBDA: return -sin(lam) * gx + cos(lam) * gy;
    case D_THETA: return -sin(th) * cos(lam) * gx - sin(th) * sin(lam) * gy + cos(th) * gz;
    case D_LSFC: {
        /* Laplace-Beltrami on the unit sphere: tr(H) - c^T H c - 2 c.grad p */
        poly_t h[3][3];
        const poly_t* g[3] = {&dx, &dy, &dz};
        double H[3][3], c[3] = {x0, y0, z0};
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) { p_d(g[i], j, &h[i][j]); H[i][j] = p_eval(&h[i][j], x0, y0, z0); }
        double tr = H[0][0] + H[1][1] + H[2][2], q = 0.;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) q += c[i] * H[i][j] * c[j];
        return tr - q - 2. * cdotg;
    }
    case D_XSFC: return gx - x0 * cdotg;
    case D_YSFC: return gy - y0 * cdotg;
    case D_ZSFC: return gz - z0 * cdotg;
    case D_HV: {
        poly_t cur = p, nxt;
        for (int k = 0; k < hv_k; k++) { p_lapl(&cur, dim, &nxt); cur = nxt; }
        return p_eval(&cur, x0, y0, z0);
    }
    default: return 0.; /* R and ALT_*: no polynomial counterpart (rbffd.cpp:527-531) */
    }
}

/* ------------------------------------------------------------------ */
/* Tangent-plane basis (poly_deg >= 2).                                 */
typedef struct { double e1[3], e2[3], s; } tframe_t;

static void tangent_frame(const double* xyz, const int* st, int n, tframe_t* F)
{
    const double* c = xyz + 3 * (size_t)st[0];
    double lam, th;
    cart2sph(c[0], c[1], c[2], &lam, &th);
    F->e1[0] = -sin(lam); F->e1[1] = cos(lam); F->e1[2] = 0.;
    F->e2[0] = -sin(th) * cos(lam); F->e2[1] = -sin(th) * sin(lam); F->e2[2] = cos(th);
    double s2 = 0.;
    for (int j = 0; j < n; j++) {
        const double* x = xyz + 3 * (size_t)st[j];
        double dx = x[0] - c[0], dy = x[1] - c[1], dz = x[2] - c[2];
        double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > s2) s2 = r2;
    }
    F->s = s2 > 0. ? sqrt(s2) : 1.;
}

static void tangent_exponents(int deg, int (*e)[2])
{
    int k = 0;
    for (int t = 0; t <= deg; t++)
        for (int a = t; a >= 0; a--) { e[k][0] = a; e[k][1] = t - a; k++; }
}

static double fact(int a) { double f = 1.; for (int i = 2; i <= a; i++) f *= i; return f; }
static double binom(int k, int i) { return fact(k) / (fact(i) * fact(k - i)); }

/* operator applied to xi^a eta^b at the centre */
static double tangent_op(unsigned which, int a, int b, const tframe_t* F, int dim, int hv_k)
{
    double s = F->s;
    int t = a + b;
    switch (which) {
    case D_INTERP: return t == 0 ? 1. : 0.;
    case D_LAMBDA: return (a == 1 && b == 0) ? 1. / s : 0.;
    case D_THETA: return (a == 0 && b == 1) ? 1. / s : 0.;
    case D_X: case D_Y: case D_Z: case D_XSFC: case D_YSFC: case D_ZSFC: {
        int ax = (which == D_X || which == D_XSFC) ? 0 : ((which == D_Y || which == D_YSFC) ? 1 : 2);
        if (a == 1 && b == 0) return F->e1[ax] / s;
        if (a == 0 && b == 1) return F->e2[ax] / s;
        return 0.;
    }
    case D_LSFC: return ((a == 2 && b == 0) || (a == 0 && b == 2)) ? 2. / (s * s) : 0.;
    case D_LAPL: {
        double q = 0.;
        for (int ax = 0; ax < dim && ax < 3; ax++) {
            if (a == 2 && b == 0) q += 2. * F->e1[ax] * F->e1[ax];
            if (a == 1 && b == 1) q += 2. * F->e1[ax] * F->e2[ax];
            if (a == 0 && b == 2) q += 2. * F->e2[ax] * F->e2[ax];
        }
        return q / (s * s);
    }
    case D_HV: {
        if (t != 2 * hv_k || (a & 1) || (b & 1)) return 0.;
        return binom(hv_k, a / 2) * fact(a) * fact(b) / pow(s, 2 * hv_k);
    }
    default: return 0.;
    }
}

/* ------------------------------------------------------------------ */
/* RHS entry j (< n) of operator `which`: rbffd.cpp:375-503.            */
static double rhs_rbf(unsigned which, const double* x0v, const double* xjv, double eps, int dim, int hv_k)
{
    double eps2 = eps * eps;
    double dx = x0v[0] - xjv[0], dy = x0v[1] - xjv[1], dz = x0v[2] - xjv[2];
    double r2 = dx * dx + dy * dy + dz * dz;
    double lam_j, th_j, lam_i, th_i;
    cart2sph(xjv[0], xjv[1], xjv[2], &lam_j, &th_j);
    cart2sph(x0v[0], x0v[1], x0v[2], &lam_i, &th_i);
    switch (which) {
    case D_X: return orc_rbf(1, eps, dim, dx, dy, dz, hv_k);
    case D_Y: return orc_rbf(2, eps, dim, dx, dy, dz, hv_k);
    case D_Z: return orc_rbf(3, eps, dim, dx, dy, dz, hv_k);
    case D_LAPL: return orc_rbf(7, eps, dim, dx, dy, dz, hv_k);
    case D_INTERP: return g_eval(eps2, r2);
    case D_R: return orc_rbf(4, eps, dim, dx, dy, dz, hv_k);
    case D_LAMBDA: {
        double drdl = cos(th_j) * sin(lam_i - lam_j);
        return fabs(drdl) > 0. ? drdl * g_rderiv_over_r(eps2, r2) : 0.;
    }
    case D_THETA: {
        double drdt = cos(th_j) * sin(th_i) * cos(lam_i - lam_j) - sin(th_j) * cos(th_i);
        return fabs(drdt) > 0. ? drdt * g_rderiv_over_r(eps2, r2) : 0.;
    }
    case D_LSFC:
        return (1. / 4.) * ((4. - r2) * g_rderiv2(eps2, r2) + (4. - 3. * r2) * g_rderiv_over_r(eps2, r2));
    case D_XSFC: case D_YSFC: case D_ZSFC: {
        double xTx = x0v[0] * xjv[0] + x0v[1] * xjv[1] + x0v[2] * xjv[2];
        int ax = which == D_XSFC ? 0 : (which == D_YSFC ? 1 : 2);
        double v = x0v[ax] * xTx - xjv[ax];
        return v * g_rderiv_over_r(eps2, r2);
    }
    case D_HV: return orc_rbf(8, eps, dim, dx, dy, dz, hv_k);
    default: return 0.; /* ALT_*: rbffd.cpp:490-494 */
    }
}

/* ------------------------------------------------------------------ */
/* dgesv restatement: Gaussian elimination with partial pivoting on the
 * augmented row-major matrix [A | B] (m x (m+nrhs)), then column-oriented
 * back substitution -- the arithmetic of dgetf2 + dgetrs (dtrsm L then U).
 * Pivot: first row of maximum |a_ik| (idamax).  Multipliers by division.
 * Returns 0, or k+1 if U(k,k) is exactly zero (dgetrf's INFO). */
int orc_gesv_aug(int m, int nrhs, double* a)
{
    int ld = m + nrhs, info = 0;
    for (int k = 0; k < m; k++) {
        int p = k;
        double best = fabs(a[k * ld + k]);
        for (int i = k + 1; i < m; i++) {
            double v = fabs(a[i * ld + k]);
            if (v > best) { best = v; p = i; }
        }
        if (p != k)
            for (int j = 0; j < ld; j++) { double t = a[k * ld + j]; a[k * ld + j] = a[p * ld + j]; a[p * ld + j] = t; }
        double piv = a[k * ld + k];
        if (piv == 0.) { if (!info) info = k + 1; continue; }
        for (int i = k + 1; i < m; i++) {
            double l = a[i * ld + k] / piv;
            a[i * ld + k] = l;
            for (int j = k + 1; j < ld; j++) a[i * ld + j] = fma(-l, a[k * ld + j], a[i * ld + j]);
        }
    }
    if (info) return info;
    /* back substitution, column oriented (dtrsm upper, non-unit) */
    for (int r = 0; r < nrhs; r++) {
        int c = m + r;
        for (int k = m - 1; k >= 0; k--) {
            double xk = a[k * ld + c] / a[k * ld + k];
            a[k * ld + c] = xk;
            for (int i = 0; i < k; i++) a[i * ld + c] = fma(-xk, a[i * ld + k], a[i * ld + c]);
        }
    }
    return 0;
}

/* Plain interface for pinning against numpy.linalg.solve: A row-major m x m,
 * B row-major m x nrhs; solution written to X (m x nrhs). */
int orc_lu_solve(int m, int nrhs, const double* A, const double* B, double* X)
{
    int ld = m + nrhs;
    double* a = (double*)malloc(sizeof(double) * (size_t)m * ld);
    if (!a) return -1;
    for (int i = 0; i < m; i++) {
        for (int j = 0; j < m; j++) a[i * ld + j] = A[i * m + j];
        for (int r = 0; r < nrhs; r++) a[i * ld + m + r] = B[i * nrhs + r];
    }
    int info = orc_gesv_aug(m, nrhs, a);
    for (int i = 0; i < m; i++)
        for (int r = 0; r < nrhs; r++) X[i * nrhs + r] = a[i * ld + m + r];
    free(a);
    return info;
}

/* ------------------------------------------------------------------ */
/* Assemble and solve one stencil: rbffd.cpp:225-352.                   */
static int popcount16(unsigned v) { int c = 0; for (int b = 0; b < 16; b++) c += (v >> b) & 1u; return c; }

/* Build the augmented system for stencil `row`; returns m, fills a (m x (m+K)). */
static int assemble_stencil(const double* xyz, const int* st, int n, int deg, double eps,
                            unsigned der_types, int dim, int hv_k, double* a)
{
    int np = orc_poly_size(deg), m = n + np, K = popcount16(der_types), ld = m + K;
    int e[32][3];
    poly_exponents(deg == 1 ? 1 : (deg == 0 ? 0 : -1), e);
    double eps2 = eps * eps;
    memset(a, 0, sizeof(double) * (size_t)m * ld);
    /* distanceMatrix: ar(j,i) = phi(x_i - x_j) (rbffd.cpp:943-966) */
    for (int j = 0; j < n; j++) {
        const double* xj = xyz + 3 * (size_t)st[j];
        for (int i = 0; i < n; i++) {
            const double* xi = xyz + 3 * (size_t)st[i];
            double dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
            a[j * ld + i] = g_eval(eps2, dx * dx + dy * dy + dz * dz);
        }
    }
    /* polynomial border: {1} or {1,x,y,z} (rbffd.cpp:150-172); tangent basis beyond */
    tframe_t F;
    int te[32][2];
    if (deg >= 2) {
        tangent_frame(xyz, st, n, &F);
        tangent_exponents(deg, te);
    }
    const double* c0 = xyz + 3 * (size_t)st[0];
    for (int q = 0; q < np; q++)
        for (int i = 0; i < n; i++) {
            const double* xi = xyz + 3 * (size_t)st[i];
            double v;
            if (deg >= 2) {
                double dx = xi[0] - c0[0], dy = xi[1] - c0[1], dz = xi[2] - c0[2];
                double u = (dx * F.e1[0] + dy * F.e1[1] + dz * F.e1[2]) / F.s;
                double w = (dx * F.e2[0] + dy * F.e2[1] + dz * F.e2[2]) / F.s;
                v = pow(u, te[q][0]) * pow(w, te[q][1]);
            } else {
                v = pow(xi[0], e[q][0]) * pow(xi[1], e[q][1]) * pow(xi[2], e[q][2]);
            }
            a[(n + q) * ld + i] = v;
            a[i * ld + (n + q)] = v;
        }
    /* right-hand sides, one column per selected type in bit order (rbffd.cpp:106-125) */
    const double* x0v = xyz + 3 * (size_t)st[0];
    int col = 0;
    for (int b = 0; b < 16; b++) {
        unsigned which = 1u << b;
        if (!(der_types & which)) continue;
        for (int j = 0; j < n; j++)
            a[j * ld + m + col] = rhs_rbf(which, x0v, xyz + 3 * (size_t)st[j], eps, dim, hv_k);
        for (int q = 0; q < np; q++) {
            double v;
            if (deg == 0) v = 0.;
            else if (deg == 1) v = poly_op(which, e[q], x0v[0], x0v[1], x0v[2], dim, hv_k);
            else v = tangent_op(which, te[q][0], te[q][1], &F, dim, hv_k);
            a[(n + q) * ld + m + col] = v;
        }
        col++;
    }
    return m;
}

/* All stencils.  w_out: [K][N][n_pad] (types in bit order), first st_len[i]
 * entries of each row = weights of the stencil nodes (the reference stores n+np
 * and applies only n, rbffd.cpp:300-306,680-684); padding = 0.  HV weights are
 * multiplied by hv_scale (= getHVScalar(), rbffd.h:227-238; rbffd.cpp:295-297).
 * deg_per_row may be NULL (all rows use poly_deg).  Returns 0 or the first
 * failing row + 1 (negated) when a pivot is exactly zero. */
int orc_weights(int N, const double* xyz, int n_pad, const int* st, const int* st_len,
                const double* eps, unsigned der_types, int dim, int poly_deg, const int* deg_per_row,
                int hv_k, double hv_scale, double* w_out, int nthreads)
{
    int K = popcount16(der_types);
    int bad = 0;
    memset(w_out, 0, sizeof(double) * (size_t)K * N * n_pad);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
    {
        int mmax = n_pad + orc_poly_size(4);
        double* a = (double*)malloc(sizeof(double) * (size_t)mmax * (mmax + K));
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
        for (int r = 0; r < N; r++) {
            const int* s = st + (size_t)r * n_pad;
            int n = st_len ? st_len[r] : n_pad;
            int deg = deg_per_row ? deg_per_row[r] : poly_deg;
            double ep = eps[s[0]]; /* var_epsilon[stencil[0]] (rbffd.cpp:395-400) */
            int m = assemble_stencil(xyz, s, n, deg, ep, der_types, dim, hv_k, a);
            int info = orc_gesv_aug(m, K, a);
            if (info) {
#ifdef _OPENMP
#pragma omp critical
#endif
                { if (!bad) bad = r + 1; }
                continue;
            }
            int col = 0, ld = m + K;
            for (int b = 0; b < 16; b++) {
                unsigned which = 1u << b;
                if (!(der_types & which)) continue;
                double scale = which == D_HV ? hv_scale : 1.;
                double* w = w_out + ((size_t)col * N + r) * n_pad;
                for (int j = 0; j < n; j++) w[j] = a[j * ld + m + col] * scale;
                col++;
            }
        }
        free(a);
    }
    return bad ? -bad : 0;
}

/* Assembled system of one stencil, for inspection: a (m x (m+K)) row-major. */
int orc_assemble(const double* xyz, const int* st, int n, int deg, double eps, unsigned der_types,
                 int dim, int hv_k, double* a)
{
    return assemble_stencil(xyz, st, n, deg, eps, der_types, dim, hv_k, a);
}

/* ------------------------------------------------------------------ */
/* applyWeightsForDeriv (rbffd.cpp:669-688): deriv[i] = sum_s w[i][s]*u[st_i[s]],
 * s in stencil order; accumulation fused (fma).  u and deriv are [N][T].      */
static int g_fused = 1;

/* 1: fused multiply-adds on the time-stepping path (the device's FP64
 * arithmetic); 0: plain products and sums (the reference's own build). */
void orc_set_fused(int fused) { g_fused = fused ? 1 : 0; }
int orc_get_fused(void) { return g_fused; }

/* a*b + c in the selected model */
static inline double madd(double a, double b, double c) { return g_fused ? fma(a, b, c) : a * b + c; }

static inline double row_dot(const double* w, const int* s, int n, const double* u, int T, int t)
{
    double der = 0.0;
    for (int k = 0; k < n; k++) der = madd(w[k], u[(size_t)s[k] * T + t], der);
    return der;
}

void orc_apply(int N, int n_pad, const int* st, const int* st_len, const double* w, int T,
               const double* u, double* deriv, int start, int count, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (int i = start; i < start + count; i++) {
        int n = st_len ? st_len[i] : n_pad;
        for (int t = 0; t < T; t++)
            deriv[(size_t)i * T + t] = row_dot(w + (size_t)i * n_pad, st + (size_t)i * n_pad, n, u, T, t);
    }
}

/* ------------------------------------------------------------------ */
/* Per-node coefficients of CosineBell::solve (cosine_bell.cpp:35-49):
 * cu = vel_u / a, cv = vel_v / a.                                       */
void orc_cosine_bell_coeffs(int N, const double* xyz, double a, double alpha, double u0, double* cu, double* cv)
{
    for (int i = 0; i < N; i++) {
        double lam, th;
        cart2sph(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], &lam, &th);
        double vel_u = u0 * (cos(th) * cos(alpha) + sin(th) * cos(lam) * sin(alpha));
        double vel_v = -u0 * (sin(lam) * sin(alpha));
        cu[i] = vel_u / a;
        cv[i] = vel_v / a;
    }
}

/* Right-hand side f(x) for one stage.
 *   kind 1 (advection, CosineBell::solve form):
 *        f = -(cu*Dlam x + cv*Dth x)  [+ Dhv x]
 *   kind 2 (heat on the sphere): f = kappa * Dlsfc x                          */
typedef struct {
    int kind, N, n_pad, T;
    const int* st; const int* st_len;
    const double *w0, *w1, *w2; /* kind 1: lambda, theta, hv (may be NULL); kind 2: lsfc */
    const double *cu, *cv;
    double kappa;
} rhs_t;

static void eval_rhs(const rhs_t* R, const double* x, double* f)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = 0; i < R->N; i++) {
        int n = R->st_len ? R->st_len[i] : R->n_pad;
        const int* s = R->st + (size_t)i * R->n_pad;
        for (int t = 0; t < R->T; t++) {
            double v;
            if (R->kind == 1) {
                double dl = row_dot(R->w0 + (size_t)i * R->n_pad, s, n, x, R->T, t);
                double dt = row_dot(R->w1 + (size_t)i * R->n_pad, s, n, x, R->T, t);
                /* -((vel_u/a) * dh_dlambda + (vel_v/a) * dh_dtheta), cosine_bell.cpp:51 */
                v = -madd(R->cu[i], dl, R->cv[i] * dt);
                if (R->w2) v = v + row_dot(R->w2 + (size_t)i * R->n_pad, s, n, x, R->T, t);
            } else {
                v = R->kappa * row_dot(R->w0 + (size_t)i * R->n_pad, s, n, x, R->T, t);
            }
            f[(size_t)i * R->T + t] = v;
        }
    }
}

/* Classical RK4 (time_dependent_pde.cpp:172-304), u updated in place. */
static int rk4(const rhs_t* R, double* u, double dt, int nsteps, int nthreads)
{
    size_t L = (size_t)R->N * R->T;
    double *s = malloc(sizeof(double) * L), *k1 = malloc(sizeof(double) * L), *k2 = malloc(sizeof(double) * L),
           *k3 = malloc(sizeof(double) * L), *k4 = malloc(sizeof(double) * L);
    if (!s || !k1 || !k2 || !k3 || !k4) { free(s); free(k1); free(k2); free(k3); free(k4); return -1; }
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    for (int step = 0; step < nsteps; step++) {
        /* s = u + 0.5*dt*(k + 0): time_dependent_pde.cpp:201-250 (the forcing
         * term f is 0, and k + 0. == k for every non-zero k) */
        eval_rhs(R, u, k1);
        for (size_t i = 0; i < L; i++) s[i] = madd(0.5 * dt, k1[i], u[i]);
        eval_rhs(R, s, k2);
        for (size_t i = 0; i < L; i++) s[i] = madd(0.5 * dt, k2[i], u[i]);
        eval_rhs(R, s, k3);
        for (size_t i = 0; i < L; i++) s[i] = madd(dt, k3[i], u[i]);
        eval_rhs(R, s, k4);
        /* u + (dt/6.)*(k1 + 2k2 + 2k3 + k4), :280-282 (2.*k is exact) */
        for (size_t i = 0; i < L; i++) u[i] = madd(dt / 6., k1[i] + 2. * k2[i] + 2. * k3[i] + k4[i], u[i]);
    }
    free(s); free(k1); free(k2); free(k3); free(k4);
    return 0;
}

int orc_rk4_advect(int N, int n_pad, const int* st, const int* st_len, const double* w_lambda,
                   const double* w_theta, const double* w_hv, const double* cu, const double* cv, int T,
                   double* u, double dt, int nsteps, int nthreads)
{
    rhs_t R = {1, N, n_pad, T, st, st_len, w_lambda, w_theta, w_hv, cu, cv, 0.};
    return rk4(&R, u, dt, nsteps, nthreads);
}

int orc_rk4_heat(int N, int n_pad, const int* st, const int* st_len, const double* w_lsfc, double kappa, int T,
                 double* u, double dt, int nsteps, int nthreads)
{
    rhs_t R = {2, N, n_pad, T, st, st_len, w_lsfc, NULL, NULL, NULL, NULL, kappa};
    return rk4(&R, u, dt, nsteps, nthreads);
}

int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_num_procs();  /* not omp_get_max_threads: a call with nthreads = 1 lowers that for the process */
#else
    return 1;
#endif
}

/* cart2sph exported for the pin against src/utils/geom/cart2sph.cpp */
void orc_cart2sph(double x, double y, double z, double* theta, double* phi)
{
    cart2sph(x, y, z, theta, phi);
}

/* ------------------------------------------------------------------------
 * Synthetic workload inputs for the CPU arm of the benchmark, so that it
 * builds its grid and initial state without the product library.  The
 * reference's maximum-determinant node files are not distributed; these are
 * the seeded stand-ins the benchmark uses on both arms.
 *
 * orc_nodes_fibonacci: the Fibonacci spiral z_i = 1 - (2i+1)/N,
 * phi_i = i*pi*(3 - sqrt 5), turned by a uniform random rotation drawn from
 * three splitmix64 uniforms (Shoemake's unit quaternion), each point
 * renormalised onto the unit sphere.
 * ------------------------------------------------------------------------ */
static uint64_t sm64_next(uint64_t* s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double sm64_unit(uint64_t* s) { return (double)(sm64_next(s) >> 11) * (1.0 / 9007199254740992.0); }

int orc_nodes_fibonacci(int N, uint64_t seed, double* xyz)
{
    if (N <= 0 || !xyz) return -1;
    uint64_t s = seed;
    double a = sm64_unit(&s), b = sm64_unit(&s), c = sm64_unit(&s);
    const double tau = 6.283185307179586476925286766559;
    /* unit quaternion (qw; qx, qy, qz) */
    double qx = sqrt(1.0 - a) * sin(tau * b), qy = sqrt(1.0 - a) * cos(tau * b);
    double qz = sqrt(a) * sin(tau * c), qw = sqrt(a) * cos(tau * c);
    double M[3][3];
    M[0][0] = 1 - 2 * (qy * qy + qz * qz); M[0][1] = 2 * (qx * qy - qz * qw); M[0][2] = 2 * (qx * qz + qy * qw);
    M[1][0] = 2 * (qx * qy + qz * qw); M[1][1] = 1 - 2 * (qx * qx + qz * qz); M[1][2] = 2 * (qy * qz - qx * qw);
    M[2][0] = 2 * (qx * qz - qy * qw); M[2][1] = 2 * (qy * qz + qx * qw); M[2][2] = 1 - 2 * (qx * qx + qy * qy);
    const double ga = 3.14159265358979323846264338327950288 * (3.0 - sqrt(5.0));
    for (int i = 0; i < N; i++) {
        double zi = 1.0 - (2.0 * i + 1.0) / N;
        double ri = 1.0 - zi * zi;
        ri = sqrt(ri > 0.0 ? ri : 0.0);
        double ph = ga * (double)i;
        double p0 = ri * cos(ph), p1 = ri * sin(ph), p2 = zi;
        double q[3];
        for (int r = 0; r < 3; r++) q[r] = M[r][0] * p0 + M[r][1] * p1 + M[r][2] * p2;
        double len = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
        for (int r = 0; r < 3; r++) xyz[3 * (size_t)i + r] = q[r] / len;
    }
    return 0;
}

/* orc_sph_heat: u(x, t) = sum_{l <= lmax, |m| <= l} c_lm exp(-kappa l(l+1) t) Y_lm(x)
 * with real orthonormal spherical harmonics, coefficients ordered (l, m = -l..l):
 * Y_l0 = P_l0(cos colat), Y_lm = sqrt 2 P_l|m|(cos colat) cos(m lon) for m > 0 and
 * sin(|m| lon) for m < 0, P the fully normalised associated Legendre functions
 * (Condon-Shortley phase) from the standard three-term recurrences.  The exact
 * solution of u_t = kappa * Laplace-Beltrami(u) on the unit sphere. */
int orc_sph_heat(int N, const double* xyz, int lmax, const double* coef, double kappa, double t, double* u)
{
    if (N < 0 || !xyz || !coef || !u || lmax < 0 || lmax > 200) return -1;
    const double PI = 3.14159265358979323846264338327950288;
    int L1 = lmax + 1;
    double* dec = (double*)malloc(sizeof(double) * L1);
    if (!dec) return -2;
    for (int l = 0; l <= lmax; l++) dec[l] = exp(-kappa * l * (l + 1.0) * t);
    int bad = 0;
#pragma omp parallel
    {
        double* P = (double*)malloc(sizeof(double) * L1 * L1);
        if (!P) {
#pragma omp atomic write
            bad = 1;
        }
#pragma omp for schedule(static)
        for (int i = 0; i < N; i++) {
            if (!P) continue;
            double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1], z = xyz[3 * (size_t)i + 2];
            double sc = sqrt(x * x + y * y), cc = z, lon = atan2(y, x);
            P[0] = sqrt(1.0 / (4.0 * PI));
            for (int m = 1; m <= lmax; m++)
                P[m * L1 + m] = -sqrt((2.0 * m + 1.0) / (2.0 * m)) * sc * P[(m - 1) * L1 + (m - 1)];
            for (int m = 0; m < lmax; m++) P[(m + 1) * L1 + m] = sqrt(2.0 * m + 3.0) * cc * P[m * L1 + m];
            for (int m = 0; m <= lmax; m++)
                for (int l = m + 2; l <= lmax; l++) {
                    double al = sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
                    double bl = sqrt(((l - 1.0) * (l - 1.0) - (double)m * m) / (4.0 * (l - 1.0) * (l - 1.0) - 1.0));
                    P[l * L1 + m] = al * (cc * P[(l - 1) * L1 + m] - bl * P[(l - 2) * L1 + m]);
                }
            double sum = 0.0;
            int k = 0;
            for (int l = 0; l <= lmax; l++) {
                double part = 0.0;
                for (int m = -l; m <= l; m++, k++) {
                    int am = m < 0 ? -m : m;
                    double y_lm = m == 0 ? P[l * L1] : sqrt(2.0) * P[l * L1 + am] * (m > 0 ? cos(am * lon) : sin(am * lon));
                    part += coef[k] * y_lm;
                }
                sum += dec[l] * part;
            }
            u[i] = sum;
        }
        free(P);
    }
    free(dec);
    return bad ? -2 : 0;
}
