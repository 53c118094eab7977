// Test infrastructure: exposes the reference's own Gaussian RBF
// (src/rbffd/rbfs/rbf_gaussian.h) and cart2sph (src/utils/geom/cart2sph.cpp)
// through C functions, so tests can pin the oracle's restatement of them.
// Built from the reference sources in place by oracle/build.py.
#include "rbfs/rbf_gaussian.h"
#include "utils/geom/cart2sph.h"

extern "C" double ref_rbf(int which, double eps, int dim, double dx, double dy, double dz, int hv_k)
{
    RBF_Gaussian r(eps, dim);
    Vec3 d(dx, dy, dz);
    switch (which) {
    case 0: return r.eval(d);
    case 1: return r.xderiv(d);
    case 2: return r.yderiv(d);
    case 3: return r.zderiv(d);
    case 4: return r.rderiv(d);
    case 5: return r.rderiv_over_r(d);
    case 6: return r.rderiv2(d);
    case 7: return r.lapl_deriv(d);
    case 8: return r.hyperviscosity(d, hv_k);
    }
    return 0.0 / 0.0;
}

extern "C" void ref_cart2sph(double x, double y, double z, double* theta, double* phi, double* r)
{
    sph_coords_type s = cart2sph(x, y, z);
    *theta = s.theta;
    *phi = s.phi;
    *r = s.r;
}
