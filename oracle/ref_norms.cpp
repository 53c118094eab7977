// Test infrastructure: the reference's own norm routines
// (src/utils/norms.cpp) with PDE::calcSolNorms' relative-norm rule
// (src/pdes/pde.cpp:467-480) through a C function.  Built from the reference
// sources in place by oracle/build.py into oracle/_ref/.
#include <cfloat>
#include <cmath>
#include <vector>

#include "norms.h"

extern "C" void ref_sol_norms(const double* sol, const double* exact, int n, double* out)
{
    std::vector<double> v(sol, sol + n), e(exact, exact + n);
    const double l1fabs = l1norm(v, e, 0, n), l1denom = l1norm(e, 0, n);
    const double l2fabs = l2norm(v, e, 0, n), l2denom = l2norm(e, 0, n);
    const double lifabs = linfnorm(v, e, 0, n), lidenom = linfnorm(e, 0, n);
    out[0] = l1fabs;
    out[1] = (l1denom > 1e-10) ? l1fabs / l1denom : (l1fabs + 1.) / (l1denom + 1.);
    out[2] = l2fabs;
    out[3] = (l2denom > 1e-10) ? l2fabs / l2denom : (l2fabs + 1.) / (l2denom + 1.);
    out[4] = lifabs;
    out[5] = (lidenom > 1e-10) ? lifabs / lidenom : (lifabs + 1.) / (lidenom + 1.);
}
