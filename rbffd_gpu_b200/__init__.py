"""B200 (sm_100a) RBF-FD hot path: batched FP64 stencil weights, fused ELL
derivative / hyperviscosity application and RK4, behind the reference's
RBFFD / TimeDependentPDE interface (src/rbffd/rbffd.h, src/pdes/time_dependent_pde.h).

The compute lives in librbffd_sm100.so (CUDA C++ for sm_100a, C ABI in
include/rbffd_sm100.h); this package is a thin Python view of that ABI used
by the tests and the benchmark.  The C++ view for drop-in use is in
rbffd_gpu_b200/cpp/.
"""
from .api import (  # noqa: F401
    F32, F64, ARITH_FUSED, ARITH_UNFUSED, ELIM_AUTO, ELIM_UNBLOCKED, ELIM_BLOCKED, ELIM_ROW_MAP, ELIM_REGISTERS, X, Y, Z, LAPL, R, HV, LAMBDA, THETA, LSFC, XSFC, YSFC, ZSFC, INTERP, ALT_XSFC, ALT_YSFC, ALT_ZSFC, RK4,
    RbffdError, Context, Grid, RBFFD, TimeDependentPDE, CosineBell, HeatSphere, Advection, VortexRollup,
    vortex_rollup_coefficients, exact_vortex_rollup, sol_norms,
    fibonacci_nodes, knn_stencils, knn_stencils_gpu, generate_stencils, generate_stencils_gpu, variable_epsilon, ST_BRUTE_FORCE, ST_KDTREE, ST_HASH,
    write_weights_file, read_weights_file, exact_cosine_bell,
    exact_sph_heat, device_count, version, eig_classify, hessenberg_eigenvalues, node_order, stencils_hash, ORDER_MORTON, ORDER_RCM, ORDER_GIVEN,
    Server, heat_params, cosine_bell_params, ERR_OOM, ERR_TIMEOUT, ERR_BUDGET, ERR_CANCELLED,
)
