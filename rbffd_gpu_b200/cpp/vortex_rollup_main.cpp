// Vortex roll-up on the sphere through the C++ classes of rbffd_cuda.hpp: the
// flow of the reference's experiment driver
// (tests/experiments/vortex_rollup_on_sphere/main.cpp:150-420) -- nodes,
// stencils, RBFFD weights for d/dlambda (+ hyperviscosity), an optional
// eigenvalue check of the operator with the time step it suggests
// (2 / max_neg_eig, main.cpp:379-394), VortexRollup, fillInitialConditions
// with the exact solution at START_TIME, advance(RK4, dt) per iteration with
// the local error printed every LOCAL_SOL_DUMP_FREQUENCY iterations, and the
// error against the exact solution at the end.
//
// Settings are KEY=VALUE arguments with the reference's test.conf names:
// GRID_SIZE, STENCIL_SIZE, EPSILON_C1, EPSILON_C2, HV_K, HV_GAMMA,
// USE_HYPERVISCOSITY, START_TIME, END_TIME, DT, MAX_NUM_ITERS,
// LOCAL_SOL_DUMP_FREQUENCY, MAX_LOCAL_REL_ERROR, USE_EIG_DT and
// DERIVATIVE_EIGENVALUE_TEST (eigenvalues of the operator; dt is lowered to
// the suggested step when USE_EIG_DT=1), STENCIL_GEN_TYPE (0 brute force,
// 1 k-d tree, 2 hash grid with NS_NB_X/Y/Z -- the driver's default,
// main.cpp:123-164), plus POLY_DEG, DTYPE (64 or 32), SEED and OUTPUT (file
// for the final solution, N doubles in node order).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "rbffd_cuda.hpp"

using namespace rbffd_sm100;

int main(int argc, char** argv)
{
    std::map<std::string, std::string> cfg;
    for (int a = 1; a < argc; a++) {
        const char* eq = std::strchr(argv[a], '=');
        if (!eq) {
            std::fprintf(stderr, "usage: %s KEY=VALUE ...\n", argv[0]);
            return 2;
        }
        cfg[std::string(argv[a], eq - argv[a])] = eq + 1;
    }
    auto num = [&](const char* k, double dflt) { return cfg.count(k) ? std::atof(cfg[k].c_str()) : dflt; };
    const int N = (int)num("GRID_SIZE", 10201);
    const int n = (int)num("STENCIL_SIZE", 50);
    const double start_time = num("START_TIME", 0.0), end_time = num("END_TIME", 3.0);
    double dt = num("DT", 0.05);
    const int max_num_iters = (int)num("MAX_NUM_ITERS", 10000);
    const int dump_every = std::max(1, (int)num("LOCAL_SOL_DUMP_FREQUENCY", 300000));
    const double max_local_rel_error = num("MAX_LOCAL_REL_ERROR", 1.0);
    const int dtype = num("DTYPE", 64) == 32 ? RBFFD_F32 : RBFFD_F64;

    // nodes: Fibonacci spiral under a seeded rotation; stencils from the
    // brute-force or k-d tree generator, or the hash grid (which renumbers
    // the nodes by cell), as Grid::generateStencils makes them
    std::vector<double> xyz(3 * (size_t)N);
    check(nullptr, rbffd_nodes_fibonacci(N, (uint64_t)num("SEED", 1), xyz.data()), "nodes");
    const int gen = (int)num("STENCIL_GEN_TYPE", 2);
    if (gen < 0 || gen > 2) {
        std::fprintf(stderr, "STENCIL_GEN_TYPE must be 0, 1 or 2\n");
        return 2;
    }
    std::vector<Vec3> nodes(N);
    for (int i = 0; i < N; i++) nodes[i] = Vec3{xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    std::vector<StencilType> stencils = generateStencils(nodes, n, (st_generator_t)gen, DBL_MAX, (int)num("NS_NB_X", 10),
                                                         (int)num("NS_NB_Y", 10), (int)num("NS_NB_Z", 10));
    for (int i = 0; i < N; i++) {
        xyz[3 * i] = nodes[i].x;
        xyz[3 * i + 1] = nodes[i].y;
        xyz[3 * i + 2] = nodes[i].z;
    }

    Context ctx(0);
    Grid_CUDA grid(ctx, nodes, stencils);
    const int useHV = (int)num("USE_HYPERVISCOSITY", 1);
    RBFFD_CUDA der(RBFFD_CUDA::LAMBDA, &grid, 2);
    der.setUseHyperviscosity(useHV);
    if (cfg.count("EPSILON_C1") || cfg.count("EPSILON_C2"))
        der.setEpsilonByParameters(num("EPSILON_C1", 0), num("EPSILON_C2", 0));
    else
        der.setEpsilonByStencilSize();
    der.setHVScalars((int)num("HV_K", 4), num("HV_GAMMA", 800));
    der.setPolynomialDegree((int)num("POLY_DEG", 0));
    der.computeAllWeightsForAllStencils();

    if (num("DERIVATIVE_EIGENVALUE_TEST", 0) != 0.0 || num("USE_EIG_DT", 0) != 0.0) {
        der.computeEigenvalues(RBFFD_CUDA::LAMBDA, false);
        const RBFFD_CUDA::EigenvalueOutput eigs = der.getEigenvalues();
        const double max_dt = 2. / eigs.max_neg_eig;
        std::printf("Suggested max_dt based on eigenvalues (1/lambda_max)= %f\n", max_dt);
        if (dt > max_dt) {
            std::printf("WARNING! your choice of timestep (%g) is TOO LARGE for to maintain stability of system. "
                        "According to eigenvalues, it must be less than %g\n", dt, max_dt);
            if (num("USE_EIG_DT", 0) != 0.0) dt = max_dt;
        }
    }
    std::printf("[MAIN] ********* USING TIMESTEP dt=%g ********** \n", dt);

    VortexRollup_CUDA pde(&grid, &der, useHV, dtype);
    pde.setStartEndTime(start_time, end_time);
    std::vector<double> h0(N);
    check(nullptr, rbffd_exact_vortex_rollup(N, xyz.data(), start_time, h0.data()), "exact solution");
    pde.fillInitialConditions(h0);

    const int num_iters = (int)((end_time - start_time) / dt);
    std::printf("NUM_ITERS = %d\n", num_iters);
    std::vector<double> exact(N);
    int iter;
    for (iter = 0; iter < num_iters && iter < max_num_iters; iter++) {
        if (!(iter % dump_every)) {
            std::printf("\n*********** Local Solution [ Iteration: %d (t = %g, dt = %g) ] *************\n", iter,
                        pde.getTime(), dt);
            check(nullptr, rbffd_exact_vortex_rollup(N, xyz.data(), pde.getTime(), exact.data()), "exact solution");
            pde.checkLocalError(exact, max_local_rel_error);
        }
        pde.advance(TimeDependentPDE_CUDA::RK4, dt);
    }
    check(nullptr, rbffd_exact_vortex_rollup(N, xyz.data(), pde.getTime(), exact.data()), "exact solution");
    std::printf("\n*********** Final Solution [ Iteration: %d (t = %g) ] *************\n", iter, pde.getTime());
    const std::vector<double> nrm = pde.checkLocalError(exact, max_local_rel_error);
    std::printf("rel L2 = %.6e, rel Linf = %.6e against the exact roll-up\n", nrm[3], nrm[5]);
    if (cfg.count("OUTPUT")) {
        const std::vector<double> h = pde.getLocalSolution();
        FILE* f = std::fopen(cfg["OUTPUT"].c_str(), "wb");
        if (!f || std::fwrite(h.data(), sizeof(double), N, f) != (size_t)N) {
            std::fprintf(stderr, "cannot write %s\n", cfg["OUTPUT"].c_str());
            return 1;
        }
        std::fclose(f);
    }
    return 0;
}
