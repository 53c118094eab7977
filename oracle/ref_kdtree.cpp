// Test infrastructure: exposes the reference's own k-d tree
// (external/kdtree/KDTree.h, used by Grid::generateStencilsKDTree,
// src/grids/grid_interface.cpp:688-725) through a C function, so tests can
// compare stencil index lists with it.  Built from the reference sources in
// place by oracle/build.py into oracle/_ref/.
#include <ctime>
#include <cstdio>
#include <iostream>
#include <sstream>
#include "KDTree.h"

extern "C" int ref_knn(const double* xyz, int N, int k, int* idx_out, double* dist_out)
{
    // KDTree prints progress to std::cout; keep the test output clean.
    std::streambuf* old = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    KDTree tree(xyz, N, 3);
    std::cout.rdbuf(old);
    for (int i = 0; i < N; i++) {
        std::vector<int> ids;
        std::vector<double> d;
        tree.k_closest_points(Vec3(xyz + 3 * (size_t)i), k, ids, d);
        if ((int)ids.size() != k) return -1;
        for (int j = 0; j < k; j++) {
            idx_out[(size_t)i * k + j] = ids[j];
            dist_out[(size_t)i * k + j] = d[j];
        }
    }
    return 0;
}
