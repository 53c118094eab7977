// Test infrastructure: exposes the reference's own hash-grid stencil generator
// (Grid::generateStencilsHash, src/grids/grid_interface.cpp:733-966) through a
// C function, so tests can compare node orders and stencils with it.  Built
// from the reference sources in place by oracle/build.py into oracle/_ref/.
// The grid's extents are set as GridReader sets them (refreshExtents from the
// default box, src/grids/grid_reader.cpp:123) unless given.
#include <ctime>
#include <cstdio>
#include <iostream>
#include <sstream>

#include "grid_interface.h"

namespace {
class HashGrid : public Grid {
public:
    explicit HashGrid(std::vector<NodeType>& nodes) : Grid(nodes) {}
    void setRadius(double r) { max_st_radius = r; }
};
}  // namespace

extern "C" int ref_stencils_hash(const double* xyz, int N, int n, int nbx, int nby, int nbz, const double* extents,
                                 double max_radius, double* xyz_sorted, int* st, int* st_len)
{
    std::streambuf* old = std::cout.rdbuf();  // the grid prints progress
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    std::vector<NodeType> nodes(N);
    for (int i = 0; i < N; i++) nodes[i] = NodeType(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    HashGrid g(nodes);
    if (extents) g.setExtents(extents[0], extents[1], extents[2], extents[3], extents[4], extents[5]);
    else g.refreshExtents();
    g.setMaxStencilSize(n);
    g.setRadius(max_radius);
    g.setNSHashDims(nbx, nby, nbz);
    g.generateStencils(Grid::ST_HASH);
    std::cout.rdbuf(old);
    std::vector<NodeType>& nl = g.getNodeList();
    for (int i = 0; i < N; i++) {
        xyz_sorted[3 * i] = nl[i].x();
        xyz_sorted[3 * i + 1] = nl[i].y();
        xyz_sorted[3 * i + 2] = nl[i].z();
        StencilType& s = g.getStencil(i);
        st_len[i] = (int)s.size();
        for (int j = 0; j < n; j++) st[(size_t)i * n + j] = j < (int)s.size() ? (int)s[j] : -1;
    }
    return 0;
}

// The reference's own Grid::generateStencilsBruteForce (method 0,
// grid_interface.cpp:637-686) and Grid::generateStencilsKDTree (method 1,
// grid_interface.cpp:688-725), both trimming at max_st_radius; the grid keeps
// the caller's numbering.  st[N][n] padded with -1.
extern "C" int ref_stencils_generate(const double* xyz, int N, int n, int method, double max_radius, int* st,
                                     int* st_len)
{
    std::streambuf* old = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    std::vector<NodeType> nodes(N);
    for (int i = 0; i < N; i++) nodes[i] = NodeType(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    HashGrid g(nodes);
    g.refreshExtents();
    g.setMaxStencilSize(n);
    g.setRadius(max_radius);
    g.generateStencils(method == 0 ? Grid::ST_BRUTE_FORCE : Grid::ST_KDTREE);
    std::cout.rdbuf(old);
    for (int i = 0; i < N; i++) {
        StencilType& s = g.getStencil(i);
        st_len[i] = (int)s.size();
        for (int j = 0; j < n; j++) st[(size_t)i * n + j] = j < (int)s.size() ? (int)s[j] : -1;
    }
    return 0;
}
