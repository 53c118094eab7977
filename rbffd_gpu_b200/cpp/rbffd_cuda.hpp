// C++ view of librbffd_sm100.so shaped like the reference's classes, for
// drivers written against them.
//
//   RBFFD_CUDA            class RBFFD (src/rbffd/rbffd.h:29-547): DerType flags,
//                         parameter setters, computeAllWeightsForAllStencils,
//                         both applyWeightsForDeriv overloads, getStencilWeights
//   TimeDependentPDE_CUDA class TimeDependentPDE (src/pdes/time_dependent_pde.h:9-126):
//                         TimeScheme, fillInitialConditions, advance(which, dt),
//                         getTime / setTime, getLocalSolution (pde.h:161)
//   CosineBell_CUDA       class CosineBell (src/pdes/hyperbolic/cosine_bell.h:31-46)
//   HeatSphere_CUDA       heat on the sphere, u_t = kappa * LSFC u
//   Advection_CUDA        advection with caller-given per-node coefficients
//   Server_CUDA           the serving loop (rbffd_server_*)
//
// The reference's GPU classes (RBFFD_CL, TimeDependentPDE_CL) subclass the CPU
// ones and override applyWeightsForDeriv / advance; these classes carry the
// same signatures over opaque handles so a driver swaps the type and keeps its
// calls.  Grid_CUDA stands in for the reference's Grid (node list and stencil
// map; getNodeList, getStencils, getStencilsSize, getMaxStencilSize).
//
// Errors: the reference prints and exits (e.g. rbffd.cpp:221,500).  These
// classes do the same at the call that failed, unless RBFFD_CUDA_THROW is
// defined, in which case they throw rbffd_sm100::Error.
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/rbffd_sm100.h"

namespace rbffd_sm100 {

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(rbffd_ctx* ctx, int rc, const char* what)
{
    if (rc == RBFFD_OK) return;
    std::string msg = std::string(what) + ": " + rbffd_status_string(rc);
    if (ctx) msg += std::string(" (") + rbffd_ctx_last_error(ctx) + ")";
#ifdef RBFFD_CUDA_THROW
    throw Error(rc, msg);
#else
    std::fprintf(stderr, "[RBFFD_CUDA] Error: %s\n", msg.c_str());
    std::exit(EXIT_FAILURE);
#endif
}

struct Vec3 {
    double x, y, z;
};

// One device; owns every device buffer created from it.
class Context {
public:
    explicit Context(int device = 0) { check(nullptr, rbffd_ctx_create(device, &h_), "rbffd_ctx_create"); }
    ~Context() { rbffd_ctx_destroy(h_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    rbffd_ctx* handle() const { return h_; }
    void synchronize() { check(h_, rbffd_ctx_synchronize(h_), "rbffd_ctx_synchronize"); }

private:
    rbffd_ctx* h_ = nullptr;
};

typedef std::vector<int> StencilType;  // src/common_typedefs.h:16

// Nodes and stencils resident on the device.
// Grid::generateStencils(st_max_size, st_generator_t) (grid_interface.h:37,
// 166-167): stencils of max_st_size nodes for a node list, with the
// reference's max_st_radius (DBL_MAX: none).  ST_HASH renumbers the nodes by
// cell, as the reference's hash generator re-sorts its grid: the node list is
// replaced by the renumbered one.
enum st_generator_t { ST_BRUTE_FORCE = 0, ST_KDTREE = 1, ST_HASH = 2 };
inline std::vector<StencilType> generateStencils(std::vector<Vec3>& nodes, unsigned max_st_size,
                                                 st_generator_t generator = ST_BRUTE_FORCE,
                                                 double max_st_radius = DBL_MAX, int ns_nx = 10, int ns_ny = 10,
                                                 int ns_nz = 10)
{
    const int N = (int)nodes.size(), n = (int)max_st_size;
    std::vector<double> xyz(3 * (size_t)N);
    for (int i = 0; i < N; i++) {
        xyz[3 * (size_t)i] = nodes[i].x;
        xyz[3 * (size_t)i + 1] = nodes[i].y;
        xyz[3 * (size_t)i + 2] = nodes[i].z;
    }
    std::vector<int> st((size_t)N * n), len(N);
    if (generator == ST_HASH) {
        std::vector<int> order(N);
        check(nullptr,
              rbffd_stencils_hash(xyz.data(), N, n, ns_nx, ns_ny, ns_nz, nullptr, max_st_radius, order.data(),
                                  st.data(), len.data()),
              "generateStencils");
        std::vector<Vec3> renumbered(N);
        for (int k = 0; k < N; k++) renumbered[k] = nodes[order[k]];
        nodes.swap(renumbered);
    } else {
        check(nullptr,
              rbffd_stencils_generate(xyz.data(), N, n,
                                      generator == ST_KDTREE ? RBFFD_ST_KDTREE : RBFFD_ST_BRUTE_FORCE, max_st_radius,
                                      st.data(), len.data(), nullptr, 0),
              "generateStencils");
    }
    std::vector<StencilType> out(N);
    for (int i = 0; i < N; i++) out[i].assign(st.begin() + (size_t)i * n, st.begin() + (size_t)i * n + len[i]);
    return out;
}

class Grid_CUDA {
public:
    Grid_CUDA(Context& ctx, const std::vector<Vec3>& nodes, const std::vector<StencilType>& stencils,
              unsigned global_nodes = 0)
        : ctx_(ctx), nodes_(nodes), stencils_(stencils), global_(global_nodes ? global_nodes : (unsigned)nodes.size())
    {
        const int N = (int)nodes.size();
        for (const StencilType& s : stencils) n_pad_ = std::max(n_pad_, (int)s.size());
        std::vector<double>& xyz = xyz_;
        xyz.resize(3 * (size_t)N);
        for (int i = 0; i < N; i++) {
            xyz[3 * i] = nodes[i].x;
            xyz[3 * i + 1] = nodes[i].y;
            xyz[3 * i + 2] = nodes[i].z;
        }
        st_.assign((size_t)N * n_pad_, 0);
        len_.assign(N, 0);
        for (int i = 0; i < N; i++) {
            len_[i] = (int)stencils[i].size();
            for (int s = 0; s < len_[i]; s++) st_[(size_t)i * n_pad_ + s] = stencils[i][s];
            for (int s = len_[i]; s < n_pad_; s++) st_[(size_t)i * n_pad_ + s] = i;
        }
        check(ctx.handle(), rbffd_grid_create(ctx.handle(), N, xyz.data(), n_pad_, st_.data(), len_.data(), &h_),
              "rbffd_grid_create");
    }
    ~Grid_CUDA() { rbffd_grid_destroy(h_); }
    Grid_CUDA(const Grid_CUDA&) = delete;
    Grid_CUDA& operator=(const Grid_CUDA&) = delete;

    std::vector<Vec3>& getNodeList() { return nodes_; }
    std::vector<StencilType>& getStencils() { return stencils_; }
    unsigned getStencilsSize() const { return (unsigned)stencils_.size(); }
    unsigned getNodeListSize() const { return (unsigned)nodes_.size(); }
    unsigned getGlobalNodeListSize() const { return global_; }
    unsigned getMaxStencilSize() const { return (unsigned)n_pad_; }
    rbffd_grid* handle() const { return h_; }
    Context& context() const { return ctx_; }
    // stencils as [N][getMaxStencilSize()] (padding = centre) and their lengths
    const std::vector<int>& paddedStencils() const { return st_; }
    const std::vector<int>& stencilLengths() const { return len_; }
    // node coordinates as [N][3]
    const std::vector<double>& coordinates() const { return xyz_; }

private:
    Context& ctx_;
    std::vector<Vec3> nodes_;
    std::vector<StencilType> stencils_;
    std::vector<int> st_, len_;
    std::vector<double> xyz_;
    unsigned global_;
    int n_pad_ = 1;
    rbffd_grid* h_ = nullptr;
};

class RBFFD_CUDA {
public:
    // identical values to RBFFD::DerType (rbffd.h:43-60)
    enum DerType {
        X = RBFFD_X, Y = RBFFD_Y, Z = RBFFD_Z, LAPL = RBFFD_LAPL, R = RBFFD_R, HV = RBFFD_HV,
        LAMBDA = RBFFD_LAMBDA, THETA = RBFFD_THETA, LSFC = RBFFD_LSFC, XSFC = RBFFD_XSFC, YSFC = RBFFD_YSFC,
        ZSFC = RBFFD_ZSFC, ALT_XSFC = RBFFD_ALT_XSFC, ALT_YSFC = RBFFD_ALT_YSFC, ALT_ZSFC = RBFFD_ALT_ZSFC,
        INTERP = RBFFD_INTERP
    };
    typedef unsigned int DerTypes;
    enum DataType { FP32 = RBFFD_F32, FP64 = RBFFD_F64 };
    // RBFFD::WeightType (rbffd.h:89): the direct solve is the one implemented
    enum WeightType { Direct = 0, ContourSVD = 1 };
    // derTypeStr of rbffd.cpp:40-58, by DerType bit
    static const char* derTypeStr(DerType which)
    {
        static const char* names[16] = {"x",    "y",        "z",        "lapl",     "r",        "hv",
                                        "lambda", "theta",  "Lsfc",     "Xsfc",     "Ysfc",     "Zsfc",
                                        "Alt_Xsfc", "Alt_Ysfc", "Alt_Zsfc", "interp"};
        for (int b = 0; b < 16; b++)
            if ((unsigned)which == (1u << b)) return names[b];
        return "unknown";
    }

    // RBFFD(DerTypes typesToCompute, Grid* grid, int dim_num, int rank=0) (rbffd.h:192)
    RBFFD_CUDA(DerTypes typesToCompute, Grid_CUDA* grid, int dim_num, int rank = 0)
        : computedTypes(typesToCompute), grid_ref(*grid), dim_num(dim_num), rank(rank),
          var_epsilon(grid->getStencilsSize(), 1.0)
    {
    }
    virtual ~RBFFD_CUDA() {}

    // -- parameters (rbffd.h:213-381) --
    void setUseHyperviscosity(int tf)
    {
        useHyperviscosity = tf;
        if (tf) computedTypes |= HV;
        else computedTypes &= ~(DerTypes)HV;
    }
    int getUseHyperviscosity() { return useHyperviscosity; }
    double getHVScalar() { return -hv_gamma * std::pow((double)grid_ref.getGlobalNodeListSize(), -(double)hv_k); }
    double setHVScalars(int k, double gamma_c)
    {
        hv_k = k;
        hv_gamma = gamma_c;
        return hv_gamma;
    }
    void appendDerTypes(DerTypes t) { computedTypes |= t; }
    void setEpsilon(double eps) { var_epsilon.assign(var_epsilon.size(), eps); }
    void setEpsilon(std::vector<double>& lst_of_epsilon)
    {
        if (lst_of_epsilon.size() != var_epsilon.size())
            check(grid_ref.context().handle(), RBFFD_ERR_INVALID, "setEpsilon: length of the list does not match");
        var_epsilon = lst_of_epsilon;
    }
    void setEpsilonByParameters(double c1, double c2)
    {
        setEpsilon(c1 * std::sqrt((double)grid_ref.getGlobalNodeListSize()) - c2);
    }
    // the reference's per-stencil-size table for the cosine bell (rbffd.h:300-345)
    // rbffd.h:376-380, rbffd.cpp:1378-1420 (Sarler 2006): eps at each centre =
    // 1 / (alpha * distance to the stencil's last node); beta unused there too
    void setVariableEpsilon(double alpha = 1.0, double beta = 1.0)
    {
        (void)beta;
        check(nullptr,
              rbffd_variable_epsilon((int)grid_ref.getStencilsSize(), grid_ref.coordinates().data(),
                                     (int)grid_ref.getMaxStencilSize(), grid_ref.paddedStencils().data(),
                                     grid_ref.stencilLengths().data(), alpha, var_epsilon.data()),
              "setVariableEpsilon");
    }
    void setEpsilonByStencilSize()
    {
        double c1, c2;
        switch (grid_ref.getMaxStencilSize()) {
        case 17: c1 = 0.026, c2 = 0.08, hv_k = 2, hv_gamma = 8e-4; break;
        case 31: c1 = 0.035, c2 = 0.1, hv_k = 4, hv_gamma = 5e-2; break;
        case 50: c1 = 0.044, c2 = 0.14, hv_k = 6, hv_gamma = 5e-1; break;
        case 101: c1 = 0.058, c2 = 0.16, hv_k = 8, hv_gamma = 5e-2; break;
        default:
            check(grid_ref.context().handle(), RBFFD_ERR_UNSUPPORTED,
                  "setEpsilonByStencilSize supports stencil sizes 17, 31, 50 and 101");
            return;
        }
        setEpsilonByParameters(c1, c2);
    }
    // Beyond the reference (which fixes one constant monomial): -1 none, 0
    // constant, 1 {1,x,y,z}, 2..4 tangent-plane polynomials; optional per row.
    void setPolynomialDegree(int deg, const std::vector<int>* deg_per_row = nullptr)
    {
        poly_deg = deg;
        deg_rows = deg_per_row ? *deg_per_row : std::vector<int>();
    }

    // -- weights --
    // rbffd.h:507-522: any ALT_*SFC type brings X, Y, Z and all three ALT types
    bool adjustForSFCTypes()
    {
        const DerTypes alt = ALT_XSFC | ALT_YSFC | ALT_ZSFC;
        if (!(computedTypes & alt)) return false;
        computedTypes |= X | Y | Z | alt;
        return true;
    }
    // rbffd.h:247-253.  Condition numbers are not computed on the device; the
    // flag is kept so reference drivers run unchanged.
    void setComputeConditionNumber(bool tf) { computeCondNums = tf; }
    bool getComputeConditionNumber() const { return computeCondNums; }
    void setWeightType(WeightType type) { weightMethod = type; }
    void computeAllWeightsForAllStencils()
    {
        if (weightMethod != Direct)
            check(nullptr, RBFFD_ERR_UNSUPPORTED,
                  "computeAllWeightsForAllStencils: ContourSVD weights are not built (WeightType Direct only)");
        adjustForSFCTypes();
        rbffd_weight_params p;
        p.der_types = computedTypes;
        p.dim = dim_num;
        p.poly_deg = poly_deg;
        p.hv_k = hv_k;
        p.hv_gamma = hv_gamma;
        p.hv_nodes = (double)grid_ref.getGlobalNodeListSize();
        check(grid_ref.context().handle(),
              rbffd_weights_compute(grid_ref.handle(), &p, var_epsilon.data(), 0.0,
                                    deg_rows.empty() ? nullptr : deg_rows.data()),
              "computeAllWeightsForAllStencils");
    }
    // weights of one operator computed elsewhere (e.g. the reference's CPU path), [N][n_pad]
    void setWeights(DerType which, const std::vector<double>& w)
    {
        check(grid_ref.context().handle(), rbffd_weights_set(grid_ref.handle(), which, w.data()), "setWeights");
    }
    std::vector<double> getWeights(DerType which)
    {
        std::vector<double> w((size_t)grid_ref.getStencilsSize() * grid_ref.getMaxStencilSize());
        check(grid_ref.context().handle(), rbffd_weights_get(grid_ref.handle(), which, w.data()), "getWeights");
        return w;
    }
    // one stencil's weights (a host copy; rbffd.h:395 returns the reference's own array)
    std::vector<double> getStencilWeights(DerType which, int st_indx)
    {
        std::vector<double> all = getWeights(which);
        const size_t n = grid_ref.getMaxStencilSize();
        return std::vector<double>(all.begin() + st_indx * n, all.begin() + (st_indx + 1) * n);
    }

    // -- weight files (rbffd.h:400-410): the reference's Matrix Market forms --
    void setAsciiWeights(int binary_or_ascii) { asciiWeights = binary_or_ascii; }
    void writeToFile(DerType which, const std::string& filename)
    {
        std::vector<double> w = getWeights(which);
        check(grid_ref.context().handle(),
              rbffd_weights_file_write(filename.c_str(), asciiWeights ? 0 : 1, (int)grid_ref.getStencilsSize(),
                                       (int)grid_ref.getMaxStencilSize(), grid_ref.paddedStencils().data(),
                                       grid_ref.stencilLengths().data(), w.data()),
              "writeToFile");
    }
    // returns 0 (the reference's loadFromFile returns nonzero codes on failure)
    int loadFromFile(DerType which, const std::string& filename)
    {
        std::vector<double> w((size_t)grid_ref.getStencilsSize() * grid_ref.getMaxStencilSize());
        check(grid_ref.context().handle(),
              rbffd_weights_file_read(filename.c_str(), asciiWeights ? 0 : 1, (int)grid_ref.getStencilsSize(),
                                      (int)grid_ref.getMaxStencilSize(), grid_ref.paddedStencils().data(),
                                      grid_ref.stencilLengths().data(), w.data()),
              "loadFromFile");
        setWeights(which, w);
        return 0;
    }
    // RBFFD::writeAllWeightsToFile / loadAllWeightsFromFile (rbffd.cpp:1212-1250):
    // every computed type, one file each named base_<derTypeStr>.mtx (ASCII)
    // or .bmtx (binary).  The reference derives base from its grid and
    // parameters (getFileDetailString); here the caller names it.  load
    // returns the number of types whose file could not be read, as the
    // reference sums loadFromFile's error codes, and keeps the weights it
    // could read.
    std::string getFilename(DerType which, const std::string& base = "weights_rbffd") const
    {
        return base + "_" + derTypeStr(which) + (asciiWeights ? ".mtx" : ".bmtx");
    }
    void writeAllWeightsToFile(const std::string& base = "weights_rbffd")
    {
        for (int b = 0; b < 16; b++)
            if (computedTypes & (1u << b)) writeToFile((DerType)(1u << b), getFilename((DerType)(1u << b), base));
    }
    int loadAllWeightsFromFile(const std::string& base = "weights_rbffd")
    {
        int err = 0;
        for (int b = 0; b < 16; b++) {
            if (!(computedTypes & (1u << b))) continue;
            const DerType t = (DerType)(1u << b);
            std::vector<double> w((size_t)grid_ref.getStencilsSize() * grid_ref.getMaxStencilSize());
            const int rc = rbffd_weights_file_read(getFilename(t, base).c_str(), asciiWeights ? 0 : 1,
                                                   (int)grid_ref.getStencilsSize(), (int)grid_ref.getMaxStencilSize(),
                                                   grid_ref.paddedStencils().data(), grid_ref.stencilLengths().data(),
                                                   w.data());
            if (rc) {
                err += 1;
                continue;
            }
            setWeights(t, w);
        }
        return err;
    }

    // -- eigenvalue stability check (rbffd.h:91-100,281,412-417; rbffd.cpp:703-873) --
    typedef rbffd_eig_output EigenvalueOutput;
    // Every eigenvalue of the operator (+ HV when hyperviscosity is on) on the
    // device; counts and extremes as the reference prints them, the eigenvalues
    // written "%+lf%+lfi" one per line to eigenvalue_file when one is named.
    // Returns max |Re| among the negative eigenvalues.  Like the reference, a
    // mix of signs or more than one zero eigenvalue is an error that exits when
    // exit_on_fail.
    double computeEigenvalues(DerType which, bool exit_on_fail, EigenvalueOutput* output = nullptr,
                              const char* eigenvalue_file = nullptr)
    {
        const int N = (int)grid_ref.getStencilsSize();
        std::vector<double> re(N), im(N);
        EigenvalueOutput o;
        double ret = 0.0;
        check(grid_ref.context().handle(),
              rbffd_eigenvalues(grid_ref.handle(), which, useHyperviscosity, re.data(), im.data(), &o, &ret),
              "computeEigenvalues");
        if (eigenvalue_file) {
            FILE* f = std::fopen(eigenvalue_file, "w");
            if (f) {
                for (int i = 0; i < N; i++) std::fprintf(f, "%+lf%+lfi\n", re[i], im[i]);
                std::fclose(f);
            }
        }
        std::printf("\n[RBFFD] ****** Number positive eigenvalues: %d (nb_bnd: 0) *******\n\n", o.nb_positive);
        std::printf("\n[RBFFD] ****** Number negative eigenvalues: %d *******\n\n", o.nb_negative);
        std::printf("\n[RBFFD] ****** Number zero (-1e-8 <= eval <= 1e-8) eigenvalues: %d *******\n\n", o.nb_zero);
        if (output) *output = o;
        cachedEigenvalues = o;
        eigenvalues_computed = true;
        const bool mixed = o.nb_negative > 0 && o.nb_positive > 0, zeros = o.nb_zero > 1;
        if (mixed || zeros) {
            std::printf("[RBFFD] Error: %s\n", mixed ? "we expect either all positive or all negative eigenvalues."
                                                     : "more than one eigenvalue is zero.");
            if (exit_on_fail) {
#ifdef RBFFD_CUDA_THROW
                throw Error(RBFFD_ERR_INVALID, "computeEigenvalues: unstable operator");
#else
                std::exit(EXIT_FAILURE);
#endif
            }
        }
        return ret;
    }
    EigenvalueOutput getEigenvalues()
    {
        if (!eigenvalues_computed) computeEigenvalues(LAPL, false);
        return cachedEigenvalues;
    }

    // -- apply (rbffd.h:257-274) --
    virtual void applyWeightsForDeriv(DerType which, std::vector<double>& u, std::vector<double>& deriv,
                                      bool isChangedU = true)
    {
        const unsigned nb_stencils = grid_ref.getStencilsSize();
        if (deriv.size() < nb_stencils) deriv.resize(nb_stencils);
        applyWeightsForDeriv(which, 0, nb_stencils, u.data(), deriv.data(), isChangedU);
    }
    virtual void applyWeightsForDeriv(DerType which, unsigned start_indx, unsigned nb_stencils, double* u,
                                      double* deriv, bool isChangedU = true)
    {
        (void)isChangedU;  // u is always copied: the device holds no stale copy
        check(grid_ref.context().handle(),
              rbffd_apply(grid_ref.handle(), which, dtype, start_indx, nb_stencils, u, deriv),
              "applyWeightsForDeriv");
    }
    // arithmetic of applyWeightsForDeriv (FP64 default; FP32 as RBFFD_CL's single-precision path)
    void setDataType(DataType t) { dtype = t; }

    DerTypes getComputedTypes() const { return computedTypes; }
    Grid_CUDA& grid() { return grid_ref; }

protected:
    DerTypes computedTypes;
    Grid_CUDA& grid_ref;
    int dim_num, rank;
    int hv_k = 2;            // ctor defaults (rbffd.cpp:26)
    double hv_gamma = 8e-4;
    int useHyperviscosity = 0;
    std::vector<double> var_epsilon;
    int poly_deg = 0;
    std::vector<int> deg_rows;
    int dtype = RBFFD_F64;
    int asciiWeights = 0;  // binary weight files unless setAsciiWeights(1)
    bool computeCondNums = false;
    WeightType weightMethod = Direct;
    EigenvalueOutput cachedEigenvalues = {};
    bool eigenvalues_computed = false;
};

class TimeDependentPDE_CUDA {
public:
    enum TimeScheme { EULER = 0, MIDPOINT, RK4 };  // time_dependent_pde.h:20

    virtual ~TimeDependentPDE_CUDA() { rbffd_pde_destroy(h_); }
    TimeDependentPDE_CUDA(const TimeDependentPDE_CUDA&) = delete;
    TimeDependentPDE_CUDA& operator=(const TimeDependentPDE_CUDA&) = delete;

    // the initial state, [N] (one tracer) or [N][T]
    virtual void fillInitialConditions(const std::vector<double>& u)
    {
        check(ctx(), rbffd_pde_set_state(h_, u.data()), "fillInitialConditions");
    }
    // advance(TimeScheme which, double delta_t) (time_dependent_pde.h:42): one step
    virtual void advance(TimeScheme which, double delta_t) { advance(which, delta_t, 1); }
    // nsteps steps in one call (captured in a CUDA graph when use_graph)
    void advance(TimeScheme which, double delta_t, int nsteps, bool use_graph = false)
    {
        check(ctx(), rbffd_pde_advance(h_, (int)which, delta_t, nsteps, use_graph ? RBFFD_ADVANCE_GRAPH : 0),
              "advance");
    }
    std::vector<double> getLocalSolution()
    {
        std::vector<double> u((size_t)grid_.getNodeListSize() * T_);
        check(ctx(), rbffd_pde_get_state(h_, u.data()), "getLocalSolution");
        return u;
    }
    void setTime(double t) { check(ctx(), rbffd_pde_set_time(h_, t), "setTime"); }
    // FP32 PDEs: carry each step's rounding of u + increment into the next (rbffd_pde_set_compensated_state)
    void setCompensatedState(bool on) { check(ctx(), rbffd_pde_set_compensated_state(h_, on ? 1 : 0), "setCompensatedState"); }
    // PDE::checkLocalError (pde.h:120-127): the solution's error norms against
    // exact values, printed as the reference prints them (no boundary nodes on
    // the sphere); a high error is reported, never fatal.  Returns the norms
    // rbffd_sol_norms gives: l1, l1 rel, l2, l2 rel, linf, linf rel.
    std::vector<double> checkLocalError(const std::vector<double>& exact, double rel_err_max = -1.)
    {
        std::vector<double> u = getLocalSolution(), nrm(6), none(6);
        check(nullptr, rbffd_sol_norms(u.data(), exact.data(), (int)u.size(), nrm.data()), "checkLocalError");
        check(nullptr, rbffd_sol_norms(nullptr, nullptr, 0, none.data()), "checkLocalError");
        const char* labels[4] = {"Boundary", "Interior Stencils w/o Boundary", "All Interior", "Interior & Boundary"};
        const char* p[3] = {"l1", "l2", "linf"};
        for (int g = 0; g < 4; g++)
            for (int k = 0; k < 3; k++) {
                const std::vector<double>& v = g == 0 ? none : nrm;
                std::printf("%s %s error (%d nodes):   Absolute = %le,    Relative = %le \n", labels[g], p[k],
                            g == 0 ? 0 : (int)u.size(), v[2 * k], v[2 * k + 1]);
            }
        if (rel_err_max > 0 && nrm[3] > rel_err_max)
            std::printf("[PDE] Error! l2 relative error (=%f%%) is too high to continue. We require %f%% or less.\n",
                        100. * nrm[3], 100. * rel_err_max);
        return nrm;
    }
    // PDE::checkGlobalError (pde.h:130-147): on one rank, checkLocalError
    std::vector<double> checkGlobalError(const std::vector<double>& exact, Grid_CUDA* global_grid = nullptr,
                                         double rel_err_max = -1., bool ignore_sol_error = true)
    {
        (void)global_grid;
        (void)ignore_sol_error;
        return checkLocalError(exact, rel_err_max);
    }
    // pde.h:161: one node's value
    double getLocalSolution(unsigned indx) { return getLocalSolution()[indx]; }
    // PDE::syncCPUtoGPU (pde.h:166): the device holds the state and every read copies it
    void syncCPUtoGPU() {}
    // TimeDependentPDE::setStartEndTime (time_dependent_pde.h:52-56)
    void setStartEndTime(double start, double end)
    {
        start_time_ = start;
        end_time_ = end;
        setTime(start);
    }
    double getTime()
    {
        double t = 0.0;
        check(ctx(), rbffd_pde_get_time(h_, &t), "getTime");
        return t;
    }
    rbffd_pde* handle() const { return h_; }

protected:
    TimeDependentPDE_CUDA(Grid_CUDA* grid, RBFFD_CUDA* der, const rbffd_pde_params& p) : grid_(*grid), T_(p.ntracers)
    {
        (void)der;  // the operators' weights live on the grid
        check(grid->context().handle(), rbffd_pde_create(grid->handle(), &p, &h_), "TimeDependentPDE");
    }
    rbffd_ctx* ctx() const { return grid_.context().handle(); }
    Grid_CUDA& grid_;
    int T_;
    rbffd_pde* h_ = nullptr;
    double start_time_ = 0., end_time_ = 0.;
};

inline rbffd_pde_params pde_params(int kind, int dtype, int ntracers)
{
    rbffd_pde_params p;
    p.rhs_kind = kind;
    p.ntracers = ntracers;
    p.dtype = dtype;
    p.use_hv = 0;
    p.sphere_radius = 1.0;
    p.alpha = 0.0;
    p.u0 = 0.0;
    p.kappa = 1.0;
    p.cu = p.cv = nullptr;
    return p;
}

// CosineBell(Domain*, RBFFD*, Communicator*, earth_radius, velocity_angle,
//            one_revolution_in_seconds, useHyperviscosity) (cosine_bell.h:36)
class CosineBell_CUDA : public TimeDependentPDE_CUDA {
public:
    CosineBell_CUDA(Grid_CUDA* grid, RBFFD_CUDA* der, double earth_radius, double velocity_angle,
                    double one_revolution_in_seconds, int useHyperviscosity, int dtype = RBFFD_F64, int ntracers = 1)
        : TimeDependentPDE_CUDA(grid, der, params(earth_radius, velocity_angle, one_revolution_in_seconds,
                                                   useHyperviscosity, dtype, ntracers))
    {
    }

private:
    static rbffd_pde_params params(double a, double alpha, double rev, int hv, int dtype, int ntracers)
    {
        rbffd_pde_params p = pde_params(RBFFD_RHS_COSINE_BELL, dtype, ntracers);
        p.use_hv = hv;
        p.sphere_radius = a;
        p.alpha = alpha;
        p.u0 = (2. * M_PI * a) / rev;  // cosine_bell.h:50
        return p;
    }
};

class HeatSphere_CUDA : public TimeDependentPDE_CUDA {
public:
    HeatSphere_CUDA(Grid_CUDA* grid, RBFFD_CUDA* der, double kappa = 1.0, int dtype = RBFFD_F64, int ntracers = 1)
        : TimeDependentPDE_CUDA(grid, der, params(kappa, dtype, ntracers))
    {
    }

private:
    static rbffd_pde_params params(double kappa, int dtype, int ntracers)
    {
        rbffd_pde_params p = pde_params(RBFFD_RHS_HEAT, dtype, ntracers);
        p.kappa = kappa;
        return p;
    }
};

class Advection_CUDA : public TimeDependentPDE_CUDA {
public:
    Advection_CUDA(Grid_CUDA* grid, RBFFD_CUDA* der, const std::vector<double>& cu, const std::vector<double>& cv,
                   int useHyperviscosity, int dtype = RBFFD_F64, int ntracers = 1)
        : TimeDependentPDE_CUDA(grid, der, params(cu, cv, useHyperviscosity, dtype, ntracers))
    {
    }

private:
    static rbffd_pde_params params(const std::vector<double>& cu, const std::vector<double>& cv, int hv, int dtype,
                                   int ntracers)
    {
        rbffd_pde_params p = pde_params(RBFFD_RHS_ADVECTION, dtype, ntracers);
        p.use_hv = hv;
        p.cu = cu.data();
        p.cv = cv.data();
        return p;
    }
};

// VortexRollup(Domain*, RBFFD*, Communicator*, int useHyperviscosity) (vortex_rollup.h:16):
// f = -w(theta) D_lambda h [+ D_hv h], w from rbffd_vortex_rollup_coefficients.
class VortexRollup_CUDA : public TimeDependentPDE_CUDA {
public:
    VortexRollup_CUDA(Grid_CUDA* grid, RBFFD_CUDA* der, int useHyperviscosity, int dtype = RBFFD_F64,
                      int ntracers = 1)
        : TimeDependentPDE_CUDA(grid, der, params(coefficients(*grid), useHyperviscosity, dtype, ntracers))
    {
    }

private:
    static const std::vector<double>& coefficients(Grid_CUDA& g)
    {
        static thread_local std::vector<double> w;  // read by rbffd_pde_create inside the base constructor
        const std::vector<double>& xyz = g.coordinates();
        w.assign(xyz.size() / 3, 0.0);
        check(nullptr, rbffd_vortex_rollup_coefficients((int)w.size(), xyz.data(), w.data()), "VortexRollup");
        return w;
    }
    static rbffd_pde_params params(const std::vector<double>& w, int hv, int dtype, int ntracers)
    {
        rbffd_pde_params p = pde_params(RBFFD_RHS_ADVECTION, dtype, ntracers);
        p.use_hv = hv;
        p.cu = w.data();
        p.cv = nullptr;
        return p;
    }
};

// The serving loop: continuous batching of requests on cached grids.
class Server_CUDA {
public:
    explicit Server_CUDA(Context& ctx, double hbm_fraction = 0.8, int max_active = 0) : ctx_(ctx)
    {
        check(ctx.handle(), rbffd_server_start(ctx.handle(), hbm_fraction, max_active, &h_), "rbffd_server_start");
    }
    ~Server_CUDA() { rbffd_server_stop(h_); }
    Server_CUDA(const Server_CUDA&) = delete;
    Server_CUDA& operator=(const Server_CUDA&) = delete;

    // out must stay valid until the request is done
    uint64_t submit(Grid_CUDA& grid, const rbffd_pde_params& p, const std::vector<double>& u0, double dt, int nsteps,
                    std::vector<double>& out)
    {
        out.resize(grid.getNodeListSize());
        rbffd_request r;
        r.grid = grid.handle();
        r.pde = p;
        r.u0 = u0.data();
        r.dt = dt;
        r.nsteps = nsteps;
        r.out = out.data();
        uint64_t id = 0;
        check(ctx_.handle(), rbffd_server_submit(h_, &r, &id), "rbffd_server_submit");
        return id;
    }
    int wait(uint64_t id, double timeout_s = 600.0) { return rbffd_server_wait(h_, id, timeout_s); }
    void waitIdle(double timeout_s = 600.0) { check(ctx_.handle(), rbffd_server_wait_idle(h_, timeout_s), "wait_idle"); }
    // RBFFD_ADMIT_ARRIVAL or RBFFD_ADMIT_SHORTEST (least work first)
    void setAdmissionOrder(int order)
    {
        check(ctx_.handle(), rbffd_server_set_admission_order(h_, order), "set_admission_order");
    }
    rbffd_server_stats stats()
    {
        rbffd_server_stats s;
        check(ctx_.handle(), rbffd_server_get_stats(h_, &s), "rbffd_server_get_stats");
        return s;
    }

private:
    Context& ctx_;
    rbffd_server* h_ = nullptr;
};

}  // namespace rbffd_sm100
