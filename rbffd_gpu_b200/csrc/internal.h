// Internal declarations shared by the translation units of librbffd_sm100.so.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/rbffd_sm100.h"

#define RBFFD_VERSION_STRING "rbffd_sm100 0.1.0 (sm_100a)"

// Index of a DerType bit (0..15) or -1.
inline int der_index(unsigned t)
{
    if (t == 0 || (t & (t - 1))) return -1;
    int i = 0;
    while (!(t & 1u)) { t >>= 1; i++; }
    return i < 16 ? i : -1;
}

struct TuneKey {
    int kernel, dtype, ntracers, N, n_pad;
    bool operator<(const TuneKey& o) const
    {
        return std::tie(kernel, dtype, ntracers, N, n_pad) < std::tie(o.kernel, o.dtype, o.ntracers, o.N, o.n_pad);
    }
};
struct Shape {
    int lanes = 0, block = 0;
    int tile = 0;  // rows per block with the halo staged in shared memory; 0 = gather from global memory
    int tma = 0;   // tiled kernel that streams weights and indices into shared memory with bulk copies
    int sched = 0; // tiled, FP32, one operator: each row reads its slots in the halo's conflict-avoiding schedule
    int pf = 0;    // tiled, one lane per row: upcoming chunks of weights and indices prefetched into L2
    int plain = 0; // FP64, one tracer, one lane per row, global gathers: the reference build's arithmetic
                   // (every multiply-add a rounded product, then a rounded sum; RBFFD_ARITH_UNFUSED)
    int pipe = 0;  // tiled, one operator, one lane group per row: weights and indices pipelined in registers
    int db = 0;    // tiled, one operator, one lane group per row: persistent blocks, next tile's halo copied in
                   // (cp.async) while the current one is computed
};

// Device status word of a context: kernels whose waits are bounded write a
// nonzero code here instead of hanging or trapping; the host reads and clears it.
enum { DEV_STATUS_OK = 0, DEV_STATUS_WAIT_TIMEOUT = 1 };

struct rbffd_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    std::mutex err_mu;  // last_error is also written by the serving loop's thread
    size_t held = 0;
    std::mutex mu;
    std::map<TuneKey, Shape> tuned;  // autotuner results per problem shape
    int* d_status = nullptr;         // DEV_STATUS_* written by kernels with bounded waits
    int arith = 0;                   // RBFFD_ARITH_*: FP64 arithmetic of rbffd_apply* and of new FP64 PDEs
    int weights_elim = 0;            // RBFFD_ELIM_*: elimination of the weight solves (0: autotuned)
};

// Read and clear the context's device status; RBFFD_ERR_TIMEOUT if a kernel gave up waiting.
int ctx_check_device_status(rbffd_ctx* ctx);

struct rbffd_grid {
    rbffd_ctx* ctx = nullptr;
    int N = 0, n_pad = 0, n4 = 0;  // n4: slots per row (n_pad rounded up to 4)
    int N32 = 0, nc = 0;           // rows rounded up to 32; chunks of 4 slots per row
    int* d_idx = nullptr;          // sliced ELL (ell.cuh), N32 x n4: node indices, padding = centre
    int* d_len = nullptr;          // [N] stencil lengths
    double4* d_xyz = nullptr;      // [N] node coordinates (w unused)
    double* d_w64[16] = {};        // per operator, sliced ELL N32 x n4: FP64 weights, padding 0
    float* d_w32[16] = {};         // FP32 copies (rounded to nearest)
    float* d_w32s[16] = {};        // FP32 copies in the 8-row slot schedule of halo sched_R
    int sched_R = 0;               // rows per block of the halo that has an 8-row slot schedule (0: none)
    unsigned w32_ver[16] = {};     // counts refreshes of d_w32[op] (copies made from it follow it)
    // Rows and nodes are stored in an internal order (a 3-D Morton curve through
    // the nodes) so that rows handled together gather from nearby nodes; the
    // stencil slot order is kept, so each row's arithmetic is unchanged.
    int* d_perm = nullptr;         // [N] internal row -> caller's node index
    std::vector<int> h_perm;       // same, on the host
    std::vector<int> h_iperm;      // caller's node index -> internal row
    std::vector<int> h_len;        // stencil lengths, internal order
    std::map<int, struct Halo*> halos;  // per rows-per-block R, built on first use
    // The cluster-resident RK4 layout (res_C CTAs of res_R rows; rk4.cu): per
    // CTA a halo of at most res_H nodes, each stencil slot's halo position, and
    // each row's push list (consumer CTA << 12 | halo position).  Built on first use.
    int res_R = 0, res_C = 0, res_H = 0, res_P = 0;
    int* d_res_pptr = nullptr;              // [res_C][res_R + 1] push-list ranges
    unsigned short* d_res_pdst = nullptr;   // [res_C][res_P]
    unsigned short* d_res_lidx = nullptr;   // [res_C][n4][res_R]
    struct WeightsWork* ww = nullptr;   // the weight solver's device workspace and captured launch (weights.cu)
    size_t bytes = 0;
};
void weights_work_free(rbffd_grid* g);
// Free the cluster-resident layout of a grid (rk4.cu).
void resident_free(rbffd_grid* g);

// Move [N][T] values (elem_bytes each) between the caller's node order and the
// grid's internal order (device arrays, on stream s).
int grid_to_internal(rbffd_grid* g, const void* src, void* dst, int T, int elem_bytes, cudaStream_t s);
int grid_to_caller(rbffd_grid* g, const void* src, void* dst, int T, int elem_bytes, cudaStream_t s);
// FP64 ELL apply with plain (unfused) multiply-adds, one lane per row (core.cu).
int grid_apply_dev_plain(rbffd_grid* g, int op, int T_tr, const double* u, double* out, int start, int count,
                         cudaStream_t s);
// Load (under lazy module loading) the device code of the permutation
// kernels / of the allocation-free heat RK4 path on the current device.
int grid_permute_preload();
int noalloc_preload();

// Row blocks of R consecutive internal rows with their halo: the unique nodes
// their stencils reference.  A block's kernel stages the halo's values in
// shared memory and reads them through 16-bit local indices (lidx, the sliced
// ELL layout of the stencils with each node index replaced by its position in
// the block's halo).  Positions are chosen so that the nodes 8 consecutive
// rows read at one slot fall in different 16-byte bank groups where possible;
// padding positions repeat a node of the block.
struct Halo {
    int R = 0, nblocks = 0, max_halo = 0;  // R: most rows in a block (blocks hold whole 32-row slices)
    int* d_rows = nullptr;       // [nblocks + 1] first row of each block
    int* d_ptr = nullptr;        // [nblocks + 1] offsets into d_nodes
    int* d_nodes = nullptr;      // node staged at each halo position (internal order)
    unsigned short* d_lidx = nullptr;  // sliced ELL, N32 x n4
    size_t b_nodes = 0, b_lidx = 0;
    // Conflict-avoiding slot schedules (built on demand, grid_halo_schedule):
    // each row's slots reordered so that at each step the P rows whose 16-byte
    // reads share one shared-memory wavefront read halo records in different
    // bank groups (position mod P) where their stencils allow; padding entries
    // (weight 0) take any free group.  P = 128 bytes / record bytes: 8 for
    // 16-byte records (four FP32 values per node), 4 for 32-byte, 2 for
    // 64-byte.  Index k = log2(P).  Changes the summation order of a row, so
    // only FP32 paths use it.
    unsigned short* d_lidx_s[4] = {};  // sliced ELL: position read at scheduled slot t
    unsigned short* d_slot_s[4] = {};  // original slot of scheduled slot t, SLOT_FREE for padding
};
constexpr unsigned short SLOT_FREE = 0xFFFF;
int grid_halo(rbffd_grid* g, int R, const Halo** out);
// The halo of R rows per block with its slot schedule for P rows per
// wavefront (P = 2, 4 or 8).
int grid_halo_schedule(rbffd_grid* g, int R, int P, const Halo** out);
// FP32 weights of operator op in the 8-row slot schedule of the halo of R
// rows per block (made on first use, refreshed with the FP32 copy; one R per
// grid).
int grid_f32_scheduled(rbffd_grid* g, int R, int op, const float** out);
// dst (sliced ELL, N32 x n4 floats) = the FP32 weights src in the slot order
// `slot` of a schedule (padding entries 0), on stream s.
int grid_schedule_weights(rbffd_grid* g, const float* src, const unsigned short* slot, float* dst, cudaStream_t s);

enum { KIND_ADVECT = 0, KIND_HEAT = 1 };

// Device-resident state of one time-dependent PDE (rk4.cu); the serving loop
// (server.cu) advances several of them in shared launches.
struct rbffd_pde {
    rbffd_grid* g = nullptr;
    rbffd_ctx* ctx = nullptr;
    int kind = 0, T = 1, dtype = RBFFD_F64, use_hv = 0;
    int op[3] = {-1, -1, -1};
    void *u = nullptr, *xa = nullptr, *xb = nullptr, *acc = nullptr;
    void *cu = nullptr, *cv = nullptr;
    // Advection with one fused operator -(cu W_lambda + cv W_theta) + W_hv
    // (sliced ELL, formed in FP64, rounded once to the PDE's dtype): the
    // stages stream one weight array instead of three
    void* wf = nullptr;  // in the PDE's dtype
    bool fused = false;
    // FP32 compensated state (rbffd_pde_set_compensated_state): [N][T] floats,
    // minus the rounding each step's u + increment lost; nullptr: off
    void* comp = nullptr;
    bool tuning = false;  // the autotuner's dt = 0 steps run: stage 3 leaves comp alone
    // The FP32 operators the stages stream (wf, or the grid's FP32 copies of
    // the one to three operators) in the slot schedule of halo ws_R for ws_P
    // rows per wavefront; each remade when its source changes (ws_src, ws_ver)
    float* ws[3] = {nullptr, nullptr, nullptr};
    int ws_R = 0, ws_P = 0;
    const void* ws_src[3] = {nullptr, nullptr, nullptr};
    unsigned ws_ver[3] = {0, 0, 0};
    void *d[3] = {nullptr, nullptr, nullptr};  // unfused path: one output per operator
    double* stage64 = nullptr;                  // FP64 staging for host state copies of an FP32 PDE
    double kappa = 1.0;
    double t = 0.0;
    Shape shape;
    bool forced = false;
    int arith = 0;  // RBFFD_ARITH_*
    cudaGraphExec_t gexec = nullptr;
    double g_dt = 0.0;
    int g_steps = 0;
    Shape g_shape;
    size_t bytes = 0;
};
// Device bytes rbffd_pde_create allocates for these parameters on grid g.
size_t pde_bytes(const rbffd_grid* g, const rbffd_pde_params* prm);
// Advection coefficients of an advection right-hand side, internal node order,
// in prm->dtype, into device arrays of N values (rk4.cu).
int advect_coefficients(rbffd_grid* g, const rbffd_pde_params* prm, void* cu_dev, void* cv_dev, cudaStream_t s);

// ---- error helpers --------------------------------------------------------
int set_error(rbffd_ctx* ctx, int status, const char* fmt, ...);
int cuda_error(rbffd_ctx* ctx, cudaError_t e, const char* what);

#define RBFFD_CUDA_TRY(ctx, call)                                     \
    do {                                                              \
        cudaError_t _e = (call);                                      \
        if (_e != cudaSuccess) return cuda_error((ctx), _e, #call);   \
    } while (0)

// Device allocation that is accounted against the context.
int dev_alloc(rbffd_ctx* ctx, void** p, size_t bytes);
void dev_free(rbffd_ctx* ctx, void* p, size_t bytes);

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

// FP32 copy of an FP64 slot-major weight array (kernel in grid.cu).
int grid_make_f32(rbffd_grid* g, int op);
