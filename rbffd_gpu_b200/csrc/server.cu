// Serving: a persistent request loop with continuous batching.
//
// A request is one time-dependent PDE solve (heat or advection on a grid whose
// weights are on the device, any step count, its own dt and kappa).
//
// Banks.  Requests on the same grid with the same right-hand side (kind,
// hyperviscosity, advection field) and dtype share a bank: state arrays u,
// xa, xb, acc (FP32: and comp, below) with room for BANK_W_F32 (FP32) or
// BANK_W_F64 (FP64) values per node (one for requests with their own per-node
// coefficients), in the grid's
// internal node order, plus the bank's advection coefficients.  The K
// requests of a bank occupy columns 0..K-1 of an interleaved [N][W] layout
// whose row stride W is K rounded up to a power of two; a stage kernel row
// reads the stencil's indices and each operator's weights once for all W
// columns and gathers a neighbour's W values with one vector load, so
// requests on a grid share both the operator stream and the gathers, and a
// lone request runs on the plain [N] layout.  When requests join or leave,
// the bank is repacked at the next step boundary (u into the free xa buffer
// at the new stride, then the two are swapped).
//
// FP32 banks keep a compensated state: a request's RK4 step moves u by a
// small fraction of itself, and rounding u + increment to FP32 every step
// drops most of the increment's bits (over 2000 steps of a serving-sized
// heat solve the FP32 state drifted 2e-5 from FP64).  Stage 3 therefore adds
// the increment with Knuth's TwoSum and keeps minus the lost part in a
// per-value compensation array that the next step adds back; a result is read
// out as u - comp.  Stages 0-2 and the gathers are unchanged.
//
// FP32 advection banks fuse their right-hand side into one operator: the
// velocity field is steady and the same for every column, so
//   f_i = -(cu_i D_lambda + cv_i D_theta) u + D_hv u = sum_s Wf[i][s] u[idx[i][s]]
// with Wf[i][s] = -(cu_i W_lambda[i][s] + cv_i W_theta[i][s]) + W_hv[i][s]
// formed once per bank in FP64 from the FP64 weights and rounded to FP32: one
// weight stream per stage instead of three.  FP64 banks keep the three
// operators and the reference's arithmetic (results equal the oracle's).
//
// Stage launches take the grid's row blocks with their halos (struct Halo,
// blocks of up to SEG_ROWS rows): a block first copies the bank values of its
// halo nodes into shared memory (one vector per node), then its rows gather
// from there through the 16-bit local indices -- half the index stream of the
// int32 indices, and gathers that never leave the SM.
//
// Two host threads per server:
//   * admission (admission_loop), in arrival order (or least work first,
//     rbffd_server_set_admission_order): a request gets a free
//     column of a matching bank, or a new bank, while the context's device
//     memory plus what the request adds stays within the HBM budget and fewer
//     than max_active requests are admitted (idle banks are freed first,
//     oldest first, when the budget is short).  Its initial state is uploaded
//     into an I/O buffer of its own; all this overlaps the running batches;
//   * stepping (worker_loop): at a step boundary, banks whose membership
//     changed are repacked, joining requests' initial states written into
//     their columns; then a batch of RK4 steps for
//     every bank with active columns, each of the four stages of a step one
//     launch of k_stage_bank per (dtype, width, operator count) over the rows
//     of all those banks (a table maps blocks to banks).  A batch is the
//     smallest remaining step count, capped at about TICK_TARGET_S of device
//     time.  Requests that reached their step count read their column out
//     and leave.
// A column's sums run over its stencil's slots in order with the rounding
// sequence of k_stage_scalar with one lane per row (rk4.cu), and free columns
// hold zeros, so a request's result does not depend on the rest of the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <new>
#include <thread>
#include <tuple>
#include <type_traits>
#include <vector>

#include "ell.cuh"
#include "internal.h"

namespace {

constexpr int SEG_ROWS = 128;               // rows (threads) per block of a stage launch
constexpr int BANK_W_F32 = 8;               // columns of an FP32 bank (32-byte rows)
constexpr int BANK_W_F64 = 4;               // columns of an FP64 bank (32-byte rows)
constexpr int BANK_W_MAX = 8;
constexpr double TICK_TARGET_S = 5e-3;      // device time aimed at per batch of steps
constexpr int TICK_MAX_STEPS = 160;
constexpr size_t TABLE_BYTES0 = 64 * 1024;  // initial capacity of the bank tables
constexpr int TILE_SMEM_MAX = 96 * 1024;    // shared memory for a block's halo values (two blocks per SM)

// One bank as a stage launch sees it.
template <typename T>
struct BankDesc {
    const int* idx;
    const T* w0;
    const T* w1;
    const T* w2;
    const T* cu;  // [N] advection coefficients (advection banks)
    const T* cv;
    T* u;  // [N][W] state and stage buffers
    T* xa;
    T* xb;
    T* acc;
    T* comp;  // FP32 banks: [N][W] compensation of u's rounding (nullptr: none)
    T c[4][BANK_W_MAX];  // per column: dt/2, dt/2, dt, dt/6 (0 for free columns)
    T kappa[BANK_W_MAX];
    // row blocks and halos of the grid (tiled launches)
    const int* hrows;             // [nblocks + 1] first row of each block
    const int* hptr;              // [nblocks + 1] offsets into hnodes
    const int* hnodes;            // halo node indices
    const unsigned short* lidx;   // sliced ELL local indices into the block's halo
    int N, nc, kind;
    int block0;  // first block of this bank in the launch
};

// W consecutive values (W * sizeof(T) = 4, 8 or a multiple of 16 bytes)
template <typename T, int W>
__device__ __forceinline__ void ldw(const T* p, T (&v)[W], bool readonly)
{
    if (W * sizeof(T) == 8) {
        float2 t = readonly ? __ldg(reinterpret_cast<const float2*>(p)) : *reinterpret_cast<const float2*>(p);
        memcpy(&v[0], &t, 8);
    } else if (W * sizeof(T) % 16 == 0) {
#pragma unroll
        for (int q = 0; q < W * (int)sizeof(T) / 16; q++) {
            float4 t = readonly ? __ldg(reinterpret_cast<const float4*>(p) + q) : reinterpret_cast<const float4*>(p)[q];
            memcpy(&v[q * 16 / sizeof(T)], &t, 16);
        }
    } else {
#pragma unroll
        for (int k = 0; k < W; k++) v[k] = readonly ? __ldg(p + k) : p[k];
    }
}

template <typename T, int W>
__device__ __forceinline__ void stw(T* p, const T (&v)[W])
{
    if (W * sizeof(T) == 8) {
        float2 t;
        memcpy(&t, &v[0], 8);
        *reinterpret_cast<float2*>(p) = t;
    } else if (W * sizeof(T) % 16 == 0) {
#pragma unroll
        for (int q = 0; q < W * (int)sizeof(T) / 16; q++) {
            float4 t;
            memcpy(&t, &v[q * 16 / sizeof(T)], 16);
            reinterpret_cast<float4*>(p)[q] = t;
        }
    } else {
#pragma unroll
        for (int k = 0; k < W; k++) p[k] = v[k];
    }
}

// Right-hand side and RK4 stage update of row i, all W columns (the
// arithmetic of stage_update in rk4.cu, per column).
template <typename T, int W, int NOPS>
__device__ __forceinline__ void bank_stage_update(const BankDesc<T>& B, int i, int stage, const T (&d0)[W],
                                                  const T (&d1)[W], const T (&d2)[W])
{
    const bool adv = B.kind == KIND_ADVECT;
    const T cu = adv ? B.cu[i] : T(0), cv = adv ? B.cv[i] : T(0);
    const size_t row = (size_t)i * W;
    T ui[W], ac[W], out[W], cm[W];
    ldw<T, W>(B.u + row, ui, false);
    if (stage > 0) ldw<T, W>(B.acc + row, ac, false);
    const bool comp = stage == 3 && B.comp != nullptr;
    if (comp) ldw<T, W>(B.comp + row, cm, false);
#pragma unroll
    for (int v = 0; v < W; v++) {
        T f;
        if (adv) {
            f = -Ar<T>::fma(cu, d0[v], Ar<T>::mul(cv, d1[v]));
            if (NOPS > 2) f = Ar<T>::add(f, d2[v]);
        } else {
            f = Ar<T>::mul(B.kappa[v], d0[v]);
        }
        const T c = B.c[stage][v];
        if (stage == 0) {
            ac[v] = f;
            out[v] = Ar<T>::fma(c, f, ui[v]);
        } else if (stage < 3) {
            ac[v] = Ar<T>::add(ac[v], Ar<T>::mul(T(2), f));
            out[v] = Ar<T>::fma(c, f, ui[v]);
        } else if (comp) {
            // compensated update: the increment is small against u, so rounding u + inc
            // loses most of its bits; cm holds minus what each step's sum lost (the exact
            // rounding error of the sum, by Knuth's TwoSum) and the next step adds it back
            const T y = Ar<T>::sub(Ar<T>::mul(c, Ar<T>::add(ac[v], f)), cm[v]);
            out[v] = Ar<T>::add(ui[v], y);
            const T yb = Ar<T>::sub(out[v], ui[v]);
            const T lost = Ar<T>::add(Ar<T>::sub(ui[v], Ar<T>::sub(out[v], yb)), Ar<T>::sub(y, yb));
            cm[v] = -lost;
        } else {
            out[v] = Ar<T>::fma(c, Ar<T>::add(ac[v], f), ui[v]);
        }
    }
    if (stage < 3) {
        stw<T, W>(B.acc + row, ac);
        stw<T, W>((stage == 1 ? B.xb : B.xa) + row, out);
    } else {
        stw<T, W>(B.u + row, out);
        if (comp) stw<T, W>(B.comp + row, cm);
    }
}

// One RK4 stage for the rows of every bank of one launch.  Stage buffers as in
// k_stage_scalar: 0: u -> xa, 1: xa -> xb, 2: xb -> xa, 3: xa -> u.  Column v
// of row i accumulates w[s] * x[idx[s]][v] over the slots s in stencil order
// with fused multiply-adds, exactly the single-request sequence.
template <typename T, int W, int NOPS>
__global__ void __launch_bounds__(SEG_ROWS) k_stage_bank(const BankDesc<T>* __restrict__ banks, int nbanks, int stage)
{
    int lo = 0, hi = nbanks - 1;  // last bank with block0 <= blockIdx.x
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (banks[mid].block0 <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const BankDesc<T>& B = banks[lo];
    const int i = ((int)blockIdx.x - B.block0) * SEG_ROWS + (int)threadIdx.x;
    if (i >= B.N) return;
    const T* x = stage == 0 ? B.u : (stage == 2 ? B.xb : B.xa);
    T d0[W], d1[W], d2[W];
#pragma unroll
    for (int v = 0; v < W; v++) d0[v] = d1[v] = d2[v] = T(0);
    for (int c = 0; c < B.nc; c++) {
        const size_t o = sell_off(i, c, B.nc);
        const int4 j4 = ld_idx4(B.idx + o);
        const int jj[4] = {j4.x, j4.y, j4.z, j4.w};
        T wa[4], wb[4], wc[4];
        ld_w4(B.w0 + o, wa);
        if (NOPS > 1) ld_w4(B.w1 + o, wb);
        if (NOPS > 2) ld_w4(B.w2 + o, wc);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            T xv[W];
            ldw<T, W>(x + (size_t)jj[e] * W, xv, true);
#pragma unroll
            for (int v = 0; v < W; v++) {
                d0[v] = Ar<T>::fma(wa[e], xv[v], d0[v]);
                if (NOPS > 1) d1[v] = Ar<T>::fma(wb[e], xv[v], d1[v]);
                if (NOPS > 2) d2[v] = Ar<T>::fma(wc[e], xv[v], d2[v]);
            }
        }
    }
    bank_stage_update<T, W, NOPS>(B, i, stage, d0, d1, d2);
}

// The same stage over a grid's halo row blocks: the block's halo values of x
// are staged in shared memory ([halo node][W]), gathers read them through the
// 16-bit local indices.  Same per-column arithmetic as k_stage_bank.
template <typename T, int W, int NOPS>
__global__ void __launch_bounds__(SEG_ROWS) k_stage_bank_tile(const BankDesc<T>* __restrict__ banks, int nbanks,
                                                              int stage)
{
    extern __shared__ __align__(16) unsigned char smem_bank[];
    T* sx = reinterpret_cast<T*>(smem_bank);
    int lo = 0, hi = nbanks - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (banks[mid].block0 <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const BankDesc<T>& B = banks[lo];
    const int b = (int)blockIdx.x - B.block0;
    const int r0 = __ldg(B.hrows + b), r1 = __ldg(B.hrows + b + 1);
    const int h0 = __ldg(B.hptr + b), hn = __ldg(B.hptr + b + 1) - h0;
    const T* x = stage == 0 ? B.u : (stage == 2 ? B.xb : B.xa);
    // 32-byte rows are staged as two 16-byte planes ([plane][halo position]):
    // each gather instruction then reads 16-byte vectors at a 16-byte stride,
    // the access the halo placement spreads over the bank groups
    constexpr int P = W * sizeof(T) == 32 ? 2 : 1, VP = W / P;
    for (int h = threadIdx.x; h < hn; h += blockDim.x) {
        T v[W];
        ldw<T, W>(x + (size_t)__ldg(B.hnodes + h0 + h) * W, v, true);
#pragma unroll
        for (int p = 0; p < P; p++) {
            T vp[VP];
#pragma unroll
            for (int q = 0; q < VP; q++) vp[q] = v[p * VP + q];
            stw<T, VP>(sx + ((size_t)p * hn + h) * VP, vp);
        }
    }
    __syncthreads();
    const int i = r0 + (int)threadIdx.x;
    if (i >= r1) return;
    T d0[W], d1[W], d2[W];
#pragma unroll
    for (int v = 0; v < W; v++) d0[v] = d1[v] = d2[v] = T(0);
    for (int c = 0; c < B.nc; c++) {
        const size_t o = sell_off(i, c, B.nc);
        const ushort4 l4 = __ldg(reinterpret_cast<const ushort4*>(B.lidx + o));
        const int ll[4] = {l4.x, l4.y, l4.z, l4.w};
        T wa[4], wb[4], wc[4];
        ld_w4(B.w0 + o, wa);
        if (NOPS > 1) ld_w4(B.w1 + o, wb);
        if (NOPS > 2) ld_w4(B.w2 + o, wc);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            T xv[W];
#pragma unroll
            for (int p = 0; p < P; p++) {
                T vp[VP];
                ldw<T, VP>(sx + ((size_t)p * hn + ll[e]) * VP, vp, false);
#pragma unroll
                for (int q = 0; q < VP; q++) xv[p * VP + q] = vp[q];
            }
#pragma unroll
            for (int v = 0; v < W; v++) {
                d0[v] = Ar<T>::fma(wa[e], xv[v], d0[v]);
                if (NOPS > 1) d1[v] = Ar<T>::fma(wb[e], xv[v], d1[v]);
                if (NOPS > 2) d2[v] = Ar<T>::fma(wc[e], xv[v], d2[v]);
            }
        }
    }
    bank_stage_update<T, W, NOPS>(B, i, stage, d0, d1, d2);
}

// A bank's new layout at a step boundary: column c of dst (row stride wdst)
// takes column from[c] of src (stride wsrc), or the initial state of a
// joining request (FP64, caller's node order, rounded to T), or zero.
constexpr int FROM_ZERO = -1, FROM_IO = -2;

template <typename T>
struct Repack {
    T* dst;
    const T* src;
    int wsrc, wdst, N;
    int from[BANK_W_MAX];
    const double* io[BANK_W_MAX];
    const int* perm;  // internal row -> caller's node index
};

template <typename T>
__global__ void k_repack(Repack<T> a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.N) return;
    for (int c = 0; c < a.wdst; c++) {
        T v = T(0);
        if (a.from[c] >= 0) v = a.src[(size_t)i * a.wsrc + a.from[c]];
        else if (a.from[c] == FROM_IO) v = (T)a.io[c][a.perm[i]];
        a.dst[(size_t)i * a.wdst + c] = v;
    }
}

// A request's column, back to FP64 in the caller's node order.
template <typename T>
__global__ void k_column_out(const T* u, const T* comp, int W, int col, double* __restrict__ io,
                             const int* __restrict__ perm, int N)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const size_t e = (size_t)i * W + col;
    // with a compensation, u - comp is the state to twice the precision of T
    io[perm[i]] = comp ? (double)u[e] - (double)comp[e] : (double)u[e];
}

// Fused advection operator of a bank, row by row over the padded rows (sliced
// ELL; padding rows and slots stay 0): Wf = -(cu W_lambda + cv W_theta) + W_hv,
// in the halo's slot schedule when slot is given (entry t of row i takes the
// row's original slot slot[t], 0 for a padding entry).
__global__ void k_fuse_advection(float* __restrict__ wf, const double* __restrict__ wl,
                                 const double* __restrict__ wt, const double* __restrict__ wh,
                                 const double* __restrict__ cu, const double* __restrict__ cv,
                                 const unsigned short* __restrict__ slot, int N, int rows, int nc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    const double a = i < N ? cu[i] : 0.0, c = i < N ? cv[i] : 0.0;
    for (int t = 0; t < 4 * nc; t++) {
        const size_t ot = sell_elem(i, t, nc);
        const int s = slot ? slot[ot] : t;
        if (i >= N || s == SLOT_FREE) {
            wf[ot] = 0.0f;
            continue;
        }
        const size_t o = sell_elem(i, s, nc);
        double w = -(a * wl[o] + c * wt[o]);
        if (wh) w += wh[o];
        wf[ot] = __double2float_rn(w);
    }
}

using Clock = std::chrono::steady_clock;

struct Bank;

struct Request {
    uint64_t id = 0;
    rbffd_request p{};
    std::vector<double> u0, cu, cv;  // copies taken at submission
    Clock::time_point t_submit, t_admit, t_done;
    bool admitted = false, cancel = false, inserted = false;
    int done = 0, status = RBFFD_OK;
    Bank* bank = nullptr;
    int col = -1;
    double* d_io = nullptr;  // [N] FP64, caller's order: initial state in, result out
    int steps_done = 0;
};

struct Bank {
    rbffd_grid* grid = nullptr;
    rbffd_pde_params prm{};  // right-hand side (coefficient pointers unused)
    uint64_t owner = 0;      // request id for a bank with caller-given coefficients
    int dtype = RBFFD_F32, kind = KIND_HEAT, nops = 1;
    int Wcap = 1;  // values per node the arrays hold
    int op[3] = {-1, -1, -1};
    void *u = nullptr, *xa = nullptr, *xb = nullptr, *acc = nullptr, *cu = nullptr, *cv = nullptr;
    void* comp = nullptr;  // FP32 banks: compensation of u's rounding, [N][Wcap]
    void* wf = nullptr;  // fused advection operator (FP32 advection banks), sliced ELL
    const Halo* halo = nullptr;  // the grid's row blocks of SEG_ROWS rows (nullptr: untiled)
    // FP32 tiled banks read the halo's conflict-avoiding slot schedule: local
    // indices d_lidx_s and weights in the same order (wf, or the grid's
    // scheduled FP32 copy wsched for heat)
    bool sched = false;
    const float* wsched = nullptr;
    size_t bytes = 0;
    int members = 0;       // admitted requests assigned to the bank (S->mu)
    bool in_plan = false;  // referenced by the stepping thread's current tables (S->mu)
    Clock::time_point idle_since;
    // layout, owned by the stepping thread
    int W = 1;                   // row stride
    std::vector<Request*> cols;  // occupant of each column 0..W-1 (nullptr: free)
    std::vector<Request*> join;  // admitted, placed at the next step boundary
    bool dirty = false;          // membership changed since the last repack
};

size_t state_bytes(const rbffd_pde_params& p) { return p.dtype == RBFFD_F64 ? 8 : 4; }

int bank_capacity(const rbffd_pde_params& p)
{
    if (p.rhs_kind == RBFFD_RHS_ADVECTION) return 1;
    return p.dtype == RBFFD_F64 ? BANK_W_F64 : BANK_W_F32;
}

bool bank_fused(const rbffd_pde_params& p) { return p.rhs_kind != RBFFD_RHS_HEAT && p.dtype == RBFFD_F32; }

size_t fused_bytes(const rbffd_grid* g) { return (size_t)g->N32 * g->n4 * sizeof(float); }

size_t bank_bytes(const rbffd_grid* g, const rbffd_pde_params& p)
{
    const size_t es = state_bytes(p), N = (size_t)g->N;
    const size_t rhs = p.rhs_kind == RBFFD_RHS_HEAT ? 0 : (bank_fused(p) ? fused_bytes(g) : 2 * N * es);
    const int arrays = p.dtype == RBFFD_F32 ? 5 : 4;  // u, xa, xb, acc (and FP32: the compensation)
    return arrays * N * bank_capacity(p) * es + rhs;
}

bool bank_fits(const Bank& b, const Request& r)
{
    const rbffd_pde_params& p = r.p.pde;
    if (b.grid != r.p.grid || b.prm.rhs_kind != p.rhs_kind || b.dtype != p.dtype) return false;
    if (p.rhs_kind == RBFFD_RHS_ADVECTION) return b.owner == r.id;  // caller-given coefficients
    if (p.rhs_kind == RBFFD_RHS_HEAT) return true;                  // kappa is per column
    return b.prm.use_hv == p.use_hv && b.prm.sphere_radius == p.sphere_radius && b.prm.alpha == p.alpha &&
           b.prm.u0 == p.u0;
}

}  // namespace

struct rbffd_server {
    rbffd_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;   // stepping thread: stage launches, repacks, column read-outs
    cudaStream_t astream = nullptr;  // admission thread: bank set-up, initial-state uploads
    cudaStream_t cstream = nullptr;  // stepping thread: results copied to the callers
    cudaEvent_t ev[2][3] = {};       // per batch slot: start, end, finished columns read out
    cudaEvent_t ev_tab = nullptr;    // the last bank tables copied to the device
    size_t budget = 0;
    int max_active = 0;
    int order = RBFFD_ADMIT_ARRIVAL;  // which pending request admission takes next (S->mu)
    std::mutex mu;  // guards everything below up to the stepping-thread state
    std::condition_variable cv_work;   // the stepping thread waits for admitted requests
    std::condition_variable cv_admit;  // the admission thread waits for requests, columns or memory
    std::condition_variable cv_done;   // callers wait for results
    std::deque<std::shared_ptr<Request>> pending;  // submitted, not yet admitted
    std::vector<std::shared_ptr<Request>> ready;   // admitted, join at the next step boundary
    std::vector<std::shared_ptr<Request>> active;  // stepping
    int finishing = 0;  // left `active` with the batch in flight, not yet completed
    std::map<uint64_t, std::shared_ptr<Request>> all;
    std::vector<std::unique_ptr<Bank>> banks;
    uint64_t next_id = 1;
    bool stop = false, admitter_done = false;
    bool paused = false;  // no batches are issued while set (admission continues)
    int inject_fail = 0;
    size_t owned = 0;  // device bytes of banks and I/O buffers (reserved or allocated)
    rbffd_server_stats st{};
    std::thread worker, admitter;
    // stepping-thread state
    void* h_tab = nullptr;  // pinned host bank tables
    void* d_tab = nullptr;
    size_t tab_cap = 0;
    double step_s = 0.0;  // device seconds per step of the last batch
};

namespace {

void finish_request(Request& r, int status)
{
    r.status = status;
    r.t_done = Clock::now();
    r.done = 1;
}

size_t ctx_held(rbffd_ctx* ctx)
{
    std::lock_guard<std::mutex> lk(ctx->mu);
    return ctx->held;
}

void ctx_account(rbffd_ctx* ctx, size_t add, size_t sub)
{
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->held += add;
    ctx->held -= std::min(ctx->held, sub);
}

void bank_free_memory(rbffd_ctx* ctx, Bank& b)
{
    const size_t es = b.dtype == RBFFD_F64 ? 8 : 4, n = (size_t)b.grid->N * b.Wcap * es, nc = (size_t)b.grid->N * es;
    dev_free(ctx, b.u, n);
    dev_free(ctx, b.xa, n);
    dev_free(ctx, b.xb, n);
    dev_free(ctx, b.acc, n);
    dev_free(ctx, b.comp, n);
    dev_free(ctx, b.cu, nc);
    dev_free(ctx, b.cv, nc);
    dev_free(ctx, b.wf, fused_bytes(b.grid));
    b.u = b.xa = b.xb = b.acc = b.comp = b.cu = b.cv = b.wf = nullptr;
}

// Device arrays of a new bank for request r (zeroed state, advection
// coefficients); called without S->mu held.
int bank_create(rbffd_server* S, const Request& r, Bank& b)
{
    rbffd_ctx* ctx = S->ctx;
    rbffd_grid* g = r.p.grid;
    const rbffd_pde_params& p = r.p.pde;
    b.grid = g;
    b.prm = p;
    b.prm.cu = b.prm.cv = nullptr;
    b.owner = p.rhs_kind == RBFFD_RHS_ADVECTION ? r.id : 0;
    b.dtype = p.dtype;
    b.Wcap = bank_capacity(p);
    if (p.rhs_kind == RBFFD_RHS_HEAT) {
        b.kind = KIND_HEAT;
        b.nops = 1;
        b.op[0] = der_index(RBFFD_LSFC);
    } else {
        b.kind = KIND_ADVECT;
        b.nops = p.use_hv ? 3 : 2;
        b.op[0] = der_index(RBFFD_LAMBDA);
        b.op[1] = der_index(RBFFD_THETA);
        if (p.use_hv) b.op[2] = der_index(RBFFD_HV);
    }
    b.bytes = bank_bytes(g, p);
    int rc;
    for (int k = 0; k < b.nops; k++)  // FP32 weight copies are made on first use
        if (b.dtype == RBFFD_F32 && !g->d_w32[b.op[k]] && (rc = grid_make_f32(g, b.op[k]))) return rc;
    const size_t es = state_bytes(p), n = (size_t)g->N * b.Wcap * es;
    if ((rc = dev_alloc(ctx, &b.u, n)) || (rc = dev_alloc(ctx, &b.xa, n)) || (rc = dev_alloc(ctx, &b.xb, n)) ||
        (rc = dev_alloc(ctx, &b.acc, n)) || (b.dtype == RBFFD_F32 && (rc = dev_alloc(ctx, &b.comp, n)))) {
        bank_free_memory(ctx, b);
        return rc;
    }
    // the grid's row blocks and halos; banks whose halos would not fit shared memory stay untiled
    const Halo* h = nullptr;
    if (grid_halo(g, SEG_ROWS, &h) == RBFFD_OK && (size_t)h->max_halo * b.Wcap * es <= (size_t)TILE_SMEM_MAX)
        b.halo = h;
    if (b.halo && b.dtype == RBFFD_F32) {  // FP32: the conflict-avoiding slot schedule
        const Halo* hs = nullptr;
        if ((rc = grid_halo_schedule(g, SEG_ROWS, 8, &hs)) ||
            (b.kind == KIND_HEAT && (rc = grid_f32_scheduled(g, SEG_ROWS, b.op[0], &b.wsched)))) {
            bank_free_memory(ctx, b);
            return rc;
        }
        b.sched = true;
    }
    cudaError_t e = cudaMemsetAsync(b.u, 0, n, S->astream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.xa, 0, n, S->astream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.xb, 0, n, S->astream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.acc, 0, n, S->astream);
    if (e == cudaSuccess && b.comp) e = cudaMemsetAsync(b.comp, 0, n, S->astream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->astream);
    if (e != cudaSuccess) {
        bank_free_memory(ctx, b);
        return cuda_error(ctx, e, "bank set-up");
    }
    if (b.kind == KIND_ADVECT) {
        rbffd_pde_params q = p;
        q.cu = r.cu.empty() ? nullptr : r.cu.data();
        q.cv = r.cv.empty() ? nullptr : r.cv.data();
        if (bank_fused(p)) {  // FP64 coefficients and weights -> one FP32 operator
            q.dtype = RBFFD_F64;
            void *cu64 = nullptr, *cv64 = nullptr;
            const size_t nc = (size_t)g->N * sizeof(double);
            if (!(rc = dev_alloc(ctx, &cu64, nc)) && !(rc = dev_alloc(ctx, &cv64, nc)) &&
                !(rc = advect_coefficients(g, &q, cu64, cv64, S->astream)) &&
                !(rc = dev_alloc(ctx, &b.wf, fused_bytes(g)))) {
                const int rows = g->N32;
                k_fuse_advection<<<(rows + 127) / 128, 128, 0, S->astream>>>(
                    (float*)b.wf, g->d_w64[b.op[0]], g->d_w64[b.op[1]], b.op[2] >= 0 ? g->d_w64[b.op[2]] : nullptr,
                    (const double*)cu64, (const double*)cv64, b.sched ? b.halo->d_slot_s[3] : nullptr, g->N, rows,
                    g->nc);
                cudaError_t e = cudaGetLastError();
                if (e == cudaSuccess) e = cudaStreamSynchronize(S->astream);
                if (e != cudaSuccess) rc = cuda_error(ctx, e, "fused advection operator");
            }
            dev_free(ctx, cu64, nc);
            dev_free(ctx, cv64, nc);
        } else {
            const size_t nc = (size_t)g->N * es;
            if (!(rc = dev_alloc(ctx, &b.cu, nc)) && !(rc = dev_alloc(ctx, &b.cv, nc)))
                rc = advect_coefficients(g, &q, b.cu, b.cv, S->astream);
        }
        if (rc) {
            bank_free_memory(ctx, b);
            return rc;
        }
    }
    return RBFFD_OK;
}

// The pending request admission takes next (S->mu held, queue not empty):
// the first, or with RBFFD_ADMIT_SHORTEST the one with the least work
// (nodes x padded stencil size x steps; the first of equals).
std::shared_ptr<Request> next_pending(rbffd_server* S)
{
    if (S->order != RBFFD_ADMIT_SHORTEST) return S->pending.front();
    auto work = [](const Request& r) { return (double)r.p.grid->N * r.p.grid->n4 * r.p.nsteps; };
    auto best = S->pending.begin();
    for (auto it = S->pending.begin(); it != S->pending.end(); ++it)
        if (work(**it) < work(**best)) best = it;
    return *best;
}

// Remove r from the pending queue (S->mu held).
void drop_pending(rbffd_server* S, const std::shared_ptr<Request>& r)
{
    for (auto it = S->pending.begin(); it != S->pending.end(); ++it)
        if (*it == r) {
            S->pending.erase(it);
            return;
        }
}

// Admission thread.  In admission order (arrival, or least work first), each
// pending request gets a column of a matching bank (a new bank when none has
// room and the budget allows; idle banks are freed first, oldest first) and
// an I/O buffer holding its initial state, then moves to the ready list.  Runs beside the stepping thread, so
// allocation and the upload overlap the running batches.
void admission_loop(rbffd_server* S)
{
    cudaSetDevice(S->ctx->device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        // cancelled requests still waiting leave now (all of them once the server stops);
        // only this thread removes requests from the queue
        for (auto it = S->pending.begin(); it != S->pending.end();)
            if ((*it)->cancel || S->stop) {
                finish_request(**it, RBFFD_ERR_CANCELLED);
                S->st.cancelled++;
                it = S->pending.erase(it);
                S->cv_done.notify_all();
            } else {
                ++it;
            }
        if (S->stop) break;
        const int running = (int)(S->active.size() + S->ready.size()) + S->finishing;
        if (S->pending.empty() || (S->max_active > 0 && running >= S->max_active)) {
            S->cv_admit.wait(lk);
            continue;
        }
        std::shared_ptr<Request> r = next_pending(S);
        if (S->inject_fail > 0) {
            S->inject_fail--;
            drop_pending(S, r);
            finish_request(*r, set_error(S->ctx, RBFFD_ERR_OOM, "injected admission failure"));
            S->st.failed++;
            S->cv_done.notify_all();
            continue;
        }
        rbffd_grid* g = r->p.grid;
        const size_t io_bytes = (size_t)g->N * sizeof(double);
        Bank* bank = nullptr;
        for (auto& b : S->banks)
            if (bank_fits(*b, *r) && b->members < b->Wcap) {
                bank = b.get();
                break;
            }
        const size_t need = io_bytes + (bank ? 0 : bank_bytes(g, r->p.pde));
        if (ctx_held(S->ctx) + need > S->budget) {
            size_t k = S->banks.size();  // the idle bank that has been idle longest
            for (size_t q = 0; q < S->banks.size(); q++)
                if (S->banks[q].get() != bank && S->banks[q]->members == 0 && !S->banks[q]->in_plan &&
                    (k == S->banks.size() || S->banks[q]->idle_since < S->banks[k]->idle_since))
                    k = q;
            if (k < S->banks.size()) {
                std::unique_ptr<Bank> b = std::move(S->banks[k]);
                S->banks.erase(S->banks.begin() + (long)k);
                S->owned -= std::min(S->owned, b->bytes);
                lk.unlock();
                bank_free_memory(S->ctx, *b);
                lk.lock();
                continue;
            }
            if (running > 0) {  // memory frees up when a running request finishes
                S->cv_admit.wait(lk);
                continue;
            }
            drop_pending(S, r);
            finish_request(*r, set_error(S->ctx, RBFFD_ERR_BUDGET,
                                         "request needing %zu bytes does not fit the budget of %zu bytes", need,
                                         S->budget));
            S->st.failed++;
            S->cv_done.notify_all();
            continue;
        }
        S->owned += need;  // reserved before allocating: submissions meanwhile count it as the server's
        if (bank) bank->members++;
        lk.unlock();
        int rc = RBFFD_OK;
        std::unique_ptr<Bank> fresh;
        if (!bank) {
            fresh.reset(new (std::nothrow) Bank());
            rc = fresh ? bank_create(S, *r, *fresh) : RBFFD_ERR_OOM;
        }
        double* io = nullptr;
        if (rc == RBFFD_OK) {
            cudaError_t e = cudaMallocAsync((void**)&io, io_bytes, S->astream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(io, r->u0.data(), io_bytes, cudaMemcpyHostToDevice, S->astream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(S->astream);
            if (e != cudaSuccess) {
                rc = cuda_error(S->ctx, e, "request upload");
                if (io) cudaFreeAsync(io, S->astream);
                io = nullptr;
            } else {
                ctx_account(S->ctx, io_bytes, 0);
            }
        }
        if (rc != RBFFD_OK && fresh) bank_free_memory(S->ctx, *fresh);  // no-op after a failed bank_create
        lk.lock();
        drop_pending(S, r);  // still queued: only this thread removes from the queue
        if (rc != RBFFD_OK) {
            S->owned -= std::min(S->owned, need);
            if (bank && --bank->members == 0) bank->idle_since = Clock::now();
            finish_request(*r, rc);
            S->st.failed++;
            S->cv_done.notify_all();
            continue;
        }
        if (!bank) {
            bank = fresh.get();
            bank->members = 1;
            S->banks.push_back(std::move(fresh));
        } else {
            S->st.slots_reused++;
        }
        r->bank = bank;
        r->d_io = io;
        r->admitted = true;
        r->t_admit = Clock::now();
        S->ready.push_back(r);
        S->cv_work.notify_one();
    }
    S->admitter_done = true;
    S->cv_work.notify_all();
}

template <typename T>
void fill_desc(BankDesc<T>& d, const Bank& b, int block0)
{
    const rbffd_grid* g = b.grid;
    auto W = [&](int k) -> const T* {
        if (b.op[k] < 0) return nullptr;
        return std::is_same<T, double>::value ? (const T*)g->d_w64[b.op[k]] : (const T*)g->d_w32[b.op[k]];
    };
    d.idx = g->d_idx;
    d.w0 = b.wf ? (const T*)b.wf : (b.sched ? (const T*)b.wsched : W(0));
    d.w1 = b.wf ? nullptr : W(1);
    d.w2 = b.wf ? nullptr : W(2);
    d.cu = (const T*)b.cu;
    d.cv = (const T*)b.cv;
    d.u = (T*)b.u;
    d.xa = (T*)b.xa;
    d.xb = (T*)b.xb;
    d.acc = (T*)b.acc;
    d.comp = (T*)b.comp;
    for (int v = 0; v < BANK_W_MAX; v++) {
        const Request* r = v < b.W ? b.cols[v] : nullptr;
        const bool on = r != nullptr;
        // the stage coefficients of rbffd_pde_advance; free columns hold zeros and stay zero
        const double dt = on ? r->p.dt : 0.0;
        d.c[0][v] = (T)(0.5 * dt);
        d.c[1][v] = (T)(0.5 * dt);
        d.c[2][v] = (T)(1.0 * dt);
        d.c[3][v] = (T)(dt / 6.);
        // a fused operator is applied as f = 1 * (Wf u)
        d.kappa[v] = on ? (b.wf ? T(1) : (T)r->p.pde.kappa) : T(0);
    }
    d.hrows = b.halo ? b.halo->d_rows : nullptr;
    d.hptr = b.halo ? b.halo->d_ptr : nullptr;
    d.hnodes = b.halo ? b.halo->d_nodes : nullptr;
    d.lidx = b.halo ? (b.sched ? b.halo->d_lidx_s[3] : b.halo->d_lidx) : nullptr;
    d.N = g->N;
    d.nc = g->nc;
    d.kind = b.wf ? KIND_HEAT : b.kind;
    d.block0 = block0;
}

// One kernel launch per stage: the banks of one dtype, width and operator count.
struct Launch {
    int dtype = 0, W = 1, nops = 1, tiled = 0, nbanks = 0, blocks = 0;
    size_t off = 0;      // byte offset of its bank table
    size_t smem = 0;     // dynamic shared memory (tiled launches)
    double bytes = 0.0;  // algorithmic bytes per stage
};

inline size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// Lay out the bank tables of every launch for the banks with active columns
// and upload them, stream-ordered before the launches that read them (the
// previous batch has completed, so the pinned host copy is free to rewrite).
// Called with S->mu held (reads bank membership); the copy is asynchronous.
int upload_tables(rbffd_server* S, std::vector<Launch>& plan)
{
    plan.clear();
    for (auto& b : S->banks) b->in_plan = false;
    std::vector<Bank*> bs;
    for (auto& b : S->banks) {
        bool any = false;
        for (const Request* r : b->cols) any |= r != nullptr;
        if (any) bs.push_back(b.get());
    }
    std::vector<std::vector<Bank*>> per_launch;
    size_t off = 0;
    for (int dt = 0; dt < 2; dt++)
        for (int W : {1, 2, 4, 8})
            for (int no = 1; no <= 3; no++)
            for (int ti = 0; ti < 2; ti++) {
                std::vector<Bank*> sel;
                for (Bank* b : bs)
                    if (b->dtype == (dt ? RBFFD_F64 : RBFFD_F32) && b->W == W && (b->wf ? 1 : b->nops) == no &&
                        (b->halo != nullptr) == (ti == 1))
                        sel.push_back(b);
                if (sel.empty()) continue;
                Launch L;
                L.dtype = dt ? RBFFD_F64 : RBFFD_F32;
                L.W = W;
                L.nops = no;
                L.tiled = ti;
                for (Bank* b : sel)
                    if (ti) L.smem = std::max(L.smem, (size_t)b->halo->max_halo * W * (dt ? 8 : 4));
                L.nbanks = (int)sel.size();
                L.off = off;
                off = align256(off + sel.size() * (dt ? sizeof(BankDesc<double>) : sizeof(BankDesc<float>)));
                plan.push_back(L);
                per_launch.push_back(sel);
            }
    if (off > S->tab_cap) {
        const size_t cap = std::max<size_t>(off * 2, TABLE_BYTES0);
        RBFFD_CUDA_TRY(S->ctx, cudaStreamSynchronize(S->stream));  // no batch reads the old tables
        if (S->h_tab) cudaFreeHost(S->h_tab);
        dev_free(S->ctx, S->d_tab, S->tab_cap);
        S->h_tab = nullptr;
        S->d_tab = nullptr;
        S->tab_cap = 0;
        RBFFD_CUDA_TRY(S->ctx, cudaMallocHost(&S->h_tab, cap));
        const int rc = dev_alloc(S->ctx, &S->d_tab, cap);
        if (rc) return rc;
        S->tab_cap = cap;
    }
    RBFFD_CUDA_TRY(S->ctx, cudaEventSynchronize(S->ev_tab));  // the previous copy has left h_tab
    char* h = (char*)S->h_tab;
    for (size_t l = 0; l < plan.size(); l++) {
        Launch& L = plan[l];
        for (size_t q = 0; q < per_launch[l].size(); q++) {
            Bank* b = per_launch[l][q];
            b->in_plan = true;
            if (L.dtype == RBFFD_F64) fill_desc(((BankDesc<double>*)(h + L.off))[q], *b, L.blocks);
            else fill_desc(((BankDesc<float>*)(h + L.off))[q], *b, L.blocks);
            L.blocks += L.tiled ? b->halo->nblocks : (b->grid->N + SEG_ROWS - 1) / SEG_ROWS;
            const double wb = L.dtype == RBFFD_F64 ? 8.0 : 4.0, ib = L.tiled ? 2.0 : 4.0;
            const bool coef = b->kind == KIND_ADVECT && !b->wf;
            L.bytes += (double)b->grid->N * (b->grid->n_pad * (L.nops * wb + ib) + wb * (4.0 * b->W + (coef ? 2.0 : 0.0)));
        }
    }
    if (off) RBFFD_CUDA_TRY(S->ctx, cudaMemcpyAsync(S->d_tab, S->h_tab, off, cudaMemcpyHostToDevice, S->stream));
    RBFFD_CUDA_TRY(S->ctx, cudaEventRecord(S->ev_tab, S->stream));
    return RBFFD_OK;
}

template <typename T, int W, int NOPS>
void launch_bank(const Launch& L, const BankDesc<T>* d, int stage, cudaStream_t s)
{
    if (L.tiled) k_stage_bank_tile<T, W, NOPS><<<L.blocks, SEG_ROWS, L.smem, s>>>(d, L.nbanks, stage);
    else k_stage_bank<T, W, NOPS><<<L.blocks, SEG_ROWS, 0, s>>>(d, L.nbanks, stage);
}

template <typename T, int W>
void launch_bank_w(const Launch& L, const BankDesc<T>* d, int stage, cudaStream_t s)
{
    switch (L.nops) {
    case 1: launch_bank<T, W, 1>(L, d, stage, s); break;
    case 2: launch_bank<T, W, 2>(L, d, stage, s); break;
    default: launch_bank<T, W, 3>(L, d, stage, s); break;
    }
}

// Allow the tiled instantiations TILE_SMEM_MAX of dynamic shared memory on the current device.
template <typename T, int W>
cudaError_t tile_attrs_w()
{
    cudaError_t e = cudaFuncSetAttribute(k_stage_bank_tile<T, W, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         TILE_SMEM_MAX);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_stage_bank_tile<T, W, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 TILE_SMEM_MAX);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_stage_bank_tile<T, W, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 TILE_SMEM_MAX);
    return e;
}

cudaError_t tile_attrs()
{
    cudaError_t e = tile_attrs_w<float, 1>();
    if (e == cudaSuccess) e = tile_attrs_w<float, 2>();
    if (e == cudaSuccess) e = tile_attrs_w<float, 4>();
    if (e == cudaSuccess) e = tile_attrs_w<float, 8>();
    if (e == cudaSuccess) e = tile_attrs_w<double, 1>();
    if (e == cudaSuccess) e = tile_attrs_w<double, 2>();
    if (e == cudaSuccess) e = tile_attrs_w<double, 4>();
    return e;
}

void launch_stage(const Launch& L, char* d, int stage, cudaStream_t s)
{
    if (L.dtype == RBFFD_F64) {
        const BankDesc<double>* t = (const BankDesc<double>*)(d + L.off);
        switch (L.W) {
        case 1: launch_bank_w<double, 1>(L, t, stage, s); break;
        case 2: launch_bank_w<double, 2>(L, t, stage, s); break;
        default: launch_bank_w<double, 4>(L, t, stage, s); break;
        }
    } else {
        const BankDesc<float>* t = (const BankDesc<float>*)(d + L.off);
        switch (L.W) {
        case 1: launch_bank_w<float, 1>(L, t, stage, s); break;
        case 2: launch_bank_w<float, 2>(L, t, stage, s); break;
        case 4: launch_bank_w<float, 4>(L, t, stage, s); break;
        default: launch_bank_w<float, 8>(L, t, stage, s); break;
        }
    }
}

// Issue nsteps RK4 steps for the planned banks between the events e0 and e1
// (returns at once; the batch runs on the stepping stream).
int launch_steps(rbffd_server* S, const std::vector<Launch>& plan, int nsteps, cudaEvent_t e0, cudaEvent_t e1,
                 long long* launches, double* bytes)
{
    char* d = (char*)S->d_tab;
    for (const Launch& L : plan) *bytes += 4.0 * nsteps * L.bytes;
    RBFFD_CUDA_TRY(S->ctx, cudaEventRecord(e0, S->stream));
    for (int step = 0; step < nsteps; step++)
        for (int stage = 0; stage < 4; stage++)
            for (const Launch& L : plan) {
                launch_stage(L, d, stage, S->stream);
                ++*launches;
            }
    RBFFD_CUDA_TRY(S->ctx, cudaGetLastError());
    RBFFD_CUDA_TRY(S->ctx, cudaEventRecord(e1, S->stream));
    return RBFFD_OK;
}

// New layout of a bank whose membership changed: its remaining requests in
// order, then the joining ones, in columns 0..K-1 at stride K rounded up to a
// power of two (written into xa, which is free between steps, then swapped
// with u).  Stepping thread, between batches.
template <typename T>
void bank_repack(Bank& b, cudaStream_t s)
{
    std::vector<Request*> keep;
    std::vector<int> from;
    for (int c = 0; c < (int)b.cols.size(); c++)
        if (b.cols[c]) {
            keep.push_back(b.cols[c]);
            from.push_back(c);
        }
    for (Request* r : b.join) {
        keep.push_back(r);
        from.push_back(FROM_IO);
    }
    b.join.clear();
    b.dirty = false;
    const int K = (int)keep.size();
    if (K == 0) {
        b.cols.clear();
        return;
    }
    int W = 1;
    while (W < K) W *= 2;
    Repack<T> a;
    a.dst = (T*)b.xa;
    a.src = (const T*)b.u;
    a.wsrc = b.W;
    a.wdst = W;
    a.N = b.grid->N;
    a.perm = b.grid->d_perm;
    for (int c = 0; c < BANK_W_MAX; c++) {
        a.from[c] = c < K ? from[c] : FROM_ZERO;
        a.io[c] = c < K ? keep[c]->d_io : nullptr;
    }
    k_repack<T><<<(a.N + 255) / 256, 256, 0, s>>>(a);
    std::swap(b.u, b.xa);
    if (b.comp) {  // the compensation follows its column into xb (also free between steps); joiners start at 0
        Repack<T> ac = a;
        ac.dst = (T*)b.xb;
        ac.src = (const T*)b.comp;
        for (int c = 0; c < BANK_W_MAX; c++)
            if (ac.from[c] == FROM_IO) ac.from[c] = FROM_ZERO;
        k_repack<T><<<(a.N + 255) / 256, 256, 0, s>>>(ac);
        std::swap(b.comp, b.xb);
    }
    b.W = W;
    b.cols.assign(W, nullptr);
    for (int c = 0; c < K; c++) {
        b.cols[c] = keep[c];
        keep[c]->col = c;
        keep[c]->inserted = true;
    }
}

template <typename T>
void column_out(const Request& r, cudaStream_t s)
{
    const Bank& b = *r.bank;
    const int N = b.grid->N;
    k_column_out<T><<<(N + 255) / 256, 256, 0, s>>>((const T*)b.u, (const T*)b.comp, b.W, r.col, r.d_io,
                                                    b.grid->d_perm, N);
}

// A batch of steps in flight.  Requests that finish with it leave the banks
// when it is issued (their columns are read out into their I/O buffers on the
// stepping stream right behind it); it completes once the next batch is
// already queued, so the device does not wait for the host between batches.
struct Flight {
    bool on = false, launched = false;
    int slot = 0, nsteps = 0, rc = RBFFD_OK;
    long long launches = 0;
    double bytes = 0.0, nu = 0.0;
    std::vector<std::shared_ptr<Request>> leave;  // finish with this batch (status set when issued)
    std::vector<Bank*> banks;                     // banks its tables reference
};

// Completes a batch (stepping thread, without S->mu): waits for it, copies
// its finished requests' results to their callers on the copy stream (behind
// the read-out), frees their I/O buffers, then publishes results, statistics
// and the banks that no queued batch references any more.
void complete(rbffd_server* S, Flight& f, const std::vector<Bank*>& still_used)
{
    double secs = 0.0;
    int rc = f.rc;
    if (f.launched) {
        cudaError_t e = cudaEventSynchronize(S->ev[f.slot][1]);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, S->ev[f.slot][0], S->ev[f.slot][1]);
        if (e != cudaSuccess && rc == RBFFD_OK) rc = cuda_error(S->ctx, e, "batch");
        secs = ms * 1e-3;
    }
    if (!f.leave.empty()) {
        cudaError_t e = cudaStreamWaitEvent(S->cstream, S->ev[f.slot][2], 0);
        for (auto& rp : f.leave) {
            Request& r = *rp;
            if (rc != RBFFD_OK && r.status == RBFFD_OK) r.status = rc;
            if (r.status == RBFFD_OK && e == cudaSuccess)
                e = cudaMemcpyAsync(r.p.out, r.d_io, (size_t)r.p.grid->N * sizeof(double), cudaMemcpyDeviceToHost,
                                    S->cstream);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(S->cstream);
        const int copy_rc = e == cudaSuccess ? RBFFD_OK : cuda_error(S->ctx, e, "request result");
        for (auto& rp : f.leave) {
            Request& r = *rp;
            if (copy_rc != RBFFD_OK && r.status == RBFFD_OK) r.status = copy_rc;
            if (r.d_io) cudaFreeAsync(r.d_io, S->cstream);
            r.d_io = nullptr;
            ctx_account(S->ctx, 0, (size_t)r.p.grid->N * sizeof(double));
        }
    }
    std::lock_guard<std::mutex> lk(S->mu);
    if (f.launched && rc == RBFFD_OK && f.nsteps > 0) S->step_s = secs / f.nsteps;
    S->st.ticks++;
    S->st.launches += f.launches;
    S->st.node_updates += f.nu;
    S->st.gpu_busy_s += secs;
    S->st.stage_bytes += f.bytes;
    for (auto& rp : f.leave) {
        Request& r = *rp;
        Bank* b = r.bank;
        S->owned -= std::min(S->owned, (size_t)r.p.grid->N * sizeof(double));
        if (--b->members == 0) b->idle_since = Clock::now();
        r.bank = nullptr;
        S->finishing--;
        finish_request(r, r.status);
        if (r.status == RBFFD_OK) S->st.completed++;
        else if (r.status == RBFFD_ERR_CANCELLED) S->st.cancelled++;
        else S->st.failed++;
    }
    for (Bank* b : f.banks)
        if (std::find(still_used.begin(), still_used.end(), b) == still_used.end()) b->in_plan = false;
    if (!f.leave.empty()) {
        S->cv_done.notify_all();
        S->cv_admit.notify_one();  // columns and memory to admit the next requests
    }
    f = Flight();
}

// Stepping thread: admitted requests join at step boundaries; batches of RK4
// steps for every bank with active columns, the next batch queued before the
// previous one is completed.
void worker_loop(rbffd_server* S)
{
    cudaSetDevice(S->ctx->device);
    std::unique_lock<std::mutex> lk(S->mu);
    bool changed = true;
    std::vector<Launch> plan;
    std::vector<Bank*> plan_banks;  // banks the current tables reference
    Flight flight;                  // the batch in flight
    int slot = 0;
    for (;;) {
        const bool hold = S->paused && !S->stop;
        std::vector<std::shared_ptr<Request>> joining;
        if (!hold) {
            joining.swap(S->ready);
            for (auto& r : joining) S->active.push_back(r);
            S->st.max_active_seen = std::max<long long>(
                S->st.max_active_seen, (long long)(S->active.size() + (flight.on ? flight.leave.size() : 0)));
        }
        if (S->active.empty() || hold) {
            if (flight.on) {  // finish the batch in flight first
                lk.unlock();
                complete(S, flight, plan_banks);
                lk.lock();
                continue;
            }
            if (S->active.empty()) {
                for (auto& b : S->banks) b->in_plan = false;  // no batch in flight
                if (S->stop && S->admitter_done && S->ready.empty()) break;
            }
            S->cv_work.wait(lk);
            continue;
        }
        for (auto& r : joining) {
            r->bank->join.push_back(r.get());
            r->bank->dirty = true;
        }
        std::vector<Bank*> dirty;  // banks with requests (not freeable meanwhile) whose membership changed
        for (auto& b : S->banks)
            if (b->dirty) {
                if (b->members > 0) dirty.push_back(b.get());
                else bank_repack<float>(*b, S->stream);  // no request left: just forget the layout
            }
        lk.unlock();
        int rc = RBFFD_OK;
        for (Bank* b : dirty) {  // new layouts and initial states, behind the batch in flight
            if (b->dtype == RBFFD_F64) bank_repack<double>(*b, S->stream);
            else bank_repack<float>(*b, S->stream);
        }
        if (!dirty.empty()) {
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) rc = cuda_error(S->ctx, e, "bank repack");
        }
        lk.lock();
        changed |= !dirty.empty();
        std::vector<std::shared_ptr<Request>> act = S->active;
        int nsteps = TICK_MAX_STEPS;
        if (S->step_s > 0.0) nsteps = std::max(1, std::min(TICK_MAX_STEPS, (int)(TICK_TARGET_S / S->step_s)));
        for (auto& r : act) nsteps = std::min(nsteps, r->p.nsteps - r->steps_done);
        if (changed && rc == RBFFD_OK) {
            rc = upload_tables(S, plan);
            changed = false;
            plan_banks.clear();
            for (auto& b : S->banks)
                if (b->in_plan) plan_banks.push_back(b.get());
        }
        for (Bank* b : flight.banks) b->in_plan = true;  // still running
        lk.unlock();
        Flight nf;
        nf.on = true;
        nf.slot = slot;
        slot ^= 1;
        nf.nsteps = nsteps;
        nf.banks = plan_banks;
        if (rc == RBFFD_OK) {
            rc = launch_steps(S, plan, nsteps, S->ev[nf.slot][0], S->ev[nf.slot][1], &nf.launches, &nf.bytes);
            nf.launched = rc == RBFFD_OK;
        }
        nf.rc = rc;
        for (auto& r : act) {
            r->steps_done += nsteps;
            nf.nu += (double)r->p.grid->N * nsteps;
            bool cancel;
            {
                std::lock_guard<std::mutex> g(S->mu);
                cancel = r->cancel;
            }
            int st;
            if (rc != RBFFD_OK) st = rc;
            else if (cancel) st = RBFFD_ERR_CANCELLED;
            else if (r->steps_done >= r->p.nsteps) st = RBFFD_OK;
            else continue;
            if (st == RBFFD_OK && r->inserted) {  // read the column out right behind the batch
                if (r->bank->dtype == RBFFD_F64) column_out<double>(*r, S->stream);
                else column_out<float>(*r, S->stream);
            }
            r->status = st;
            nf.leave.push_back(r);
        }
        cudaEventRecord(S->ev[nf.slot][2], S->stream);
        if (cudaGetLastError() != cudaSuccess)
            for (auto& r : nf.leave)
                if (r->status == RBFFD_OK) r->status = set_error(S->ctx, RBFFD_ERR_CUDA, "result read-out");
        lk.lock();
        for (auto& rp : nf.leave) {  // leave the banks now: the next layouts are built without them
            Bank* b = rp->bank;
            if (rp->col >= 0 && rp->col < (int)b->cols.size() && b->cols[rp->col] == rp.get()) b->cols[rp->col] = nullptr;
            b->dirty = true;
            S->active.erase(std::find(S->active.begin(), S->active.end(), rp));
            S->finishing++;
            changed = true;
        }
        lk.unlock();
        if (flight.on) complete(S, flight, plan_banks);
        flight = std::move(nf);
        lk.lock();
    }
}

}  // namespace

extern "C" int rbffd_server_start(rbffd_ctx* ctx, double hbm_fraction, int max_active, rbffd_server** out)
{
    if (!ctx || !out || !(hbm_fraction > 0.0 && hbm_fraction <= 1.0)) return RBFFD_ERR_INVALID;
    *out = nullptr;
    cudaSetDevice(ctx->device);
    size_t free_b = 0, total_b = 0;
    RBFFD_CUDA_TRY(ctx, cudaMemGetInfo(&free_b, &total_b));
    rbffd_server* S = new (std::nothrow) rbffd_server();
    if (!S) return RBFFD_ERR_OOM;
    S->ctx = ctx;
    S->budget = (size_t)(hbm_fraction * (double)total_b);
    S->max_active = max_active > 0 ? max_active : 0;
    // bank tables for a few hundred banks, held from the start so that they
    // count against the budget before the first admission
    const size_t tab = TABLE_BYTES0;
    cudaError_t e = cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->astream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->cstream, cudaStreamNonBlocking);
    for (int k = 0; k < 2; k++)
        for (int j = 0; j < 3 && e == cudaSuccess; j++)
            e = j < 2 ? cudaEventCreate(&S->ev[k][j]) : cudaEventCreateWithFlags(&S->ev[k][j], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->ev_tab, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost(&S->h_tab, tab);
    if (e == cudaSuccess) e = tile_attrs();
    int rc = e == cudaSuccess ? RBFFD_OK : cuda_error(ctx, e, "rbffd_server_start");
    if (rc == RBFFD_OK && (rc = dev_alloc(ctx, &S->d_tab, tab)) == RBFFD_OK) S->tab_cap = tab;
    if (rc != RBFFD_OK) {
        dev_free(ctx, S->d_tab, S->tab_cap);
        if (S->h_tab) cudaFreeHost(S->h_tab);
        for (int k = 0; k < 2; k++)
            for (int j = 0; j < 3; j++)
                if (S->ev[k][j]) cudaEventDestroy(S->ev[k][j]);
        if (S->ev_tab) cudaEventDestroy(S->ev_tab);
        if (S->cstream) cudaStreamDestroy(S->cstream);
        if (S->astream) cudaStreamDestroy(S->astream);
        if (S->stream) cudaStreamDestroy(S->stream);
        delete S;
        return rc;
    }
    S->st.budget_bytes = (double)S->budget;
    S->worker = std::thread(worker_loop, S);
    S->admitter = std::thread(admission_loop, S);
    *out = S;
    return RBFFD_OK;
}

extern "C" int rbffd_server_submit(rbffd_server* S, const rbffd_request* req, uint64_t* id)
{
    if (!S || !req || !id) return RBFFD_ERR_INVALID;
    rbffd_ctx* ctx = S->ctx;
    rbffd_grid* g = req->grid;
    if (!g || !req->u0 || !req->out || req->nsteps < 0 || !(req->dt == req->dt))
        return set_error(ctx, RBFFD_ERR_INVALID, "a request needs a grid, u0, out, nsteps >= 0 and a dt");
    if (g->ctx != ctx) return set_error(ctx, RBFFD_ERR_INVALID, "request grid belongs to another context");
    const rbffd_pde_params& p = req->pde;
    if (p.ntracers != 1) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "served requests carry one tracer");
    if (p.dtype != RBFFD_F32 && p.dtype != RBFFD_F64) return set_error(ctx, RBFFD_ERR_INVALID, "bad dtype %d", p.dtype);
    unsigned ops;
    if (p.rhs_kind == RBFFD_RHS_HEAT) {
        ops = RBFFD_LSFC;
    } else if (p.rhs_kind == RBFFD_RHS_COSINE_BELL || p.rhs_kind == RBFFD_RHS_ADVECTION) {
        ops = RBFFD_LAMBDA | RBFFD_THETA | (p.use_hv ? RBFFD_HV : 0u);
        if (p.rhs_kind == RBFFD_RHS_ADVECTION && (!p.cu || !p.cv))
            return set_error(ctx, RBFFD_ERR_INVALID, "advection needs per-node coefficients cu and cv");
        if (p.rhs_kind == RBFFD_RHS_COSINE_BELL && p.sphere_radius == 0.0)
            return set_error(ctx, RBFFD_ERR_INVALID, "cosine bell needs a nonzero sphere radius");
    } else {
        return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "rhs_kind %d", p.rhs_kind);
    }
    for (int b = 0; b < 16; b++)
        if ((ops >> b & 1u) && !g->d_w64[b])
            return set_error(ctx, RBFFD_ERR_STATE, "weights of operator 0x%x are not on the device", 1u << b);
    // the most a request can add: a new bank and its I/O buffer
    const size_t need = bank_bytes(g, p) + (size_t)g->N * sizeof(double);
    auto r = std::make_shared<Request>();
    r->p = *req;
    const int N = g->N;
    r->u0.assign(req->u0, req->u0 + N);
    if (p.rhs_kind == RBFFD_RHS_ADVECTION) {
        r->cu.assign(p.cu, p.cu + N);
        r->cv.assign(p.cv, p.cv + N);
    }
    r->p.pde.cu = r->p.pde.cv = nullptr;
    r->p.u0 = r->u0.data();
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return set_error(ctx, RBFFD_ERR_STATE, "server is stopping");
    // memory the server cannot free (grids, the caller's own PDEs) plus this request
    const size_t held = ctx_held(ctx);
    if (held - std::min(held, S->owned) + need > S->budget)
        return set_error(ctx, RBFFD_ERR_BUDGET, "request needing %zu bytes can never fit the budget of %zu bytes", need,
                         S->budget);
    r->id = S->next_id++;
    r->t_submit = Clock::now();
    S->st.submitted++;
    if (req->nsteps == 0) {  // nothing to advance: the result is the initial state
        memcpy(req->out, req->u0, (size_t)N * sizeof(double));
        r->t_admit = r->t_submit;
        r->admitted = true;
        finish_request(*r, RBFFD_OK);
        S->st.completed++;
    } else {
        S->pending.push_back(r);
        S->cv_admit.notify_one();
    }
    S->all[r->id] = r;
    *id = r->id;
    return RBFFD_OK;
}

extern "C" int rbffd_server_poll(rbffd_server* S, uint64_t id, int* done, int* status, double* latency_s,
                                 double* queue_s)
{
    if (!S || !done) return RBFFD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->all.find(id);
    if (it == S->all.end()) return set_error(S->ctx, RBFFD_ERR_INVALID, "unknown request %llu", (unsigned long long)id);
    const Request& r = *it->second;
    *done = r.done;
    if (status) *status = r.done ? r.status : RBFFD_OK;
    if (latency_s) *latency_s = r.done ? std::chrono::duration<double>(r.t_done - r.t_submit).count() : -1.0;
    if (queue_s) *queue_s = r.admitted ? std::chrono::duration<double>(r.t_admit - r.t_submit).count() : -1.0;
    return RBFFD_OK;
}

extern "C" int rbffd_server_wait(rbffd_server* S, uint64_t id, double timeout_s)
{
    if (!S || !(timeout_s >= 0.0)) return RBFFD_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->all.find(id);
    if (it == S->all.end()) return set_error(S->ctx, RBFFD_ERR_INVALID, "unknown request %llu", (unsigned long long)id);
    std::shared_ptr<Request> r = it->second;
    if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return r->done != 0; }))
        return RBFFD_ERR_TIMEOUT;
    return r->status;
}

extern "C" int rbffd_server_wait_idle(rbffd_server* S, double timeout_s)
{
    if (!S || !(timeout_s >= 0.0)) return RBFFD_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                             [&] {
                                 return S->pending.empty() && S->ready.empty() && S->active.empty() &&
                                        S->finishing == 0;
                             }))
        return RBFFD_ERR_TIMEOUT;
    return RBFFD_OK;
}

extern "C" int rbffd_server_cancel(rbffd_server* S, uint64_t id)
{
    if (!S) return RBFFD_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->all.find(id);
    if (it == S->all.end()) return set_error(S->ctx, RBFFD_ERR_INVALID, "unknown request %llu", (unsigned long long)id);
    std::shared_ptr<Request> r = it->second;
    if (r->done) return RBFFD_OK;
    r->cancel = true;
    S->cv_admit.notify_one();
    S->cv_work.notify_one();
    S->cv_done.wait(lk, [&] { return r->done != 0; });
    return RBFFD_OK;
}

extern "C" int rbffd_server_get_stats(rbffd_server* S, rbffd_server_stats* out)
{
    if (!S || !out) return RBFFD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->st;
    out->pending = (long long)S->pending.size();
    out->active = (long long)(S->active.size() + S->ready.size()) + S->finishing;
    out->held_bytes = (double)ctx_held(S->ctx);
    return RBFFD_OK;
}

extern "C" int rbffd_server_set_admission_order(rbffd_server* S, int order)
{
    if (!S || (order != RBFFD_ADMIT_ARRIVAL && order != RBFFD_ADMIT_SHORTEST)) return RBFFD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    S->order = order;
    S->cv_admit.notify_all();
    return RBFFD_OK;
}

extern "C" int rbffd_server_pause(rbffd_server* S, int paused)
{
    if (!S) return RBFFD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    S->paused = paused != 0;
    S->cv_work.notify_all();
    return RBFFD_OK;
}

extern "C" int rbffd_server_inject_admission_failures(rbffd_server* S, int count)
{
    if (!S || count < 0) return RBFFD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    S->inject_fail = count;
    return RBFFD_OK;
}

extern "C" int rbffd_server_stop(rbffd_server* S)
{
    if (!S) return RBFFD_ERR_INVALID;
    {
        // the admission thread cancels the pending requests; the stepping thread
        // finishes the admitted ones
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_admit.notify_all();
    S->cv_work.notify_all();
    if (S->admitter.joinable()) S->admitter.join();
    if (S->worker.joinable()) S->worker.join();
    cudaSetDevice(S->ctx->device);
    cudaStreamSynchronize(S->stream);
    cudaStreamSynchronize(S->astream);
    cudaStreamSynchronize(S->cstream);
    for (auto& b : S->banks) bank_free_memory(S->ctx, *b);
    S->banks.clear();
    if (S->h_tab) cudaFreeHost(S->h_tab);
    dev_free(S->ctx, S->d_tab, S->tab_cap);
    for (int k = 0; k < 2; k++)
        for (int j = 0; j < 3; j++) cudaEventDestroy(S->ev[k][j]);
    cudaEventDestroy(S->ev_tab);
    cudaStreamDestroy(S->cstream);
    cudaStreamDestroy(S->astream);
    cudaStreamDestroy(S->stream);
    delete S;
    return RBFFD_OK;
}
