// K3: classical RK4 with the derivative application and the PDE right-hand
// side fused into each stage (TimeDependentPDE::advanceRungeKutta4,
// src/pdes/time_dependent_pde.cpp:172-304; the reference GPU form is
// evaluateRK4_classic / advanceRK4_classic, src/cl_kernels/rk4_thread_per_stencil.cl).
//
// One launch per stage.  Stage kernel, per stencil row i (and tracer t):
//   d_k   = sum_s W_k[s][i] * x[idx[s][i]]            (K = 1..3 operators)
//   f     = RHS(d_0, d_1, d_2)                         (cosine bell / heat / advection)
//   stage 0:  acc = f;           xnext = u + (dt/2) f
//   stage 1:  acc = acc + 2 f;   xnext = u + (dt/2) f
//   stage 2:  acc = acc + 2 f;   xnext = u + dt f
//   stage 3:  u   = u + (dt/6)(acc + f)
// which is the reference's update u + dt/6 (k1 + 2k2 + 2k3 + k4) with the sum
// evaluated in the same left-to-right order.  Four state buffers (u, two
// ping-pong stage inputs, acc) replace the reference's eight
// (time_dependent_pde_cl.cpp:677-708).  The stage input x is gathered while
// xnext is written, so the two never alias; stage 3 writes u[i] only from row
// i, which no other row of that launch gathers (it gathers x).
//
// FP64 arithmetic uses explicit round-to-nearest intrinsics so the order of
// operations is fixed: with one lane per row the result equals a CPU loop
// that fuses the same multiply-adds.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <type_traits>

#include "ell.cuh"
#include "internal.h"
#include "tma.cuh"

int grid_apply_dev(rbffd_grid* g, int op, int dtype, int T_tr, const void* u, void* out, int start, int count, int G,
                   cudaStream_t s);

template <typename T>
struct StageParams {
    const int* __restrict__ idx;
    const T* __restrict__ w0;
    const T* __restrict__ w1;
    const T* __restrict__ w2;
    const T* __restrict__ cu;
    const T* __restrict__ cv;
    const T* x;   // gathered stage input (never written during a launch)
    T* u;         // u_n (written in stage 3)
    T* xnext;     // next stage input
    T* acc;       // RK accumulator
    T c;          // dt/2, dt/2, dt, dt/6 for stages 0..3
    T kappa;
    int N, nc, T_tr, stage;  // nc: 4-slot chunks per row (sliced ELL, ell.cuh)
    T* comp = nullptr;       // stage 3 of an FP32 PDE with a compensated state: minus what u lost
};

// Right-hand side and the stage update for one (row, tracer) value.  PLAIN:
// every multiply-add rounded twice (madd, ell.cuh), the reference build's
// arithmetic; otherwise fused.
template <typename T, int KIND, bool HV, bool PLAIN = false>
__device__ __forceinline__ void stage_update(const StageParams<T>& p, int i, size_t e, T d0, T d1, T d2, T cu, T cv)
{
    T f;
    if (KIND == KIND_ADVECT) {
        // CosineBell::solve: f = -((vel_u/a) * dlambda + (vel_v/a) * dtheta) (+ hv), cosine_bell.cpp:47-57
        f = -madd<T, PLAIN>(cu, d0, Ar<T>::mul(cv, d1));
        if (HV) f = Ar<T>::add(f, d2);
    } else {
        f = Ar<T>::mul(p.kappa, d0);
    }
    T ui = p.u[e];
    switch (p.stage) {
    case 0:
        p.acc[e] = f;
        p.xnext[e] = madd<T, PLAIN>(p.c, f, ui);
        break;
    case 1:
    case 2:
        p.acc[e] = Ar<T>::add(p.acc[e], Ar<T>::mul(T(2), f));
        p.xnext[e] = madd<T, PLAIN>(p.c, f, ui);
        break;
    default:
        if (!std::is_same<T, double>::value && p.comp) {
            // compensated: add the increment with Knuth's TwoSum and keep minus the part
            // the rounded sum lost; the next step adds it back (u - comp is the state)
            const T y = Ar<T>::sub(Ar<T>::mul(p.c, Ar<T>::add(p.acc[e], f)), p.comp[e]);
            const T s = Ar<T>::add(ui, y);
            const T yb = Ar<T>::sub(s, ui);
            const T lost = Ar<T>::add(Ar<T>::sub(ui, Ar<T>::sub(s, yb)), Ar<T>::sub(y, yb));
            p.u[e] = s;
            p.comp[e] = -lost;
        } else {
            p.u[e] = madd<T, PLAIN>(p.c, Ar<T>::add(p.acc[e], f), ui);
        }
        break;
    }
}

// Single tracer, G lanes per row; lane g handles the 4-slot chunks g, g+G, ...
// With G == 1 the slots are accumulated in stencil order.
template <typename T, int KIND, bool HV, int G, bool PLAIN = false>
__global__ void __launch_bounds__(512) k_stage_scalar(StageParams<T> p)
{
    int gt = blockIdx.x * blockDim.x + threadIdx.x;
    int i = gt / G, lane = gt % G;
    bool active = i < p.N;
    int ii = active ? i : 0;
    T d0 = T(0), d1 = T(0), d2 = T(0);
#pragma unroll 2
    for (int c = lane; c < p.nc; c += G) {
        const size_t o = sell_off(ii, c, p.nc);
        int4 j = ld_idx4(p.idx + o);
        T x[4] = {__ldg(p.x + j.x), __ldg(p.x + j.y), __ldg(p.x + j.z), __ldg(p.x + j.w)};
        T w[4];
        ld_w4(p.w0 + o, w);
#pragma unroll
        for (int k = 0; k < 4; k++) d0 = madd<T, PLAIN>(w[k], x[k], d0);
        if (KIND == KIND_ADVECT) {
            ld_w4(p.w1 + o, w);
#pragma unroll
            for (int k = 0; k < 4; k++) d1 = madd<T, PLAIN>(w[k], x[k], d1);
            if (HV) {
                ld_w4(p.w2 + o, w);
#pragma unroll
                for (int k = 0; k < 4; k++) d2 = madd<T, PLAIN>(w[k], x[k], d2);
            }
        }
    }
    if (G > 1) {
        d0 = group_sum<G>(d0);
        if (KIND == KIND_ADVECT) {
            d1 = group_sum<G>(d1);
            if (HV) d2 = group_sum<G>(d2);
        }
    }
    if (!active || lane != 0) return;
    T cu = T(0), cv = T(0);
    if (KIND == KIND_ADVECT) {
        cu = p.cu[i];
        cv = p.cv[i];
    }
    stage_update<T, KIND, HV, PLAIN>(p, i, (size_t)i, d0, d1, d2, cu, cv);
}

// ---------------------------------------------------------------------------
// Cluster-resident RK4: every step of an advance in one launch of one
// thread-block cluster of C CTAs.  CTA q holds rows q R .. q R + R-1 (one
// thread per row): the rows' weights of every operator, their stencils as
// positions in the CTA's halo (the unique nodes its rows read, each held by
// its owning CTA and local row) in shared memory for the whole launch, and
// its rows of u, the two stage inputs and the accumulator.  Every row sums
// its slots in stencil order from the CTA's halo buffer and applies
// stage_update, the per-stage kernels' arithmetic, so the result is
// k_stage_scalar's with one lane per row bit for bit; it then stores its new
// value straight into the other halo buffer of every CTA whose halo holds the
// row (distributed shared memory; a host-built push list per row), and one
// cluster barrier (release / acquire) separates the stages: stage s reads
// halo buffer s mod 2 and fills buffer s + 1 mod 2.  u is read at the start
// and written back at the end.
constexpr int RES_MAX_CLUSTER = 16;

template <typename T>
struct ResidentParams {
    const int* pptr;               // [C][R + 1]: each row's range in pdst
    const unsigned short* pdst;    // [C][P]: halo positions a row's value goes to, consumer CTA << 12 | position
    const unsigned short* lidx;    // [C][n4][R]: halo position of each stencil slot
    const T* w[3];                 // the operators streamed (sliced ELL)
    const T* cu;
    const T* cv;
    T* u;                          // state, internal order
    T c[4];                        // dt/2, dt/2, dt, dt/6 (rounded to T as the per-stage launches do)
    T kappa;
    int N, nc, R, K, H, P, nsteps;
};

// Body of the cluster-resident kernels.  NCR = 0: each row's weights and halo
// positions in shared memory (any stencil size); NCR > 0: stencils of exactly
// NCR 4-slot chunks with the row's weights and halo positions in registers for
// the whole launch (at most 256 rows per CTA), so a slot costs one
// shared-memory load (the halo value) instead of up to four.
template <typename T, int KIND, bool HV, bool PLAIN, int NCR>
__device__ __forceinline__ void rk4_cluster_body(const ResidentParams<T>& rp)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int KC = KIND == KIND_HEAT ? 1 : (HV ? 3 : 2);
    constexpr int N4R = 4 * NCR;
    const int R = rp.R, n4 = NCR > 0 ? N4R : 4 * rp.nc, H = rp.H, P = rp.P;
    const int K = NCR > 0 ? 0 : rp.K;          // operators kept in shared memory
    T* ws = reinterpret_cast<T*>(smem_raw);  // [K][n4][R]
    T* xs = ws + (size_t)K * n4 * R;           // u, xa, xb, acc, cu, cv: [6][R]
    T* us = xs;
    T* xa = xs + R;
    T* xb = xs + 2 * R;
    T* acc = xs + 3 * R;
    T* cus = xs + 4 * R;
    T* cvs = xs + 5 * R;
    T* hb0 = xs + 6 * R;                                                  // [2][H] halo buffers
    T* hb1 = hb0 + H;
    unsigned short* pd = reinterpret_cast<unsigned short*>(hb1 + H);     // [P] this CTA's push list
    unsigned short* lx = pd + P;                                          // [n4][R] (NCR = 0)
    const int q = (int)cl.block_rank(), r = threadIdx.x;
    const int i = q * R + r;
    const bool active = i < rp.N;
    T wr[NCR > 0 ? KC : 1][NCR > 0 ? N4R : 1];
    unsigned lr[NCR > 0 ? N4R / 2 : 1];  // two 16-bit halo positions per register
    for (int e = r; e < P; e += R) pd[e] = rp.pdst[(size_t)q * P + e];
    const int pb = rp.pptr[(size_t)q * (R + 1) + r], pe = rp.pptr[(size_t)q * (R + 1) + r + 1];
    if constexpr (NCR > 0) {
#pragma unroll
        for (int sl = 0; sl < N4R; sl++) {
            const size_t o = active ? sell_elem(i, sl, NCR) : 0;
            const unsigned v = rp.lidx[((size_t)q * N4R + sl) * R + r];
            if (sl % 2 == 0)
                lr[sl / 2] = v;
            else
                lr[sl / 2] |= v << 16;
#pragma unroll
            for (int k = 0; k < KC; k++) wr[k][sl] = active ? rp.w[k][o] : T(0);
        }
    } else {
        for (int sl = 0; sl < n4; sl++) {
            const size_t o = active ? sell_elem(i, sl, rp.nc) : 0;
            lx[(size_t)sl * R + r] = rp.lidx[((size_t)q * n4 + sl) * R + r];
#pragma unroll
            for (int k = 0; k < 3; k++)
                if (k < K) ws[((size_t)k * n4 + sl) * R + r] = active ? rp.w[k][o] : T(0);
        }
    }
    const T u0 = active ? rp.u[i] : T(0);
    us[r] = u0;
    xa[r] = xb[r] = acc[r] = T(0);
    cus[r] = active && KIND == KIND_ADVECT ? rp.cu[i] : T(0);
    cvs[r] = active && KIND == KIND_ADVECT ? rp.cv[i] : T(0);
    cl.sync();  // every CTA of the cluster runs: its shared memory may be written
    auto push = [&](T* buf, T value) {
        for (int e = pb; e < pe; e++) {
            const unsigned v = pd[e];
            cl.map_shared_rank(buf, (int)(v >> 12))[v & 4095u] = value;
        }
    };
    push(hb0, u0);
    cl.sync();
    StageParams<T> p = {};
    p.kappa = rp.kappa;
    p.u = us;
    p.acc = acc;
    for (int step = 0; step < rp.nsteps; step++)
        for (int stage = 0; stage < 4; stage++) {
            const T* hin = (stage & 1) ? hb1 : hb0;
            p.xnext = stage == 0 ? xa : (stage == 1 ? xb : (stage == 2 ? xa : nullptr));
            p.c = stage == 0 ? rp.c[0] : (stage == 1 ? rp.c[1] : (stage == 2 ? rp.c[2] : rp.c[3]));
            p.stage = stage;
            if (active) {
                T d0 = T(0), d1 = T(0), d2 = T(0);
                if constexpr (NCR > 0) {
#pragma unroll
                    for (int c4 = 0; c4 < N4R; c4 += 4) {
                        T xj[4];
#pragma unroll
                        for (int k = 0; k < 4; k++) xj[k] = hin[(lr[(c4 + k) / 2] >> (16 * ((c4 + k) % 2))) & 0xFFFFu];
#pragma unroll
                        for (int k = 0; k < 4; k++) {
                            d0 = madd<T, PLAIN>(wr[0][c4 + k], xj[k], d0);
                            if constexpr (KC > 1) d1 = madd<T, PLAIN>(wr[KC > 1 ? 1 : 0][c4 + k], xj[k], d1);
                            if constexpr (KC > 2) d2 = madd<T, PLAIN>(wr[KC > 2 ? 2 : 0][c4 + k], xj[k], d2);
                        }
                    }
                } else {
                    for (int c4 = 0; c4 < n4; c4 += 4) {
                        T xj[4];
#pragma unroll
                        for (int k = 0; k < 4; k++) xj[k] = hin[lx[(size_t)(c4 + k) * R + r]];
#pragma unroll
                        for (int k = 0; k < 4; k++) {
                            const size_t e = (size_t)(c4 + k) * R + r;
                            d0 = madd<T, PLAIN>(ws[e], xj[k], d0);
                            if (KIND == KIND_ADVECT) {
                                d1 = madd<T, PLAIN>(ws[(size_t)n4 * R + e], xj[k], d1);
                                if (HV) d2 = madd<T, PLAIN>(ws[(size_t)2 * n4 * R + e], xj[k], d2);
                            }
                        }
                    }
                }
                stage_update<T, KIND, HV, PLAIN>(p, i, (size_t)r, d0, d1, d2, cus[r], cvs[r]);
                push((stage & 1) ? hb0 : hb1, stage == 3 ? us[r] : p.xnext[r]);  // the next stage's input
            }
            cl.sync();
        }
    if (active) rp.u[i] = us[r];
}

template <typename T, int KIND, bool HV, bool PLAIN>
__global__ void __launch_bounds__(1024) k_rk4_cluster(ResidentParams<T> rp)
{
    rk4_cluster_body<T, KIND, HV, PLAIN, 0>(rp);
}

// Register-resident weights: one CTA of at most 256 threads per SM, up to 255 registers each.
template <typename T, int KIND, bool HV, bool PLAIN, int NCR>
__global__ void __launch_bounds__(256, 1) k_rk4_cluster_rw(ResidentParams<T> rp)
{
    rk4_cluster_body<T, KIND, HV, PLAIN, NCR>(rp);
}

// Stencil chunk counts with a register-resident variant, and the register
// budget of a row's weights (32-bit registers).
constexpr int RES_RW_NC0 = 8, RES_RW_NC1 = 13, RES_RW_MAX_REGS = 192;

template <typename T, int KIND, bool HV>
constexpr bool res_rw_fits(int ncr)
{
    return (KIND == KIND_HEAT ? 1 : (HV ? 3 : 2)) * 4 * ncr * (int)sizeof(T) / 4 <= RES_RW_MAX_REGS;
}

// The kernel for ncr chunks held in registers (0, or a combination over the
// register budget: weights in shared memory).
template <typename T, int KIND, bool HV, bool PLAIN, int NCR>
static void (*res_kernel())(ResidentParams<T>)
{
    if constexpr (NCR > 0 && res_rw_fits<T, KIND, HV>(NCR))
        return k_rk4_cluster_rw<T, KIND, HV, PLAIN, NCR>;
    else
        return k_rk4_cluster<T, KIND, HV, PLAIN>;
}

// Shared memory of k_rk4_cluster for R rows per CTA, H halo positions, P push
// entries and K operators of n4 slots in shared memory.
template <typename T>
static size_t resident_smem(int K, int n4, int R, int H, int P)
{
    return ((size_t)K * n4 * R + 6 * (size_t)R + 2 * (size_t)H) * sizeof(T) +
           ((size_t)(K ? n4 : 0) * R + P) * sizeof(unsigned short);
}

template <typename T, int KIND, bool HV, bool PLAIN>
static int launch_resident_t(rbffd_pde* P, const ResidentParams<T>& rp, int C, size_t smem, cudaStream_t s,
                             bool check_only, int ncr)
{
    rbffd_ctx* ctx = P->ctx;
    auto kern = ncr == RES_RW_NC0   ? res_kernel<T, KIND, HV, PLAIN, RES_RW_NC0>()
                : ncr == RES_RW_NC1 ? res_kernel<T, KIND, HV, PLAIN, RES_RW_NC1>()
                                    : res_kernel<T, KIND, HV, PLAIN, 0>();
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess ||
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "cluster-resident RK4: kernel attributes refused");
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(rp.R, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) != cudaSuccess || nclusters < 1) {
        cudaGetLastError();
        return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "cluster-resident RK4: a cluster of %d CTAs with %zu bytes "
                         "of shared memory each does not fit", C, smem);
    }
    if (check_only) return RBFFD_OK;
    RBFFD_CUDA_TRY(ctx, cudaLaunchKernelEx(&cfg, kern, rp));
    return RBFFD_OK;
}

// Multiple tracers: state [N][T_tr]; VEC consecutive tracers per lane, loaded
// as one 16-byte vector; T_tr / VEC lanes per row share the row's weights and
// indices (same addresses: one transaction per chunk for the group).
template <typename T, int VEC>
struct VecT;
template <>
struct VecT<float, 4> { typedef float4 type; };
template <>
struct VecT<double, 2> { typedef double2 type; };
template <>
struct VecT<float, 1> { typedef float type; };
template <>
struct VecT<double, 1> { typedef double type; };

template <typename T, int VEC>
__device__ __forceinline__ void vload(const T* p, T (&v)[VEC])
{
    typedef typename VecT<T, VEC>::type V;
    static_assert(sizeof(V) == VEC * sizeof(T), "vector width");
    V t = __ldg(reinterpret_cast<const V*>(p));
    memcpy(v, &t, sizeof(V));
}

template <typename T, int VEC, int KIND, bool HV>
__global__ void __launch_bounds__(512) k_stage_vec(StageParams<T> p)
{
    int lpr = p.T_tr / VEC;
    int gt = blockIdx.x * blockDim.x + threadIdx.x;
    int i = gt / lpr, lane = gt % lpr;
    if (i >= p.N) return;
    T d0[VEC], d1[VEC], d2[VEC];
#pragma unroll
    for (int v = 0; v < VEC; v++) d0[v] = d1[v] = d2[v] = T(0);
    const size_t toff = (size_t)lane * VEC;
    for (int c = 0; c < p.nc; c++) {
        const size_t o = sell_off(i, c, p.nc);
        int4 j4 = ld_idx4(p.idx + o);
        const int jj[4] = {j4.x, j4.y, j4.z, j4.w};
        T wa[4], wb[4], wc[4];
        ld_w4(p.w0 + o, wa);
        if (KIND == KIND_ADVECT) {
            ld_w4(p.w1 + o, wb);
            if (HV) ld_w4(p.w2 + o, wc);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            T xj[VEC];
            vload<T, VEC>(p.x + (size_t)jj[k] * p.T_tr + toff, xj);
#pragma unroll
            for (int v = 0; v < VEC; v++) {
                d0[v] = Ar<T>::fma(wa[k], xj[v], d0[v]);
                if (KIND == KIND_ADVECT) {
                    d1[v] = Ar<T>::fma(wb[k], xj[v], d1[v]);
                    if (HV) d2[v] = Ar<T>::fma(wc[k], xj[v], d2[v]);
                }
            }
        }
    }
    T cu = T(0), cv = T(0);
    if (KIND == KIND_ADVECT) {
        cu = p.cu[i];
        cv = p.cv[i];
    }
#pragma unroll
    for (int v = 0; v < VEC; v++)
        stage_update<T, KIND, HV>(p, i, (size_t)i * p.T_tr + toff + v, d0[v], d1[v], d2[v], cu, cv);
}

// Tiled stage kernel: one CTA per block of R consecutive internal rows.  The
// CTA first copies the values of its halo (the unique nodes its rows' stencils
// reference, struct Halo) from global memory into shared memory -- each node's
// T values once, as 16-byte vectors -- then every row gathers from shared
// memory through 16-bit local indices.  The per-row arithmetic is that of
// k_stage_vec / k_stage_scalar: lane group (T/VEC lanes) x G chunk lanes per
// row, chunks in stencil order per lane.
struct TileParams {
    const int* __restrict__ ptr;
    const int* __restrict__ nodes;
    const unsigned short* __restrict__ lidx;
    const int* __restrict__ rows;  // [nblocks + 1]: block b owns rows [rows[b], rows[b+1])
    int R;                         // most rows in a block
    int N32;                       // rows of the sliced ELL arrays (N rounded up to 32)
};

// Chunks ahead that the prefetching variant of k_stage_tile asks L2 for.
constexpr int TILE_PF_DIST = 2;

// PF > 0: while working on chunk c, one lane per 128-byte line of a chunk's
// weights asks L2 for chunk c + PF * G (weights and local indices).  It pays
// where the weight stream comes from HBM and the kernel waits on it (FP64
// multi-tracer stages); where the weights stay in L2 the extra instructions
// cost more, so the autotuner decides.
// NV > 0: the vectors per node (T_tr / VEC) known at compile time, so node
// offsets in shared memory and state indices are shifts, not multiplies.
template <typename T, int VEC, int G, int KIND, bool HV, int PF = 0, int NV = 0>
__global__ void __launch_bounds__(1024) k_stage_tile(StageParams<T> p, TileParams tp)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sx = reinterpret_cast<T*>(smem_raw);
    typedef typename VecT<T, VEC>::type V;
    const int vpn = NV > 0 ? NV : p.T_tr / VEC;  // vectors per node (= lanes per tracer group of a row)
    const int ntr = NV > 0 ? NV * VEC : p.T_tr;
    const int L = vpn * G;         // threads per row
    const int b = blockIdx.x;
    const int h0 = __ldg(tp.ptr + b), hn = __ldg(tp.ptr + b + 1) - h0;
    for (int e = threadIdx.x; e < hn * vpn; e += blockDim.x) {
        const int h = e / vpn, v = e - h * vpn;
        const int node = __ldg(tp.nodes + h0 + h);
        reinterpret_cast<V*>(sx)[(size_t)h * vpn + v] =
            __ldg(reinterpret_cast<const V*>(p.x + (size_t)node * ntr) + v);
    }
    __syncthreads();
    const int lr = threadIdx.x % L, rl = threadIdx.x / L;
    const int i = __ldg(tp.rows + b) + rl;
    const bool active = i < __ldg(tp.rows + b + 1);
    const int tv = lr % vpn, g = lr / vpn;
    T d0[VEC], d1[VEC], d2[VEC];
#pragma unroll
    for (int v = 0; v < VEC; v++) d0[v] = d1[v] = d2[v] = T(0);
    if (active) {
        constexpr int RPL = 128 / (4 * (int)sizeof(T));  // rows per 128-byte line of one chunk
        const bool lead = PF > 0 && lr == 0 && (i % RPL) == 0;
#pragma unroll 2
        for (int c = g; c < p.nc; c += G) {
            const size_t o = sell_off(i, c, p.nc);
            if (PF > 0 && lead && c + PF * G < p.nc) {
                const size_t q = sell_off(i, c + PF * G, p.nc);
                prefetch_l2(p.w0 + q);
                if (KIND == KIND_ADVECT) {
                    prefetch_l2(p.w1 + q);
                    if (HV) prefetch_l2(p.w2 + q);
                }
                prefetch_l2(tp.lidx + q);
            }
            const ushort4 l4 = __ldg(reinterpret_cast<const ushort4*>(tp.lidx + o));
            const int ll[4] = {l4.x, l4.y, l4.z, l4.w};
            T wa[4], wb[4], wc[4];
            ld_w4(p.w0 + o, wa);
            if (KIND == KIND_ADVECT) {
                ld_w4(p.w1 + o, wb);
                if (HV) ld_w4(p.w2 + o, wc);
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                T xj[VEC];
                const V t = reinterpret_cast<const V*>(sx)[(size_t)ll[k] * vpn + tv];
                memcpy(xj, &t, sizeof(V));
#pragma unroll
                for (int v = 0; v < VEC; v++) {
                    d0[v] = Ar<T>::fma(wa[k], xj[v], d0[v]);
                    if (KIND == KIND_ADVECT) {
                        d1[v] = Ar<T>::fma(wb[k], xj[v], d1[v]);
                        if (HV) d2[v] = Ar<T>::fma(wc[k], xj[v], d2[v]);
                    }
                }
            }
        }
    }
    if (G > 1) {
#pragma unroll
        for (int m = G / 2; m > 0; m >>= 1)
#pragma unroll
            for (int v = 0; v < VEC; v++) {
                d0[v] += __shfl_xor_sync(0xffffffffu, d0[v], m * vpn, L);
                if (KIND == KIND_ADVECT) {
                    d1[v] += __shfl_xor_sync(0xffffffffu, d1[v], m * vpn, L);
                    if (HV) d2[v] += __shfl_xor_sync(0xffffffffu, d2[v], m * vpn, L);
                }
            }
    }
    if (!active || g != 0) return;
    T cu = T(0), cv = T(0);
    if (KIND == KIND_ADVECT) {
        cu = p.cu[i];
        cv = p.cv[i];
    }
#pragma unroll
    for (int v = 0; v < VEC; v++)
        stage_update<T, KIND, HV>(p, i, (size_t)i * ntr + (size_t)tv * VEC + v, d0[v], d1[v], d2[v], cu, cv);
}

// Tiled stage kernel with the weight and index stream software-pipelined in
// registers: one operator (heat, or a fused advection operator), one lane
// group of NV lanes per row, each lane keeping the local indices and weights
// of its row's next RD chunks in flight while it works on the current one
// (loads issued RD chunks ahead, a ring of registers indexed statically by an
// unrolled loop).  The per-row arithmetic -- chunks in order, slots in order,
// the same fused multiply-adds -- is k_stage_tile's with G = 1, so the results
// are the same bits.
template <typename T, int VEC, int NV, int RD>
__global__ void __launch_bounds__(1024) k_stage_tile_pipe(StageParams<T> p, TileParams tp)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sx = reinterpret_cast<T*>(smem_raw);
    typedef typename VecT<T, VEC>::type V;
    constexpr int ntr = NV * VEC;
    const int b = blockIdx.x;
    const int h0 = __ldg(tp.ptr + b), hn = __ldg(tp.ptr + b + 1) - h0;
    for (int e = threadIdx.x; e < hn * NV; e += blockDim.x) {
        const int h = e / NV, v = e - h * NV;
        const int node = __ldg(tp.nodes + h0 + h);
        reinterpret_cast<V*>(sx)[(size_t)h * NV + v] = __ldg(reinterpret_cast<const V*>(p.x + (size_t)node * ntr) + v);
    }
    __syncthreads();
    const int tv = threadIdx.x % NV, rl = threadIdx.x / NV;
    const int i = __ldg(tp.rows + b) + rl;
    if (i >= __ldg(tp.rows + b + 1)) return;
    const int nc = p.nc;
    const size_t o0 = sell_off(i, 0, nc);  // chunk c of row i sits at o0 + 128 c (sliced ELL)
    T d0[VEC];
#pragma unroll
    for (int v = 0; v < VEC; v++) d0[v] = T(0);
    ushort4 lq[RD];
    T wq[RD][4];
#pragma unroll
    for (int r = 0; r < RD; r++)
        if (r < nc) {
            lq[r] = __ldg(reinterpret_cast<const ushort4*>(tp.lidx + o0 + 128 * (size_t)r));
            ld_w4(p.w0 + o0 + 128 * (size_t)r, wq[r]);
        }
    for (int c0 = 0; c0 < nc; c0 += RD) {
#pragma unroll
        for (int r = 0; r < RD; r++) {
            const int c = c0 + r;
            if (c < nc) {
                const ushort4 l4 = lq[r];
                T w[4];
#pragma unroll
                for (int k = 0; k < 4; k++) w[k] = wq[r][k];
                if (c + RD < nc) {
                    const size_t o = o0 + 128 * (size_t)(c + RD);
                    lq[r] = __ldg(reinterpret_cast<const ushort4*>(tp.lidx + o));
                    ld_w4(p.w0 + o, wq[r]);
                }
                const int ll[4] = {l4.x, l4.y, l4.z, l4.w};
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    T xj[VEC];
                    const V t = reinterpret_cast<const V*>(sx)[(size_t)ll[k] * NV + tv];
                    memcpy(xj, &t, sizeof(V));
#pragma unroll
                    for (int v = 0; v < VEC; v++) d0[v] = Ar<T>::fma(w[k], xj[v], d0[v]);
                }
            }
        }
    }
#pragma unroll
    for (int v = 0; v < VEC; v++)
        stage_update<T, KIND_HEAT, false>(p, i, (size_t)i * ntr + (size_t)tv * VEC + v, d0[v], T(0), T(0), T(0),
                                          T(0));
}

// Asynchronous global -> shared copies of one node record's vector (16, 8 or
// 4 bytes; cp.async), committed as a group and waited for by group count.
template <int BYTES>
__device__ __forceinline__ void cp_async_vec(void* smem_dst, const void* gsrc)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    if (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(gsrc), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Halo slots a thread stages per tile in k_stage_tile_db (max halo x NV / threads, rounded up).
constexpr int DB_SLOTS = 8;

// Persistent tiled stage kernel for one streamed operator (heat, or a fused
// advection operator), one lane group of NV lanes per row: each block takes
// tiles b = blockIdx.x, blockIdx.x + gridDim.x, ... and keeps two halo
// buffers, so the node values of its next tile are copied in (cp.async, 16
// bytes per lane) while it works on the current one; the node indices of the
// tile after that are loaded into registers a tile ahead, so issuing the
// copies never waits on them.  The per-row arithmetic is k_stage_tile's with
// G = 1 (chunks and slots in order, the same fused multiply-adds), so the
// results are the same bits.
template <typename T, int VEC, int NV>
__global__ void __launch_bounds__(1024) k_stage_tile_db(StageParams<T> p, TileParams tp, int nblocks, int buf_vecs)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    typedef typename VecT<T, VEC>::type V;
    constexpr int ntr = NV * VEC;
    V* const buf0 = reinterpret_cast<V*>(smem_raw);  // buffer k of the two at buf0 + k * buf_vecs
    const int tid = threadIdx.x, nt = blockDim.x;
    int nodes_next[DB_SLOTS];  // node of each of this thread's halo slots, for the tile to be copied next
    auto load_nodes = [&](int tb) {
        if (tb >= nblocks) return;
        const int h0 = __ldg(tp.ptr + tb), hn = __ldg(tp.ptr + tb + 1) - h0;
#pragma unroll
        for (int q = 0; q < DB_SLOTS; q++) {
            const int e = tid + q * nt;
            nodes_next[q] = e < hn * NV ? __ldg(tp.nodes + h0 + e / NV) : -1;
        }
    };
    auto issue = [&](int tb, V* dst) {  // copies of tile tb's halo (node indices from nodes_next)
        if (tb < nblocks) {
#pragma unroll
            for (int q = 0; q < DB_SLOTS; q++) {
                const int e = tid + q * nt;
                if (nodes_next[q] >= 0)
                    cp_async_vec<sizeof(V)>(dst + e, reinterpret_cast<const V*>(p.x + (size_t)nodes_next[q] * ntr) +
                                                         (e % NV));
            }
        }
        cp_async_commit();  // an empty group past the last tile keeps the group count regular
    };
    int b = blockIdx.x;
    load_nodes(b);
    issue(b, buf0);
    load_nodes(b + gridDim.x);
    const int tv = tid % NV, rl = tid / NV;
    const int nc = p.nc;
    for (int it = 0; b < nblocks; it++, b += gridDim.x) {
        issue(b + gridDim.x, buf0 + ((it + 1) & 1) * (size_t)buf_vecs);
        load_nodes(b + 2 * gridDim.x);
        cp_async_wait<1>();  // this thread's copies of tile b have landed
        __syncthreads();     // ... and everyone's
        const V* sx = buf0 + (it & 1) * (size_t)buf_vecs;
        const int i = __ldg(tp.rows + b) + rl;
        if (i < __ldg(tp.rows + b + 1)) {
            T d0[VEC];
#pragma unroll
            for (int v = 0; v < VEC; v++) d0[v] = T(0);
            const size_t o0 = sell_off(i, 0, nc);
#pragma unroll 2
            for (int c = 0; c < nc; c++) {
                const size_t o = o0 + 128 * (size_t)c;
                const ushort4 l4 = __ldg(reinterpret_cast<const ushort4*>(tp.lidx + o));
                const int ll[4] = {l4.x, l4.y, l4.z, l4.w};
                T w[4];
                ld_w4(p.w0 + o, w);
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    T xj[VEC];
                    const V t = sx[(size_t)ll[k] * NV + tv];
                    memcpy(xj, &t, sizeof(V));
#pragma unroll
                    for (int v = 0; v < VEC; v++) d0[v] = Ar<T>::fma(w[k], xj[v], d0[v]);
                }
            }
#pragma unroll
            for (int v = 0; v < VEC; v++)
                stage_update<T, KIND_HEAT, false>(p, i, (size_t)i * ntr + (size_t)tv * VEC + v, d0[v], T(0), T(0),
                                                  T(0), T(0));
        }
        __syncthreads();  // tile b's buffer is free for the copies issued next iteration
    }
    cp_async_wait<0>();
}

// Tiled stage kernel with bulk-copy streaming.  Same per-row arithmetic as
// k_stage_tile with one chunk lane per row, but the block's weights and local
// indices -- in the sliced layout one contiguous run per operator per 32-row
// slice -- are streamed into a ring of TMA_NB shared-memory stage buffers by
// asynchronous bulk copies (cp.async.bulk, completion counted on an mbarrier),
// TMA_CS chunks per stage, so the copy engine keeps TMA_NB stages of the weight
// stream in flight per block without holding them in registers.  Thread 0
// issues the copies; a stage buffer is refilled after the block's barrier
// that ends its use.  Every wait is bounded: on timeout the block records
// DEV_STATUS_WAIT_TIMEOUT in *status, waits (bounded) for its copies still in
// flight and returns.
constexpr int TMA_CS = 4;
constexpr int TMA_NB = 3;
constexpr long long TMA_WAIT_LIMIT = 1ll << 22;

template <typename T, int VEC, int KIND, bool HV>
__global__ void __launch_bounds__(1024) k_stage_tma(StageParams<T> p, TileParams tp, int* status, int halo_bytes,
                                                   int stage_bytes)
{
    extern __shared__ __align__(128) unsigned char smem_tma[];
    constexpr int K = KIND == KIND_ADVECT ? (HV ? 3 : 2) : 1;
    typedef typename VecT<T, VEC>::type V;
    T* sx = reinterpret_cast<T*>(smem_tma);
    unsigned char* ring = smem_tma + halo_bytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(ring + (size_t)TMA_NB * stage_bytes);
    const int R = tp.R, nc = p.nc, vpn = p.T_tr / VEC;
    const int b = blockIdx.x, tid = threadIdx.x;
    const int r0 = __ldg(tp.rows + b), r1 = __ldg(tp.rows + b + 1);  // r0 is a multiple of 32
    const int nslices = (min(tp.N32, (r1 + 31) & ~31) - r0) >> 5;
    const int nstages = (nc + TMA_CS - 1) / TMA_CS;
    const size_t op_bytes = (size_t)R * TMA_CS * 4 * sizeof(T);       // one operator's region of a stage
    const size_t slice_w = (size_t)TMA_CS * 32 * 4 * sizeof(T);        // one slice in an operator region
    const size_t slice_l = (size_t)TMA_CS * 32 * 4 * sizeof(unsigned short);
    const T* wsrc[3] = {p.w0, p.w1, p.w2};

    auto issue = [&](int j) {  // thread 0: copies of stage j into buffer j % TMA_NB
        unsigned char* buf = ring + (size_t)(j % TMA_NB) * stage_bytes;
        if (j >= TMA_NB) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // after the block's reads
        const int c0 = j * TMA_CS, cs = min(TMA_CS, nc - c0);
        const uint32_t bw = (uint32_t)(cs * 32 * 4 * sizeof(T)), bl = (uint32_t)(cs * 32 * 4 * sizeof(unsigned short));
        mbar_arrive_expect_tx(&bars[j % TMA_NB], (uint32_t)nslices * (K * bw + bl));
        for (int q = 0; q < nslices; q++) {
            const size_t off = sell_off(r0 + 32 * q, c0, nc);
            for (int k = 0; k < K; k++) bulk_load(buf + k * op_bytes + q * slice_w, wsrc[k] + off, bw, &bars[j % TMA_NB]);
            bulk_load(buf + K * op_bytes + q * slice_l, tp.lidx + off, bl, &bars[j % TMA_NB]);
        }
    };

    if (tid == 0) {
        for (int s = 0; s < TMA_NB; s++) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int j = 0; j < min(TMA_NB, nstages); j++) issue(j);
    // stage the halo's node values while the first copies are in flight
    const int h0 = __ldg(tp.ptr + b), hn = __ldg(tp.ptr + b + 1) - h0;
    for (int e = tid; e < hn * vpn; e += blockDim.x) {
        const int h = e / vpn, v = e - h * vpn;
        const int node = __ldg(tp.nodes + h0 + h);
        reinterpret_cast<V*>(sx)[(size_t)h * vpn + v] = __ldg(reinterpret_cast<const V*>(p.x + (size_t)node * p.T_tr) + v);
    }
    __syncthreads();

    const int rl = tid / vpn, tv = tid - rl * vpn;
    const int i = r0 + rl;
    const bool active = i < r1;
    const int q = rl >> 5, l = rl & 31;
    T d0[VEC], d1[VEC], d2[VEC];
#pragma unroll
    for (int v = 0; v < VEC; v++) d0[v] = d1[v] = d2[v] = T(0);
    for (int j = 0; j < nstages; j++) {
        const int s = j % TMA_NB;
        const bool ok = mbar_wait_bounded(&bars[s], (uint32_t)((j / TMA_NB) & 1), TMA_WAIT_LIMIT);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(status, DEV_STATUS_WAIT_TIMEOUT);
                for (int jj = j; jj < min(j + TMA_NB, nstages); jj++)
                    mbar_wait_bounded(&bars[jj % TMA_NB], (uint32_t)((jj / TMA_NB) & 1), TMA_WAIT_LIMIT);
            }
            return;
        }
        const unsigned char* buf = ring + (size_t)s * stage_bytes;
        const int cs = min(TMA_CS, nc - j * TMA_CS);
        if (active) {
            for (int cc = 0; cc < cs; cc++) {
                const size_t cell = ((size_t)q * TMA_CS + cc) * 32 + l;  // this row's chunk in a region
                const ushort4 l4 = reinterpret_cast<const ushort4*>(buf + K * op_bytes)[cell];
                const int ll[4] = {l4.x, l4.y, l4.z, l4.w};
                T wa[4], wb[4], wc[4];
                ld_w4_shared(reinterpret_cast<const T*>(buf) + cell * 4, wa);
                if (KIND == KIND_ADVECT) {
                    ld_w4_shared(reinterpret_cast<const T*>(buf + op_bytes) + cell * 4, wb);
                    if (HV) ld_w4_shared(reinterpret_cast<const T*>(buf + 2 * op_bytes) + cell * 4, wc);
                }
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    T xj[VEC];
                    const V t = reinterpret_cast<const V*>(sx)[(size_t)ll[k] * vpn + tv];
                    memcpy(xj, &t, sizeof(V));
#pragma unroll
                    for (int v = 0; v < VEC; v++) {
                        d0[v] = Ar<T>::fma(wa[k], xj[v], d0[v]);
                        if (KIND == KIND_ADVECT) {
                            d1[v] = Ar<T>::fma(wb[k], xj[v], d1[v]);
                            if (HV) d2[v] = Ar<T>::fma(wc[k], xj[v], d2[v]);
                        }
                    }
                }
            }
        }
        __syncthreads();  // buffer s is free again
        if (tid == 0 && j + TMA_NB < nstages) issue(j + TMA_NB);
    }
    if (!active) return;
    T cu = T(0), cv = T(0);
    if (KIND == KIND_ADVECT) {
        cu = p.cu[i];
        cv = p.cv[i];
    }
#pragma unroll
    for (int v = 0; v < VEC; v++)
        stage_update<T, KIND, HV>(p, i, (size_t)i * p.T_tr + (size_t)tv * VEC + v, d0[v], d1[v], d2[v], cu, cv);
}

// Unfused right-hand side + stage update from per-operator outputs (the plain path).
template <typename T, int KIND, bool HV, bool PLAIN = false>
__global__ void k_rhs_axpy(StageParams<T> p, const T* __restrict__ d0, const T* __restrict__ d1, const T* __restrict__ d2)
{
    size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)p.N * p.T_tr) return;
    int i = (int)(e / p.T_tr);
    T cu = T(0), cv = T(0);
    if (KIND == KIND_ADVECT) {
        cu = p.cu[i];
        cv = p.cv[i];
    }
    stage_update<T, KIND, HV, PLAIN>(p, i, e, d0[e], KIND == KIND_ADVECT ? d1[e] : T(0), HV ? d2[e] : T(0), cu, cv);
}

// ---------------------------------------------------------------------------
// launch helpers

template <typename T>
static StageParams<T> make_params(rbffd_pde* P, int stage, double dt)
{
    rbffd_grid* g = P->g;
    StageParams<T> p;
    auto W = [&](int k) -> const T* {
        if (k < 0 || P->op[k] < 0) return nullptr;
        return std::is_same<T, double>::value ? (const T*)g->d_w64[P->op[k]] : (const T*)g->d_w32[P->op[k]];
    };
    p.idx = g->d_idx;
    p.w0 = W(0);
    p.w1 = W(1);
    p.w2 = W(2);
    if (P->fused) {  // the heat stage with kappa = 1 over the fused operator
        p.w0 = (const T*)P->wf;
        p.w1 = p.w2 = nullptr;
    }
    p.cu = (const T*)P->cu;
    p.cv = (const T*)P->cv;
    T* u = (T*)P->u;
    T* xa = (T*)P->xa;
    T* xb = (T*)P->xb;
    static const double cfac[4] = {0.5, 0.5, 1.0, 0.0};
    double c = stage == 3 ? dt / 6. : cfac[stage] * dt;
    p.c = (T)c;
    p.kappa = P->fused ? T(1) : (T)P->kappa;
    p.x = stage == 0 ? u : (stage == 1 ? xa : (stage == 2 ? xb : xa));
    p.xnext = stage == 0 ? xa : (stage == 1 ? xb : (stage == 2 ? xa : nullptr));
    p.u = u;
    p.acc = (T*)P->acc;
    p.comp = stage == 3 && !P->tuning ? (T*)P->comp : nullptr;
    p.N = g->N;
    p.nc = g->nc;
    p.T_tr = P->T;
    p.stage = stage;
    return p;
}

// Tiled launch geometry for a shape, or false if the tiled kernel cannot run it.
struct TileGeom {
    const Halo* h = nullptr;
    int vec = 1, vpn = 1, G = 1, threads = 0;
    int tma = 0, halo_bytes = 0, stage_bytes = 0;
    int sched = -1;  // index of the halo's slot schedule the rows read (-1: stencil order)
    int pf = 0;      // L2 prefetch of upcoming chunks
    int pipe = 0;    // k_stage_tile_pipe: weights and indices pipelined in registers
    int db = 0;      // k_stage_tile_db: persistent blocks with two halo buffers
    size_t smem = 0;
};

// Rows per 16-byte-load wavefront of the FP32 tiled kernel with one lane group
// per row: 128 bytes / (T * 4)-byte node records (8, 4 or 2 for T = 4, 8, 16),
// or 0 where a slot schedule does not apply (FP32, four values per vector).
static int sched_rows(const rbffd_pde* P)
{
    if (P->dtype != RBFFD_F32) return 0;
    return P->T == 4 ? 8 : (P->T == 8 ? 4 : (P->T == 16 ? 2 : 0));
}

// Operators a stage streams: one for heat and the fused advection operator,
// two or three (hyperviscosity) for advection.
static int streamed_operators(const rbffd_pde* P)
{
    return (P->kind == KIND_HEAT || P->fused) ? 1 : (P->use_hv ? 3 : 2);
}

static int log2_rows(int Pw) { return Pw == 2 ? 1 : (Pw == 4 ? 2 : 3); }

// The halo schedule of R rows per block and the PDE's operators in its slot
// order (P->ws), made or refreshed before launches that read them.
static int pde_sched_prepare(rbffd_pde* P, int R)
{
    rbffd_grid* g = P->g;
    rbffd_ctx* ctx = P->ctx;
    const int Pw = sched_rows(P);
    if (!Pw) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "a slot schedule needs FP32 and 4, 8 or 16 tracers");
    const Halo* h = nullptr;
    int rc = grid_halo_schedule(g, R, Pw, &h);
    if (rc) return rc;
    const size_t bytes = (size_t)g->N32 * g->n4 * sizeof(float);
    const int K = streamed_operators(P);
    const bool fresh_layout = P->ws_R != R || P->ws_P != Pw;
    for (int k = 0; k < K; k++) {
        const float* src = P->fused ? (const float*)P->wf : g->d_w32[P->op[k]];
        const unsigned ver = P->fused ? 0u : g->w32_ver[P->op[k]];
        if (!src) return set_error(ctx, RBFFD_ERR_STATE, "no FP32 weights for the slot schedule");
        if (!P->ws[k]) {
            if ((rc = dev_alloc(ctx, (void**)&P->ws[k], bytes))) return rc;
            P->bytes += bytes;
            P->ws_src[k] = nullptr;
        }
        if (fresh_layout || P->ws_src[k] != src || P->ws_ver[k] != ver) {
            if ((rc = grid_schedule_weights(g, src, h->d_slot_s[log2_rows(Pw)], P->ws[k], ctx->stream))) return rc;
            P->ws_src[k] = src;
            P->ws_ver[k] = ver;
        }
    }
    P->ws_R = R;
    P->ws_P = Pw;
    return RBFFD_OK;
}

static bool tile_geom(rbffd_pde* P, Shape sh, TileGeom* tg)
{
    if (sh.tile <= 0) return false;
    auto it = P->g->halos.find(sh.tile);
    if (it == P->g->halos.end()) return false;
    const int es = P->dtype == RBFFD_F64 ? 8 : 4;
    const int V = P->dtype == RBFFD_F64 ? 2 : 4;
    TileGeom t;
    t.h = it->second;
    if (P->T == 1)
        t.vec = 1;
    else if (P->T % V == 0)
        t.vec = V;
    else
        return false;
    t.vpn = P->T / t.vec;
    t.G = sh.lanes > 0 ? sh.lanes : 1;
    if (t.G != 1 && t.G != 2 && t.G != 4) return false;
    const int L = t.vpn * t.G;
    if (L > 32 || (L & (L - 1))) return false;
    t.threads = sh.tile * L;
    if (t.threads > 1024) return false;
    t.smem = (size_t)t.h->max_halo * P->T * es;
    if (sh.sched) {  // prepared by pde_sched_prepare for this block size
        const int Pw = sched_rows(P);
        if (!Pw || t.G != 1 || t.vec != 4 || sh.tma || P->ws_R != sh.tile || P->ws_P != Pw ||
            !t.h->d_lidx_s[log2_rows(Pw)])
            return false;
        for (int k = 0; k < streamed_operators(P); k++)
            if (!P->ws[k]) return false;
        t.sched = log2_rows(Pw);
    }
    if (sh.pf) {
        if (t.G != 1 || sh.tma || sh.sched) return false;
        t.pf = 1;
    }
    if (sh.pipe) {  // one operator streamed, one lane group per row, a compile-time node width
        if (t.G != 1 || sh.tma || sh.pf || !(P->kind == KIND_HEAT || P->fused) ||
            !(t.vpn == 1 || t.vpn == 2 || t.vpn == 4 || t.vpn == 8))
            return false;
        t.pipe = 1;
    }
    if (sh.db) {  // as pipe, and every block's halo within DB_SLOTS copies per thread
        if (t.G != 1 || sh.tma || sh.pf || sh.pipe || !(P->kind == KIND_HEAT || P->fused) ||
            !(t.vpn == 1 || t.vpn == 2 || t.vpn == 4 || t.vpn == 8) || t.h->max_halo > DB_SLOTS * sh.tile)
            return false;
        t.db = 1;
        t.smem *= 2;
    }
    if (sh.tma) {
        if (t.G != 1) return false;
        const int K = P->kind == KIND_HEAT ? 1 : (P->use_hv ? 3 : 2);
        t.tma = 1;
        t.halo_bytes = round_up((int)t.smem, 128);
        t.stage_bytes = round_up(K * sh.tile * TMA_CS * 4 * es + sh.tile * TMA_CS * 4 * 2, 128);
        t.smem = (size_t)t.halo_bytes + (size_t)TMA_NB * t.stage_bytes + TMA_NB * sizeof(uint64_t);
    }
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, P->ctx->device);
    if (t.smem > (size_t)optin) return false;
    *tg = t;
    return true;
}

template <typename T, int VEC, int KIND, bool HV>
static void launch_tile_v(const StageParams<T>& p, const TileParams& tp, const TileGeom& t, cudaStream_t s)
{
    const int nb = t.h->nblocks;
    if (t.pf) {
        cudaFuncSetAttribute(k_stage_tile<T, VEC, 1, KIND, HV, TILE_PF_DIST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)t.smem);
        k_stage_tile<T, VEC, 1, KIND, HV, TILE_PF_DIST><<<nb, t.threads, t.smem, s>>>(p, tp);
        return;
    }
    // one lane per row with the common node widths: compile-time vectors per node
    if (t.G == 1 && (t.vpn == 1 || t.vpn == 4 || t.vpn == 8)) {
        if (t.vpn == 1) {
            cudaFuncSetAttribute(k_stage_tile<T, VEC, 1, KIND, HV, 0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)t.smem);
            k_stage_tile<T, VEC, 1, KIND, HV, 0, 1><<<nb, t.threads, t.smem, s>>>(p, tp);
        } else if (t.vpn == 4) {
            cudaFuncSetAttribute(k_stage_tile<T, VEC, 1, KIND, HV, 0, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)t.smem);
            k_stage_tile<T, VEC, 1, KIND, HV, 0, 4><<<nb, t.threads, t.smem, s>>>(p, tp);
        } else {
            cudaFuncSetAttribute(k_stage_tile<T, VEC, 1, KIND, HV, 0, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)t.smem);
            k_stage_tile<T, VEC, 1, KIND, HV, 0, 8><<<nb, t.threads, t.smem, s>>>(p, tp);
        }
        return;
    }
    switch (t.G) {
    case 1:
        cudaFuncSetAttribute(k_stage_tile<T, VEC, 1, KIND, HV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem);
        k_stage_tile<T, VEC, 1, KIND, HV><<<nb, t.threads, t.smem, s>>>(p, tp);
        break;
    case 2:
        cudaFuncSetAttribute(k_stage_tile<T, VEC, 2, KIND, HV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem);
        k_stage_tile<T, VEC, 2, KIND, HV><<<nb, t.threads, t.smem, s>>>(p, tp);
        break;
    default:
        cudaFuncSetAttribute(k_stage_tile<T, VEC, 4, KIND, HV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem);
        k_stage_tile<T, VEC, 4, KIND, HV><<<nb, t.threads, t.smem, s>>>(p, tp);
        break;
    }
}

// Depth of the register pipeline of k_stage_tile_pipe (chunks in flight per lane).
constexpr int PIPE_RD = 4;

template <typename T, int VEC>
static void launch_pipe_v(const StageParams<T>& p, const TileParams& tp, const TileGeom& t, cudaStream_t s)
{
    const int nb = t.h->nblocks;
    if (t.vpn == 1) {
        cudaFuncSetAttribute(k_stage_tile_pipe<T, VEC, 1, PIPE_RD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)t.smem);
        k_stage_tile_pipe<T, VEC, 1, PIPE_RD><<<nb, t.threads, t.smem, s>>>(p, tp);
    } else if (t.vpn == 2) {
        cudaFuncSetAttribute(k_stage_tile_pipe<T, VEC, 2, PIPE_RD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)t.smem);
        k_stage_tile_pipe<T, VEC, 2, PIPE_RD><<<nb, t.threads, t.smem, s>>>(p, tp);
    } else if (t.vpn == 4) {
        cudaFuncSetAttribute(k_stage_tile_pipe<T, VEC, 4, PIPE_RD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)t.smem);
        k_stage_tile_pipe<T, VEC, 4, PIPE_RD><<<nb, t.threads, t.smem, s>>>(p, tp);
    } else {
        cudaFuncSetAttribute(k_stage_tile_pipe<T, VEC, 8, PIPE_RD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)t.smem);
        k_stage_tile_pipe<T, VEC, 8, PIPE_RD><<<nb, t.threads, t.smem, s>>>(p, tp);
    }
}

// Persistent grid of k_stage_tile_db: as many blocks as fit on the device at
// once (occupancy x SMs), at most one per tile.
template <typename T, int VEC, int NV>
static void launch_db_nv(const StageParams<T>& p, const TileParams& tp, const TileGeom& t, int device, cudaStream_t s)
{
    auto kern = k_stage_tile_db<T, VEC, NV>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem);
    int per_sm = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, t.threads, t.smem);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int nb = t.h->nblocks;
    const int grid = std::max(1, std::min(nb, std::max(per_sm, 1) * sms));
    kern<<<grid, t.threads, t.smem, s>>>(p, tp, nb, (int)(t.smem / 2 / sizeof(typename VecT<T, VEC>::type)));
}

template <typename T, int VEC>
static void launch_db_v(const StageParams<T>& p, const TileParams& tp, const TileGeom& t, int device, cudaStream_t s)
{
    if constexpr (VEC == 1) {  // one value per node
        launch_db_nv<T, 1, 1>(p, tp, t, device, s);
        return;
    }
    if (t.vpn == 1)
        launch_db_nv<T, VEC, 1>(p, tp, t, device, s);
    else if (t.vpn == 2)
        launch_db_nv<T, VEC, 2>(p, tp, t, device, s);
    else if (t.vpn == 4)
        launch_db_nv<T, VEC, 4>(p, tp, t, device, s);
    else
        launch_db_nv<T, VEC, 8>(p, tp, t, device, s);
}

template <typename T, int VEC, int KIND, bool HV>
static void launch_tma_v(const StageParams<T>& p, const TileParams& tp, const TileGeom& t, int* status, cudaStream_t s)
{
    cudaFuncSetAttribute(k_stage_tma<T, VEC, KIND, HV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem);
    k_stage_tma<T, VEC, KIND, HV><<<t.h->nblocks, t.threads, t.smem, s>>>(p, tp, status, t.halo_bytes, t.stage_bytes);
}

template <typename T, int KIND, bool HV>
static void launch_stage_t(rbffd_pde* P, const StageParams<T>& p, Shape sh, cudaStream_t s)
{
    TileGeom tg;
    if (tile_geom(P, sh, &tg)) {
        TileParams tp{tg.h->d_ptr, tg.h->d_nodes, tg.h->d_lidx, tg.h->d_rows, tg.h->R, P->g->N32};
        constexpr int VV = std::is_same<T, float>::value ? 4 : 2;
        if (tg.sched >= 0) {  // slot-scheduled rows: local indices and the operators in that order
            StageParams<T> ps = p;
            ps.w0 = (const T*)P->ws[0];
            ps.w1 = (const T*)P->ws[1];
            ps.w2 = (const T*)P->ws[2];
            tp.lidx = tg.h->d_lidx_s[tg.sched];
            if (tg.pipe)
                launch_pipe_v<T, VV>(ps, tp, tg, s);
            else
                launch_tile_v<T, VV, KIND, HV>(ps, tp, tg, s);
            return;
        }
        if (tg.db) {
            if (tg.vec == 1)
                launch_db_v<T, 1>(p, tp, tg, P->ctx->device, s);
            else
                launch_db_v<T, VV>(p, tp, tg, P->ctx->device, s);
            return;
        }
        if (tg.pipe) {
            if (tg.vec == 1)
                launch_pipe_v<T, 1>(p, tp, tg, s);
            else
                launch_pipe_v<T, VV>(p, tp, tg, s);
            return;
        }
        if (tg.tma) {
            if (tg.vec == 1)
                launch_tma_v<T, 1, KIND, HV>(p, tp, tg, P->ctx->d_status, s);
            else
                launch_tma_v<T, VV, KIND, HV>(p, tp, tg, P->ctx->d_status, s);
        } else if (tg.vec == 1) {
            launch_tile_v<T, 1, KIND, HV>(p, tp, tg, s);
        } else {
            launch_tile_v<T, VV, KIND, HV>(p, tp, tg, s);
        }
        return;
    }
    int B = sh.block > 0 ? sh.block : 256;
    if constexpr (std::is_same<T, double>::value) {
        if (sh.plain) {  // the reference build's arithmetic: one tracer, one lane per row
            k_stage_scalar<T, KIND, HV, 1, true><<<(P->g->N + B - 1) / B, B, 0, s>>>(p);
            return;
        }
    }
    if (P->T == 1) {
        int G = sh.lanes > 0 ? sh.lanes : 1;
        long long threads = (long long)P->g->N * G;
        int nb = (int)((threads + B - 1) / B);
        switch (G) {
        case 1: k_stage_scalar<T, KIND, HV, 1><<<nb, B, 0, s>>>(p); break;
        case 2: k_stage_scalar<T, KIND, HV, 2><<<nb, B, 0, s>>>(p); break;
        case 4: k_stage_scalar<T, KIND, HV, 4><<<nb, B, 0, s>>>(p); break;
        case 8: k_stage_scalar<T, KIND, HV, 8><<<nb, B, 0, s>>>(p); break;
        default: k_stage_scalar<T, KIND, HV, 16><<<nb, B, 0, s>>>(p); break;
        }
        return;
    }
    const int V = std::is_same<T, float>::value ? 4 : 2;
    if (P->T % V == 0) {
        long long threads = (long long)P->g->N * (P->T / V);
        k_stage_vec<T, std::is_same<T, float>::value ? 4 : 2, KIND, HV><<<(int)((threads + B - 1) / B), B, 0, s>>>(p);
    } else {
        long long threads = (long long)P->g->N * P->T;
        k_stage_vec<T, 1, KIND, HV><<<(int)((threads + B - 1) / B), B, 0, s>>>(p);
    }
}

template <typename T>
static void launch_stage(rbffd_pde* P, int stage, double dt, Shape sh, cudaStream_t s)
{
    StageParams<T> p = make_params<T>(P, stage, dt);
    if (P->kind == KIND_HEAT || P->fused)
        launch_stage_t<T, KIND_HEAT, false>(P, p, sh, s);
    else if (P->use_hv)
        launch_stage_t<T, KIND_ADVECT, true>(P, p, sh, s);
    else
        launch_stage_t<T, KIND_ADVECT, false>(P, p, sh, s);
}

static void launch_stage_any(rbffd_pde* P, int stage, double dt, Shape sh, cudaStream_t s)
{
    if (P->dtype == RBFFD_F64)
        launch_stage<double>(P, stage, dt, sh, s);
    else
        launch_stage<float>(P, stage, dt, sh, s);
}

template <typename T, bool PLAIN>
static int unfused_stage_t(rbffd_pde* P, int stage, double dt, cudaStream_t s)
{
    int nops = P->kind == KIND_HEAT ? 1 : (P->use_hv ? 3 : 2);
    for (int k = 0; k < nops; k++) {
        StageParams<T> p = make_params<T>(P, stage, dt);
        int rc;
        if constexpr (PLAIN)
            rc = grid_apply_dev_plain(P->g, P->op[k], P->T, p.x, (double*)P->d[k], 0, P->g->N, s);
        else
            rc = grid_apply_dev(P->g, P->op[k], P->dtype, P->T, p.x, P->d[k], 0, P->g->N, 1, s);
        if (rc) return rc;
    }
    StageParams<T> p = make_params<T>(P, stage, dt);
    size_t n = (size_t)P->g->N * P->T;
    int nb = (int)((n + 255) / 256);
    const T *d0 = (const T*)P->d[0], *d1 = (const T*)P->d[1], *d2 = (const T*)P->d[2];
    if (P->kind == KIND_HEAT)
        k_rhs_axpy<T, KIND_HEAT, false, PLAIN><<<nb, 256, 0, s>>>(p, d0, d1, d2);
    else if (P->use_hv)
        k_rhs_axpy<T, KIND_ADVECT, true, PLAIN><<<nb, 256, 0, s>>>(p, d0, d1, d2);
    else
        k_rhs_axpy<T, KIND_ADVECT, false, PLAIN><<<nb, 256, 0, s>>>(p, d0, d1, d2);
    return RBFFD_OK;
}

template <typename T>
static int unfused_stage(rbffd_pde* P, int stage, double dt, cudaStream_t s)
{
    if constexpr (std::is_same<T, double>::value)
        if (P->arith == RBFFD_ARITH_UNFUSED) return unfused_stage_t<double, true>(P, stage, dt, s);
    return unfused_stage_t<T, false>(P, stage, dt, s);
}

// ---------------------------------------------------------------------------
// autotuner.  A first pass times every candidate shape on the stage
// sequence 0, 1, 2 (the stages that write only the scratch buffers xa, xb and
// acc).  A second pass times the three fastest as the solver runs them: 25
// full RK4 steps in one CUDA graph, with dt = 0 (every stage then writes u
// back unchanged, u + 0 * f) and u saved and restored around the timing
// besides, so the caller's state is untouched.  The fastest of the second
// pass is kept per problem shape.

static Shape autotune(rbffd_pde* P)
{
    rbffd_ctx* ctx = P->ctx;
    TuneKey key{P->fused ? KIND_HEAT * 4 : P->kind * 4 + (P->use_hv ? 2 : 0), P->dtype, P->T, P->g->N, P->g->n_pad};
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto it = ctx->tuned.find(key);
        if (it != ctx->tuned.end()) return it->second;
    }
    // tuning steps (dt = 0, state saved and restored) leave a compensated state's correction alone
    struct TuningFlag {
        rbffd_pde* P;
        explicit TuningFlag(rbffd_pde* q) : P(q) { P->tuning = true; }
        ~TuningFlag() { P->tuning = false; }
    } tuning_flag(P);
    std::vector<Shape> cands;
    const int blocks[3] = {128, 256, 512};
    if (P->T == 1) {
        const int lanes[5] = {1, 2, 4, 8, 16};
        for (int G : lanes)
            for (int B : blocks) cands.push_back(Shape{G, B});
    } else {
        for (int B : blocks) cands.push_back(Shape{0, B});
    }
    // tiled candidates: halo staged in shared memory, R rows per block
    const int rows_per_block[3] = {64, 128, 256};
    for (int R : rows_per_block) {
        const Halo* h = nullptr;
        if (grid_halo(P->g, R, &h) != RBFFD_OK) continue;
        for (int G : {1, 2, 4}) {
            Shape c{G, 0, R, 0};
            TileGeom tg;
            if (tile_geom(P, c, &tg)) cands.push_back(c);
        }
        Shape c{1, 0, R, 1};  // weights and indices streamed by bulk copies
        TileGeom tg;
        if (tile_geom(P, c, &tg)) cands.push_back(c);
        Shape cp{1, 0, R, 0, 0, 1};  // upcoming chunks prefetched into L2
        if (tile_geom(P, cp, &tg)) cands.push_back(cp);
        Shape cq{1, 0, R};  // weights and indices pipelined in registers
        cq.pipe = 1;
        if (tile_geom(P, cq, &tg)) cands.push_back(cq);
        Shape cd{1, 0, R};  // persistent blocks, next tile's halo copied in during the current one
        cd.db = 1;
        if (tile_geom(P, cd, &tg)) cands.push_back(cd);
        if (sched_rows(P) && pde_sched_prepare(P, R) == RBFFD_OK) {  // rows in the conflict-avoiding slot order
            Shape cs{1, 0, R, 0, 1};
            if (tile_geom(P, cs, &tg)) cands.push_back(cs);
            cs.pipe = 1;
            if (tile_geom(P, cs, &tg)) cands.push_back(cs);
        }
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const bool log = getenv("RBFFD_TUNE_LOG") != nullptr;
    // Launches captured in a CUDA graph, one warm replay, then the fastest of
    // `trials` timed replays, per launch in ms (negative if the shape failed).
    auto time_graph = [&](const Shape& c, int launches, bool full_steps, int trials) -> float {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        if (c.sched && pde_sched_prepare(P, c.tile) != RBFFD_OK) return -1.f;
        if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return -1.f;
        }
        for (int r = 0; r < launches; r++) launch_stage_any(P, full_steps ? r % 4 : r % 3, 0.0, c, ctx->stream);
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        float ms = 1e30f;
        for (int trial = 0; e == cudaSuccess && trial <= trials; trial++) {
            cudaEventRecord(e0, ctx->stream);
            e = cudaGraphLaunch(exec, ctx->stream);
            cudaEventRecord(e1, ctx->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float t = 0;
            cudaEventElapsedTime(&t, e0, e1);
            if (trial > 0) ms = std::min(ms, t);  // trial 0 warms caches and clocks
        }
        if (exec) cudaGraphExecDestroy(exec);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return -1.f;
        }
        if (log)
            fprintf(stderr,
                    "[rbffd tune] kind=%d hv=%d dtype=%d T=%d N=%d n_pad=%d lanes=%d block=%d tile=%d tma=%d sched=%d "
                    "pf=%d%s: %.2f us\n",
                    P->kind, P->use_hv, P->dtype, P->T, P->g->N, P->g->n_pad, c.lanes, c.block, c.tile, c.tma, c.sched, c.pf,
                    full_steps ? " (full steps)" : "", 1e3f * ms / launches);
        return ms / launches;
    };
    std::vector<std::pair<float, int>> first_pass;
    for (int k = 0; k < (int)cands.size(); k++) {
        const float t = time_graph(cands[k], 21, false, 2);
        if (t >= 0.f) first_pass.push_back({t, k});
    }
    std::sort(first_pass.begin(), first_pass.end());
    Shape best = first_pass.empty() ? cands[0] : cands[first_pass[0].second];
    const size_t ubytes = (size_t)P->g->N * P->T * (P->dtype == RBFFD_F64 ? 8 : 4);
    void* saved = nullptr;
    if (first_pass.size() > 1 && dev_alloc(ctx, &saved, ubytes) == RBFFD_OK) {
        if (cudaMemcpyAsync(saved, P->u, ubytes, cudaMemcpyDeviceToDevice, ctx->stream) == cudaSuccess) {
            float best_ms = 1e30f;
            for (int r = 0; r < (int)first_pass.size() && r < 3; r++) {
                const float t = time_graph(cands[first_pass[r].second], 100, true, 3);
                if (t >= 0.f && t < best_ms) {
                    best_ms = t;
                    best = cands[first_pass[r].second];
                }
            }
            cudaMemcpyAsync(P->u, saved, ubytes, cudaMemcpyDeviceToDevice, ctx->stream);
        }
        cudaStreamSynchronize(ctx->stream);
        dev_free(ctx, saved, ubytes);
    }
    cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->tuned[key] = best;
    return best;
}

// ---------------------------------------------------------------------------
// C ABI

// Per-node advection coefficients cu = vel_u / a and cv = vel_v / a in the
// grid's internal order, stored in prm->dtype at cu_dev / cv_dev.  The cosine
// bell's are computed on the host in FP64 exactly as CosineBell::solve does
// every stage (cosine_bell.cpp:35-49; the velocity field is steady);
// RBFFD_RHS_ADVECTION's are the caller's, reordered.
int advect_coefficients(rbffd_grid* g, const rbffd_pde_params* prm, void* cu_dev, void* cv_dev, cudaStream_t s)
{
    rbffd_ctx* ctx = g->ctx;
    const int N = g->N;
    std::vector<double> cu(N), cv(N);
    if (prm->rhs_kind == RBFFD_RHS_COSINE_BELL) {
        std::vector<double> xyz((size_t)N * 4);
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(xyz.data(), g->d_xyz, (size_t)N * sizeof(double4), cudaMemcpyDeviceToHost, s));
        RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
        const double a = prm->sphere_radius, alpha = prm->alpha, u0 = prm->u0;
        for (int i = 0; i < N; i++) {
            const double x = xyz[4 * (size_t)i], y = xyz[4 * (size_t)i + 1], z = xyz[4 * (size_t)i + 2];
            const double lambda = atan2(y, x);
            const double theta = atan2(z, sqrt(x * x + y * y));
            const double vel_u = u0 * (cos(theta) * cos(alpha) + sin(theta) * cos(lambda) * sin(alpha));
            const double vel_v = -u0 * (sin(lambda) * sin(alpha));
            cu[i] = vel_u / a;
            cv[i] = vel_v / a;
        }
    } else {
        for (int i = 0; i < N; i++) {  // caller's node order -> internal row order
            cu[i] = prm->cu[g->h_perm[i]];
            cv[i] = prm->cv ? prm->cv[g->h_perm[i]] : 0.0;
        }
    }
    if (prm->dtype == RBFFD_F64) {
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(cu_dev, cu.data(), (size_t)N * 8, cudaMemcpyHostToDevice, s));
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(cv_dev, cv.data(), (size_t)N * 8, cudaMemcpyHostToDevice, s));
        RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    } else {
        std::vector<float> fu(N), fv(N);
        for (int i = 0; i < N; i++) {
            fu[i] = (float)cu[i];
            fv[i] = (float)cv[i];
        }
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(cu_dev, fu.data(), (size_t)N * 4, cudaMemcpyHostToDevice, s));
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(cv_dev, fv.data(), (size_t)N * 4, cudaMemcpyHostToDevice, s));
        RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    }
    return RBFFD_OK;
}

size_t pde_bytes(const rbffd_grid* g, const rbffd_pde_params* prm)
{
    const size_t es = prm->dtype == RBFFD_F64 ? 8 : 4, nt = (size_t)g->N * (prm->ntracers > 0 ? prm->ntracers : 1);
    size_t b = 4 * nt * es;                     // u, xa, xb, acc
    if (prm->dtype == RBFFD_F32) b += nt * 8;  // FP64 staging
    if (prm->rhs_kind != RBFFD_RHS_HEAT) b += 2 * (size_t)g->N * es;
    return b;
}

static void pde_free(rbffd_pde* P)
{
    if (!P) return;
    rbffd_ctx* ctx = P->ctx;
    size_t es = (P->dtype == RBFFD_F64 ? 8 : 4);
    size_t n = (size_t)P->g->N * P->T * es;
    if (P->gexec) cudaGraphExecDestroy(P->gexec);
    dev_free(ctx, P->u, n);
    dev_free(ctx, P->xa, n);
    dev_free(ctx, P->xb, n);
    dev_free(ctx, P->acc, n);
    for (int k = 0; k < 3; k++) dev_free(ctx, P->d[k], n);
    dev_free(ctx, P->stage64, (size_t)P->g->N * P->T * 8);
    dev_free(ctx, P->cu, (size_t)P->g->N * es);
    dev_free(ctx, P->cv, (size_t)P->g->N * es);
    dev_free(ctx, P->wf, (size_t)P->g->N32 * P->g->n4 * (P->dtype == RBFFD_F64 ? sizeof(double) : sizeof(float)));
    for (int k = 0; k < 3; k++) dev_free(ctx, P->ws[k], (size_t)P->g->N32 * P->g->n4 * sizeof(float));
    dev_free(ctx, P->comp, (size_t)P->g->N * P->T * sizeof(float));
    delete P;
}

// Fused advection operator, row by row over the padded rows (padding rows
// and slots 0): Wf = -(cu W_lambda + cv W_theta) (+ W_hv) in FP64 from the
// FP64 weights and the PDE's coefficients (in its dtype T), rounded once to T.
template <typename T>
__global__ void k_fuse_operator(T* __restrict__ wf, const double* __restrict__ wl, const double* __restrict__ wt,
                                const double* __restrict__ wh, const T* __restrict__ cu, const T* __restrict__ cv,
                                int N, int rows, int nc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    const double a = i < N ? (double)cu[i] : 0.0, c = i < N ? (double)cv[i] : 0.0;
    for (int s = 0; s < 4 * nc; s++) {
        const size_t o = sell_elem(i, s, nc);
        double w = -__fma_rn(a, wl[o], __dmul_rn(c, wt[o]));
        if (wh) w = __dadd_rn(w, wh[o]);
        wf[o] = i < N ? (T)w : T(0);
    }
}

extern "C" int rbffd_pde_set_fused_operator(rbffd_pde* P, int on)
{
    if (!P) return RBFFD_ERR_INVALID;
    rbffd_ctx* ctx = P->ctx;
    if (!on) {
        if (P->fused && P->gexec) {
            cudaGraphExecDestroy(P->gexec);
            P->gexec = nullptr;
        }
        P->fused = false;
        return RBFFD_OK;
    }
    if (P->kind != KIND_ADVECT)
        return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "a fused operator is built for advection only");
    if (P->arith == RBFFD_ARITH_UNFUSED)
        return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "the unfused (reference) arithmetic keeps the three operators");
    if (P->fused) return RBFFD_OK;
    rbffd_grid* g = P->g;
    cudaSetDevice(ctx->device);
    const bool f64 = P->dtype == RBFFD_F64;
    const size_t bytes = (size_t)g->N32 * g->n4 * (f64 ? sizeof(double) : sizeof(float));
    if (!P->wf) {
        int rc = dev_alloc(ctx, (void**)&P->wf, bytes);
        if (rc) return rc;
        P->bytes += bytes;
    }
    const double* wh = P->op[2] >= 0 ? g->d_w64[P->op[2]] : nullptr;
    if (f64)
        k_fuse_operator<double><<<(g->N32 + 127) / 128, 128, 0, ctx->stream>>>(
            (double*)P->wf, g->d_w64[P->op[0]], g->d_w64[P->op[1]], wh, (const double*)P->cu, (const double*)P->cv,
            g->N, g->N32, g->nc);
    else
        k_fuse_operator<float><<<(g->N32 + 127) / 128, 128, 0, ctx->stream>>>(
            (float*)P->wf, g->d_w64[P->op[0]], g->d_w64[P->op[1]], wh, (const float*)P->cu, (const float*)P->cv,
            g->N, g->N32, g->nc);
    RBFFD_CUDA_TRY(ctx, cudaGetLastError());
    P->ws_src[0] = nullptr;  // a scheduled copy of the previous operator is stale
    if (P->gexec) {
        cudaGraphExecDestroy(P->gexec);
        P->gexec = nullptr;
    }
    P->fused = true;
    return RBFFD_OK;
}

// FP32 state with a compensated update: a per-value FP32 array holds minus
// the part of u + increment that each step's rounding lost (Knuth's TwoSum in
// stage 3 of the per-stage kernels), added back by the next step; the state
// read out is u - comp.  Off: the array is freed and the plain update returns.
extern "C" int rbffd_pde_set_compensated_state(rbffd_pde* P, int on)
{
    if (!P) return RBFFD_ERR_INVALID;
    rbffd_ctx* ctx = P->ctx;
    const size_t bytes = (size_t)P->g->N * P->T * sizeof(float);
    if (on && P->dtype != RBFFD_F32)
        return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "a compensated state is for FP32 PDEs (FP64 rounds 2^29 times finer)");
    if (!on == !P->comp) return RBFFD_OK;
    cudaSetDevice(ctx->device);
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));  // no launch of the old setting still running
    if (P->gexec) {  // captured launches carry the array's address
        cudaGraphExecDestroy(P->gexec);
        P->gexec = nullptr;
    }
    if (!on) {
        dev_free(ctx, P->comp, bytes);
        P->comp = nullptr;
        P->bytes -= bytes;
        return RBFFD_OK;
    }
    int rc = dev_alloc(ctx, &P->comp, bytes);
    if (rc) return rc;
    P->bytes += bytes;
    RBFFD_CUDA_TRY(ctx, cudaMemsetAsync(P->comp, 0, bytes, ctx->stream));
    return RBFFD_OK;
}

extern "C" int rbffd_pde_create(rbffd_grid* g, const rbffd_pde_params* prm, rbffd_pde** out)
{
    if (!g || !prm || !out) return RBFFD_ERR_INVALID;
    *out = nullptr;
    rbffd_ctx* ctx = g->ctx;
    if (prm->dtype != RBFFD_F32 && prm->dtype != RBFFD_F64)
        return set_error(ctx, RBFFD_ERR_INVALID, "bad dtype %d", prm->dtype);
    if (prm->ntracers < 1 || prm->ntracers > 1024)
        return set_error(ctx, RBFFD_ERR_INVALID, "ntracers %d outside [1, 1024]", prm->ntracers);
    int kind;
    int ops[3] = {-1, -1, -1};
    if (prm->rhs_kind == RBFFD_RHS_HEAT) {
        kind = KIND_HEAT;
        ops[0] = der_index(RBFFD_LSFC);
    } else if (prm->rhs_kind == RBFFD_RHS_COSINE_BELL || prm->rhs_kind == RBFFD_RHS_ADVECTION) {
        kind = KIND_ADVECT;
        ops[0] = der_index(RBFFD_LAMBDA);
        ops[1] = der_index(RBFFD_THETA);
        if (prm->use_hv) ops[2] = der_index(RBFFD_HV);
        if (prm->rhs_kind == RBFFD_RHS_ADVECTION && !prm->cu)
            return set_error(ctx, RBFFD_ERR_INVALID, "advection needs per-node coefficients cu");
        // no cv: f = -cu D_lambda h (+ HV), as VortexRollup::solve (vortex_rollup.cpp:27-57); the
        // D_theta slot reads the D_lambda weights again with cv = 0 (the same bits: 0 * d = 0)
        if (prm->rhs_kind == RBFFD_RHS_ADVECTION && !prm->cv) ops[1] = ops[0];
        if (prm->rhs_kind == RBFFD_RHS_COSINE_BELL && prm->sphere_radius == 0.0)
            return set_error(ctx, RBFFD_ERR_INVALID, "cosine bell needs a nonzero sphere radius");
    } else {
        return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "rhs_kind %d", prm->rhs_kind);
    }
    for (int k = 0; k < 3; k++)
        if (ops[k] >= 0 && !g->d_w64[ops[k]])
            return set_error(ctx, RBFFD_ERR_STATE, "weights of operator 0x%x are not on the device", 1u << ops[k]);
    cudaSetDevice(ctx->device);
    rbffd_pde* P = new (std::nothrow) rbffd_pde();
    if (!P) return RBFFD_ERR_OOM;
    P->g = g;
    P->ctx = ctx;
    P->kind = kind;
    P->T = prm->ntracers;
    P->dtype = prm->dtype;
    P->use_hv = kind == KIND_ADVECT && prm->use_hv;
    P->kappa = prm->kappa;
    memcpy(P->op, ops, sizeof ops);
    int N = g->N;
    size_t es = (P->dtype == RBFFD_F64 ? 8 : 4);
    size_t n = (size_t)N * P->T * es;
    int rc;
    if ((rc = dev_alloc(ctx, &P->u, n)) || (rc = dev_alloc(ctx, &P->xa, n)) || (rc = dev_alloc(ctx, &P->xb, n)) ||
        (rc = dev_alloc(ctx, &P->acc, n))) {
        pde_free(P);
        return rc;
    }
    P->bytes = 4 * n;
    if (P->dtype == RBFFD_F32) {
        if ((rc = dev_alloc(ctx, (void**)&P->stage64, (size_t)N * P->T * 8))) {
            pde_free(P);
            return rc;
        }
        P->bytes += (size_t)N * P->T * 8;
    }
    cudaStream_t s = ctx->stream;
    if (kind == KIND_ADVECT) {
        if ((rc = dev_alloc(ctx, &P->cu, N * es)) || (rc = dev_alloc(ctx, &P->cv, N * es)) ||
            (rc = advect_coefficients(g, prm, P->cu, P->cv, s))) {
            pde_free(P);
            return rc;
        }
        P->bytes += 2 * N * es;
    }
    // FP32 weight copies exist whenever FP64 weights do (grid_make_f32).
    for (int k = 0; k < 3; k++)
        if (ops[k] >= 0 && !g->d_w32[ops[k]] && (rc = grid_make_f32(g, ops[k]))) {
            pde_free(P);
            return rc;
        }
    RBFFD_CUDA_TRY(ctx, cudaMemsetAsync(P->u, 0, n, s));
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    // the context's FP64 arithmetic (rbffd_ctx_set_arithmetic) for PDEs it applies to
    if (ctx->arith == RBFFD_ARITH_UNFUSED && P->dtype == RBFFD_F64 && P->T == 1)
        rbffd_pde_set_arithmetic(P, RBFFD_ARITH_UNFUSED);
    *out = P;
    return RBFFD_OK;
}

extern "C" int rbffd_pde_destroy(rbffd_pde* P)
{
    if (!P) return RBFFD_ERR_INVALID;
    cudaSetDevice(P->ctx->device);
    cudaStreamSynchronize(P->ctx->stream);
    pde_free(P);
    return RBFFD_OK;
}

__global__ void k_to_dtype_f(const double* __restrict__ a, float* __restrict__ b, size_t n)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __double2float_rn(a[i]);
}
__global__ void k_from_f(const float* __restrict__ a, double* __restrict__ b, size_t n)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
}
// b = a - c in FP64 (a compensated FP32 state and its correction)
__global__ void k_from_f_compensated(const float* __restrict__ a, const float* __restrict__ c, double* __restrict__ b,
                                     size_t n)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i] - (double)c[i];
}

extern "C" int rbffd_pde_set_state(rbffd_pde* P, const double* u)
{
    if (!P || !u) return RBFFD_ERR_INVALID;
    rbffd_ctx* ctx = P->ctx;
    cudaSetDevice(ctx->device);
    size_t n = (size_t)P->g->N * P->T;
    cudaStream_t s = ctx->stream;
    // the stage buffers xa/xb are free between steps and serve as staging
    int rc;
    if (P->dtype == RBFFD_F64) {
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(P->xa, u, n * 8, cudaMemcpyHostToDevice, s));
        if ((rc = grid_to_internal(P->g, P->xa, P->u, P->T, 8, s))) return rc;
    } else {
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(P->stage64, u, n * 8, cudaMemcpyHostToDevice, s));
        k_to_dtype_f<<<(int)((n + 255) / 256), 256, 0, s>>>(P->stage64, (float*)P->xb, n);
        RBFFD_CUDA_TRY(ctx, cudaGetLastError());
        if ((rc = grid_to_internal(P->g, P->xb, P->u, P->T, 4, s))) return rc;
        if (P->comp) RBFFD_CUDA_TRY(ctx, cudaMemsetAsync(P->comp, 0, n * sizeof(float), s));
    }
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    return RBFFD_OK;
}

extern "C" int rbffd_pde_get_state(rbffd_pde* P, double* u)
{
    if (!P || !u) return RBFFD_ERR_INVALID;
    rbffd_ctx* ctx = P->ctx;
    cudaSetDevice(ctx->device);
    size_t n = (size_t)P->g->N * P->T;
    cudaStream_t s = ctx->stream;
    int rc;
    if (P->dtype == RBFFD_F64) {
        if ((rc = grid_to_caller(P->g, P->u, P->xa, P->T, 8, s))) return rc;
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(u, P->xa, n * 8, cudaMemcpyDeviceToHost, s));
    } else {
        if ((rc = grid_to_caller(P->g, P->u, P->xb, P->T, 4, s))) return rc;
        if (P->comp) {  // u - comp, the compensated state
            if ((rc = grid_to_caller(P->g, P->comp, P->xa, P->T, 4, s))) return rc;
            k_from_f_compensated<<<(int)((n + 255) / 256), 256, 0, s>>>((const float*)P->xb, (const float*)P->xa,
                                                                         P->stage64, n);
        } else {
            k_from_f<<<(int)((n + 255) / 256), 256, 0, s>>>((const float*)P->xb, P->stage64, n);
        }
        RBFFD_CUDA_TRY(ctx, cudaGetLastError());
        RBFFD_CUDA_TRY(ctx, cudaMemcpyAsync(u, P->stage64, n * 8, cudaMemcpyDeviceToHost, s));
    }
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    return RBFFD_OK;
}

extern "C" int rbffd_pde_set_time(rbffd_pde* P, double t)
{
    if (!P) return RBFFD_ERR_INVALID;
    P->t = t;
    return RBFFD_OK;
}

extern "C" int rbffd_pde_get_time(rbffd_pde* P, double* t)
{
    if (!P || !t) return RBFFD_ERR_INVALID;
    *t = P->t;
    return RBFFD_OK;
}

extern "C" int rbffd_pde_set_shape(rbffd_pde* P, int lanes, int block)
{
    if (!P) return RBFFD_ERR_INVALID;
    if (!(lanes == 0 || lanes == 1 || lanes == 2 || lanes == 4 || lanes == 8 || lanes == 16)) return RBFFD_ERR_INVALID;
    if (!(block == 0 || block == 64 || block == 128 || block == 256 || block == 512)) return RBFFD_ERR_INVALID;
    if (P->arith == RBFFD_ARITH_UNFUSED) {  // one lane per row in stencil order; only the block size is free
        if (lanes > 1)
            return set_error(P->ctx, RBFFD_ERR_UNSUPPORTED, "the unfused (reference) arithmetic uses one lane per row");
        P->shape = Shape{1, block ? block : 256};
        P->shape.plain = 1;
        P->forced = true;
        return RBFFD_OK;
    }
    if (lanes == 0 && block == 0) {
        P->forced = false;
        P->shape = Shape{};
        return RBFFD_OK;
    }
    if (P->T > 1 && lanes > 1) return set_error(P->ctx, RBFFD_ERR_UNSUPPORTED, "lanes per row apply to one tracer only");
    P->shape = Shape{lanes ? lanes : 1, block ? block : 256, 0};
    P->forced = true;
    return RBFFD_OK;
}

extern "C" int rbffd_pde_set_arithmetic(rbffd_pde* P, int arith)
{
    if (!P) return RBFFD_ERR_INVALID;
    if (arith != RBFFD_ARITH_FUSED && arith != RBFFD_ARITH_UNFUSED)
        return set_error(P->ctx, RBFFD_ERR_INVALID, "unknown arithmetic %d", arith);
    if (arith == RBFFD_ARITH_UNFUSED && (P->dtype != RBFFD_F64 || P->T != 1))
        return set_error(P->ctx, RBFFD_ERR_UNSUPPORTED, "the unfused (reference) arithmetic is FP64 with one tracer");
    if (arith == RBFFD_ARITH_UNFUSED && P->fused)
        return set_error(P->ctx, RBFFD_ERR_UNSUPPORTED, "the unfused (reference) arithmetic keeps the three operators");
    P->arith = arith;
    P->forced = false;
    P->shape = Shape{};
    if (arith == RBFFD_ARITH_UNFUSED) return rbffd_pde_set_shape(P, 1, 256);
    return RBFFD_OK;
}

extern "C" int rbffd_pde_get_arithmetic(rbffd_pde* P, int* arith)
{
    if (!P || !arith) return RBFFD_ERR_INVALID;
    *arith = P->arith;
    return RBFFD_OK;
}

extern "C" int rbffd_pde_get_shape(rbffd_pde* P, int* lanes, int* block)
{
    if (!P || !lanes || !block) return RBFFD_ERR_INVALID;
    *lanes = P->shape.lanes;
    *block = P->shape.block;
    return RBFFD_OK;
}

extern "C" int rbffd_pde_set_tiled_shape(rbffd_pde* P, int rows_per_block, int lanes, int flags)
{
    if (!P) return RBFFD_ERR_INVALID;
    if (P->arith == RBFFD_ARITH_UNFUSED)
        return set_error(P->ctx, RBFFD_ERR_UNSUPPORTED, "the unfused (reference) arithmetic gathers from global memory");
    if (rows_per_block < 32 || rows_per_block > 1024 || rows_per_block % 32 || !(lanes == 1 || lanes == 2 || lanes == 4))
        return set_error(P->ctx, RBFFD_ERR_INVALID, "rows_per_block must be a multiple of 32, lanes 1, 2 or 4");
    if (flags & ~(RBFFD_TILE_STREAM_WEIGHTS | RBFFD_TILE_SLOT_SCHEDULE | RBFFD_TILE_PREFETCH | RBFFD_TILE_PIPELINE |
                  RBFFD_TILE_DOUBLE_BUFFER))
        return set_error(P->ctx, RBFFD_ERR_INVALID, "unknown tiled-shape flags 0x%x", flags);
    const bool stream_weights = flags & RBFFD_TILE_STREAM_WEIGHTS, sched = flags & RBFFD_TILE_SLOT_SCHEDULE,
               pf = flags & RBFFD_TILE_PREFETCH, pipe = flags & RBFFD_TILE_PIPELINE,
               db = flags & RBFFD_TILE_DOUBLE_BUFFER;
    if ((stream_weights || sched || pf || pipe || db) && lanes != 1)
        return set_error(P->ctx, RBFFD_ERR_INVALID,
                         "streamed weights, slot schedules, prefetch, the register pipeline and double-buffered "
                         "halos use one lane per row");
    if (db && (stream_weights || sched || pf || pipe))
        return set_error(P->ctx, RBFFD_ERR_INVALID, "double-buffered halos combine with no other tiled-shape flag");
    if ((int)stream_weights + (int)sched + (int)pf > 1 || (pipe && (stream_weights || pf)))
        return set_error(P->ctx, RBFFD_ERR_INVALID,
                         "streamed weights, a slot schedule and prefetch do not combine; the register pipeline "
                         "combines with a slot schedule only");
    cudaSetDevice(P->ctx->device);
    const Halo* h = nullptr;
    int rc = grid_halo(P->g, rows_per_block, &h);
    if (rc) return rc;
    if (sched && (rc = pde_sched_prepare(P, rows_per_block))) return rc;
    Shape c{lanes, 0, rows_per_block, stream_weights ? 1 : 0, sched ? 1 : 0, pf ? 1 : 0};
    c.pipe = pipe ? 1 : 0;
    c.db = db ? 1 : 0;
    TileGeom tg;
    if (!tile_geom(P, c, &tg))
        return set_error(P->ctx, RBFFD_ERR_UNSUPPORTED, "tiled shape (%d rows, %d lanes) does not fit this PDE",
                         rows_per_block, lanes);
    P->shape = c;
    P->forced = true;
    return RBFFD_OK;
}

extern "C" int rbffd_pde_get_tiling(rbffd_pde* P, int* rows_per_block)
{
    if (!P || !rows_per_block) return RBFFD_ERR_INVALID;
    *rows_per_block = P->shape.tile;
    return RBFFD_OK;
}

extern "C" int rbffd_pde_get_tile_flags(rbffd_pde* P, int* flags)
{
    if (!P || !flags) return RBFFD_ERR_INVALID;
    *flags = (P->shape.tma ? RBFFD_TILE_STREAM_WEIGHTS : 0) | (P->shape.sched ? RBFFD_TILE_SLOT_SCHEDULE : 0) |
             (P->shape.pf ? RBFFD_TILE_PREFETCH : 0) | (P->shape.pipe ? RBFFD_TILE_PIPELINE : 0) |
             (P->shape.db ? RBFFD_TILE_DOUBLE_BUFFER : 0);
    return RBFFD_OK;
}

static void run_steps(rbffd_pde* P, double dt, int nsteps, Shape sh)
{
    for (int k = 0; k < nsteps; k++)
        for (int st = 0; st < 4; st++) launch_stage_any(P, st, dt, sh, P->ctx->stream);
}

// The cluster-resident layout (C CTAs of R rows), built on the host from the
// device's stencil array the first time it is used: each CTA's halo (the
// sorted unique nodes its rows read), each stencil slot's halo position, and
// each row's push list (the CTAs and halo positions its value goes to).
void resident_free(rbffd_grid* g)
{
    rbffd_ctx* ctx = g->ctx;
    dev_free(ctx, g->d_res_pptr, (size_t)g->res_C * (g->res_R + 1) * sizeof(int));
    dev_free(ctx, g->d_res_pdst, (size_t)g->res_C * g->res_P * sizeof(unsigned short));
    dev_free(ctx, g->d_res_lidx, (size_t)g->res_C * g->n4 * g->res_R * sizeof(unsigned short));
    g->d_res_pptr = nullptr;
    g->d_res_pdst = g->d_res_lidx = nullptr;
    g->res_R = g->res_C = g->res_H = g->res_P = 0;
}

static int resident_halo(rbffd_grid* g, int R, int C)
{
    if (g->res_R == R && g->res_C == C) return RBFFD_OK;
    rbffd_ctx* ctx = g->ctx;
    const int N = g->N, nc = g->nc, n4 = g->n4;
    std::vector<int> idx((size_t)g->N32 * n4);
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    RBFFD_CUDA_TRY(ctx, cudaMemcpy(idx.data(), g->d_idx, idx.size() * sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<std::vector<int>> halo(C);
    int H = 1;
    for (int q = 0; q < C; q++) {
        std::vector<int>& v = halo[q];
        for (int i = q * R; i < std::min(N, q * R + R); i++)
            for (int sl = 0; sl < n4; sl++) v.push_back(idx[sell_elem(i, sl, nc)]);
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        H = std::max(H, (int)v.size());
    }
    if (H > 4096) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "cluster-resident RK4: a CTA's halo exceeds 4096 nodes");
    std::vector<unsigned short> lidx((size_t)C * n4 * R, 0);
    std::vector<std::vector<unsigned short>> dst((size_t)C * R);  // push targets of each row
    for (int q = 0; q < C; q++) {
        const std::vector<int>& v = halo[q];
        for (size_t h = 0; h < v.size(); h++) dst[v[h]].push_back((unsigned short)((q << 12) | (int)h));
        for (int i = q * R; i < std::min(N, q * R + R); i++)
            for (int sl = 0; sl < n4; sl++) {
                const int j = idx[sell_elem(i, sl, nc)];
                lidx[((size_t)q * n4 + sl) * R + (i - q * R)] =
                    (unsigned short)(std::lower_bound(v.begin(), v.end(), j) - v.begin());
            }
    }
    int Pm = 1;
    for (int q = 0; q < C; q++) {
        int cnt = 0;
        for (int r = 0; r < R; r++) cnt += (int)dst[(size_t)q * R + r].size();
        Pm = std::max(Pm, cnt);
    }
    std::vector<int> pptr((size_t)C * (R + 1), 0);
    std::vector<unsigned short> pdst((size_t)C * Pm, 0);
    for (int q = 0; q < C; q++) {
        int e = 0;
        for (int r = 0; r < R; r++) {
            pptr[(size_t)q * (R + 1) + r] = e;
            for (unsigned short d : dst[(size_t)q * R + r]) pdst[(size_t)q * Pm + e++] = d;
        }
        pptr[(size_t)q * (R + 1) + R] = e;
    }
    resident_free(g);
    int rc = dev_alloc(ctx, (void**)&g->d_res_pptr, pptr.size() * sizeof(int));
    if (!rc) rc = dev_alloc(ctx, (void**)&g->d_res_pdst, pdst.size() * sizeof(unsigned short));
    if (!rc) rc = dev_alloc(ctx, (void**)&g->d_res_lidx, lidx.size() * sizeof(unsigned short));
    if (rc) {
        dev_free(ctx, g->d_res_pptr, pptr.size() * sizeof(int));
        dev_free(ctx, g->d_res_pdst, pdst.size() * sizeof(unsigned short));
        g->d_res_pptr = nullptr;
        g->d_res_pdst = nullptr;
        return rc;
    }
    RBFFD_CUDA_TRY(ctx, cudaMemcpy(g->d_res_pptr, pptr.data(), pptr.size() * sizeof(int), cudaMemcpyHostToDevice));
    RBFFD_CUDA_TRY(ctx, cudaMemcpy(g->d_res_pdst, pdst.data(), pdst.size() * sizeof(unsigned short),
                                   cudaMemcpyHostToDevice));
    RBFFD_CUDA_TRY(ctx, cudaMemcpy(g->d_res_lidx, lidx.data(), lidx.size() * sizeof(unsigned short),
                                   cudaMemcpyHostToDevice));
    g->res_R = R;
    g->res_C = C;
    g->res_H = H;
    g->res_P = Pm;
    return RBFFD_OK;
}

// nsteps RK4 steps in one cluster-resident launch (k_rk4_cluster), one
// tracer; check_only: report whether the PDE fits without launching.
template <typename T>
static int advance_resident_t(rbffd_pde* P, double dt, int nsteps, cudaStream_t s, bool check_only)
{
    rbffd_ctx* ctx = P->ctx;
    rbffd_grid* g = P->g;
    const bool heat = P->kind == KIND_HEAT || P->fused;
    const int K = heat ? 1 : (P->use_hv ? 3 : 2);
    const int C = std::min(RES_MAX_CLUSTER, (g->N + 31) / 32), n4 = 4 * g->nc;
    const int R = ((g->N + C - 1) / C + 31) / 32 * 32;
    if (R > 1024)
        return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "cluster-resident RK4: %d nodes exceed %d CTAs of 1024 rows",
                         g->N, C);
    int rc = resident_halo(g, R, C);
    if (rc) return rc;
    // weights and halo positions in registers where the stencil size has a variant and the budget allows
    const int ncr =
        (R <= 256 && (g->nc == RES_RW_NC0 || g->nc == RES_RW_NC1) && K * n4 * (int)sizeof(T) / 4 <= RES_RW_MAX_REGS)
            ? g->nc
            : 0;
    const size_t smem =
        ncr ? resident_smem<T>(0, 0, R, g->res_H, g->res_P) : resident_smem<T>(K, n4, R, g->res_H, g->res_P);
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
    if (smem > (size_t)optin)
        return set_error(ctx, RBFFD_ERR_UNSUPPORTED,
                         "cluster-resident RK4: %zu bytes of weights, halo and state per CTA exceed shared memory",
                         smem);
    ResidentParams<T> rp;
    for (int k = 0; k < 3; k++)
        rp.w[k] = k < K ? (P->fused ? (const T*)P->wf
                                    : (std::is_same<T, double>::value ? (const T*)g->d_w64[P->op[k]]
                                                                      : (const T*)g->d_w32[P->op[k]]))
                        : nullptr;
    rp.cu = (const T*)P->cu;
    rp.cv = (const T*)P->cv;
    rp.u = (T*)P->u;
    static const double cfac[4] = {0.5, 0.5, 1.0, 0.0};
    for (int st = 0; st < 4; st++) rp.c[st] = (T)(st == 3 ? dt / 6. : cfac[st] * dt);
    rp.kappa = P->fused ? T(1) : (T)P->kappa;
    rp.N = g->N;
    rp.nc = g->nc;
    rp.R = R;
    rp.K = K;
    rp.H = g->res_H;
    rp.P = g->res_P;
    rp.pptr = g->d_res_pptr;
    rp.pdst = g->d_res_pdst;
    rp.lidx = g->d_res_lidx;
    rp.nsteps = nsteps;
    const bool plain = P->arith == RBFFD_ARITH_UNFUSED;
    if (heat)
        return plain ? launch_resident_t<T, KIND_HEAT, false, true>(P, rp, C, smem, s, check_only, ncr)
                     : launch_resident_t<T, KIND_HEAT, false, false>(P, rp, C, smem, s, check_only, ncr);
    if (P->use_hv)
        return plain ? launch_resident_t<T, KIND_ADVECT, true, true>(P, rp, C, smem, s, check_only, ncr)
                     : launch_resident_t<T, KIND_ADVECT, true, false>(P, rp, C, smem, s, check_only, ncr);
    return plain ? launch_resident_t<T, KIND_ADVECT, false, true>(P, rp, C, smem, s, check_only, ncr)
                 : launch_resident_t<T, KIND_ADVECT, false, false>(P, rp, C, smem, s, check_only, ncr);
}

static int advance_resident(rbffd_pde* P, double dt, int nsteps, int flags)
{
    rbffd_ctx* ctx = P->ctx;
    if (P->T != 1) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "cluster-resident RK4 serves one tracer");
    if (P->comp) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "cluster-resident RK4 keeps no compensated state");
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const int rc = P->dtype == RBFFD_F64 ? advance_resident_t<double>(P, dt, nsteps, s, false)
                                         : advance_resident_t<float>(P, dt, nsteps, s, false);
    if (rc) return rc;
    P->t += dt * nsteps;
    if (!(flags & RBFFD_ADVANCE_ASYNC)) RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    return RBFFD_OK;
}

extern "C" int rbffd_pde_advance(rbffd_pde* P, int scheme, double dt, int nsteps, int flags)
{
    if (!P) return RBFFD_ERR_INVALID;
    rbffd_ctx* ctx = P->ctx;
    if (scheme != 2) return set_error(ctx, RBFFD_ERR_UNSUPPORTED, "time scheme %d (only RK4 = 2)", scheme);
    if (nsteps < 0) return set_error(ctx, RBFFD_ERR_INVALID, "nsteps < 0");
    if (nsteps == 0) return RBFFD_OK;
    if (flags & RBFFD_ADVANCE_RESIDENT) return advance_resident(P, dt, nsteps, flags);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    if (flags & RBFFD_ADVANCE_UNFUSED) {
        // plain path: per-operator SpMV launches, separate RHS/axpy, host sync per step
        size_t n = (size_t)P->g->N * P->T * (P->dtype == RBFFD_F64 ? 8 : 4);
        int nops = P->kind == KIND_HEAT ? 1 : (P->use_hv ? 3 : 2);
        for (int k = 0; k < nops; k++)
            if (!P->d[k]) {
                int rc = dev_alloc(ctx, &P->d[k], n);
                if (rc) return rc;
                P->bytes += n;
            }
        for (int k = 0; k < nsteps; k++) {
            for (int st = 0; st < 4; st++) {
                int rc = P->dtype == RBFFD_F64 ? unfused_stage<double>(P, st, dt, s) : unfused_stage<float>(P, st, dt, s);
                if (rc) return rc;
            }
            RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
            P->t += dt;
        }
        return RBFFD_OK;
    }
    if (!P->forced && P->shape.block == 0 && P->shape.tile == 0) P->shape = autotune(P);
    Shape sh = P->shape;
    if (sh.tile > 0) {  // the halo must exist before any capture (building it copies to the device)
        const Halo* h = nullptr;
        int rc = grid_halo(P->g, sh.tile, &h);
        if (rc) return rc;
        if (sh.sched && (rc = pde_sched_prepare(P, sh.tile))) return rc;
    }
    if (flags & RBFFD_ADVANCE_GRAPH) {
        const int chunk = 25;
        int full = nsteps / chunk, rest = nsteps % chunk;
        if (full > 0) {
            if (!P->gexec || P->g_dt != dt || P->g_steps != chunk || P->g_shape.lanes != sh.lanes ||
                P->g_shape.block != sh.block || P->g_shape.tile != sh.tile || P->g_shape.tma != sh.tma ||
                P->g_shape.sched != sh.sched || P->g_shape.pf != sh.pf || P->g_shape.plain != sh.plain ||
                P->g_shape.pipe != sh.pipe || P->g_shape.db != sh.db) {
                if (P->gexec) {
                    cudaGraphExecDestroy(P->gexec);
                    P->gexec = nullptr;
                }
                cudaGraph_t graph;
                RBFFD_CUDA_TRY(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                run_steps(P, dt, chunk, sh);
                cudaError_t e = cudaStreamEndCapture(s, &graph);
                if (e != cudaSuccess) return cuda_error(ctx, e, "graph capture");
                e = cudaGraphInstantiate(&P->gexec, graph, 0);
                cudaGraphDestroy(graph);
                if (e != cudaSuccess) {
                    P->gexec = nullptr;
                    return cuda_error(ctx, e, "graph instantiate");
                }
                P->g_dt = dt;
                P->g_steps = chunk;
                P->g_shape = sh;
            }
            for (int r = 0; r < full; r++) RBFFD_CUDA_TRY(ctx, cudaGraphLaunch(P->gexec, s));
        }
        run_steps(P, dt, rest, sh);
    } else {
        run_steps(P, dt, nsteps, sh);
    }
    RBFFD_CUDA_TRY(ctx, cudaGetLastError());
    P->t += dt * nsteps;
    if (!(flags & RBFFD_ADVANCE_ASYNC)) {
        RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(s));
        if (sh.tma) return ctx_check_device_status(ctx);
    }
    return RBFFD_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free RK4 for the heat equation.
//
// Some callers cannot let a library allocate device memory: applications that
// reserve (almost) all of the GPU's memory up front for their own pool, so a
// cudaMalloc inside the library would fail or fragment that pool, and callers
// on latency-critical paths, where cudaMalloc/cudaFree may synchronise the
// device.  rbffd_heat_rk4_noalloc serves them: the caller passes the state
// vector in its own device memory; the copy of the state in the grid's
// internal node order and the three stage buffers RK4 needs live in the
// file-scope array below.  rbffd_ctx_create loads the device code this path
// uses (this array, the stage kernels, the permutation kernels) on the
// context's GPU, so the array is reserved then and held until the process
// exits, and no call of this entry point loads a module (which would take
// device memory) even under the CUDA runtime's lazy loading.  A caller that
// reserves the GPU's memory for its own pool creates its context first.
//
// Limits and sharing: NOALLOC_MAX_NODES nodes in FP64 (twice that in FP32);
// larger grids are rejected.  Every call on a device uses the same array, so
// calls that overlap on that GPU (other streams, other threads, other
// contexts of this process) overwrite each other's buffers: serialise them.
// Each call first writes the whole state copy, and stage 0 writes every stage
// element a later stage reads, so the array needs no clearing between calls.
constexpr int NOALLOC_MAX_NODES = 262144;
static __device__ __align__(256) double g_noalloc_scratch[4 * NOALLOC_MAX_NODES];  // 8 MiB per GPU

// The host-side name g_noalloc_scratch is not a device address: the address a
// kernel may use is looked up with the context's device current, on every
// call (cheap, allocates nothing), so a context recreated after a
// cudaDeviceReset -- where the module reloads at a new address -- is served
// its current address.
static int noalloc_scratch(rbffd_ctx* ctx, void** out)
{
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return cuda_error(ctx, e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress");
    *out = p;
    return RBFFD_OK;
}

// Called by rbffd_ctx_create with the context's device current: loads the
// allocation-free path's device code (see above).  cudaFuncGetAttributes
// loads a kernel; cudaGetSymbolAddress loads the array's module.
int noalloc_preload()
{
    void* p = nullptr;
    cudaFuncAttributes a;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess ||
        cudaFuncGetAttributes(&a, k_stage_scalar<double, KIND_HEAT, false, 1>) != cudaSuccess ||
        cudaFuncGetAttributes(&a, k_stage_scalar<float, KIND_HEAT, false, 1>) != cudaSuccess)
        return RBFFD_ERR_CUDA;
    return grid_permute_preload();
}

// u: the state in the grid's internal order (a region of the scratch array)
template <typename T>
static void noalloc_steps(rbffd_grid* g, const T* w, T* u, T* scratch, T kappa, double dt, int nsteps, cudaStream_t s)
{
    const int N = g->N;
    T* xa = scratch;
    T* xb = scratch + N;
    T* acc = scratch + 2 * (size_t)N;
    StageParams<T> p;
    p.idx = g->d_idx;
    p.w0 = w;
    p.w1 = nullptr;
    p.w2 = nullptr;
    p.cu = nullptr;
    p.cv = nullptr;
    p.u = u;
    p.acc = acc;
    p.kappa = kappa;
    p.N = N;
    p.nc = g->nc;
    p.T_tr = 1;
    const int B = 256, nb = (N + B - 1) / B;
    for (int k = 0; k < nsteps; k++)
        for (int st = 0; st < 4; st++) {
            static const double cfac[3] = {0.5, 0.5, 1.0};
            p.c = (T)(st == 3 ? dt / 6. : cfac[st] * dt);
            p.x = st == 0 ? u : (st == 1 ? xa : (st == 2 ? xb : xa));
            p.xnext = st == 0 ? xa : (st == 1 ? xb : (st == 2 ? xa : nullptr));
            p.stage = st;
            k_stage_scalar<T, KIND_HEAT, false, 1><<<nb, B, 0, s>>>(p);
        }
}

extern "C" int rbffd_heat_rk4_noalloc(rbffd_grid* g, int dtype, double kappa, double dt, int nsteps, void* u_dev)
{
    if (!g || !u_dev || nsteps < 0) return RBFFD_ERR_INVALID;
    rbffd_ctx* ctx = g->ctx;
    if (dtype != RBFFD_F32 && dtype != RBFFD_F64) return set_error(ctx, RBFFD_ERR_INVALID, "bad dtype %d", dtype);
    const int max_nodes = dtype == RBFFD_F64 ? NOALLOC_MAX_NODES : 2 * NOALLOC_MAX_NODES;
    if (g->N > max_nodes)
        return set_error(ctx, RBFFD_ERR_INVALID,
                         "rbffd_heat_rk4_noalloc: grid has %d nodes, the fixed scratch holds at most %d (%s)", g->N,
                         max_nodes, dtype == RBFFD_F64 ? "FP64" : "FP32");
    const int op = der_index(RBFFD_LSFC);
    const void* w = dtype == RBFFD_F64 ? (const void*)g->d_w64[op] : (const void*)g->d_w32[op];
    if (!w) return set_error(ctx, RBFFD_ERR_STATE, "Laplace-Beltrami (LSFC) weights are not on the device");
    if (nsteps == 0) return RBFFD_OK;
    RBFFD_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    void* scratch = nullptr;
    int rc = noalloc_scratch(ctx, &scratch);
    if (rc) return rc;
    // scratch layout (elements of dtype): [xa | xb | acc | state in internal order], N each
    const int es = dtype == RBFFD_F64 ? 8 : 4;
    void* u_int = (char*)scratch + 3 * (size_t)g->N * es;
    if ((rc = grid_to_internal(g, u_dev, u_int, 1, es, ctx->stream))) return rc;
    if (dtype == RBFFD_F64)
        noalloc_steps<double>(g, (const double*)w, (double*)u_int, (double*)scratch, kappa, dt, nsteps, ctx->stream);
    else
        noalloc_steps<float>(g, (const float*)w, (float*)u_int, (float*)scratch, (float)kappa, dt, nsteps, ctx->stream);
    RBFFD_CUDA_TRY(ctx, cudaGetLastError());
    if ((rc = grid_to_caller(g, u_int, u_dev, 1, es, ctx->stream))) return rc;
    RBFFD_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RBFFD_OK;
}
