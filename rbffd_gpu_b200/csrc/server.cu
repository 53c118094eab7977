// Serving: a persistent request loop with continuous batching.
//
// A request is one time-dependent PDE solve (heat or advection on a grid whose
// weights are on the device, any step count).  One host thread per server runs
// the loop:
//   1. admission, in arrival order: a request is admitted while fewer than
//      max_active requests run and the context's device memory plus the
//      request's buffers stays within the HBM budget.  Its buffers are an
//      rbffd_pde; a finished request's rbffd_pde with the same grid and
//      right-hand side is reused (a "slot") instead of allocating, and idle
//      slots are released first when the budget is short;
//   2. a batch of RK4 steps for every active request: each of the four stages
//      of a step is ONE launch of k_stage_batched over the concatenated rows
//      of all active requests (per dtype), a segment table mapping blocks to
//      requests.  The batch length is the smallest remaining step count,
//      capped so a batch takes about TICK_TARGET_S of device time: requests
//      that arrive meanwhile join at the next batch;
//   3. requests that reached their step count copy their state to the
//      caller's buffer and leave; their rbffd_pde becomes an idle slot.
// Each row is computed by one thread in stencil order with the rounding
// sequence of k_stage_scalar with one lane per row (rk4.cu), so a request's
// result does not depend on the rest of the batch.
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
#include <type_traits>
#include <vector>

#include "ell.cuh"
#include "internal.h"

namespace {

constexpr int SEG_ROWS = 128;            // rows (threads) per block of the batched launch
constexpr double TICK_TARGET_S = 2e-3;   // device time aimed at per batch of steps
constexpr int TICK_MAX_STEPS = 64;
constexpr size_t TABLE_BYTES0 = 64 * 1024;  // initial segment-table capacity

template <typename T>
struct Segment {
    const int* idx;
    const T* w0;
    const T* w1;
    const T* w2;
    const T* cu;
    const T* cv;
    T* u;
    T* xa;
    T* xb;
    T* acc;
    T c[4];  // dt/2, dt/2, dt, dt/6
    T kappa;
    int N, nc, kind, use_hv;
    int block0;  // first block of this request in the launch
};

// One RK4 stage for the rows of all requests of one dtype.  Stage inputs:
// 0: u -> xa, 1: xa -> xb, 2: xb -> xa, 3: xa -> u (the buffers of k_stage_*).
template <typename T>
__global__ void __launch_bounds__(SEG_ROWS) k_stage_batched(const Segment<T>* __restrict__ segs, int nseg, int stage)
{
    int lo = 0, hi = nseg - 1;  // last segment with block0 <= blockIdx.x
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segs[mid].block0 <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const Segment<T>& S = segs[lo];
    const int i = ((int)blockIdx.x - S.block0) * SEG_ROWS + (int)threadIdx.x;
    if (i >= S.N) return;
    const T* x = stage == 0 ? S.u : (stage == 2 ? S.xb : S.xa);
    const bool adv = S.kind == KIND_ADVECT, hv = adv && S.use_hv;
    T d0 = T(0), d1 = T(0), d2 = T(0);
    for (int c = 0; c < S.nc; c++) {
        const size_t o = sell_off(i, c, S.nc);
        const int4 j = ld_idx4(S.idx + o);
        const T xv[4] = {__ldg(x + j.x), __ldg(x + j.y), __ldg(x + j.z), __ldg(x + j.w)};
        T w[4];
        ld_w4(S.w0 + o, w);
#pragma unroll
        for (int k = 0; k < 4; k++) d0 = Ar<T>::fma(w[k], xv[k], d0);
        if (adv) {
            ld_w4(S.w1 + o, w);
#pragma unroll
            for (int k = 0; k < 4; k++) d1 = Ar<T>::fma(w[k], xv[k], d1);
            if (hv) {
                ld_w4(S.w2 + o, w);
#pragma unroll
                for (int k = 0; k < 4; k++) d2 = Ar<T>::fma(w[k], xv[k], d2);
            }
        }
    }
    T f;
    if (adv) {
        f = -Ar<T>::fma(S.cu[i], d0, Ar<T>::mul(S.cv[i], d1));
        if (hv) f = Ar<T>::add(f, d2);
    } else {
        f = Ar<T>::mul(S.kappa, d0);
    }
    const T ui = S.u[i];
    const T c = S.c[stage];
    switch (stage) {
    case 0:
        S.acc[i] = f;
        S.xa[i] = Ar<T>::fma(c, f, ui);
        break;
    case 1:
        S.acc[i] = Ar<T>::add(S.acc[i], Ar<T>::mul(T(2), f));
        S.xb[i] = Ar<T>::fma(c, f, ui);
        break;
    case 2:
        S.acc[i] = Ar<T>::add(S.acc[i], Ar<T>::mul(T(2), f));
        S.xa[i] = Ar<T>::fma(c, f, ui);
        break;
    default:
        S.u[i] = Ar<T>::fma(c, Ar<T>::add(S.acc[i], f), ui);
        break;
    }
}

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    rbffd_request p{};
    std::vector<double> u0, cu, cv;  // copies taken at submission
    Clock::time_point t_submit, t_admit, t_done;
    bool admitted = false, cancel = false;
    int done = 0, status = RBFFD_OK;
    rbffd_pde* pde = nullptr;
    size_t bytes = 0;
    int steps_done = 0;
};

// An idle rbffd_pde kept for reuse by a later request with the same grid and
// right-hand side (per-node coefficients included).
struct Slot {
    rbffd_pde* pde;
    rbffd_pde_params prm;
    rbffd_grid* grid;
    size_t bytes;
};

bool slot_fits(const Slot& s, const rbffd_grid* g, const rbffd_pde_params& p)
{
    if (s.grid != g || s.prm.rhs_kind != p.rhs_kind || s.prm.dtype != p.dtype) return false;
    if (p.rhs_kind == RBFFD_RHS_HEAT) return true;        // kappa is a per-request scalar
    if (p.rhs_kind == RBFFD_RHS_ADVECTION) return false;  // caller-given coefficients: never shared
    return s.prm.use_hv == p.use_hv && s.prm.sphere_radius == p.sphere_radius && s.prm.alpha == p.alpha &&
           s.prm.u0 == p.u0;
}

enum { ADMIT_WAIT = 1 };

}  // namespace

struct rbffd_server {
    rbffd_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    size_t budget = 0;
    int max_active = 0;
    std::mutex mu;  // guards everything below that the worker and callers share
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> pending;
    std::vector<std::shared_ptr<Request>> active;
    std::map<uint64_t, std::shared_ptr<Request>> all;
    uint64_t next_id = 1;
    bool stop = false;
    int inject_fail = 0;
    size_t owned = 0;  // device bytes of the server's rbffd_pde objects (active + idle slots)
    rbffd_server_stats st{};
    std::thread worker;
    // worker-only state
    std::vector<Slot> slots;
    void* h_tab = nullptr;  // pinned host segment tables
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

// Give a request's rbffd_pde back as an idle slot, or free it.
void retire_pde(rbffd_server* S, Request& r, bool keep)
{
    if (!r.pde) return;
    if (keep) {
        S->slots.push_back(Slot{r.pde, r.p.pde, r.p.grid, r.bytes});
    } else {
        rbffd_pde_destroy(r.pde);
        std::lock_guard<std::mutex> lk(S->mu);
        S->owned -= std::min(S->owned, r.bytes);
    }
    r.pde = nullptr;
}

void drop_slot(rbffd_server* S, size_t k)
{
    rbffd_pde_destroy(S->slots[k].pde);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->owned -= std::min(S->owned, S->slots[k].bytes);
    }
    S->slots.erase(S->slots.begin() + (long)k);
}

// Give the request device buffers holding its initial state.  RBFFD_OK,
// ADMIT_WAIT (the budget frees up when active requests finish) or an error.
int admit(rbffd_server* S, Request& r, bool nothing_active, bool* reused)
{
    *reused = false;
    rbffd_grid* g = r.p.grid;
    rbffd_pde* P = nullptr;
    for (size_t k = 0; k < S->slots.size(); k++)
        if (slot_fits(S->slots[k], g, r.p.pde)) {
            P = S->slots[k].pde;
            r.bytes = S->slots[k].bytes;
            S->slots.erase(S->slots.begin() + (long)k);
            *reused = true;
            break;
        }
    if (!P) {
        const size_t need = pde_bytes(g, &r.p.pde);
        while (ctx_held(S->ctx) + need > S->budget && !S->slots.empty()) drop_slot(S, 0);  // oldest idle first
        if (ctx_held(S->ctx) + need > S->budget) {
            if (!nothing_active) return ADMIT_WAIT;
            return set_error(S->ctx, RBFFD_ERR_BUDGET, "request of %zu bytes does not fit the budget of %zu bytes",
                             need, S->budget);
        }
        {
            // reserve before allocating: submissions meanwhile see these bytes as the server's
            std::lock_guard<std::mutex> lk(S->mu);
            S->owned += need;
        }
        const int rc = rbffd_pde_create(g, &r.p.pde, &P);
        std::lock_guard<std::mutex> lk(S->mu);
        S->owned -= std::min(S->owned, need);
        if (rc) return rc;
        r.bytes = P->bytes;
        S->owned += r.bytes;
    }
    P->kappa = r.p.pde.kappa;
    P->t = 0.0;
    const int rc = rbffd_pde_set_state(P, r.u0.data());
    r.pde = P;
    if (rc) {
        retire_pde(S, r, false);
        return rc;
    }
    return RBFFD_OK;
}

template <typename T>
void fill_segment(Segment<T>& s, const Request& r, int block0)
{
    const rbffd_pde* P = r.pde;
    const rbffd_grid* g = P->g;
    auto W = [&](int k) -> const T* {
        if (P->op[k] < 0) return nullptr;
        return std::is_same<T, double>::value ? (const T*)g->d_w64[P->op[k]] : (const T*)g->d_w32[P->op[k]];
    };
    s.idx = g->d_idx;
    s.w0 = W(0);
    s.w1 = W(1);
    s.w2 = W(2);
    s.cu = (const T*)P->cu;
    s.cv = (const T*)P->cv;
    s.u = (T*)P->u;
    s.xa = (T*)P->xa;
    s.xb = (T*)P->xb;
    s.acc = (T*)P->acc;
    // the stage coefficients of rbffd_pde_advance
    const double dt = r.p.dt;
    s.c[0] = (T)(0.5 * dt);
    s.c[1] = (T)(0.5 * dt);
    s.c[2] = (T)(1.0 * dt);
    s.c[3] = (T)(dt / 6.);
    s.kappa = (T)P->kappa;
    s.N = g->N;
    s.nc = g->nc;
    s.kind = P->kind;
    s.use_hv = P->use_hv;
    s.block0 = block0;
}

struct Tables {
    int n32 = 0, n64 = 0, blocks32 = 0, blocks64 = 0;
    size_t off64 = 0;  // byte offset of the FP64 table
};

// Build the segment tables of the active set and upload them (stream-ordered
// before the launches that read them; the previous batch has completed, so
// the pinned host copy is free to rewrite).
int upload_tables(rbffd_server* S, const std::vector<std::shared_ptr<Request>>& act, Tables& t)
{
    t = Tables{};
    for (auto& r : act) (r->pde->dtype == RBFFD_F64 ? t.n64 : t.n32)++;
    const size_t b32 = (size_t)t.n32 * sizeof(Segment<float>), b64 = (size_t)t.n64 * sizeof(Segment<double>);
    t.off64 = (b32 + 255) / 256 * 256;
    const size_t need = t.off64 + b64;
    if (need > S->tab_cap) {
        const size_t cap = std::max<size_t>(need * 2, TABLE_BYTES0);
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
    Segment<float>* s32 = (Segment<float>*)S->h_tab;
    Segment<double>* s64 = (Segment<double>*)((char*)S->h_tab + t.off64);
    int k32 = 0, k64 = 0;
    for (auto& r : act) {
        const int nb = (r->pde->g->N + SEG_ROWS - 1) / SEG_ROWS;
        if (r->pde->dtype == RBFFD_F64) {
            fill_segment(s64[k64++], *r, t.blocks64);
            t.blocks64 += nb;
        } else {
            fill_segment(s32[k32++], *r, t.blocks32);
            t.blocks32 += nb;
        }
    }
    RBFFD_CUDA_TRY(S->ctx, cudaMemcpyAsync(S->d_tab, S->h_tab, need, cudaMemcpyHostToDevice, S->stream));
    return RBFFD_OK;
}

// Issue nsteps RK4 steps for the active set; returns after they complete.
int run_steps(rbffd_server* S, const Tables& t, int nsteps, double* seconds, long long* launches)
{
    const Segment<float>* d32 = (const Segment<float>*)S->d_tab;
    const Segment<double>* d64 = (const Segment<double>*)((char*)S->d_tab + t.off64);
    RBFFD_CUDA_TRY(S->ctx, cudaEventRecord(S->ev0, S->stream));
    for (int step = 0; step < nsteps; step++)
        for (int stage = 0; stage < 4; stage++) {
            if (t.n32) {
                k_stage_batched<float><<<t.blocks32, SEG_ROWS, 0, S->stream>>>(d32, t.n32, stage);
                ++*launches;
            }
            if (t.n64) {
                k_stage_batched<double><<<t.blocks64, SEG_ROWS, 0, S->stream>>>(d64, t.n64, stage);
                ++*launches;
            }
        }
    RBFFD_CUDA_TRY(S->ctx, cudaGetLastError());
    RBFFD_CUDA_TRY(S->ctx, cudaEventRecord(S->ev1, S->stream));
    RBFFD_CUDA_TRY(S->ctx, cudaEventSynchronize(S->ev1));
    float ms = 0.f;
    RBFFD_CUDA_TRY(S->ctx, cudaEventElapsedTime(&ms, S->ev0, S->ev1));
    *seconds = ms * 1e-3;
    return RBFFD_OK;
}

void worker_loop(rbffd_server* S)
{
    cudaSetDevice(S->ctx->device);
    std::unique_lock<std::mutex> lk(S->mu);
    bool changed = true;
    Tables tab;
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
        // admission in arrival order
        while (!S->stop && !S->pending.empty() && (S->max_active <= 0 || (int)S->active.size() < S->max_active)) {
            std::shared_ptr<Request> r = S->pending.front();
            int rc;
            bool reused = false;
            if (S->inject_fail > 0) {
                S->inject_fail--;
                rc = set_error(S->ctx, RBFFD_ERR_OOM, "injected admission failure");
            } else {
                const bool nothing_active = S->active.empty();
                lk.unlock();
                rc = admit(S, *r, nothing_active, &reused);
                lk.lock();
            }
            if (rc == ADMIT_WAIT) break;
            S->pending.pop_front();
            if (rc != RBFFD_OK) {
                finish_request(*r, rc);
                S->st.failed++;
                S->cv_done.notify_all();
                continue;
            }
            r->admitted = true;
            r->t_admit = Clock::now();
            if (reused) S->st.slots_reused++;
            S->active.push_back(r);
            S->st.max_active_seen = std::max<long long>(S->st.max_active_seen, (long long)S->active.size());
            changed = true;
        }
        if (S->active.empty()) {
            if (S->stop && S->pending.empty()) break;
            S->cv_work.wait(lk);
            continue;
        }
        // one batch of steps for every active request
        std::vector<std::shared_ptr<Request>> act = S->active;
        int nsteps = TICK_MAX_STEPS;
        if (S->step_s > 0.0) nsteps = std::max(1, std::min(TICK_MAX_STEPS, (int)(TICK_TARGET_S / S->step_s)));
        for (auto& r : act) nsteps = std::min(nsteps, r->p.nsteps - r->steps_done);
        lk.unlock();
        int rc = RBFFD_OK;
        if (changed) {
            rc = upload_tables(S, act, tab);
            changed = false;
        }
        double secs = 0.0;
        long long launches = 0;
        if (rc == RBFFD_OK) rc = run_steps(S, tab, nsteps, &secs, &launches);
        if (rc == RBFFD_OK) S->step_s = secs / nsteps;
        double nu = 0.0;
        std::vector<std::shared_ptr<Request>> left;
        for (auto& r : act) {
            r->steps_done += nsteps;
            nu += (double)r->pde->g->N * nsteps;
            bool cancel;
            {
                std::lock_guard<std::mutex> g(S->mu);
                cancel = r->cancel;
            }
            if (rc != RBFFD_OK) {
                retire_pde(S, *r, false);
                r->status = rc;
            } else if (cancel) {
                retire_pde(S, *r, true);
                r->status = RBFFD_ERR_CANCELLED;
            } else if (r->steps_done >= r->p.nsteps) {
                r->pde->t = r->p.dt * r->p.nsteps;
                const int grc = rbffd_pde_get_state(r->pde, r->p.out);
                retire_pde(S, *r, grc == RBFFD_OK);
                r->status = grc;
            } else {
                continue;
            }
            left.push_back(r);
        }
        lk.lock();
        S->st.ticks++;
        S->st.launches += launches;
        S->st.node_updates += nu;
        S->st.gpu_busy_s += secs;
        for (auto& r : left) {
            finish_request(*r, r->status);
            if (r->status == RBFFD_OK) S->st.completed++;
            else if (r->status == RBFFD_ERR_CANCELLED) S->st.cancelled++;
            else S->st.failed++;
            S->active.erase(std::find(S->active.begin(), S->active.end(), r));
            changed = true;
        }
        if (!left.empty()) S->cv_done.notify_all();
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
    // segment tables for a few hundred active requests, held from the start so
    // that they count against the budget before the first admission
    const size_t tab = TABLE_BYTES0;
    cudaError_t e = cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&S->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&S->ev1);
    if (e == cudaSuccess) e = cudaMallocHost(&S->h_tab, tab);
    int rc = e == cudaSuccess ? RBFFD_OK : cuda_error(ctx, e, "rbffd_server_start");
    if (rc == RBFFD_OK && (rc = dev_alloc(ctx, &S->d_tab, tab)) == RBFFD_OK) S->tab_cap = tab;
    if (rc != RBFFD_OK) {
        if (S->h_tab) cudaFreeHost(S->h_tab);
        if (S->ev0) cudaEventDestroy(S->ev0);
        if (S->ev1) cudaEventDestroy(S->ev1);
        if (S->stream) cudaStreamDestroy(S->stream);
        delete S;
        return rc;
    }
    S->st.budget_bytes = (double)S->budget;
    S->worker = std::thread(worker_loop, S);
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
    const size_t need = pde_bytes(g, &p);
    auto r = std::make_shared<Request>();
    r->p = *req;
    const int N = g->N;
    r->u0.assign(req->u0, req->u0 + N);
    if (p.rhs_kind == RBFFD_RHS_ADVECTION) {
        r->cu.assign(p.cu, p.cu + N);
        r->cv.assign(p.cv, p.cv + N);
        r->p.pde.cu = r->cu.data();
        r->p.pde.cv = r->cv.data();
    } else {
        r->p.pde.cu = r->p.pde.cv = nullptr;
    }
    r->p.u0 = r->u0.data();
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return set_error(ctx, RBFFD_ERR_STATE, "server is stopping");
    // memory the server cannot free (grids, the caller's own PDEs) plus this request
    const size_t held = ctx_held(ctx);
    if (held - std::min(held, S->owned) + need > S->budget)
        return set_error(ctx, RBFFD_ERR_BUDGET, "request of %zu bytes can never fit the budget of %zu bytes", need,
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
        S->cv_work.notify_one();
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
                             [&] { return S->pending.empty() && S->active.empty(); }))
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
    out->active = (long long)S->active.size();
    out->held_bytes = (double)ctx_held(S->ctx);
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
        // the worker cancels the pending requests and finishes the active ones
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    if (S->worker.joinable()) S->worker.join();
    cudaSetDevice(S->ctx->device);
    while (!S->slots.empty()) drop_slot(S, S->slots.size() - 1);
    cudaStreamSynchronize(S->stream);
    if (S->h_tab) cudaFreeHost(S->h_tab);
    dev_free(S->ctx, S->d_tab, S->tab_cap);
    cudaEventDestroy(S->ev0);
    cudaEventDestroy(S->ev1);
    cudaStreamDestroy(S->stream);
    delete S;
    return RBFFD_OK;
}
