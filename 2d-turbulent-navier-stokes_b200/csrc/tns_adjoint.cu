// tns_adjoint.cu -- the discrete adjoint of one FP64 RK4 iteration on the device.
//
// tns_adjoint_step(h, Q_n, lambda) recomputes the iteration from the checkpoint Q_n with
// the solver's own FP64 kernels (dissipation + DT, viscous flux, the port mass flux,
// stages 1-3, keeping every stage input) and the state-only passes of the reverse (field
// sets, node averages, dissipation pre-pass), then runs the hand-derived reverse of
// tns_adjoint.cuh: stages 4..1 (residual / update / source reverse, gather into the
// stage input, ghosts, port lines), the viscous flux reverse inside stage 1 (faces,
// nodes, slots), and the dissipation / time-step reverse.  A step -- about 30 kernels,
// with three short branches beside the main reverse -- is one CUDA graph per (forward
// set, mode, sensitivity level), captured on first use and replayed on the handle's
// stream for every checkpoint.  TNS_ADJ_FROZEN replays only the reverse (fixed-point
// adjoint); tns_adjoint_step_next adds the next checkpoint's forward values on a branch.
#include <cuda_runtime.h>

#include <vector>

#include "tns_adjoint.cuh"
#include "tns_handle.h"

using namespace tns::adj;

namespace {

// 128-thread blocks: the reverse kernels hold 100-170 registers a thread, so a block of
// 128 fills the SM in finer steps (measured: 371 us per 512 x 192 step vs 429 us with
// 256-thread blocks and no register caps).
#ifndef TNS_ADJ_THREADS
#define TNS_ADJ_THREADS 128
#endif
constexpr int ADJ_THREADS = TNS_ADJ_THREADS;

// One thread per point; minb = resident blocks per SM the register budget is sized for.
#define TNS_ADJ_KERNEL(name, fn, minb)                                                  \
    __global__ void __launch_bounds__(ADJ_THREADS, minb) name(AdjArgs a, long long n) { \
        const long long i = (long long)blockIdx.x * ADJ_THREADS + threadIdx.x;          \
        if (i < n) fn(a, i);                                                             \
    }

// Stream priorities for the reverse (high) and the prefetch branch (low).
#ifndef TNS_ADJ_PRIORITY
#define TNS_ADJ_PRIORITY 1
#endif
#ifndef TNS_ADJ_STAGE_MINB
#define TNS_ADJ_STAGE_MINB 3
#endif
#ifndef TNS_ADJ_GATHER_MINB
#define TNS_ADJ_GATHER_MINB 4
#endif
#ifndef TNS_ADJ_FACE_MINB
#define TNS_ADJ_FACE_MINB 2
#endif

TNS_ADJ_KERNEL(k_adj_fields, s0_point, 1)
TNS_ADJ_KERNEL(k_adj_stage, s1_point, TNS_ADJ_STAGE_MINB)
TNS_ADJ_KERNEL(k_adj_gather, s3_point, TNS_ADJ_GATHER_MINB)
TNS_ADJ_KERNEL(k_adj_gather_ghosts, s3g_point, 1)
TNS_ADJ_KERNEL(k_adj_nodes, v0_point, 1)
TNS_ADJ_KERNEL(k_adj_faces, v1_point, TNS_ADJ_FACE_MINB)
TNS_ADJ_KERNEL(k_adj_node_bar, v2_point, 1)
TNS_ADJ_KERNEL(k_adj_slot_bar, v3_point, 1)
TNS_ADJ_KERNEL(k_adj_diss_pre, d0_point, 1)
TNS_ADJ_KERNEL(k_adj_diss_faces, d1_point, 1)
TNS_ADJ_KERNEL(k_adj_diss_gather, d2_point, 1)
TNS_ADJ_KERNEL(k_adj_dtmin, dtmin_point, 1)
TNS_ADJ_KERNEL(k_adj_final, final_point, 1)
TNS_ADJ_KERNEL(k_adj_centroids, centroid_point, 1)
TNS_ADJ_KERNEL(k_adj_geo, geo_point, 1)
TNS_ADJ_KERNEL(k_adj_port, port_point, 1)
TNS_ADJ_KERNEL(k_adj_port_nodes, port_node_point, 1)

// LOCAL = 0: sum of the per-cell dt adjoints (block sums, one atomic per block).
__global__ void __launch_bounds__(ADJ_THREADS) k_adj_dtsum(const double* __restrict__ v, long long n,
                                                           double* __restrict__ out) {
    __shared__ double red[ADJ_THREADS / 32];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * ADJ_THREADS + threadIdx.x; i < n; i += (long long)gridDim.x * ADJ_THREADS)
        s += v[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < ADJ_THREADS / 32 ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) atomicAdd(out, s);
    }
}

template <class K>
void launch_points(K kernel, const AdjArgs& a, long long n, cudaStream_t s) {
    const long long blocks = (n + ADJ_THREADS - 1) / ADJ_THREADS;
    kernel<<<(unsigned)blocks, ADJ_THREADS, 0, s>>>(a, n);
}

}  // namespace

// The forward values of one state (checkpoint): stage inputs, D, VIS, DT, the four
// stages' field sets, node averages and the dissipation pre-pass.  Two sets, so that
// the next checkpoint's forward values are computed while this one's reverse runs.
struct AdjForward {
    DevBuf<double> q0, rec, w, navg, dpre;
    DevBuf<int> ninfo;
    // one record (tns_adjoint_record): stage inputs 1-3, D, VIS, DT, DTMIN and the four
    // stages' port mass flux, carved from `rec` in this order
    double *q1 = nullptr, *q2 = nullptr, *q3 = nullptr, *d = nullptr, *vis = nullptr, *dt = nullptr,
           *dtmin = nullptr, *gport = nullptr;
    void carve(long long n) {
        double* p = rec.p;
        q1 = p; p += 5 * n;
        q2 = p; p += 5 * n;
        q3 = p; p += 5 * n;
        d = p; p += 5 * n;
        vis = p; p += 4 * n;
        dt = p; p += n;
        dtmin = p; p += 1;
        gport = p;
    }
};

long long record_size(long long n, long long ng) { return 25 * n + 1 + 4 * ng; }

// Device buffers and graphs of the adjoint of one handle.
struct tns_adjoint_state {
    AdjForward set[2];
    int cur = 0;                         // the set of the last step's state
    bool have_forward = false;           // set[cur] holds forward values
    int pre_set = -1;                    // a set prefetched by the last step ...
    const double* pre_ptr = nullptr;     // ... for the state at this device address
    DevBuf<double> lam, lamA, lamB, lamold, lamg, lamd, gbar, srcn, srcg, wself, wvisc, dbar, visbar, dtbar, dout,
        nbar, vfi, vfj, dtsum, sens, xcs, ycs, gportb, portacc;  // gportb [4][nghost], portacc [3][nghost]
    long long nsens = 0;
    // branches of a step: dissipation reverse, ghost gather, face-vector sensitivities,
    // forward values of the next checkpoint
    cudaStream_t side[4] = {nullptr, nullptr, nullptr, nullptr};
    // the reverse runs on high-priority streams (main + side 0-2), the prefetch branch on
    // the lowest priority, so that the reverse -- the critical path -- keeps its SMs
    cudaStream_t hp = nullptr;
    cudaEvent_t ev = nullptr;
    // [set][mode: bit 0 forward first, bit 1 prefetch the other set, bit 2 state-only
    // passes first (recorded forward values)][sensitivities: none, scalars, all]
    cudaGraphExec_t graph[2][8][3] = {};
    long long per_step[2][8][3] = {};
    long long launches = 0;
};

namespace {

AdjArgs base_args(tns_handle* h, tns_adjoint_state* s, int set, int geo) {
    AdjArgs a{};
    const AdjForward& f = s->set[set];
    a.P = h->P;
    a.M = h->M;
    a.ni = h->ni;
    a.nj = h->nj;
    a.ncell = (long long)h->ni * h->nj;
    a.npad = (long long)(h->ni + 2) * (h->nj + 2);
    a.nnode = (long long)(h->ni + 1) * (h->nj + 1);
    a.nif = (long long)(h->ni + 1) * h->nj;
    a.njf = (long long)h->ni * (h->nj + 1);
    a.qold = f.q0.p;
    a.d = f.d;
    a.vis = f.vis;
    a.dt = f.dt;
    a.dtmin = f.dtmin;
    a.w = f.w.p;
    a.w4 = f.w.p;
    a.navg = f.navg.p;
    a.ninfo = f.ninfo.p;
    a.dpre = f.dpre.p;
    a.gport = f.gport;
    a.qst[0] = f.q0.p;
    a.qst[1] = f.q1;
    a.qst[2] = f.q2;
    a.qst[3] = f.q3;
    a.gportb = s->gportb.p;
    a.gportb4 = s->gportb.p;
    a.portacc = s->portacc.p;
    a.xcs = s->xcs.p;
    a.ycs = s->ycs.p;
    a.lam_old = s->lamold.p;
    a.lamg = s->lamg.p;
    a.lamd = s->lamd.p;
    a.gbar = s->gbar.p;
    a.gbar4 = s->gbar.p;
    a.srcn = s->srcn.p;
    a.srcg = s->srcg.p;
    a.wself = s->wself.p;
    a.wvisc = s->wvisc.p;
    a.dbar = s->dbar.p;
    a.visbar = s->visbar.p;
    a.dtbar = s->dtbar.p;
    a.dout = s->dout.p;
    a.nbar = s->nbar.p;
    a.vfi = s->vfi.p;
    a.vfj = s->vfj.p;
    a.dtsum = s->dtsum.p;
    a.sens = geo >= 1;  // geo: 0 none, 1 scalars (RTOLERANCE, T0, S0), 2 everything
    a.geo = geo >= 2;
    double* sp = s->sens.p;
    const long long n = a.ncell;
    a.sxbar = sp; sp += 4 * n;
    a.sybar = sp; sp += 4 * n;
    a.volbar = sp; sp += n;
    a.dlbar = sp; sp += n;
    a.xcbar = sp; sp += a.npad;
    a.ycbar = sp; sp += a.npad;
    a.xnbar = sp; sp += a.nnode;
    a.ynbar = sp; sp += a.nnode;
    a.rtolc = sp; sp += n;
    a.rtoln = sp; sp += a.nnode;
    a.t0bar = sp; sp += n;
    a.s0bar = sp;
    return a;
}

long long sens_size(long long n, long long npad, long long nnode) {
    return 8 * n + 2 * n + 2 * npad + 2 * nnode + n + nnode + 2 * n;
}

const double kAlpha[4] = {0.25, 1.0 / 3.0, 0.5, 1.0};  // constants.f90:30-33

// Forward values of the state in set `set` (its q0), on stream st: the iteration with the
// solver's kernels (stages 1-3 keep their outputs), then every pass of the reverse that
// depends on the state alone.  Returns the number of kernels launched.
long long enqueue_forward_primal(tns_handle* h, tns_adjoint_state* s, int set, cudaStream_t st,
                                 const AdjForward* into = nullptr) {
    const Params& P = h->P;
    const Mesh& M = h->M;
    const AdjForward& f = into ? *into : s->set[set];
    long long nl = 0;
    if (!P.local) {
        tns::launch_dtmin(P, M, f.q0.p, h->partial.p, h->counter.p, f.dtmin, st);
        nl++;
    }
    // the type-6 ghosts read the port mass flux of each stage's input (one slice per stage)
    const int np = (int)h->port_ghosts.size();
    const size_t ng = (size_t)M.nghosts();
    Mesh Ms[4] = {M, M, M, M};
    double* qs[4] = {f.q0.p, f.q1, f.q2, f.q3};
    for (int k = 0; k < 4; k++) Ms[k].gport = f.gport + k * ng;
    auto gport = [&](int k) {
        if (np) {
            tns::launch_gport(P, Ms[k], qs[k], h->ports.p, np, f.gport + k * ng, st);
            nl++;
        }
    };
    tns::launch_dissipation(P, M, f.q0.p, f.d, f.dt, f.dtmin, st);
    gport(0);
    tns::launch_viscous(P, Ms[0], f.q0.p, f.vis, st);
    for (int k = 0; k < 3; k++) {
        if (k) gport(k);
        tns::launch_stage(P, Ms[k], qs[k], f.q0.p, qs[k + 1], f.d, f.vis, f.dt, f.dtmin, kAlpha[k], nullptr,
                          nullptr, h->status.p, st);
    }
    gport(3);
    return nl + 5;
}

// The passes of the reverse that depend on the state alone: the four stages' field sets,
// the node averages and the dissipation pre-pass.
long long enqueue_forward_state(tns_handle* h, tns_adjoint_state* s, int set, cudaStream_t st) {
    AdjForward& f = s->set[set];
    const size_t ng = (size_t)h->M.nghosts();
    double* qs[4] = {f.q0.p, f.q1, f.q2, f.q3};
    AdjArgs a = base_args(h, s, set, 0);
    for (int k = 0; k < 4; k++) {
        a.qin = qs[k];
        a.gport = f.gport + k * ng;
        a.w = f.w.p + (size_t)k * NWROW * a.npad;  // one field set per stage
        launch_points(k_adj_fields, a, a.npad, st);
    }
    a.w = f.w.p;
    a.gport = f.gport;
    launch_points(k_adj_nodes, a, a.nnode, st);
    launch_points(k_adj_diss_pre, a, a.ncell, st);
    return 6;
}

long long enqueue_forward(tns_handle* h, tns_adjoint_state* s, int set, cudaStream_t st) {
    const long long nl = enqueue_forward_primal(h, s, set, st);
    return nl + enqueue_forward_state(h, s, set, st);
}

// The reverse of the iteration whose forward values are in set `set`: lambda (s->lam)
// -> lambda dG/dQ_n, written back to s->lam.
long long enqueue_reverse(tns_handle* h, tns_adjoint_state* s, int set, int geo, cudaStream_t st) {
    const Params& P = h->P;
    AdjForward& f = s->set[set];
    long long nl = 0;
    AdjArgs a = base_args(h, s, set, geo);
    auto fork = [&](cudaStream_t to) {
        cudaEventRecord(s->ev, st);
        cudaStreamWaitEvent(to, s->ev, 0);
    };
    auto join = [&](cudaStream_t from) {
        cudaEventRecord(s->ev, from);
        cudaStreamWaitEvent(st, s->ev, 0);
    };
    double* qs[4] = {f.q0.p, f.q1, f.q2, f.q3};
    double* lam_stage[5] = {nullptr, s->lamA.p, s->lamB.p, s->lamA.p, s->lam.p};
    for (int k = 3; k >= 0; k--) {
        a.qin = qs[k];
        a.alpha = kAlpha[k];
        a.first = k == 3;
        a.stage1 = k == 0;
        a.lam_in = lam_stage[k + 1];
        a.lam_out = lam_stage[k];
        a.w = f.w.p + (size_t)k * NWROW * a.npad;     // this stage's field set
        a.gbar = s->gbar.p + (size_t)k * 5 * a.npad;  // one residual adjoint per stage
        a.gport = f.gport + (size_t)k * a.M.nghosts();
        a.gportb = s->gportb.p + (size_t)k * a.M.nghosts();
        launch_points(k_adj_stage, a, a.ncell, st);
        nl++;
        if (k == 0) {
            // dissipation / time-step reverse on a branch (it needs only D_bar, DT_bar)
            fork(s->side[0]);
            launch_points(k_adj_diss_faces, a, a.ncell, s->side[0]);
            launch_points(k_adj_diss_gather, a, a.ncell, s->side[0]);
            nl += 2;
            if (!P.local) {
                cudaMemsetAsync(s->dtsum.p, 0, sizeof(double), s->side[0]);
                k_adj_dtsum<<<148, ADJ_THREADS, 0, s->side[0]>>>(s->dtbar.p, a.ncell, s->dtsum.p);
                launch_points(k_adj_dtmin, a, a.ncell, s->side[0]);
                nl += 2;
            }
            // viscous reverse on the main stream
            launch_points(k_adj_faces, a, a.nif + a.njf, st);
            launch_points(k_adj_node_bar, a, a.nnode, st);
            launch_points(k_adj_slot_bar, a, a.npad, st);
            nl += 3;
        }
        fork(s->side[1]);
        launch_points(k_adj_gather_ghosts, a, band_count(a), s->side[1]);
        launch_points(k_adj_gather, a, a.ncell, st);
        nl += 2;
        join(s->side[1]);
        if (!h->port_ghosts.empty()) {
            // the port mass flux's adjoint down each port line
            launch_points(k_adj_port, a, a.ncell, st);
            nl++;
        }
    }
    if (geo >= 2) {
        // face-vector (and port) sensitivities of the whole step on their own branch
        fork(s->side[2]);
        launch_points(k_adj_geo, a, a.ncell, s->side[2]);
        nl++;
        if (!h->port_ghosts.empty()) {
            launch_points(k_adj_port_nodes, a, a.nnode, s->side[2]);
            nl++;
        }
    }
    join(s->side[0]);
    if (geo >= 2) join(s->side[2]);
    a.lam_out = s->lam.p;
    launch_points(k_adj_final, a, a.ncell, st);
    return nl + 1;
}

// One step: [forward of set X], the reverse of set X, and (mode bit 1) the forward of
// the other set on a branch beside the reverse.
long long enqueue_step(tns_handle* h, tns_adjoint_state* s, int set, int mode, int geo, cudaStream_t user) {
    long long nl = 0;
    cudaStream_t st = s->hp;
    cudaEventRecord(s->ev, user);
    cudaStreamWaitEvent(st, s->ev, 0);
    if (mode & 1) nl += enqueue_forward(h, s, set, st);
    else if (mode & 4) nl += enqueue_forward_state(h, s, set, st);
    if (mode & 2) {
        cudaEventRecord(s->ev, st);
        cudaStreamWaitEvent(s->side[3], s->ev, 0);
        nl += enqueue_forward(h, s, set ^ 1, s->side[3]);
    }
    nl += enqueue_reverse(h, s, set, geo, st);
    if (mode & 2) {
        cudaEventRecord(s->ev, s->side[3]);
        cudaStreamWaitEvent(st, s->ev, 0);
    }
    cudaEventRecord(s->ev, st);
    cudaStreamWaitEvent(user, s->ev, 0);
    return nl;
}

int check_mesh(tns_handle* h) {
    if (h->unstructured) return h->fail(TNS_ERR_UNSUPPORTED, "the adjoint needs one structured i x j block");
    if (h->precision != 0) return h->fail(TNS_ERR_ARG, "the adjoint runs on FP64 handles (precision 0)");
    if (!h->identity) return h->fail(TNS_ERR_ARG, "the adjoint needs cells numbered in (i, j) order");
    if (h->ni < 3 || h->nj < 3) return h->fail(TNS_ERR_ARG, "the adjoint needs at least 3 x 3 cells");
    for (int t : h->hgtype)
        if (t < 2 || t > 7) return h->fail(TNS_ERR_ARG, "BC type %d: the adjoint covers types 2-7", t);
    return TNS_OK;
}

}  // namespace

namespace tns_rt {
void adjoint_release(tns_handle* h) {
    tns_adjoint_state* s = h->adj;
    if (!s) return;
    for (auto& a : s->graph)
        for (auto& b : a)
            for (auto& g : b)
                if (g) cudaGraphExecDestroy(g);
    for (auto& x : s->side)
        if (x) {
            cudaStreamSynchronize(x);
            cudaStreamDestroy(x);
        }
    if (s->hp) {
        cudaStreamSynchronize(s->hp);
        cudaStreamDestroy(s->hp);
    }
    if (s->ev) cudaEventDestroy(s->ev);
    for (auto& f : s->set) {
        for (auto* b : {&f.q0, &f.rec, &f.w, &f.navg, &f.dpre})
            b->release();
        f.ninfo.release();
    }
    for (auto* b : {&s->lam, &s->lamA, &s->lamB, &s->lamold, &s->lamg, &s->lamd, &s->gbar, &s->srcn, &s->srcg,
                    &s->wself, &s->wvisc, &s->dbar, &s->visbar, &s->dtbar, &s->dout, &s->nbar, &s->vfi, &s->vfj,
                    &s->dtsum, &s->sens, &s->xcs, &s->ycs, &s->gportb, &s->portacc})
        b->release();
    delete s;
    h->adj = nullptr;
}
}  // namespace tns_rt

extern "C" {

int tns_adjoint_enable(tns_handle* h) {
    if (!h) return TNS_ERR_ARG;
    if (h->adj) return TNS_OK;
    int rc;
    if ((rc = check_mesh(h))) return rc;
    tns_adjoint_state* s = new tns_adjoint_state();
    h->adj = s;
    const long long n = (long long)h->ni * h->nj, npad = (long long)(h->ni + 2) * (h->nj + 2);
    const long long nnode = (long long)(h->ni + 1) * (h->nj + 1);
    const long long nif = (long long)(h->ni + 1) * h->nj, njf = (long long)h->ni * (h->nj + 1);
    s->nsens = sens_size(n, npad, nnode);
    struct Req {
        DevBuf<double>* b;
        long long count;
    };
    std::vector<Req> reqs = {{&s->lam, 5 * n}, {&s->lamA, 5 * n}, {&s->lamB, 5 * n}, {&s->lamold, 5 * n},
                             {&s->lamg, 5 * n}, {&s->lamd, 5 * n}, {&s->gbar, 4 * 5 * npad}, {&s->srcn, 16 * n},
                             {&s->srcg, 8 * n}, {&s->wself, 5 * n}, {&s->wvisc, 5 * npad}, {&s->dbar, 5 * n},
                             {&s->visbar, 4 * n}, {&s->dtbar, n}, {&s->dout, NDOUT * n}, {&s->nbar, 5 * nnode},
                             {&s->vfi, NVF * nif}, {&s->vfj, NVF * njf}, {&s->dtsum, 1}, {&s->sens, s->nsens},
                             {&s->xcs, npad}, {&s->ycs, npad}, {&s->gportb, 4 * (2 * (h->ni + h->nj))},
                             {&s->portacc, 3 * (2 * (h->ni + h->nj))}};
    for (auto& f : s->set)
        for (Req r : std::vector<Req>{{&f.q0, 5 * n}, {&f.rec, record_size(n, 2 * (h->ni + h->nj))},
                                      {&f.w, 4 * NWROW * npad}, {&f.navg, NNA * nnode}, {&f.dpre, NDPRE * n}})
            reqs.push_back(r);
    for (auto& r : reqs) {
        if ((rc = h->cuda(r.b->alloc((size_t)r.count), "cudaMalloc (adjoint)"))) {
            tns_rt::adjoint_release(h);
            return rc;
        }
    }
    rc = 0;
    for (auto& f : s->set)
        if (!rc) rc = h->cuda(f.ninfo.alloc((size_t)nnode), "cudaMalloc (adjoint)");
    int prio_low = 0, prio_high = 0;
    cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
#if !TNS_ADJ_PRIORITY
    prio_high = prio_low;
#endif
    for (int k = 0; k < 4; k++)
        if (!rc)
            rc = h->cuda(cudaStreamCreateWithPriority(&s->side[k], cudaStreamNonBlocking, k == 3 ? prio_low : prio_high),
                         "cudaStreamCreate");
    if (!rc) rc = h->cuda(cudaStreamCreateWithPriority(&s->hp, cudaStreamNonBlocking, prio_high), "cudaStreamCreate");
    if (!rc) rc = h->cuda(cudaEventCreateWithFlags(&s->ev, cudaEventDisableTiming), "cudaEventCreate");
    if (rc) {
        tns_rt::adjoint_release(h);
        return rc;
    }
    // the ghost ring of the residual adjoints stays zero; the sensitivities start at zero
    cudaMemsetAsync(s->gbar.p, 0, sizeof(double) * 4 * 5 * npad, h->stream);
    cudaMemsetAsync(s->wvisc.p, 0, sizeof(double) * 5 * npad, h->stream);
    cudaMemsetAsync(s->sens.p, 0, sizeof(double) * s->nsens, h->stream);
    cudaMemsetAsync(s->portacc.p, 0, sizeof(double) * s->portacc.n, h->stream);
    cudaMemsetAsync(s->gportb.p, 0, sizeof(double) * s->gportb.n, h->stream);
    for (auto& f : s->set) {
        f.carve(n);
        cudaMemsetAsync(f.rec.p, 0, sizeof(double) * f.rec.n, h->stream);
    }
    const AdjArgs a = base_args(h, s, 0, 0);
    launch_points(k_adj_centroids, a, npad, h->stream);
    return h->cuda(cudaStreamSynchronize(h->stream), "tns_adjoint_enable");
}

static int adjoint_step_impl(tns_handle* h, const double* d_q, const double* d_q_next, const double* d_rec,
                             double* d_lam, int flags) {
    if (!h || !d_lam || (!d_q && !(flags & TNS_ADJ_FROZEN))) return TNS_ERR_ARG;
    int rc;
    if (!h->adj && (rc = tns_adjoint_enable(h))) return rc;
    tns_adjoint_state* s = h->adj;
    const int geo = (flags & TNS_ADJ_SENSITIVITIES) ? 2 : ((flags & TNS_ADJ_SCALARS) ? 1 : 0);
    const int frozen = flags & TNS_ADJ_FROZEN ? 1 : 0;
    if (frozen && !s->have_forward)
        return h->fail(TNS_ERR_STATE, "tns_adjoint_step: TNS_ADJ_FROZEN before any step without it");
    if (frozen && d_q_next)
        return h->fail(TNS_ERR_ARG, "tns_adjoint_step: TNS_ADJ_FROZEN takes no next state");
    const size_t bytes = sizeof(double) * 5 * (size_t)h->ni * h->nj;
    cudaStream_t st = h->stream;
    int set = s->cur, mode = 0;
    if (d_rec && (frozen || d_q_next))
        return h->fail(TNS_ERR_ARG, "tns_adjoint_step_recorded: no TNS_ADJ_FROZEN, no next state");
    if (d_rec) {
        // forward values from the record: only the state-only passes run
        set = s->cur;
        mode = 4;
        AdjForward& f = s->set[set];
        if ((rc = h->cuda(cudaMemcpyAsync(f.q0.p, d_q, bytes, cudaMemcpyDeviceToDevice, st), "adjoint: state in")) ||
            (rc = h->cuda(cudaMemcpyAsync(f.rec.p, d_rec, sizeof(double) * f.rec.n, cudaMemcpyDeviceToDevice, st),
                          "adjoint: record in")))
            return rc;
    } else if (!frozen) {
        if (s->pre_set >= 0 && s->pre_ptr == d_q) {
            set = s->pre_set;  // prefetched by the previous step
        } else {
            set = s->cur;
            mode |= 1;
            if ((rc = h->cuda(cudaMemcpyAsync(s->set[set].q0.p, d_q, bytes, cudaMemcpyDeviceToDevice, st),
                              "adjoint: state in")))
                return rc;
        }
    }
    if (d_q_next) {
        mode |= 2;
        if ((rc = h->cuda(cudaMemcpyAsync(s->set[set ^ 1].q0.p, d_q_next, bytes, cudaMemcpyDeviceToDevice, st),
                          "adjoint: next state in")))
            return rc;
    }
    if ((rc = h->cuda(cudaMemcpyAsync(s->lam.p, d_lam, bytes, cudaMemcpyDeviceToDevice, st), "adjoint: lambda in")))
        return rc;
    if (h->profile) {
        s->launches += enqueue_step(h, s, set, mode, geo, st);
    } else {
        cudaGraphExec_t& ge = s->graph[set][mode][geo];
        if (!ge) {
            cudaGraph_t g;
            if ((rc = h->cuda(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "adjoint capture")))
                return rc;
            s->per_step[set][mode][geo] = enqueue_step(h, s, set, mode, geo, st);
            if ((rc = h->cuda(cudaStreamEndCapture(st, &g), "adjoint capture"))) return rc;
            rc = h->cuda(cudaGraphInstantiateWithFlags(&ge, g, TNS_ADJ_PRIORITY ? cudaGraphInstantiateFlagUseNodePriority : 0),
                         "adjoint graph instantiate");
            cudaGraphDestroy(g);
            if (rc) return rc;
        }
        if ((rc = h->cuda(cudaGraphLaunch(ge, st), "adjoint graph launch"))) return rc;
        s->launches += s->per_step[set][mode][geo];
    }
    s->cur = set;
    s->have_forward = true;
    s->pre_set = d_q_next ? (set ^ 1) : -1;
    s->pre_ptr = d_q_next;
    if ((rc = h->cuda(cudaMemcpyAsync(d_lam, s->lam.p, bytes, cudaMemcpyDeviceToDevice, st), "adjoint: lambda out")))
        return rc;
    return h->cuda(cudaGetLastError(), "tns_adjoint_step");
}

int tns_adjoint_step_next(tns_handle* h, const double* d_q, const double* d_q_next, double* d_lam, int flags) {
    return adjoint_step_impl(h, d_q, d_q_next, nullptr, d_lam, flags);
}

int tns_adjoint_step(tns_handle* h, const double* d_q, double* d_lam, int flags) {
    return adjoint_step_impl(h, d_q, nullptr, nullptr, d_lam, flags);
}

int tns_adjoint_step_recorded(tns_handle* h, const double* d_q, const double* d_rec, double* d_lam, int flags) {
    if (!d_rec) return TNS_ERR_ARG;
    return adjoint_step_impl(h, d_q, nullptr, d_rec, d_lam, flags);
}

long long tns_adjoint_record_size(tns_handle* h) {
    if (!h) return -1;
    return record_size((long long)h->ni * h->nj, 2LL * (h->ni + h->nj));
}

int tns_adjoint_record(tns_handle* h, const double* d_q, double* d_q_next, double* d_rec) {
    if (!h || !d_q || !d_q_next || !d_rec) return TNS_ERR_ARG;
    int rc;
    if (!h->adj && (rc = tns_adjoint_enable(h))) return rc;
    tns_adjoint_state* s = h->adj;
    const int set = s->cur;
    cudaStream_t st = h->stream;
    // the iteration with the solver's kernels, reading d_q and writing its forward values
    // straight into the record (stages 1-3, D, VIS, DT, DTMIN, port flux) and Q_{n+1}
    // into d_q_next
    AdjForward r;
    r.q0.p = const_cast<double*>(d_q);
    r.rec.p = d_rec;
    r.carve((long long)h->ni * h->nj);
    s->launches += enqueue_forward_primal(h, s, set, st, &r);
    Mesh M3 = h->M;
    M3.gport = r.gport + 3 * (size_t)h->M.nghosts();
    tns::launch_stage(h->P, M3, r.q3, r.q0.p, d_q_next, r.d, r.vis, r.dt, r.dtmin, kAlpha[3], nullptr, nullptr,
                      h->status.p, st);
    s->launches++;
    r.q0.p = nullptr;  // borrowed: not released by the DevBuf
    r.rec.p = nullptr;
    return h->cuda(cudaGetLastError(), "tns_adjoint_record");
}

long long tns_adjoint_sensitivity_size(tns_handle* h) {
    if (!h) return -1;
    const long long n = (long long)h->ni * h->nj;
    return sens_size(n, (long long)(h->ni + 2) * (h->nj + 2), (long long)(h->ni + 1) * (h->nj + 1));
}

int tns_adjoint_sensitivities(tns_handle* h, double* out, long long count, int reset) {
    if (!h || !out) return TNS_ERR_ARG;
    if (!h->adj) return h->fail(TNS_ERR_STATE, "tns_adjoint_sensitivities: the adjoint is not enabled");
    tns_adjoint_state* s = h->adj;
    if (count != s->nsens)
        return h->fail(TNS_ERR_ARG, "sensitivity buffer holds %lld values, not %lld", count, s->nsens);
    int rc;
    if ((rc = h->cuda(cudaMemcpyAsync(out, s->sens.p, sizeof(double) * s->nsens, cudaMemcpyDeviceToHost, h->stream),
                      "adjoint sensitivities")))
        return rc;
    if (reset) cudaMemsetAsync(s->sens.p, 0, sizeof(double) * s->nsens, h->stream);
    return h->cuda(cudaStreamSynchronize(h->stream), "adjoint sensitivities");
}

long long tns_adjoint_launch_count(tns_handle* h) { return h && h->adj ? h->adj->launches : 0; }

int tns_copy_state_device(tns_handle* h, double* d_buf, int direction) {
    if (!h || !d_buf || (direction != 0 && direction != 1)) return TNS_ERR_ARG;
    if (h->precision != 0) return h->fail(TNS_ERR_ARG, "tns_copy_state_device: FP64 handles only");
    if (!h->identity) return h->fail(TNS_ERR_ARG, "tns_copy_state_device: cells must be numbered in (i, j) order");
    const size_t bytes = sizeof(double) * 5 * (size_t)h->ni * h->nj;
    int rc;
    if (direction == 0) {
        rc = h->cuda(cudaMemcpyAsync(d_buf, h->qa.p, bytes, cudaMemcpyDeviceToDevice, h->stream), "state to device");
    } else {
        rc = h->cuda(cudaMemcpyAsync(h->qa.p, d_buf, bytes, cudaMemcpyDeviceToDevice, h->stream), "state from device");
        if (!rc) h->have_state = true;
    }
    return rc;
}

}  // extern "C"
