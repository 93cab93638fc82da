// tns_adjoint.cu -- the discrete adjoint of one FP64 RK4 iteration on the device.
//
// tns_adjoint_step(h, Q_n, lambda) recomputes the iteration from the checkpoint Q_n with
// the solver's own FP64 kernels (dissipation + DT, viscous flux, stages 1-3, keeping every
// stage input), then runs the hand-derived reverse of tns_adjoint.cuh: stages 4..1 (field
// set, residual / update / source reverse, gather into the stage input), the viscous flux
// reverse inside stage 1 (node averages, faces, nodes, slots), and the dissipation / time
// step reverse.  The whole step -- recompute and reverse, 25 to 30 kernels -- is one CUDA
// graph per handle (one with and one without the parameter sensitivities), replayed on
// the handle's stream for every checkpoint.
#include <cuda_runtime.h>

#include <cstring>
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

// Device buffers and graphs of the adjoint of one handle.
struct tns_adjoint_state {
    DevBuf<double> q0, q1, q2, q3, d, vis, dt, dtmin, lam, lamA, lamB, lamold, lamg, lamd, w, gbar, srcn, srcg,
        wself, wvisc, dbar, visbar, dtbar, dpre, dout, navg, nbar, vfi, vfj, dtsum, sens, xcs, ycs;
    // branches of a step: the ghost gather beside the interior gather, the dissipation
    // reverse beside the viscous reverse
    cudaStream_t side[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev = nullptr;
    DevBuf<int> ninfo;
    long long nsens = 0;
    cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};  // [frozen][sensitivities]
    long long per_step[4] = {0, 0, 0, 0};
    bool have_forward = false;  // the buffers hold the forward values of the last state
    long long launches = 0;
};

namespace {

AdjArgs base_args(tns_handle* h, tns_adjoint_state* s, int geo) {
    AdjArgs a{};
    a.P = h->P;
    a.M = h->M;
    a.ni = h->ni;
    a.nj = h->nj;
    a.ncell = (long long)h->ni * h->nj;
    a.npad = (long long)(h->ni + 2) * (h->nj + 2);
    a.nnode = (long long)(h->ni + 1) * (h->nj + 1);
    a.nif = (long long)(h->ni + 1) * h->nj;
    a.njf = (long long)h->ni * (h->nj + 1);
    a.qold = s->q0.p;
    a.d = s->d.p;
    a.vis = s->vis.p;
    a.dt = s->dt.p;
    a.dtmin = s->dtmin.p;
    a.w = s->w.p;
    a.xcs = s->xcs.p;
    a.ycs = s->ycs.p;
    a.lam_old = s->lamold.p;
    a.lamg = s->lamg.p;
    a.lamd = s->lamd.p;
    a.gbar = s->gbar.p;
    a.gbar4 = s->gbar.p;
    a.w4 = s->w.p;
    a.srcn = s->srcn.p;
    a.srcg = s->srcg.p;
    a.wself = s->wself.p;
    a.wvisc = s->wvisc.p;
    a.dbar = s->dbar.p;
    a.visbar = s->visbar.p;
    a.dtbar = s->dtbar.p;
    a.dpre = s->dpre.p;
    a.dout = s->dout.p;
    a.navg = s->navg.p;
    a.ninfo = s->ninfo.p;
    a.nbar = s->nbar.p;
    a.vfi = s->vfi.p;
    a.vfj = s->vfj.p;
    a.dtsum = s->dtsum.p;
    a.geo = geo;
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

// One reverse step, enqueued on stream st: recompute from q0, reverse into lamold, copy
// the result to lam.  With `frozen` the forward values of the previous step's state are
// reused: no recompute, no field sets, node averages or dissipation pre-pass.  Returns
// the number of kernels launched.
long long enqueue_step(tns_handle* h, tns_adjoint_state* s, int geo, int frozen, cudaStream_t st) {
    const Params& P = h->P;
    const Mesh& M = h->M;
    long long nl = 0;
    static const double alpha[4] = {0.25, 1.0 / 3.0, 0.5, 1.0};  // constants.f90:30-33
    double* qs[4] = {s->q0.p, s->q1.p, s->q2.p, s->q3.p};
    if (!frozen) {
        // forward recompute with the solver's kernels
        if (!P.local) {
            tns::launch_dtmin(P, M, s->q0.p, h->partial.p, h->counter.p, s->dtmin.p, st);
            nl++;
        }
        tns::launch_dissipation(P, M, s->q0.p, s->d.p, s->dt.p, s->dtmin.p, st);
        tns::launch_viscous(P, M, s->q0.p, s->vis.p, st);
        for (int k = 0; k < 3; k++)
            tns::launch_stage(P, M, qs[k], s->q0.p, qs[k + 1], s->d.p, s->vis.p, s->dt.p, s->dtmin.p, alpha[k],
                              nullptr, nullptr, st);
        nl += 5;
    }
    // reverse
    AdjArgs a = base_args(h, s, geo);
    auto fork = [&](cudaStream_t to) {
        cudaEventRecord(s->ev, st);
        cudaStreamWaitEvent(to, s->ev, 0);
    };
    auto join = [&](cudaStream_t from) {
        cudaEventRecord(s->ev, from);
        cudaStreamWaitEvent(st, s->ev, 0);
    };
    double* lam_stage[5] = {nullptr, s->lamA.p, s->lamB.p, s->lamA.p, s->lam.p};
    for (int k = 3; k >= 0; k--) {
        a.qin = qs[k];
        a.alpha = alpha[k];
        a.first = k == 3;
        a.stage1 = k == 0;
        a.lam_in = lam_stage[k + 1];
        a.lam_out = lam_stage[k];
        a.w = s->w.p + (size_t)k * NWROW * a.npad;  // one field set per stage
        a.gbar = s->gbar.p + (size_t)k * 5 * a.npad;  // one residual adjoint per stage
        if (!frozen) {
            launch_points(k_adj_fields, a, a.npad, st);
            nl++;
        }
        launch_points(k_adj_stage, a, a.ncell, st);
        nl++;
        if (k == 0) {
            // dissipation / time-step reverse on a branch (it needs only D_bar, DT_bar)
            fork(s->side[0]);
            if (!frozen) {
                launch_points(k_adj_diss_pre, a, a.ncell, s->side[0]);
                nl++;
            }
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
            if (!frozen) {
                launch_points(k_adj_nodes, a, a.nnode, st);
                nl++;
            }
            launch_points(k_adj_faces, a, a.nif + a.njf, st);
            if (geo) {
                // face-vector sensitivities of the whole step on their own branch
                fork(s->side[2]);
                launch_points(k_adj_geo, a, a.ncell, s->side[2]);
                nl++;
            }
            launch_points(k_adj_node_bar, a, a.nnode, st);
            launch_points(k_adj_slot_bar, a, a.npad, st);
            nl += 3;
        }
        fork(s->side[1]);
        launch_points(k_adj_gather_ghosts, a, band_count(a), s->side[1]);
        launch_points(k_adj_gather, a, a.ncell, st);
        nl += 2;
        join(s->side[1]);
    }
    join(s->side[0]);
    if (geo) join(s->side[2]);
    a.lam_out = s->lam.p;
    launch_points(k_adj_final, a, a.ncell, st);
    nl++;
    return nl;
}

int check_mesh(tns_handle* h) {
    if (h->precision != 0) return h->fail(TNS_ERR_ARG, "the adjoint runs on FP64 handles (precision 0)");
    if (!h->identity) return h->fail(TNS_ERR_ARG, "the adjoint needs cells numbered in (i, j) order");
    if (h->ni < 3 || h->nj < 3) return h->fail(TNS_ERR_ARG, "the adjoint needs at least 3 x 3 cells");
    for (int t : h->hgtype)
        if (t < 2 || t > 5) return h->fail(TNS_ERR_ARG, "BC type %d: the adjoint covers types 2-5", t);
    return TNS_OK;
}

}  // namespace

namespace tns_rt {
void adjoint_release(tns_handle* h) {
    tns_adjoint_state* s = h->adj;
    if (!s) return;
    for (auto& g : s->graph)
        if (g) cudaGraphExecDestroy(g);
    for (auto& x : s->side)
        if (x) {
            cudaStreamSynchronize(x);
            cudaStreamDestroy(x);
        }
    if (s->ev) cudaEventDestroy(s->ev);
    for (auto* b : {&s->q0, &s->q1, &s->q2, &s->q3, &s->d, &s->vis, &s->dt, &s->dtmin, &s->lam, &s->lamA, &s->lamB,
                    &s->lamold, &s->lamg, &s->lamd, &s->w, &s->gbar, &s->srcn, &s->srcg, &s->wself, &s->wvisc, &s->dbar, &s->visbar,
                    &s->dtbar, &s->dpre, &s->dout, &s->navg, &s->nbar, &s->vfi, &s->vfj, &s->dtsum, &s->sens, &s->xcs,
                    &s->ycs})
        b->release();
    s->ninfo.release();
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
    } reqs[] = {{&s->q0, 5 * n}, {&s->q1, 5 * n}, {&s->q2, 5 * n}, {&s->q3, 5 * n}, {&s->d, 5 * n},
                {&s->vis, 4 * n}, {&s->dt, n}, {&s->dtmin, 1}, {&s->lam, 5 * n}, {&s->lamA, 5 * n},
                {&s->lamB, 5 * n}, {&s->lamold, 5 * n}, {&s->lamg, 5 * n}, {&s->lamd, 5 * n},
                {&s->w, 4 * NWROW * npad}, {&s->gbar, 4 * 5 * npad},
                {&s->srcn, 16 * n}, {&s->srcg, 8 * n}, {&s->wself, 5 * n}, {&s->wvisc, 5 * npad},
                {&s->dbar, 5 * n}, {&s->visbar, 4 * n}, {&s->dtbar, n}, {&s->dpre, NDPRE * n},
                {&s->dout, NDOUT * n}, {&s->navg, NNA * nnode}, {&s->nbar, 5 * nnode}, {&s->vfi, NVF * nif},
                {&s->vfj, NVF * njf}, {&s->dtsum, 1}, {&s->sens, s->nsens}, {&s->xcs, npad}, {&s->ycs, npad}};
    for (auto& r : reqs) {
        if ((rc = h->cuda(r.b->alloc((size_t)r.count), "cudaMalloc (adjoint)"))) {
            tns_rt::adjoint_release(h);
            return rc;
        }
    }
    if ((rc = h->cuda(s->ninfo.alloc((size_t)nnode), "cudaMalloc (adjoint)")) ||
        (rc = h->cuda(cudaStreamCreateWithFlags(&s->side[0], cudaStreamNonBlocking), "cudaStreamCreate")) ||
        (rc = h->cuda(cudaStreamCreateWithFlags(&s->side[1], cudaStreamNonBlocking), "cudaStreamCreate")) ||
        (rc = h->cuda(cudaStreamCreateWithFlags(&s->side[2], cudaStreamNonBlocking), "cudaStreamCreate")) ||
        (rc = h->cuda(cudaEventCreateWithFlags(&s->ev, cudaEventDisableTiming), "cudaEventCreate"))) {
        tns_rt::adjoint_release(h);
        return rc;
    }
    // the ghost ring of the residual adjoint stays zero; the sensitivities start at zero
    cudaMemsetAsync(s->gbar.p, 0, sizeof(double) * 4 * 5 * npad, h->stream);
    cudaMemsetAsync(s->wvisc.p, 0, sizeof(double) * 5 * npad, h->stream);
    cudaMemsetAsync(s->sens.p, 0, sizeof(double) * s->nsens, h->stream);
    const AdjArgs a = base_args(h, s, 0);
    launch_points(k_adj_centroids, a, npad, h->stream);
    return h->cuda(cudaStreamSynchronize(h->stream), "tns_adjoint_enable");
}

int tns_adjoint_step(tns_handle* h, const double* d_q, double* d_lam, int flags) {
    if (!h || !d_q || !d_lam) return TNS_ERR_ARG;
    int rc;
    if (!h->adj && (rc = tns_adjoint_enable(h))) return rc;
    tns_adjoint_state* s = h->adj;
    const int geo = flags & TNS_ADJ_SENSITIVITIES ? 1 : 0;
    const int frozen = flags & TNS_ADJ_FROZEN ? 1 : 0;
    if (frozen && !s->have_forward)
        return h->fail(TNS_ERR_STATE, "tns_adjoint_step: TNS_ADJ_FROZEN before any step without it");
    const size_t bytes = sizeof(double) * 5 * (size_t)h->ni * h->nj;
    cudaStream_t st = h->stream;
    if ((!frozen &&
         (rc = h->cuda(cudaMemcpyAsync(s->q0.p, d_q, bytes, cudaMemcpyDeviceToDevice, st), "adjoint: state in"))) ||
        (rc = h->cuda(cudaMemcpyAsync(s->lam.p, d_lam, bytes, cudaMemcpyDeviceToDevice, st), "adjoint: lambda in")))
        return rc;
    const int gi = frozen * 2 + geo;
    if (h->profile) {
        s->launches += enqueue_step(h, s, geo, frozen, st);
    } else {
        if (!s->graph[gi]) {
            cudaGraph_t g;
            if ((rc = h->cuda(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "adjoint capture")))
                return rc;
            s->per_step[gi] = enqueue_step(h, s, geo, frozen, st);
            if ((rc = h->cuda(cudaStreamEndCapture(st, &g), "adjoint capture"))) return rc;
            rc = h->cuda(cudaGraphInstantiate(&s->graph[gi], g, 0), "adjoint graph instantiate");
            cudaGraphDestroy(g);
            if (rc) return rc;
        }
        if ((rc = h->cuda(cudaGraphLaunch(s->graph[gi], st), "adjoint graph launch"))) return rc;
        s->launches += s->per_step[gi];
    }
    s->have_forward = true;
    if ((rc = h->cuda(cudaMemcpyAsync(d_lam, s->lam.p, bytes, cudaMemcpyDeviceToDevice, st), "adjoint: lambda out")))
        return rc;
    return h->cuda(cudaGetLastError(), "tns_adjoint_step");
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
