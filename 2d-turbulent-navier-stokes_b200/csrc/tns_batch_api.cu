// tns_batch_api.cu -- batch runtime: many solver handles advanced together.
//
// A batch co-schedules cases created with tns_create (any sizes, any parameters, one
// precision mode).  Each kernel phase of an RK4 iteration (dissipation pre-pass, frozen
// viscous flux, four stages) is ONE launch over a table of (case, tile j, tile i)
// entries covering every active case, so small cases share the GPU instead of each
// paying a full set of launches on a mostly idle device.  One iteration per state parity
// (mixed ping-pong) and monitor mode is captured as a CUDA graph; the graphs are
// re-captured when the set of active cases changes, with the tile table compacted to
// the active cases.  Per-case residual records drive a per-case stop criterion
// (convergence masking) and a case whose state turns non-finite is masked off while the
// others carry on.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "tns_handle.h"
#include "tns_tile.cuh"

using tns::BatchCase;

#ifndef TNS_BATCH_BLOCK
#define TNS_BATCH_BLOCK 8
#endif

struct tns_batch {
    std::string err;
    std::vector<tns_handle*> cases;
    int precision = 0;
    cudaStream_t stream = nullptr;
    std::vector<BatchCase> desc;          // host copy of the device descriptors
    std::vector<int> cur_at_desc;         // mixed: member parity the descriptors map
    std::vector<int> active, failed;      // host masks
    std::vector<int> active_at_capture;
    DevBuf<BatchCase> d_desc;
    DevBuf<int> d_active;
    DevBuf<int4> d_tiles;
    DevBuf<unsigned long long> d_cdiff;   // [ncases][5]
    DevBuf<unsigned int> d_status;        // [ncases]
    unsigned long long* h_cdiff = nullptr;  // pinned [ncases][5]
    unsigned int* h_status = nullptr;       // pinned [ncases]
    int ntiles = 0;
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [monitor][parity]
    // schedule 2: BLOCK unmonitored iterations in one graph per starting parity; each
    // case's chain runs ahead on its stream with no join between the iterations
    static constexpr int BLOCK = TNS_BATCH_BLOCK;
    cudaGraphExec_t block[2] = {nullptr, nullptr};
    long long per_block = 0;
    // schedule: 0 = one launch per phase over the tile table of all active cases;
    // 1 = each case's own single-case launches on one of several streams, captured as
    // parallel branches of one graph (cases run concurrently, kernels as for tns_run);
    // 2 = as 1, with BLOCK unmonitored iterations per graph; 3 = one persistent
    // cooperative launch per run of up to PERSIST unmonitored iterations (grid barriers
    // between the phases), monitored iterations as schedule 0
    int mode = 0;
    bool general = false;  // a case is a general mesh: per-case schedules (1, 2) only
    static constexpr int PERSIST = 256;
    int persist_grid = 0;               // resident blocks of the persistent kernel
    DevBuf<unsigned int> d_bar;         // its grid barrier: arrival counter, generation
    DevBuf<unsigned int> d_error;       // bit 2: a grid barrier gave up
    unsigned int* h_error = nullptr;    // pinned
    std::vector<cudaStream_t> branch;
    std::vector<int> branch_of;  // case -> branch stream (largest cases spread first)
    std::vector<cudaEvent_t> join;
    cudaEvent_t fork = nullptr;
    long long per_iter[2] = {0, 0};
    long long launches = 0;

    int fail(int code, const char* fmt, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        err = buf;
        return code;
    }
    int cuda(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return TNS_OK;
        return fail(TNS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    }
    void drop_graphs() {
        for (auto& row : graph)
            for (auto& g : row)
                if (g) {
                    cudaGraphExecDestroy(g);
                    g = nullptr;
                }
        for (auto& g : block)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    }
};

namespace {

// Descriptor of case k: every argument block of its launches (the ones
// enqueue_iteration_f64 / enqueue_iteration_mx in tns_api.cu pass), with parity 0 of the
// mixed ping-pong reading the member's current state buffer.
BatchCase describe(tns_batch* b, int k) {
    tns_handle* h = b->cases[k];
    BatchCase c{};
    c.P = h->P;
    c.M = h->M;
    c.dtmin = h->dtmin.p;
    unsigned long long* cdiff = b->d_cdiff.p + 5 * (size_t)k;
    unsigned int* status = b->d_status.p + k;
    if (h->precision == 0) {
        double *A = h->qa.p, *B = h->qb.p, *Cq = h->qc.p;
        c.diss = tns::DissArgs<double>{A, h->d.p, h->dt.p, h->dtmin.p};
        c.q = A;
        c.vis = h->vis.p;
        const double alpha[4] = {0.25, 1.0 / 3.0, 0.5, 1.0};  // constants.f90:30-33
        const double* in[4] = {A, B, Cq, B};
        double* out[4] = {B, Cq, B, A};
        for (int mon = 0; mon < 2; mon++)
            for (int st = 0; st < 4; st++)
                c.stage[mon][st] = tns::StageArgs{in[st], A, out[st], h->d.p, h->vis.p, h->dt.p, h->dtmin.p,
                                                  alpha[st], (mon && st == 3) ? cdiff : nullptr,
                                                  st == 3 ? status : nullptr, status};
    } else {
        double* q[2] = {h->state(), h->other_state()};
        c.qmx[0] = q[0];
        c.qmx[1] = q[1];
        c.df = h->df.p;
        c.dtf = h->dtf.p;
        c.visf = h->visf.p;
        const float alpha[4] = {0.25f, 1.0f / 3.0f, 0.5f, 1.0f};
        const float* in[4] = {nullptr, h->dqb.p, h->dqc.p, h->dqb.p};
        float* out[4] = {h->dqb.p, h->dqc.p, h->dqb.p, nullptr};
        for (int par = 0; par < 2; par++)
            for (int mon = 0; mon < 2; mon++)
                for (int st = 0; st < 4; st++)
                    c.stage_mx[par][mon][st] = tns::StageArgsMx{
                        q[par], in[st], out[st], st == 3 ? q[1 - par] : nullptr, h->df.p, h->visf.p, h->dtf.p,
                        h->dtmin.p, alpha[st], (mon && st == 3) ? cdiff : nullptr, st == 3 ? status : nullptr,
                        status};
    }
    return c;
}

int upload_descriptors(tns_batch* b) {
    const int n = (int)b->cases.size();
    b->desc.resize(n);
    b->cur_at_desc.resize(n);
    for (int k = 0; k < n; k++) {
        b->desc[k] = describe(b, k);
        b->cur_at_desc[k] = b->cases[k]->cur;
    }
    b->drop_graphs();
    int rc;
    if ((rc = b->cuda(cudaMemcpyAsync(b->d_desc.p, b->desc.data(), n * sizeof(BatchCase), cudaMemcpyHostToDevice,
                                      b->stream), "cudaMemcpyAsync")))
        return rc;
    return b->cuda(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize");
}

// Tile table of the active cases, case by case, j tiles fastest (the single-case grid
// order).
int upload_tiles(tns_batch* b) {
    std::vector<int4> t;
    const int n = (int)b->cases.size();
    for (int k = 0; k < n; k++) {
        if (!b->active[k] || b->cases[k]->unstructured) continue;
        const tns::Mesh& M = b->cases[k]->M;
        const int tj = (M.nj + tns::TJ - 1) / tns::TJ, ti = (M.ni + tns::TI - 1) / tns::TI;
        for (int y = 0; y < ti; y++)
            for (int x = 0; x < tj; x++) t.push_back(make_int4(k, x, y, 0));
    }
    b->ntiles = (int)t.size();
    int rc;
    // the stream is idle here (masks change only between synchronised iterations)
    if (!t.empty() && (rc = b->cuda(cudaMemcpyAsync(b->d_tiles.p, t.data(), t.size() * sizeof(int4),
                                                    cudaMemcpyHostToDevice, b->stream), "cudaMemcpyAsync")))
        return rc;
    if ((rc = b->cuda(cudaMemcpyAsync(b->d_active.p, b->active.data(), n * sizeof(int), cudaMemcpyHostToDevice,
                                      b->stream), "cudaMemcpyAsync")) ||
        (rc = b->cuda(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize")))
        return rc;
    b->active_at_capture = b->active;
    b->drop_graphs();
    return TNS_OK;
}

// One RK4 iteration of every active case (the phases of enqueue_iteration_f64 /
// enqueue_iteration_mx in tns_api.cu, each over the whole tile table).  The global
// time step (LOCAL=0) and the type-6 port columns are per-case reductions, launched
// per case that needs them.
void enqueue_batch_iteration(tns_batch* b, int parity, bool monitor) {
    cudaStream_t s = b->stream;
    const bool mixed = b->precision == 1;
    const int n = (int)b->cases.size();
    const int nt = b->ntiles;
    auto state = [&](int k) { return mixed ? b->desc[k].qmx[parity] : b->desc[k].q; };
    for (int k = 0; k < n; k++) {
        if (!b->active[k]) continue;
        tns_handle* h = b->cases[k];
        if (!h->P.local) {
            tns::launch_dtmin(h->P, h->M, state(k), h->partial.p, h->counter.p, h->dtmin.p, s);
            b->launches++;
        }
    }
    auto phase = [&](int kernel, int stage) {
        if (mixed)
            tns::launch_batch_mx(b->d_desc.p, b->d_tiles.p, b->d_active.p, nt, kernel, parity, stage,
                                 monitor ? 1 : 0, s);
        else
            tns::launch_batch_f64(b->d_desc.p, b->d_tiles.p, b->d_active.p, nt, kernel, stage, monitor ? 1 : 0, s);
        b->launches++;
    };
    phase(0, 0);
    if (monitor) cudaMemsetAsync(b->d_cdiff.p, 0, 5 * (size_t)n * sizeof(unsigned long long), s);
    for (int st = 0; st < 4; st++) {
        for (int k = 0; k < n; k++) {
            tns_handle* h = b->cases[k];
            const int np = (int)h->port_ghosts.size();
            if (!b->active[k] || !np) continue;
            if (mixed) {
                const float* in[4] = {nullptr, h->dqb.p, h->dqc.p, h->dqb.p};
                tns::launch_gport_mx(h->P, h->M, state(k), in[st], h->ports.p, np, h->gport.p, s);
            } else {
                const double* in[4] = {b->desc[k].q, h->qb.p, h->qc.p, h->qb.p};
                tns::launch_gport(h->P, h->M, in[st], h->ports.p, np, h->gport.p, s);
            }
            b->launches++;
        }
        if (st == 0) phase(1, 0);
        phase(2, st);
    }
}

// Per-case launches on branch streams (schedule 1): ``iters`` single-case iterations of
// every active case (state parity alternating from ``parity``), forked from and joined
// back to the batch stream.
void enqueue_branches(tns_batch* b, int parity, bool monitor, int iters = 1) {
    const int n = (int)b->cases.size();
    const int nb = (int)b->branch.size();
    cudaEventRecord(b->fork, b->stream);
    std::vector<char> used(nb, 0);
    for (int k = 0; k < n; k++) {
        if (!b->active[k]) continue;
        tns_handle* h = b->cases[k];
        const int bi = b->branch_of[k];
        if (!used[bi]) {
            cudaStreamWaitEvent(b->branch[bi], b->fork, 0);
            used[bi] = 1;
        }
        cudaStream_t keep = h->stream, keep_side = h->side;
        const bool prof = h->profile;
        const long long before = h->launches;
        h->stream = b->branch[bi];
        h->side = nullptr;   // the case's pre-passes in order: the batch is parallel enough
        h->profile = false;  // no event synchronisation inside a capture
        for (int i = 0; i < iters; i++) {
            const int par = parity ^ (i & 1);
            if (b->precision == 1)
                tns_rt::enqueue_iteration_mx(h, monitor, const_cast<double*>(b->desc[k].qmx[par]),
                                             const_cast<double*>(b->desc[k].qmx[1 - par]));
            else
                tns_rt::enqueue_iteration_f64(h, monitor);
        }
        b->launches += h->launches - before;
        h->launches = before;
        h->stream = keep;
        h->side = keep_side;
        h->profile = prof;
    }
    for (int bi = 0; bi < nb; bi++)
        if (used[bi]) {
            cudaEventRecord(b->join[bi], b->branch[bi]);
            cudaStreamWaitEvent(b->stream, b->join[bi], 0);
        }
}

// Status words (and, on a monitored iteration, the CDIFF slots) of every case into the
// pinned host arrays; the caller synchronises the batch stream.
int fetch_monitor(tns_batch* b, bool monitor) {
    const int n = (int)b->cases.size();
    int rc;
    if (b->mode == 0 || b->mode == 3) {  // the tile-table kernels write the batch's own slots
        if ((rc = b->cuda(cudaMemcpyAsync(b->h_status, b->d_status.p, n * sizeof(unsigned int),
                                          cudaMemcpyDeviceToHost, b->stream), "cudaMemcpyAsync")))
            return rc;
        if (b->mode == 3 && (rc = b->cuda(cudaMemcpyAsync(b->h_error, b->d_error.p, sizeof(unsigned int),
                                                          cudaMemcpyDeviceToHost, b->stream), "cudaMemcpyAsync")))
            return rc;
        if (monitor && (rc = b->cuda(cudaMemcpyAsync(b->h_cdiff, b->d_cdiff.p, 5 * n * sizeof(unsigned long long),
                                                     cudaMemcpyDeviceToHost, b->stream), "cudaMemcpyAsync")))
            return rc;
        return TNS_OK;
    }
    for (int k = 0; k < n; k++) {
        if (!b->active[k]) continue;
        tns_handle* h = b->cases[k];
        if ((rc = b->cuda(cudaMemcpyAsync(b->h_status + k, h->status.p, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                          b->stream), "cudaMemcpyAsync")))
            return rc;
        if (monitor && (rc = b->cuda(cudaMemcpyAsync(b->h_cdiff + 5 * k, h->cdiff.p, 5 * sizeof(unsigned long long),
                                                     cudaMemcpyDeviceToHost, b->stream), "cudaMemcpyAsync")))
            return rc;
    }
    return TNS_OK;
}

int ensure_block_graph(tns_batch* b, int parity) {
    cudaGraphExec_t* g = &b->block[parity];
    if (*g) return TNS_OK;
    int rc;
    if ((rc = b->cuda(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "capture"))) return rc;
    const long long before = b->launches;
    enqueue_branches(b, parity, false, tns_batch::BLOCK);
    b->per_block = b->launches - before;
    b->launches = before;
    cudaGraph_t graph;
    if ((rc = b->cuda(cudaStreamEndCapture(b->stream, &graph), "capture"))) return rc;
    rc = b->cuda(cudaGraphInstantiate(g, graph, 0), "cudaGraphInstantiate");
    cudaGraphDestroy(graph);
    return rc;
}

int ensure_batch_graph(tns_batch* b, int monitor, int parity) {
    cudaGraphExec_t* g = &b->graph[monitor][parity];
    if (*g) return TNS_OK;
    int rc;
    if ((rc = b->cuda(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "capture"))) return rc;
    const long long before = b->launches;
    if (b->mode == 1 || b->mode == 2)
        enqueue_branches(b, parity, monitor != 0);
    else
        enqueue_batch_iteration(b, parity, monitor != 0);
    b->per_iter[monitor] = b->launches - before;
    b->launches = before;
    cudaGraph_t graph;
    if ((rc = b->cuda(cudaStreamEndCapture(b->stream, &graph), "capture"))) return rc;
    rc = b->cuda(cudaGraphInstantiate(g, graph, 0), "cudaGraphInstantiate");
    cudaGraphDestroy(graph);
    return rc;
}

}  // namespace

extern "C" {

int tns_batch_create(tns_handle* const* cases, int ncases, tns_batch** out) {
    if (!out) return TNS_ERR_ARG;
    *out = nullptr;
    if (!cases || ncases <= 0) return TNS_ERR_ARG;
    tns_batch* b = new tns_batch();
    *out = b;
    for (int k = 0; k < ncases; k++) {
        if (!cases[k]) return b->fail(TNS_ERR_ARG, "tns_batch_create: case %d is a null handle", k);
        for (int j = 0; j < k; j++)
            if (cases[j] == cases[k]) return b->fail(TNS_ERR_ARG, "tns_batch_create: case %d repeats case %d", k, j);
        if (!cases[k]->qa.p) return b->fail(TNS_ERR_STATE, "tns_batch_create: case %d was not created", k);
        if (cases[k]->unstructured) b->general = true;
    }
    b->cases.assign(cases, cases + ncases);
    b->precision = cases[0]->precision;
    for (int k = 1; k < ncases; k++)
        if (cases[k]->precision != b->precision)
            return b->fail(TNS_ERR_ARG, "tns_batch_create: case %d has precision %d, case 0 has %d", k,
                           cases[k]->precision, b->precision);
    long long ntiles = 0;
    for (tns_handle* h : b->cases)
        if (!h->unstructured)
            ntiles += (long long)((h->M.nj + tns::TJ - 1) / tns::TJ) * ((h->M.ni + tns::TI - 1) / tns::TI);
    if (ntiles > 0x7fffffffLL) return b->fail(TNS_ERR_TOO_LARGE, "tns_batch_create: %lld tiles", ntiles);
    int rc;
    if ((rc = b->cuda(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate")) ||
        (rc = b->cuda(b->d_desc.alloc(ncases), "cudaMalloc")) || (rc = b->cuda(b->d_active.alloc(ncases), "cudaMalloc")) ||
        (rc = b->cuda(b->d_tiles.alloc((size_t)ntiles), "cudaMalloc")) ||
        (rc = b->cuda(b->d_cdiff.alloc(5 * (size_t)ncases), "cudaMalloc")) ||
        (rc = b->cuda(b->d_status.alloc(ncases), "cudaMalloc")) ||
        (rc = b->cuda(cudaMallocHost((void**)&b->h_cdiff, 5 * ncases * sizeof(unsigned long long)), "cudaMallocHost")) ||
        (rc = b->cuda(cudaMallocHost((void**)&b->h_status, ncases * sizeof(unsigned int)), "cudaMallocHost")) ||
        (rc = b->cuda(cudaMemset(b->d_status.p, 0, ncases * sizeof(unsigned int)), "cudaMemset")))
        return rc;
    b->active.assign(ncases, 1);
    b->failed.assign(ncases, 0);
    if ((rc = upload_descriptors(b)) || (rc = upload_tiles(b))) return rc;
    // general meshes have no tile table: their cases run through their own iterations
    return b->general ? tns_batch_set_schedule(b, 2) : TNS_OK;
}

int tns_batch_set_active(tns_batch* b, const int* active) {
    if (!b || !active) return TNS_ERR_ARG;
    const int n = (int)b->cases.size();
    bool cleared = false;
    for (int k = 0; k < n; k++) {
        b->active[k] = active[k] ? 1 : 0;
        if (active[k] && b->failed[k]) {  // re-activating a failed case clears its status words
            b->failed[k] = 0;
            b->h_status[k] = 0;
            cleared = true;
            int rc;
            if ((rc = b->cuda(cudaMemsetAsync(b->cases[k]->status.p, 0, sizeof(unsigned int), b->stream),
                              "cudaMemsetAsync")))
                return rc;
        }
    }
    int rc;
    if (cleared && ((rc = b->cuda(cudaMemcpyAsync(b->d_status.p, b->h_status, n * sizeof(unsigned int),
                                                  cudaMemcpyHostToDevice, b->stream), "cudaMemcpyAsync")) ||
                    (rc = b->cuda(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize"))))
        return rc;
    return upload_tiles(b);
}

int tns_batch_get_active(tns_batch* b, int* active) {
    if (!b || !active) return TNS_ERR_ARG;
    for (size_t k = 0; k < b->cases.size(); k++) active[k] = b->active[k];
    return TNS_OK;
}

int tns_batch_run(tns_batch* b, int niter, int monitor_every, double stop_ratio, double* cdiff_ref,
                  double* cdiff_out, int max_records, int* n_records, int* iterations, int* case_status) {
    if (!b) return TNS_ERR_ARG;
    const int n = (int)b->cases.size();
    if (n_records)
        for (int k = 0; k < n; k++) n_records[k] = 0;
    if (iterations)
        for (int k = 0; k < n; k++) iterations[k] = 0;
    if (case_status)
        for (int k = 0; k < n; k++) case_status[k] = b->failed[k] ? TNS_ERR_NONFINITE : TNS_OK;
    if (stop_ratio > 0.0 && monitor_every <= 0)
        return b->fail(TNS_ERR_ARG, "tns_batch_run: a stop ratio needs monitor_every > 0");
    int rc;
    for (int k = 0; k < n; k++) {
        tns_handle* h = b->cases[k];
        if (!h->have_state) return b->fail(TNS_ERR_STATE, "tns_batch_run: case %d has no state uploaded", k);
        // work a member has queued on its own stream finishes first
        if ((rc = b->cuda(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize"))) return rc;
    }
    if (niter <= 0) return TNS_OK;
    // mixed ping-pong: when every member's state sits in the other buffer than the
    // descriptors' parity 0 (an odd number of iterations since), start at parity 1; a
    // mixed picture needs new descriptors (and graphs)
    int parity = 0;
    if (b->precision == 1) {
        const int f0 = b->cases[0]->cur ^ b->cur_at_desc[0];
        bool same = true;
        for (int k = 1; k < n; k++) same &= (b->cases[k]->cur ^ b->cur_at_desc[k]) == f0;
        if (same) {
            parity = f0;
        } else if ((rc = upload_descriptors(b))) {
            return rc;
        }
    }
    const int parity0 = parity;
    if (b->active != b->active_at_capture && (rc = upload_tiles(b))) return rc;

    std::vector<int> ran(n, 0), nrec(n, 0);
    std::vector<double> ref(5 * (size_t)n, 0.0);
    const bool stop = stop_ratio > 0.0;
    if (stop)
        for (int k = 0; k < n; k++)
            for (int m = 0; m < 5; m++) ref[5 * k + m] = cdiff_ref ? cdiff_ref[5 * k + m] : 0.0;
    auto set_ref = [&](int k) {
        for (int m = 0; m < 5; m++) if (!(ref[5 * k + m] > 0.0)) return false;
        return true;
    };
    bool any_failed = false;
    auto active_count = [&]() {
        int a = 0;
        for (int k = 0; k < n; k++) a += b->active[k];
        return a;
    };
    for (int it = 1; it <= niter && active_count() > 0;) {
        // the run's first iteration is monitored when it sets the stop reference
        bool needs_ref = false;
        if (stop)
            for (int k = 0; k < n; k++) needs_ref |= b->active[k] && !set_ref(k);
        auto monitored = [&](int j) {
            return (monitor_every > 0 && j % monitor_every == 0) || (j == 1 && needs_ref);
        };
        const bool monitor = monitored(it);
        if (b->active != b->active_at_capture && (rc = upload_tiles(b))) return rc;
        // schedule 1: a block of unmonitored iterations in one graph where one fits
        int step = 1;
        if (b->mode == 2 && it + tns_batch::BLOCK - 1 <= niter) {
            step = tns_batch::BLOCK;
            for (int j = it; j < it + tns_batch::BLOCK; j++)
                if (monitored(j)) step = 1;
        }
        if (b->mode == 3 && !monitor) {
            // the run of unmonitored iterations from here, in one persistent launch
            step = 1;
            while (step < tns_batch::PERSIST && it + step <= niter && !monitored(it + step)) step++;
            const int grid = std::min(b->persist_grid, 2 * b->ntiles);
            if ((rc = b->cuda(cudaMemsetAsync(b->d_bar.p, 0, 2 * sizeof(unsigned int), b->stream), "cudaMemsetAsync")) ||
                (rc = b->cuda(tns::launch_persistent(b->precision == 1, b->d_desc.p, b->d_tiles.p, b->d_active.p,
                                                     b->ntiles, step, parity, grid, b->d_bar.p, b->d_error.p,
                                                     b->stream), "persistent launch")))
                return rc;
            b->launches++;
        } else if (step > 1) {
            if ((rc = ensure_block_graph(b, parity))) return rc;
            if ((rc = b->cuda(cudaGraphLaunch(b->block[parity], b->stream), "cudaGraphLaunch"))) return rc;
            b->launches += b->per_block;
        } else {
            if ((rc = ensure_batch_graph(b, monitor ? 1 : 0, parity))) return rc;
            if ((rc = b->cuda(cudaGraphLaunch(b->graph[monitor ? 1 : 0][parity], b->stream), "cudaGraphLaunch")))
                return rc;
            b->launches += b->per_iter[monitor ? 1 : 0];
        }
        for (int k = 0; k < n; k++) ran[k] += step * b->active[k];
        if (b->precision == 1) parity ^= (step & 1);
        it += step;
        const int last = it - 1;  // the iteration the check below follows
        if (!monitor && last != niter) continue;
        // residual records, status words and the masks, at the monitor cadence and at the end
        if ((rc = fetch_monitor(b, monitor))) return rc;
        if ((rc = b->cuda(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize"))) return rc;
        if (b->mode == 3 && (*b->h_error & 4u))
            return b->fail(TNS_ERR_CUDA, "a grid barrier of the persistent batch launch did not complete in its bounded wait");
        for (int k = 0; k < n; k++) {
            if (!b->active[k]) continue;
            if (b->h_status[k] & 3u) {
                // bit 0: non-finite state; bit 1: a tile's static-data copy did not complete
                b->failed[k] = 1;
                b->active[k] = 0;
                any_failed = true;
                if (case_status) case_status[k] = (b->h_status[k] & 1u) ? TNS_ERR_NONFINITE : TNS_ERR_CUDA;
                continue;
            }
            if (!monitor) continue;
            double v[5];
            for (int m = 0; m < 5; m++) {
                std::memcpy(&v[m], &b->h_cdiff[5 * k + m], 8);
                const double init = m < 4 ? 1.0e-10 : 1.0e-20;  // constants.f90:44-45
                v[m] = v[m] >= init ? v[m] : init;
            }
            const bool record = monitor_every > 0 && last % monitor_every == 0;
            if (record) {
                if (cdiff_out && nrec[k] < max_records)
                    for (int m = 0; m < 5; m++) cdiff_out[((size_t)k * max_records + nrec[k]) * 5 + m] = v[m];
                nrec[k]++;
            }
            if (!stop) continue;
            if (!set_ref(k)) {
                for (int m = 0; m < 5; m++) ref[5 * k + m] = v[m];
                continue;
            }
            double worst = 0.0;
            for (int m = 0; m < 5; m++) worst = std::fmax(worst, v[m] / ref[5 * k + m]);
            if (worst <= stop_ratio) b->active[k] = 0;  // converged: masked off
        }
    }
    // members continue from where the batch left them
    for (int k = 0; k < n; k++) {
        tns_handle* h = b->cases[k];
        if (b->precision == 1) h->cur = b->cur_at_desc[k] ^ parity0 ^ (ran[k] & 1);
        if (ran[k]) h->have_run = true;
        if (iterations) iterations[k] = ran[k];
        if (n_records) n_records[k] = std::min(nrec[k], max_records);
    }
    if (stop && cdiff_ref)
        for (int k = 0; k < n; k++)
            for (int m = 0; m < 5; m++) cdiff_ref[5 * k + m] = ref[5 * k + m];
    if ((rc = b->cuda(cudaGetLastError(), "kernel launch"))) return rc;
    if (any_failed) return b->fail(TNS_ERR_NONFINITE, "a case's state became non-finite (NaN/Inf); it was masked off");
    return TNS_OK;
}

int tns_batch_set_schedule(tns_batch* b, int schedule) {
    if (!b) return TNS_ERR_ARG;
    if (schedule < 0 || schedule > 3) return b->fail(TNS_ERR_ARG, "schedule %d is not 0, 1, 2 or 3", schedule);
    if (b->general && (schedule == 0 || schedule == 3))
        return b->fail(TNS_ERR_UNSUPPORTED, "schedule %d needs every case to be one structured i x j block", schedule);
    int rc;
    if (schedule == 3) {
        for (size_t k = 0; k < b->cases.size(); k++) {
            const tns_handle* h = b->cases[k];
            if (!h->P.local || !h->port_ghosts.empty())
                return b->fail(TNS_ERR_UNSUPPORTED,
                               "schedule 3 needs LOCAL=1 and no type-6 port in every case (case %zu)", k);
        }
        int dev = 0, coop = 0;
        if ((rc = b->cuda(cudaGetDevice(&dev), "cudaGetDevice")) ||
            (rc = b->cuda(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev), "cudaDeviceGetAttribute")))
            return rc;
        b->persist_grid = coop ? tns::persistent_grid(b->precision == 1) : 0;
        if (b->persist_grid <= 0)
            return b->fail(TNS_ERR_UNSUPPORTED, "schedule 3 needs a cooperative launch of the persistent kernel");
        if (!b->d_bar.p && ((rc = b->cuda(b->d_bar.alloc(2), "cudaMalloc")) ||
                            (rc = b->cuda(b->d_error.alloc(1), "cudaMalloc")) ||
                            (rc = b->cuda(cudaMemset(b->d_error.p, 0, sizeof(unsigned int)), "cudaMemset")) ||
                            (rc = b->cuda(cudaMallocHost((void**)&b->h_error, sizeof(unsigned int)), "cudaMallocHost"))))
            return rc;
        *b->h_error = 0;
    }
    if (schedule >= 1 && b->branch.empty()) {
        const int n = (int)b->cases.size();
        const int nb = std::min<int>(n, 64);
        // longest-first assignment of cases (by cell count) to the least-loaded branch
        std::vector<int> order(n);
        for (int k = 0; k < n; k++) order[k] = k;
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int c) { return b->cases[a]->ncell() > b->cases[c]->ncell(); });
        std::vector<double> load(nb, 0.0);
        b->branch_of.assign(n, 0);
        for (int k : order) {
            const int bi = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            b->branch_of[k] = bi;
            load[bi] += (double)b->cases[k]->ncell();
        }
        if ((rc = b->cuda(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "cudaEventCreate"))) return rc;
        b->branch.resize(nb);
        b->join.resize(nb);
        for (int i = 0; i < nb; i++)
            if ((rc = b->cuda(cudaStreamCreateWithFlags(&b->branch[i], cudaStreamNonBlocking), "cudaStreamCreate")) ||
                (rc = b->cuda(cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming), "cudaEventCreate")))
                return rc;
    }
    if (schedule != b->mode) {
        b->mode = schedule;
        b->drop_graphs();
    }
    return TNS_OK;
}

int tns_batch_get_schedule(tns_batch* b) { return b ? b->mode : TNS_ERR_ARG; }

int tns_batch_prepare(tns_batch* b) {
    if (!b) return TNS_ERR_ARG;
    const int n = (int)b->cases.size();
    int rc;
    for (int k = 0; k < n; k++) {
        tns_handle* h = b->cases[k];
        if (!h->have_state) return b->fail(TNS_ERR_STATE, "tns_batch_prepare: case %d has no state uploaded", k);
        if ((rc = b->cuda(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize"))) return rc;
    }
    // the descriptors and the tile table tns_batch_run would start from
    if (b->precision == 1) {
        const int f0 = b->cases[0]->cur ^ b->cur_at_desc[0];
        bool same = true;
        for (int k = 1; k < n; k++) same &= (b->cases[k]->cur ^ b->cur_at_desc[k]) == f0;
        if (!same && (rc = upload_descriptors(b))) return rc;
    }
    if (b->active != b->active_at_capture && (rc = upload_tiles(b))) return rc;
    bool any = false;
    for (int k = 0; k < n; k++) any |= b->active[k] != 0;
    if (!any) return TNS_OK;  // tns_batch_run launches nothing either
    const int nparity = b->precision == 1 ? 2 : 1;
    for (int par = 0; par < nparity; par++) {
        // schedule 3 launches a graph only for its monitored iterations
        if (b->mode != 3 && (rc = ensure_batch_graph(b, 0, par))) return rc;
        if ((rc = ensure_batch_graph(b, 1, par))) return rc;
        if (b->mode == 2 && (rc = ensure_block_graph(b, par))) return rc;
    }
    return TNS_OK;
}

long long tns_batch_launch_count(tns_batch* b) { return b ? b->launches : -1; }

const char* tns_batch_last_error(tns_batch* b) { return b ? b->err.c_str() : "null batch"; }

void tns_batch_destroy(tns_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    b->drop_graphs();
    b->d_desc.release();
    b->d_active.release();
    b->d_tiles.release();
    b->d_cdiff.release();
    b->d_status.release();
    b->d_bar.release();
    b->d_error.release();
    if (b->h_error) cudaFreeHost(b->h_error);
    if (b->h_cdiff) cudaFreeHost(b->h_cdiff);
    if (b->h_status) cudaFreeHost(b->h_status);
    for (cudaStream_t st : b->branch)
        if (st) cudaStreamDestroy(st);
    for (cudaEvent_t e : b->join)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

}  // extern "C"
