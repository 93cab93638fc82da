// tns_handle.h -- the solver handle behind include/tnsgpu.h: the host layout of one
// case's mesh, its device buffers, captured iteration graphs and error state.  Shared by
// the single-case runtime (tns_api.cu) and the batch runtime (tns_batch_api.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/tnsgpu.h"
#include "tns_kernels.h"

using tns::Mesh;
using tns::Params;

namespace tns_rt {

enum KernelId { K_DISS = 0, K_VISC = 1, K_STAGE = 2, K_DTMIN = 3, K_GPORT = 4, K_NKERNEL = 5 };

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count) {
        n = count;
        return cudaMalloc((void**)&p, std::max<size_t>(count, 1) * sizeof(T));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
    }
};

}  // namespace tns_rt

using namespace tns_rt;

struct tns_adjoint_state;  // tns_adjoint.cu
struct tns_umesh_state;    // tns_unstructured.cu

struct tns_handle {
    std::string err;
    Params P{};
    Mesh M{};
    int ni = 0, nj = 0, neles = 0, nods = 0, nghosts = 0, maxid = 0;
    std::vector<int> cell_of;   // structured index k -> 0-based original cell id
    bool identity = true;
    std::vector<int> ghost_line;  // device ghost index -> bc.in line
    std::vector<int> ghost_id;    // bc.in line -> Fortran ghost id
    std::vector<int> port_ghosts;
    std::vector<double> hX, hY, hcfldl, hgxc, hgyc, hginj;  // host layout (device order)
    std::vector<double> hcvol, hstile, hfgi, hfgj;  // static geometry (VOL, stage tiles, faces)
    std::vector<int> hgtype, hgrank;
    std::vector<int> node_of;   // structured node index -> 1-based node id
    cudaStream_t own = nullptr, stream = nullptr;
    // second branch of an iteration: the dissipation pre-pass runs beside the viscous flux
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    DevBuf<double> x, y, cfldl, gxc, gyc, ginj, gport, qa, qb, qc, d, vis, dt, dtmin, partial,
        primout, cvol, stile, fgi, fgj;
    // mixed FP32/FP64 path: FP64 state ping-pong (qa, qa2) and FP32 scratch
    int precision = 0;
    int cur = 0;  // mixed: which of qa / qa2 holds the state
    DevBuf<double> qa2;
    DevBuf<float> dqb, dqc, df, visf, dtf;
    DevBuf<double> tref;  // per stage tile reference state (TileRefMx words)
    cudaGraphExec_t graph_mx[2] = {nullptr, nullptr};
    // monitored iteration (CDIFF reduction in stage 4): FP64, mixed per parity
    cudaGraphExec_t graph_mon = nullptr;
    cudaGraphExec_t graph_mon_mx[2] = {nullptr, nullptr};
    DevBuf<int> gtype, grank, ports;
    DevBuf<unsigned int> counter, status;
    DevBuf<unsigned long long> cdiff;
    double* pinned = nullptr;  // 5*ncell staging
    bool have_state = false, have_run = false;
    cudaGraphExec_t graph = nullptr;
    long long per_iter = 0, per_iter_mon = 0;
    unsigned int* status_host = nullptr;  // pinned
    // caller's page-locked CDIFF record of the last tns_enqueue_monitored, given the
    // reference's floor at the next synchronisation
    double* cdiff_pending = nullptr;
    bool profile = false;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    double kms[K_NKERNEL] = {0};
    long long kcount[K_NKERNEL] = {0};
    long long launches = 0;
    tns_adjoint_state* adj = nullptr;  // discrete adjoint buffers (tns_adjoint_enable)
    // a general quad mesh (not one i x j block): cells in reverse Cuthill-McKee order,
    // ni = NELES and nj = 1, laid out and iterated by tns_unstructured.cu
    bool unstructured = false;
    tns_umesh_state* umesh = nullptr;

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
    size_t ncell() const { return (size_t)ni * nj; }
    double* state() { return precision == 1 && cur ? qa2.p : qa.p; }
    double* other_state() { return precision == 1 && !cur ? qa2.p : qa.p; }
};


namespace tns_rt {
// Enqueues f() (nk kernel launches of kernel kind kid) on h->stream; with per-kernel
// profiling on (tns_profile), brackets it with CUDA events and adds its device time.
template <class F>
void launch(tns_handle* h, int kid, F&& f, int nk = 1) {
    if (h->profile) cudaEventRecord(h->ev[0], h->stream);
    f();
    h->launches += nk;
    if (h->profile) {
        cudaEventRecord(h->ev[1], h->stream);
        cudaEventSynchronize(h->ev[1]);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]);
        h->kms[kid] += ms;
        h->kcount[kid]++;
    }
}
// One RK4 iteration of a handle on h->stream (tns_api.cu): FP64 in place, mixed from
// state buffer A to Aout.  The batch runtime captures these per case.
void enqueue_iteration_f64(tns_handle* h, bool monitor);
void enqueue_iteration_mx(tns_handle* h, bool monitor, double* A, double* Aout);
// Frees the adjoint buffers of a handle (tns_adjoint.cu).
void adjoint_release(tns_handle* h);
}  // namespace tns_rt
