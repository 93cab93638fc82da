// tns_batch.cuh -- descriptor of one case of a batched multi-case solve.  The batched
// kernels read their case's parameters, mesh view and buffers from an array of these,
// indexed through a table of (case, tile i, tile j) entries: one launch advances every
// active case.
#pragma once

#include "tns_device.cuh"

namespace tns {

struct BatchCase {
    Params P;
    Mesh M;
    // FP64 path: state qa (in place), stage scratch qb/qc, frozen d/vis/dt
    double *qa, *qb, *qc, *d, *vis, *dt;
    // mixed path: state ping-pong qa/qa2, FP32 increments and frozen terms
    double* qa2;
    float *dqb, *dqc, *df, *visf, *dtf;
    const double* dtmin;
    unsigned long long* cdiff;  // 5 slots
    unsigned int* status;
};

// Shared-memory copy of a batched block's case: every thread reads it many times.
struct BatchBlock {
    Params P;
    Mesh M;
    int active;
};

__device__ __forceinline__ int4 batch_prologue(const BatchCase* __restrict__ cases,
                                              const int4* __restrict__ tiles,
                                              const int* __restrict__ active, BatchBlock& B) {
    static_assert(sizeof(Params) % 4 == 0 && sizeof(Mesh) % 4 == 0, "word copy");
    constexpr int NP = sizeof(Params) / 4, NM = sizeof(Mesh) / 4;
    const int4 t = tiles[blockIdx.x];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const BatchCase* c = cases + t.x;
    // one word per thread: the block's case parameters and mesh view
    if (tid < NP)
        reinterpret_cast<int*>(&B.P)[tid] = reinterpret_cast<const int*>(&c->P)[tid];
    else if (tid < NP + NM)
        reinterpret_cast<int*>(&B.M)[tid - NP] = reinterpret_cast<const int*>(&c->M)[tid - NP];
    else if (tid == NP + NM)
        B.active = active[t.x];
    __syncthreads();
    return t;
}

}  // namespace tns
