// tns_batch.cuh -- argument blocks of the tile kernels and the descriptor of one case
// of a batched multi-case solve.
//
// A single-case launch passes its argument block by value (kernel parameter space).  A
// batched launch finds, per block, its case in an array of BatchCase descriptors in
// global memory, indexed through a table of (case, tile j, tile i) entries; each
// descriptor holds every argument block the case's launches need, precomputed on the
// host (per stage, monitor mode and, on the mixed path, state parity), so a block reads
// one read-only block instead of assembling pointers in registers.
#pragma once

#include "tns_device.cuh"
#include "tns_tile.cuh"

namespace tns {

struct StageArgs {
    const double* qin;   // stage input state [5][ncell]
    const double* qold;  // state at the start of the iteration [5][ncell]
    double* qout;        // stage output [5][ncell] (may alias qold: own-cell reads only)
    const double* d;     // dissipation [5][ncell]
    const double* vis;   // viscous flux [4][ncell]
    const double* dt;    // per-cell DT (LOCAL=1)
    const double* dtmin; // DTMIN (LOCAL=0)
    double alpha;
    unsigned long long* cdiff;  // 5 slots, ordered bits of max|Q_old-Q_new| (or null)
    unsigned int* status;       // bit 0: non-finite state (checked where non-null)
    unsigned int* error;        // bit 1: a tile's static-block copy did not complete
};

template <class OutT>
struct DissArgs {
    const double* q;     // Q_old [5][ncell]
    OutT* d;             // out: D [5][ncell] (FP64, or FP32 on the mixed path)
    OutT* dt;            // out: DT per cell (LOCAL=1)
    const double* dtmin; // DTMIN (LOCAL=0)
};

struct StageArgsMx {
    const double* cold;   // state at the start of the iteration [5][ncell]
    const float* dqin;    // stage input increment (null in stage 1)
    float* dqout;         // stage output increment (stages 1-3)
    double* qout;         // new state (stage 4) [5][ncell]
    const float* d;       // dissipation [5][ncell]
    const float* vis;     // viscous flux [4][ncell]
    const float* dt;      // per-cell DT (LOCAL=1)
    const double* dtmin;  // DTMIN (LOCAL=0)
    float alpha;
    unsigned long long* cdiff;
    unsigned int* status;
    unsigned int* error;  // bit 1: a tile's static-block copy did not complete
};

struct BatchCase {
    Params P;
    Mesh M;
    // FP64 path
    DissArgs<double> diss;
    StageArgs stage[2][4];  // [monitor][stage]
    const double* q;        // state (viscous-flux input)
    double* vis;
    // mixed path; parity p reads the state from qmx[p] and writes it to qmx[1-p]
    const double* qmx[2];
    float *df, *dtf, *visf;
    StageArgsMx stage_mx[2][2][4];  // [parity][monitor][stage]
    const double* dtmin;
};

// The batched stage kernels copy their case's arguments into shared memory: loads from
// constant shared addresses instead of through a descriptor pointer held in registers.
// The mixed one then runs 4 blocks per SM like the single-case kernel (64-case sweep,
// schedule 0: 0.235 -> 0.206 s); the viscous kernels are better off without (spills).
#ifndef TNS_BATCH_SMEM_ARGS
#define TNS_BATCH_SMEM_ARGS 1
#endif
static_assert(sizeof(Params) % 8 == 0 && sizeof(Mesh) % 8 == 0 && sizeof(StageArgs) % 4 == 0 &&
                  sizeof(StageArgsMx) % 4 == 0,
              "descriptors are copied as 4-byte words and laid out at 8-byte offsets");
// Block-wide copy of a descriptor (a multiple of 4 bytes) into shared memory.
__device__ __forceinline__ void copy_words(void* dst, const void* src, size_t bytes, int tid) {
    const unsigned* s = reinterpret_cast<const unsigned*>(src);
    unsigned* d = reinterpret_cast<unsigned*>(dst);
    for (int k = tid; k < (int)(bytes / 4); k += NTHREADS) d[k] = s[k];
}

}  // namespace tns
