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

}  // namespace tns
