// tns_tile.cuh -- tile geometry and the helpers every tile kernel shares: bulk copies,
// programmatic dependent launch, halo classification, primitive variables of a cell, and the ghost state of a halo
// position (BC of boundary.f90:24-327 from the parent and its opposite neighbour).
#pragma once

#include <utility>

#include <cuda.h>

#include "tns_device.cuh"

namespace tns {

#ifndef TNS_TI
#define TNS_TI 8
#endif
#ifndef TNS_STAGE_MINB
#define TNS_STAGE_MINB 3
#endif
#ifndef TNS_STAGE_BATCH_MINB
#define TNS_STAGE_BATCH_MINB 3  // with its arguments in shared memory (tns_batch.cuh)
#endif
#ifndef TNS_VISC_MINB
#define TNS_VISC_MINB 3  // 80 registers: 3 blocks/SM beat 2 blocks without the cap
#endif
#ifndef TNS_VISC_BATCH_MINB
#define TNS_VISC_BATCH_MINB 1  // descriptor-fed arguments spill at 3 blocks/SM
#endif
// Resident blocks per SM of a kernel tuned at TI = 8, for the compiled TI: the same
// threads per SM at every tile height.
#define TNS_PER_SM(n) ((n) * 8 / TNS_TI > 0 ? (n) * 8 / TNS_TI : 1)
constexpr int TJ = 32;      // tile extent along j (contiguous in memory)
constexpr int GP_THREADS = 128;  // threads per port line of the type-6 port-flux kernels
constexpr int TI = TNS_TI;  // tile extent along i
constexpr int NTHREADS = TJ * TI;
// The viscous kernels may run one extra row of threads: a tile has (TI+1)*TJ + TI*(TJ+1)
// faces, which TI+1 rows of threads cover in two rounds.
#ifndef TNS_VISC_EXTRA_ROW
#define TNS_VISC_EXTRA_ROW 0
#endif
constexpr int VROWS = TI + TNS_VISC_EXTRA_ROW;
constexpr int VNT = TJ * VROWS;


// Halo-1 slot grid (TI+2) x (TJ+2).
constexpr int SW = TJ + 2;
constexpr int NSLOT = (TI + 2) * SW;
// The halo ring of the slot grid, 2 (TI + 2) + 2 TJ + 4 positions as ring slots r:
// position (li, lj) of r runs along the first and last slot rows, then along the first
// and last slot columns between them.
constexpr int NRING = 2 * SW + 2 * TI;
__device__ __forceinline__ void ring_slot(int r, int& li, int& lj) {
    if (r < SW) { li = 0; lj = r; }
    else if (r < 2 * SW) { li = TI + 1; lj = r - SW; }
    else if (r < 2 * SW + TI) { li = 1 + r - 2 * SW; lj = 0; }
    else { li = 1 + r - 2 * SW - TI; lj = SW - 1; }
}
constexpr int AW = TJ + 1;  // node-average grid (TI+1) x (TJ+1)
constexpr int NAVG = (TI + 1) * AW;

// Static block of one stage tile (tile (bx, by) at M.stile + (by * ntiles_j + bx) * STILE),
// built on the host: the nodes of the tile's cells, (i0..i0+TI) x (j0..j0+TJ), x then y
// (index la * SNW + lb), then per cell (index ti * TJ + tj) the source-gradient
// coefficients GA..GD, 1/VOL and 1/YCC (see source_terms).  Positions outside the mesh
// hold zeros.  A multiple of 16 bytes, so a tile's block is one bulk copy.
constexpr int SNW = TJ + 1;
constexpr int SNN = (TI + 1) * SNW;
enum StageTileField { ST_GA, ST_GB, ST_GC, ST_GD, ST_RVOL, ST_RYCC, ST_NF };
constexpr int STILE = 2 * SNN + ST_NF * TI * TJ;
static_assert(STILE % 2 == 0, "a stage tile block must be a multiple of 16 bytes");

// Programmatic dependent launch: a tile kernel lets the next kernel in the stream start
// as soon as all its blocks are running (pdl_trigger), and waits for the previous one
// to finish, with its memory visible, before it touches data that kernel produced
// (pdl_wait).  Static data, which nothing writes, may load before the wait.  Both are
// no-ops when the kernel was not launched with the attribute.
#ifndef TNS_PDL
#define TNS_PDL 1
#endif
__device__ __forceinline__ void pdl_trigger() {
#if TNS_PDL
    asm volatile("griddepcontrol.launch_dependents;");
#endif
}
__device__ __forceinline__ void pdl_wait() {
#if TNS_PDL
    asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

// One-shot bulk copy global -> shared through the TMA engine, completed on an mbarrier
// (cp.async.bulk with mbarrier::complete_tx).  Both addresses 16-byte aligned, bytes a
// multiple of 16.  bulk_copy_start: one thread, after it initialised the barrier
// (bulk_barrier_init); the block's other threads may wait on it after a __syncthreads.
__device__ __forceinline__ void bulk_barrier_init(unsigned long long* bar) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void bulk_copy_start(void* dst, const void* src, unsigned bytes,
                                                unsigned long long* bar) {
    const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;"
                 ::"r"(b), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(d), "l"(src), "r"(bytes), "r"(b) : "memory");
}
// One-shot tiled tensor copy global -> shared (cp.async.bulk.tensor, 3-D, no multicast):
// the box of `map` at element coordinates (x, y, z), x the innermost; x * element size a
// multiple of 16 bytes; the shared destination 128-byte aligned; `bytes` the whole box
// (out-of-range elements arrive as zeros and count).  `map` is the address of a
// __grid_constant__ kernel parameter.  One thread, after bulk_barrier_init.
__device__ __forceinline__ void tensor_copy_3d_start(void* dst, const CUtensorMap* map, int x, int y, int z,
                                                     unsigned bytes, unsigned long long* bar) {
    const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;"
                 ::"r"(b), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];"
                 ::"r"(d), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(b)
                 : "memory");
}
// Waits for phase 0 of the barrier with a bounded number of polls; false if the copy did
// not complete in that many (the caller reports it and skips the tile).
__device__ __forceinline__ bool bulk_wait(unsigned long long* bar, int max_polls = 1 << 20) {
    const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    for (int k = 0; k < max_polls; k++) {
        unsigned done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(b) : "memory");
        if (done) return true;
    }
    return false;
}

// Grid-wide barrier of a cooperative launch (every block resident): an arrival counter
// and a generation word in global memory, both zero before the launch.  The last block
// to arrive resets the counter and advances the generation; the others poll the
// generation at most max_polls times.  Returns false when the wait gave up (the caller
// reports it and leaves the kernel).
__device__ __forceinline__ bool grid_barrier(unsigned int* count, unsigned int* gen, int max_polls = 1 << 22) {
    __shared__ int passed;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const unsigned int g = *(volatile unsigned int*)gen;
        __threadfence();
        const unsigned int nb = gridDim.x * gridDim.y;
        if (atomicAdd(count, 1u) == nb - 1) {
            atomicExch(count, 0u);
            __threadfence();
            atomicAdd(gen, 1u);
            passed = 1;
        } else {
            int k = 0;
            while (*(volatile unsigned int*)gen == g && k < max_polls) {
                __nanosleep(64);
                k++;
            }
            passed = *(volatile unsigned int*)gen != g;
        }
        __threadfence();
    }
    __syncthreads();
    return passed != 0;
}

// Launch of a tile kernel that may overlap its predecessor's tail (see pdl_wait).
template <class... Exp, class... Act>
inline cudaError_t launch_tile(void (*kernel)(Exp...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                               Act&&... args) {
#if TNS_PDL
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Act>(args)...);
#else
    kernel<<<grid, block, smem, s>>>(std::forward<Act>(args)...);
    return cudaGetLastError();
#endif
}

// How a kernel reads the conservative state of cell c: FP64 array, or FP64 COLD plus an
// FP32 stage increment (the mixed-precision path).
struct StateF64 {
    const double* __restrict__ q;
    size_t n;
    __device__ __forceinline__ double c(int m, size_t cell) const { return q[m * n + cell]; }
};
struct StateMixed {
    const double* __restrict__ cold;
    const float* __restrict__ dq;  // null in stage 1 (state = COLD)
    size_t n;
    __device__ __forceinline__ double c(int m, size_t cell) const {
        const double v = cold[m * n + cell];
        return dq ? v + (double)dq[m * n + cell] : v;
    }
};

template <class St>
__device__ __forceinline__ void cell_prim(const Params& P, const St& st, size_t c, Prim& p) {
    primitive(P, st.c(0, c), st.c(1, c), st.c(2, c), st.c(3, c), st.c(4, c), p);
}

__device__ __forceinline__ void cell_prim(const Params& P, const double* __restrict__ q, size_t ncell,
                                          size_t c, Prim& p) {
    cell_prim(P, StateF64{q, ncell}, c, p);
}

// Classifies halo position (i, j): 0 = cell, 1..4 = ghost on that side, -1 = unused.
__device__ __forceinline__ int classify(const Mesh& M, int i, int j, int& along) {
    const bool in_i = i >= 0 && i < M.ni, in_j = j >= 0 && j < M.nj;
    if (in_i && in_j) return 0;
    if (in_i && j == -1) { along = i; return 1; }
    if (in_j && i == M.ni) { along = j; return 2; }
    if (in_i && j == M.nj) { along = i; return 3; }
    if (in_j && i == -1) { along = j; return 4; }
    return -1;
}

// BC state of the ghost on `side` at `along`, from the parent and the parent's opposite
// neighbour, whose primitives cell(i, j, Prim&) evaluates (bit-identical to their
// PRIMITIVE_VARS).
template <class CellPrim>
__device__ void ghost_state_at(const Params& P, const Mesh& M, int side, int along, CellPrim cell,
                               Prim& gh) {
    int ip, jp, io, jo;
    if (side == 1) { ip = along; jp = 0; io = along; jo = 1; }
    else if (side == 2) { ip = M.ni - 1; jp = along; io = M.ni - 2; jo = along; }
    else if (side == 3) { ip = along; jp = M.nj - 1; io = along; jo = M.nj - 2; }
    else { ip = 0; jp = along; io = 1; jo = along; }
    const int g = M.ghost_index(side, along);
    const int type = M.gtype[g];
    Prim par, opp;
    cell(ip, jp, par);
    if (type == 3) cell(io, jo, opp);
    else opp = par;
    const size_t n1 = (size_t)ip * (M.nj + 1) + jp;
    const double X[4] = {M.x[n1], M.x[n1 + M.nj + 1], M.x[n1 + M.nj + 2], M.x[n1 + 1]};
    const double Y[4] = {M.y[n1], M.y[n1 + M.nj + 1], M.y[n1 + M.nj + 2], M.y[n1 + 1]};
    double psx = 0.0, psy = 0.0;
    if (type == 6) face_vector(P.iaxis, side, X, Y, psx, psy);
    const double ycc_p = (Y[0] + Y[1] + Y[2] + Y[3]) * 0.25;
    boundary_ghost(P, type, par, opp, psx, psy, M.gyc[g], ycc_p, type == 6 ? M.gport[g] : 0.0,
                   M.ginj[g], gh);
}

// The same, with both cells read straight from the state array.
template <class St>
__device__ __forceinline__ void ghost_state(const Params& P, const Mesh& M, const St& st, int side, int along,
                                            Prim& gh) {
    ghost_state_at(P, M, side, along,
                   [&](int i, int j, Prim& p) { cell_prim(P, st, (size_t)i * M.nj + j, p); }, gh);
}

__device__ __forceinline__ void ghost_state(const Params& P, const Mesh& M, const double* __restrict__ q,
                                            size_t ncell, int side, int along, Prim& gh) {
    ghost_state(P, M, StateF64{q, ncell}, side, along, gh);
}

}  // namespace tns
