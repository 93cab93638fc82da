// tns_kernels.cu -- FP64 kernels of one RK4 iteration on a structured i x j block.
//
// Per iteration (turbnstwod.f90:95-168):
//   [k_dtmin]      global time step (LOCAL=0 only): per-cell DT and a grid-wide min
//   k_dissipation  DT (LOCAL=1) and the frozen JST dissipation D of Q_old
//                  (solver_state.f90:70-225), radius-2 shared-memory tile
//   k_stage<1>     primitives + ghost BCs + nodal averages + viscous flux (frozen VIS)
//                  + source + residual + update with alpha=1/4
//   k_stage<0> x3  primitives + ghost BCs + source + residual + update (alpha 1/3,1/2,1);
//                  the last one also reduces CDIFF and checks the state is finite.
//   [k_gport]      type-6 port mass flux of the stage input (only if such ghosts exist)
// Ghost cells are never stored: each tile evaluates the BC of the ghosts in its halo
// from the parent and the parent's opposite neighbour, both already in the tile.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>

#include "tns_device.cuh"
#include "tns_kernels.h"
#include "tns_tile.cuh"
#include "tns_batch.cuh"

namespace tns {

// ------------------------------------------------------------------ stage kernel

// Shared-memory fields of the stage tile, paired for 16-byte loads; the tile's static
// block (nodes, gradient coefficients, 1/VOL, 1/YCC) arrives by one bulk copy.  The TMA
// variant also receives the five Q planes of the tile's halo box by one tiled tensor
// copy: rows i0-1 .. i0+TI, columns j0-2 .. j0+TJ+1 (the box starts one column early so
// that its first column is a multiple of 16 bytes; out-of-mesh positions arrive as
// zeros), and evaluates its slots from there.
// Off by default: measured on 1024 x 384 (B200, FP64), the TMA variant took 157-159 us
// for a RK4 iteration's four stage launches against 145 us with plain loads (same
// results bit for bit).  A block waits for its whole box before its first slot, where
// plain loads let each warp start as its own rows arrive.
#ifndef TNS_STAGE_TMA
#define TNS_STAGE_TMA 0
#endif
// Three blocks of the TMA variant fit an SM at TI >= 8 (at TI = 4 its box would cost the
// sixth block).
#define TNS_STAGE_TMA_ON (TNS_STAGE_TMA && TNS_TI >= 8)
constexpr int QH = TI + 2, QW = TJ + 4;
static_assert(QW % 2 == 0, "the Q box rows must be a multiple of 16 bytes");

// Slot order: each thread first evaluates the slot of its own cell and keeps that cell's
// T, P and RHO in registers (the only slot values read for the cell alone), then the
// first NRING threads evaluate the halo ring's slots (tns_tile.cuh).
static_assert(NRING <= NTHREADS, "one ring slot per thread at most");

template <bool TMA>
struct StageSmemT {
    double qs[TMA ? 5 * QH * QW : 2];  // (TMA) Q planes [5][QH][QW], 128-byte aligned
    double st[STILE];                  // static block (tns_tile.cuh)
    double2 fg[5][NSLOT];              // (F_m, G_m)
    double2 uv[NSLOT];                 // (U, V)
    double2 rq[NSLOT];                 // (C5/C1, |V|)
    unsigned long long bar;   // completion of the static block's copy
    unsigned long long qbar;  // (TMA) completion of the Q box
};
using StageSmem = StageSmemT<false>;
static_assert(sizeof(double) * 5 * QH * QW % 16 == 0, "the static block follows the Q box at 16 bytes");

size_t stage_smem_bytes() { return sizeof(StageSmem); }
#if TNS_STAGE_TMA_ON
// (+128: the kernel aligns the Q box to 128 bytes inside its dynamic shared memory)
static size_t stage_tma_smem_bytes() { return sizeof(StageSmemT<true>) + 128; }
#endif

template <bool TMA>
__device__ __forceinline__ void put_slot(StageSmemT<TMA>& S, int s, const Prim& p) {
#pragma unroll
    for (int m = 0; m < 5; m++) S.fg[m][s] = make_double2(p.f[m], p.g[m]);
    S.uv[s] = make_double2(p.u, p.v);
    S.rq[s] = make_double2(p.ri, p.qm);
}

// One RK stage (turbnstwod.f90:204-227, boundary.f90:24-48, source_terms.f90:24-104,
// residual.f90:23-83) on a TI x TJ tile with its halo staged in shared memory.
// TMA: qmap is the tensor map of A.qin ([5][NI][NJ] doubles, box [5][QH][QW]).
template <bool TMA>
__device__ __forceinline__ void stage_tile(const Params& P, const Mesh& M, const StageArgs& A, int bx, int by,
                                           const CUtensorMap* qmap = nullptr) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* base = smem_raw;
    if (TMA) base += (128u - ((unsigned)__cvta_generic_to_shared(smem_raw) & 127u)) & 127u;
    StageSmemT<TMA>& S = *reinterpret_cast<StageSmemT<TMA>*>(base);
    const size_t ncell = (size_t)M.ni * M.nj;
    const int j0 = bx * TJ, i0 = by * TI;
    const int tid = threadIdx.y * TJ + threadIdx.x;
    pdl_trigger();
    // the static block is written by nothing: its copy overlaps the previous kernel's tail
    if (tid == 0) {
        bulk_barrier_init(&S.bar);
        if (TMA) bulk_barrier_init(&S.qbar);
        const size_t tile = (size_t)by * ((M.nj + TJ - 1) / TJ) + bx;
        bulk_copy_start(S.st, M.stile + tile * STILE, STILE * sizeof(double), &S.bar);
    }
    pdl_wait();
    if (TMA && tid == 0)
        tensor_copy_3d_start(S.qs, qmap, j0 - 2, i0 - 1, 0, (unsigned)(sizeof(double) * 5 * QH * QW), &S.qbar);
    __syncthreads();
    if (TMA) {
        // a block-uniform decision: every thread leaves, or none
        const bool ok = bulk_wait(&S.qbar);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(A.error, 2u);
            bulk_wait(&S.qbar);
            bulk_wait(&S.bar);
            return;
        }
    }
    // primitives of a cell of the Q box, by mesh position
    auto box_prim = [&](int ci, int cj, Prim& q) {
        const double* b = S.qs + (ci - i0 + 1) * QW + (cj - j0 + 2);
        primitive(P, b[0], b[QH * QW], b[2 * QH * QW], b[3 * QH * QW], b[4 * QH * QW], q);
    };
    // the slot at (li, lj): false where the position is neither a cell nor a ghost
    auto slot_prim = [&](int li, int lj, Prim& p) -> bool {
        int along = 0;
        const int kind = classify(M, i0 - 1 + li, j0 - 1 + lj, along);
        if (kind < 0) return false;
        if (TMA) {
            if (kind == 0) box_prim(i0 - 1 + li, j0 - 1 + lj, p);
            else ghost_state_at(P, M, kind, along, box_prim, p);
        } else if (kind == 0) {
            cell_prim(P, A.qin, ncell, (size_t)(i0 - 1 + li) * M.nj + (j0 - 1 + lj), p);
        } else {
            ghost_state(P, M, A.qin, ncell, kind, along, p);
        }
        return true;
    };
    // own cell first (its T, P, RHO kept), then the ring
    double own_t = 0.0, own_p = 0.0, own_rho = 0.0;
    {
        Prim p;
        if (slot_prim(threadIdx.y + 1, threadIdx.x + 1, p)) {
            put_slot(S, (threadIdx.y + 1) * SW + threadIdx.x + 1, p);
            own_t = kept(p.t);
            own_p = kept(p.p);
            own_rho = kept(p.rho);
        }
    }
    if (tid < NRING) {
        int li, lj;
        ring_slot(tid, li, lj);
        Prim p;
        if (slot_prim(li, lj, p)) put_slot(S, li * SW + lj, p);
    }
    __syncthreads();
    if (!bulk_wait(&S.bar)) {
        // the copy did not complete: report it, give it one more bounded wait (it writes
        // this block's shared memory) and leave the tile
        if (tid == 0) atomicOr(A.error, 2u);
        bulk_wait(&S.bar);
        return;
    }

    const int tj = threadIdx.x, ti = threadIdx.y;
    const int i = i0 + ti, j = j0 + tj;
    const bool valid = i < M.ni && j < M.nj;
    double dv[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (valid) {
        const size_t cell = (size_t)i * M.nj + j;
        const int c = (ti + 1) * SW + (tj + 1);
        const int nb[4] = {c - 1, c + SW, c + 1, c - SW};  // NC1..NC4
        const int n1 = ti * SNW + tj;  // node 1 of the cell in the static block
        const int gc = 2 * SNN + ti * TJ + tj;
        const double* X0 = S.st;
        const double* Y0 = S.st + SNN;

        // source terms first (source_terms.f90:24-104): only src3 / src5 stay live into
        // the residual
        double src3, src5;
        {
            SrcIn s;
            s.ga = S.st[gc + ST_GA * NTHREADS]; s.gb = S.st[gc + ST_GB * NTHREADS];
            s.gc = S.st[gc + ST_GC * NTHREADS]; s.gd = S.st[gc + ST_GD * NTHREADS];
            const double2 ua = S.uv[nb[0]], ub = S.uv[nb[1]], uc = S.uv[nb[2]], ud = S.uv[nb[3]];
            const double2 ra = S.rq[nb[0]], rb = S.rq[nb[1]], rc = S.rq[nb[2]], rd = S.rq[nb[3]];
            s.ua = ua.x; s.ub = ub.x; s.uc = uc.x; s.ud = ud.x;
            s.va = ua.y; s.vb = ub.y; s.vc = uc.y; s.vd = ud.y;
            s.ra = ra.x; s.rb = rb.x; s.rc = rc.x; s.rd = rd.x;
            s.qa = ra.y; s.qb = rb.y; s.qc = rc.y; s.qd = rd.y;
            const double2 tp = make_double2(own_t, own_p);
            const double RHOC = own_rho;
            const double YCCI = (Y0[n1] + Y0[n1 + SNW] + Y0[n1 + SNW + 1] + Y0[n1 + 1]) * 0.25;
            source_terms(P, s, RHOC, S.rq[c].x, tp.x, tp.y, S.uv[c].y, YCCI,
                         S.st[gc + ST_RYCC * NTHREADS], src3, src5);
        }

        // inviscid residual (residual.f90:23-62) with the sources (residual.f90:54,58)
        const double X[4] = {X0[n1], X0[n1 + SNW], X0[n1 + SNW + 1], X0[n1 + 1]};
        const double Y[4] = {Y0[n1], Y0[n1 + SNW], Y0[n1 + SNW + 1], Y0[n1 + 1]};
        double SX[4], SY[4];
#pragma unroll
        for (int k = 0; k < 4; k++) face_vector(P.iaxis, k + 1, X, Y, SX[k], SY[k]);
        double R[5];
#pragma unroll
        for (int m = 0; m < 5; m++) {
            const double2 I = S.fg[m][c], a = S.fg[m][nb[0]], b = S.fg[m][nb[1]],
                          e = S.fg[m][nb[2]], d = S.fg[m][nb[3]];
            R[m] = HALF * ((I.x + a.x) * SX[0] + (I.y + a.y) * SY[0] + (I.x + b.x) * SX[1] +
                           (I.y + b.y) * SY[1] + (I.x + e.x) * SX[2] + (I.y + e.y) * SY[2] +
                           (I.x + d.x) * SX[3] + (I.y + d.y) * SY[3]);
        }
        const double VOL = M.cvol[cell];
        R[4] = R[4] - VOL * src5;
        if (P.iaxis == 1) R[2] = R[2] - VOL * src3;

        // update (residual.f90:67-83)
        const double DT = P.local ? A.dt[cell] : *A.dtmin;
        const double DTBYVOL = DT * S.st[gc + ST_RVOL * NTHREADS];
        const double al = A.alpha;
        double Cn[5], Co[5], vis[4], dd[5];
#pragma unroll
        for (int m = 0; m < 5; m++) {
            Co[m] = A.qold[m * ncell + cell];
            dd[m] = A.d[m * ncell + cell];
        }
#pragma unroll
        for (int k = 0; k < 4; k++) vis[k] = A.vis[k * ncell + cell];
        Cn[0] = Co[0] - al * DTBYVOL * (R[0] - dd[0]);
        Cn[1] = Co[1] - al * DTBYVOL * (R[1] - vis[0] - dd[1]);
        Cn[2] = Co[2] - al * DTBYVOL * (R[2] - vis[1] - dd[2]);
        Cn[3] = Co[3] - al * DTBYVOL * (R[3] - vis[2] - dd[3]);
        Cn[4] = Co[4] - al * DTBYVOL * CFLTURB * (R[4] - vis[3] - dd[4]);
        Cn[4] = Cn[0] * dmax1(P.rtol, Cn[4] / Cn[0]);
#pragma unroll
        for (int m = 0; m < 5; m++) A.qout[m * ncell + cell] = Cn[m];
        if (A.status) {
            bool bad = false;
#pragma unroll
            for (int m = 0; m < 5; m++) bad |= !isfinite(Cn[m]);
            if (bad) atomicOr(A.status, 1u);
        }
#pragma unroll
        for (int m = 0; m < 5; m++) dv[m] = fabs(Co[m] - Cn[m]);
    }
    if (A.cdiff) {
        // max |COLD - C| per component: warp max, then one atomic per warp on the ordered
        // bit pattern (non-negative doubles order like their bits)
#pragma unroll
        for (int m = 0; m < 5; m++) {
            double v = dv[m];
            for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
            if ((threadIdx.x & 31) == 0)
                atomicMax(&A.cdiff[m], (unsigned long long)__double_as_longlong(v));
        }
    }
}

// Specialised on the residual monitor, so the CDIFF reduction is compiled only where it
// runs.
template <int MONITOR, bool TMA>
__global__ void __launch_bounds__(NTHREADS, TNS_PER_SM(TNS_STAGE_MINB))
k_stage(Params P, Mesh M, StageArgs A, const __grid_constant__ CUtensorMap qmap) {
    StageArgs Ac = A;
    if (!MONITOR) Ac.cdiff = nullptr;
    stage_tile<TMA>(P, M, Ac, blockIdx.x, blockIdx.y, &qmap);
}

// ---------------------------------------------------------------- viscous kernel

// Faces owned by a tile: i-faces (between cells (i-1,j) and (i,j)) for i in i0..i0+TI,
// j-faces (between (i,j-1) and (i,j)) for j in j0..j0+TJ.
constexpr int NIF = (TI + 1) * TJ;
constexpr int NJF = TI * (TJ + 1);

struct ViscSmem {
    double u[NSLOT], v[NSLOT], t[NSLOT], rho[NSLOT], ri[NSLOT];
    double au[NAVG], av[NAVG], at[NAVG], arho[NAVG], ar[NAVG];
    double fi[4][NIF], fj[4][NJF];
};

size_t visc_smem_bytes() { return sizeof(ViscSmem); }

// One face flux (viscous.f90:130-217) in the orientation of cell A (slot sa): C = slot
// sc, B/D = the face's nodes in node-average coordinates, geometry from the face's
// stored row fg[k * nf] (FG_*).
__device__ __forceinline__ void face_flux(const Params& P, const ViscSmem& S, int sa, int sc,
                                          int ab, int ad, const double* __restrict__ fg,
                                          size_t nf, double out[4]) {
    FaceVals f;
    f.ua = S.u[sa]; f.va = S.v[sa]; f.ta = S.t[sa];
    f.uc = S.u[sc]; f.vc = S.v[sc]; f.tc = S.t[sc];
    f.ub = S.au[ab]; f.vb = S.av[ab]; f.tb = S.at[ab];
    f.ud = S.au[ad]; f.vd = S.av[ad]; f.td = S.at[ad];
    f.rhoa = S.rho[sa]; f.rhoc = S.rho[sc]; f.rhob = S.arho[ab]; f.rhod = S.arho[ad];
    f.ra = S.ri[sa]; f.rc = S.ri[sc]; f.rb = S.ar[ab]; f.rd = S.ar[ad];
    viscous_face(P, f, fg[FG_SX * nf], fg[FG_SY * nf], fg[FG_GA * nf], fg[FG_GB * nf],
                 fg[FG_GC * nf], fg[FG_GD * nf], P.iaxis == 1 ? fg[FG_RYAVG * nf] : 0.0, out);
}

// Frozen viscous flux VIS of Q_old (viscous.f90:29-217): nodal averages, then each face
// of the tile once; a cell adds its four faces in order 1..4, negating the faces that
// were evaluated in the neighbour's orientation.
__device__ __forceinline__ void viscous_tile(const Params& P, const Mesh& M, const double* __restrict__ q,
                                             double* __restrict__ vis, int bx, int by) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ViscSmem& S = *reinterpret_cast<ViscSmem*>(smem_raw);
    const size_t ncell = (size_t)M.ni * M.nj;
    const int j0 = bx * TJ, i0 = by * TI;
    const int tid = threadIdx.y * TJ + threadIdx.x;
    pdl_trigger();
    pdl_wait();
    for (int s = tid; s < NSLOT; s += VNT) {
        const int li = s / SW, lj = s % SW;
        int along = 0;
        const int kind = classify(M, i0 - 1 + li, j0 - 1 + lj, along);
        if (kind < 0) continue;
        Prim p;
        if (kind == 0)
            cell_prim(P, q, ncell, (size_t)(i0 - 1 + li) * M.nj + (j0 - 1 + lj), p);
        else
            ghost_state(P, M, q, ncell, kind, along, p);
        S.u[s] = p.u; S.v[s] = p.v; S.t[s] = p.t; S.rho[s] = p.rho; S.ri[s] = p.ri;
    }
    __syncthreads();
    // nodal averages (viscous.f90:40-59,77-124) of nodes (i0..i0+TI, j0..j0+TJ)
    for (int s = tid; s < NAVG; s += VNT) {
        const int la = s / AW, lb = s % AW;
        const int a = i0 + la, b = j0 + lb;
        if (a > M.ni || b > M.nj) continue;
        double un = 0.0, vn = 0.0, tn = 0.0, rhon = 0.0, rn = 0.0;
        int cnt = 0, ng = 0, gs[2] = {0, 0}, gr[2] = {0, 0};
        // the four surrounding positions in ascending cell-id order
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int pi = a - 1 + (k >> 1), pj = b - 1 + (k & 1);
            const int sl = (la + (k >> 1)) * SW + lb + (k & 1);
            int along = 0;
            const int kind = classify(M, pi, pj, along);
            if (kind == 0) {
                un = un + S.u[sl]; vn = vn + S.v[sl]; tn = tn + S.t[sl];
                rhon = rhon + S.rho[sl]; rn = rn + S.ri[sl];
                cnt++;
            } else if (kind > 0) {
                gs[ng] = sl;
                gr[ng] = M.ghost_index(kind, along);
                ng++;
            }
        }
        if (ng == 2 && M.grank[gr[1]] < M.grank[gr[0]]) {
            int t = gs[0]; gs[0] = gs[1]; gs[1] = t;
            t = gr[0]; gr[0] = gr[1]; gr[1] = t;
        }
        for (int k = 0; k < ng; k++) {
            const int sl = gs[k];
            un = un + S.u[sl]; vn = vn + S.v[sl]; tn = tn + S.t[sl];
            rhon = rhon + S.rho[sl]; rn = rn + S.ri[sl];
            const int type = M.gtype[gr[k]];
            if (type == 4) {
                vn = 0.0;
            } else if (type == 5) {
                un = 0.0; vn = 0.0; rn = P.rtol_rtred;
            }
            cnt++;
        }
        const double idf = cnt == 4 ? 0.25 : 1.0 / (double)cnt;
        S.au[s] = un * idf; S.av[s] = vn * idf; S.at[s] = tn * idf; S.arho[s] = rhon * idf;
        S.ar[s] = dmax1(P.rtol, rn * idf);
    }
    __syncthreads();
    // all faces of the tile in one loop (i-faces first): at most three faces per thread,
    // one inlined copy of the face flux
    const size_t nfi = (size_t)(M.ni + 1) * M.nj, nfj = (size_t)M.ni * (M.nj + 1);
    for (int f = tid; f < NIF + NJF; f += VNT) {
        int sa, sc, ab, ad;
        const double* fg;
        size_t nf;
        if (f < NIF) {
            // i-face: orientation of cell (i-1, j) as its face 2, or of (0, j) as its face 4
            const int ii = f / TJ, jj = f % TJ;
            const int i = i0 + ii, j = j0 + jj;
            if (i > M.ni || j >= M.nj) continue;
            const int sL = ii * SW + jj + 1, sR = sL + SW;  // cells (i-1, j), (i, j)
            const int aLo = ii * AW + jj, aHi = aLo + 1;    // nodes (i, j), (i, j+1)
            if (i == 0) {  // face 4: B=N4, D=N1
                sa = sR; sc = sL; ab = aHi; ad = aLo;
            } else {  // face 2: B=N2, D=N3
                sa = sL; sc = sR; ab = aLo; ad = aHi;
            }
            fg = M.fgi + ((size_t)i * M.nj + j);
            nf = nfi;
        } else {
            // j-face: orientation of cell (i, j-1) as its face 3, or of (i, 0) as its face 1
            const int g = f - NIF;
            const int ii = g / AW, jj = g % AW;
            const int i = i0 + ii, j = j0 + jj;
            if (i >= M.ni || j > M.nj) continue;
            const int sB = (ii + 1) * SW + jj, sT = sB + 1;  // cells (i, j-1), (i, j)
            const int aL = ii * AW + jj, aR = aL + AW;       // nodes (i, j), (i+1, j)
            if (j == 0) {  // face 1: B=N1, D=N2
                sa = sT; sc = sB; ab = aL; ad = aR;
            } else {  // face 3: B=N3, D=N4
                sa = sB; sc = sT; ab = aR; ad = aL;
            }
            fg = M.fgj + ((size_t)i * (M.nj + 1) + j);
            nf = nfj;
        }
        double out[4];
        face_flux(P, S, sa, sc, ab, ad, fg, nf, out);
        if (f < NIF) {
#pragma unroll
            for (int k = 0; k < 4; k++) S.fi[k][f] = out[k];
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) S.fj[k][f - NIF] = out[k];
        }
    }
    __syncthreads();
    const int tj = threadIdx.x, ti = threadIdx.y;
    const int i = i0 + ti, j = j0 + tj;
    if (ti >= TI || i >= M.ni || j >= M.nj) return;
    const size_t cell = (size_t)i * M.nj + j;
    const int f1 = ti * AW + tj, f3 = f1 + 1;          // j-faces j, j+1
    const int f4 = ti * TJ + tj, f2 = f4 + TJ;         // i-faces i, i+1
    const double s1 = (j == 0) ? 1.0 : -1.0, s4 = (i == 0) ? 1.0 : -1.0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        double acc = s1 * S.fj[k][f1];
        acc = acc + S.fi[k][f2];
        acc = acc + S.fj[k][f3];
        acc = acc + s4 * S.fi[k][f4];
        vis[k * ncell + cell] = acc;
    }
}

__global__ void __launch_bounds__(VNT, TNS_PER_SM(TNS_VISC_MINB)) k_viscous(Params P, Mesh M, const double* __restrict__ q,
                                                      double* __restrict__ vis) {
    viscous_tile(P, M, q, vis, blockIdx.x, blockIdx.y);
}

// --------------------------------------------------------- dissipation kernel

constexpr int DW = TJ + 4;             // halo-2 slot grid (TI+4) x (TJ+4)
constexpr int NDSLOT = (TI + 4) * DW;
constexpr int RW = TJ + 2;             // ring-1 grid (TI+2) x (TJ+2)
constexpr int NRSLOT = (TI + 2) * RW;
enum DField { DC0, DC1, DC2, DC3, DC4, DP, NDF };
enum RField { RVBD, RANU, RANURT, RQ0, RQ1, RQ2, RQ3, RQ4, NRF };

size_t diss_smem_bytes() {
    return sizeof(double) * ((size_t)NDF * NDSLOT + (size_t)NRF * NRSLOT);
}

__device__ __forceinline__ double local_dt(const Params& P, double c1, double c2, double c3,
                                           double c4, double cfldl) {
    // turbnstwod.f90:97-108
    const double RHO = c1;
    const double rr = 1.0 / RHO;
    const double U = c2 * rr, V = c3 * rr;
    const double VEL = sqrt(U * U + V * V);
    const double E = c4 * rr;
    const double T = (E - 0.5 * (U * U + V * V)) * P.inv_cv;
    return cfldl / (fabs(VEL) + sqrt(P.gamrr * T));
}

template <class OutT>
__device__ __forceinline__ void dissipation_tile(const Params& P, const Mesh& M, const DissArgs<OutT>& A,
                                                 int bx, int by) {
    extern __shared__ double smem[];
    double* sd = smem;                  // NDF x NDSLOT
    double* sr = sd + NDF * NDSLOT;     // NRF x NRSLOT
    const size_t ncell = (size_t)M.ni * M.nj;
    const int j0 = bx * TJ, i0 = by * TI;
    const int tid = threadIdx.y * TJ + threadIdx.x;

    pdl_trigger();
    pdl_wait();
    for (int s = tid; s < NDSLOT; s += NTHREADS) {
        const int i = i0 - 2 + s / DW, j = j0 - 2 + s % DW;
        if (i >= 0 && i < M.ni && j >= 0 && j < M.nj) {
            const size_t c = (size_t)i * M.nj + j;
            double C[5];
#pragma unroll
            for (int m = 0; m < 5; m++) {
                C[m] = A.q[m * ncell + c];
                sd[(DC0 + m) * NDSLOT + s] = C[m];
            }
            // P as in the DT loop (turbnstwod.f90:98-104)
            const double RHO = C[0];
            const double rr = 1.0 / RHO;
            const double U = C[1] * rr, V = C[2] * rr;
            const double E = C[3] * rr;
            const double T = (E - 0.5 * (U * U + V * V)) * P.inv_cv;
            sd[DP * NDSLOT + s] = RHO * P.rr * T;
        }
    }
    __syncthreads();

    // ring-1 cells: VOL/DT, sensors, Laplacians (ghost neighbours read as the cell itself)
    for (int s = tid; s < NRSLOT; s += NTHREADS) {
        const int ri = s / RW, rj = s % RW;
        const int i = i0 - 1 + ri, j = j0 - 1 + rj;
        if (!(i >= 0 && i < M.ni && j >= 0 && j < M.nj)) continue;
        const int d = (ri + 1) * DW + (rj + 1);  // same cell in the halo-2 grid
        int nbs[4] = {d - 1, d + DW, d + 1, d - DW};
        if (j == 0) nbs[0] = d;
        if (i == M.ni - 1) nbs[1] = d;
        if (j == M.nj - 1) nbs[2] = d;
        if (i == 0) nbs[3] = d;
        const double* Pp = sd + DP * NDSLOT;
        const double* C5 = sd + DC4 * NDSLOT;
        const double PIE = Pp[d], C1I = sd[DC0 * NDSLOT + d], C5I = C5[d];
        double ANUN = fabs(Pp[nbs[0]] - PIE) + fabs(Pp[nbs[1]] - PIE) + fabs(Pp[nbs[2]] - PIE) +
                      fabs(Pp[nbs[3]] - PIE);
        double ANUD = fabs(Pp[nbs[0]] + PIE) + fabs(Pp[nbs[1]] + PIE) + fabs(Pp[nbs[2]] + PIE) +
                      fabs(Pp[nbs[3]] + PIE);
        sr[RANU * NRSLOT + s] = ANUN / ANUD;
        ANUN = fabs(C5[nbs[0]] - C5I) + fabs(C5[nbs[1]] - C5I) + fabs(C5[nbs[2]] - C5I) +
               fabs(C5[nbs[3]] - C5I);
        ANUD = fabs(C5[nbs[0]] + C5I) + fabs(C5[nbs[1]] + C5I) + fabs(C5[nbs[2]] + C5I) +
               fabs(C5[nbs[3]] + C5I);
        sr[RANURT * NRSLOT + s] = ANUN / dmax1(ANUD, 8.0 * C1I * P.rtol);
#pragma unroll
        for (int m = 0; m < 5; m++) {
            const double* Cm = sd + (DC0 + m) * NDSLOT;
            sr[(RQ0 + m) * NRSLOT + s] = Cm[nbs[0]] + Cm[nbs[1]] + Cm[nbs[2]] + Cm[nbs[3]] - 4.0 * Cm[d];
        }
        // time step and VOL/DT
        const size_t c = (size_t)i * M.nj + j;
        double DT;
        if (P.local) {
            DT = local_dt(P, sd[DC0 * NDSLOT + d], sd[DC1 * NDSLOT + d], sd[DC2 * NDSLOT + d],
                          sd[DC3 * NDSLOT + d], M.cfldl[c]);
            if (ri >= 1 && ri <= TI && rj >= 1 && rj <= TJ) A.dt[c] = (OutT)DT;
        } else {
            DT = *A.dtmin;
        }
        sr[RVBD * NRSLOT + s] = M.cvol[c] / DT;
    }
    __syncthreads();

    const int tj = threadIdx.x, ti = threadIdx.y;
    const int i = i0 + ti, j = j0 + tj;
    if (i >= M.ni || j >= M.nj) return;
    const size_t cell = (size_t)i * M.nj + j;
    const int r = (ti + 1) * RW + (tj + 1);
    const int d = (ti + 2) * DW + (tj + 2);
    const int rn[4] = {r - 1, r + RW, r + 1, r - RW};
    const int dn[4] = {d - 1, d + DW, d + 1, d - DW};
    const bool has[4] = {j > 0, i < M.ni - 1, j < M.nj - 1, i > 0};
    const double VOLBYDT = sr[RVBD * NRSLOT + r];
    // per-face blend coefficients (identical for the four equations)
    double D2c[4], D4c[4], D2t[4], D4t[4];
    const double ANUI = sr[RANU * NRSLOT + r], ANURTI = sr[RANURT * NRSLOT + r];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const double D24N = HALF * (VOLBYDT + sr[RVBD * NRSLOT + rn[k]]);
        double E2N = C02 * dmax1(ANUI, sr[RANU * NRSLOT + rn[k]]);
        double E4N = dmax1(0.0, C04 - E2N);
        D2c[k] = E2N * D24N;
        D4c[k] = E4N * D24N;
        E2N = C02 * dmax1(ANURTI, sr[RANURT * NRSLOT + rn[k]]);
        E4N = dmax1(0.0, C04 - E2N);
        D2t[k] = E2N * D24N;
        D4t[k] = E4N * D24N;
    }
#pragma unroll
    for (int m = 0; m < 5; m++) {
        const double* Cm = sd + (DC0 + m) * NDSLOT;
        const double* Qm = sr + (RQ0 + m) * NRSLOT;
        const double CI = Cm[d], D2I = Qm[r];
        double D2 = 0.0, D4 = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!has[k]) continue;  // ghost face: exactly zero contribution
            const double a2 = (m == 4) ? D2t[k] : D2c[k];
            const double a4 = (m == 4) ? D4t[k] : D4c[k];
            D2 = D2 + a2 * (Cm[dn[k]] - CI);
            D4 = D4 + a4 * (Qm[rn[k]] - D2I);
        }
        A.d[m * ncell + cell] = (OutT)(D2 - D4);
    }
}

template <class OutT>
__global__ void __launch_bounds__(NTHREADS) k_dissipation(Params P, Mesh M, DissArgs<OutT> A) {
    dissipation_tile<OutT>(P, M, A, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------- time step min

__global__ void __launch_bounds__(256)
k_dtmin(Params P, Mesh M, const double* __restrict__ q, double* dt, double* partial,
        unsigned int* counter, double* dtmin) {
    const size_t ncell = (size_t)M.ni * M.nj;
    double mn = 100000.0;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < ncell;
         c += (size_t)gridDim.x * blockDim.x) {
        const double v = local_dt(P, q[c], q[ncell + c], q[2 * ncell + c], q[3 * ncell + c],
                                  M.cfldl[c]);
        mn = dmin1(mn, v);
    }
    for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    __shared__ double wmin[8];
    __shared__ bool last;
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = mn;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = wmin[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) b = fmin(b, wmin[w]);
        partial[blockIdx.x] = b;
        __threadfence();
        const unsigned int done = atomicAdd(counter, 1u);
        last = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double b = 100000.0;
        for (unsigned int k = 0; k < gridDim.x; k++) b = fmin(b, ((volatile double*)partial)[k]);
        *dtmin = b;
        *counter = 0u;
    }
}

// Variant of k_dtmin for caller-provided device buffers (tns_time_step_noalloc): also
// stores the per-cell DT, and reduces through the scratch the launcher is handed
// (`partial`: one double per block, `counter`: zero on entry, left at zero on exit).
__global__ void __launch_bounds__(256)
k_time_step_scratch(Params P, const double* __restrict__ q, const double* __restrict__ cfldl,
                    long long ncell, double* __restrict__ dt, double* partial,
                    unsigned int* counter, double* dtmin) {
    double mn = 100000.0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x) {
        const double v = local_dt(P, q[c], q[ncell + c], q[2 * ncell + c], q[3 * ncell + c],
                                  cfldl[c]);
        dt[c] = v;
        mn = dmin1(mn, v);
    }
    for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    __shared__ double wmin[8];
    __shared__ bool last;
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = mn;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = wmin[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) b = fmin(b, wmin[w]);
        partial[blockIdx.x] = b;
        __threadfence();
        last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double b = 100000.0;
        for (unsigned int k = 0; k < gridDim.x; k++) b = fmin(b, ((volatile double*)partial)[k]);
        *dtmin = b;
        *counter = 0u;
    }
}

void launch_time_step_scratch(const Params& P, const double* q, const double* cfldl,
                              long long ncell, double* dt, double* partial,
                              unsigned int* counter, double* dtmin, int nblocks,
                              cudaStream_t s) {
    k_time_step_scratch<<<nblocks, 256, 0, s>>>(P, q, cfldl, ncell, dt, partial, counter, dtmin);
}

// ------------------------------------------------------------ port mass flux

// One block per type-6 ghost: sum of C1*U*DELY(*YCC) along the mesh line through the
// parent, across to the opposite boundary (the repaired GPORT walk); its threads stride
// the line, then a warp and block reduction in fixed order.
__global__ void k_gport(Params P, Mesh M, const double* __restrict__ q, const int* ghosts,
                        int nport, double* gport) {
    const int w = blockIdx.x;  // one block per port ghost
    const int lane = threadIdx.x & 31;
    if (w >= nport) return;  // whole block
    const size_t ncell = (size_t)M.ni * M.nj;
    const int g = ghosts[w];
    int side, along;
    if (g < M.ni) { side = 1; along = g; }
    else if (g < M.ni + M.nj) { side = 2; along = g - M.ni; }
    else if (g < 2 * M.ni + M.nj) { side = 3; along = g - M.ni - M.nj; }
    else { side = 4; along = g - 2 * M.ni - M.nj; }
    const int len = (side == 1 || side == 3) ? M.nj : M.ni;
    double sum = 0.0;
    for (int k = threadIdx.x; k < len; k += GP_THREADS) {
        const int i = (side == 1 || side == 3) ? along : k;
        const int j = (side == 1 || side == 3) ? k : along;
        const size_t c = (size_t)i * M.nj + j;
        const size_t n1 = (size_t)i * (M.nj + 1) + j;
        const double y1 = M.y[n1], y2 = M.y[n1 + M.nj + 1], y3 = M.y[n1 + M.nj + 2],
                     y4 = M.y[n1 + 1];
        double dely;
        if (side == 1) dely = HALF * ((y1 + y2) - (y3 + y4));
        else if (side == 2) dely = HALF * ((y2 + y3) - (y1 + y4));
        else if (side == 3) dely = HALF * ((y3 + y4) - (y1 + y2));
        else dely = HALF * ((y4 + y1) - (y2 + y3));
        const double c1 = q[c], u = q[ncell + c] / c1;
        double term = c1 * u * dely;
        if (P.iaxis == 1) term = term * ((y1 + y2 + y3 + y4) * 0.25);
        sum += term;
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    __shared__ double part[GP_THREADS / 32];
    if (lane == 0) part[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = part[0];
#pragma unroll
        for (int k = 1; k < GP_THREADS / 32; k++) t += part[k];
        gport[g] = t;
    }
}

// ------------------------------------------------------ primitive output

// U, V, T, P of every cell and ghost computed from q (the last stage's input), the
// arrays COMPUTE_PRIMITIVE_VARS / APPLY_BOUNDARY leave behind.  Output layout:
// [4][ncell + nghost] with ghosts in side-array order.
__global__ void k_prim_out(Params P, Mesh M, const double* __restrict__ q, double* out) {
    const size_t ncell = (size_t)M.ni * M.nj;
    const size_t ng = M.nghosts(), ntot = ncell + ng;
    const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k >= ntot) return;
    Prim p;
    if (k < ncell) {
        cell_prim(P, q, ncell, k, p);
    } else {
        const int g = (int)(k - ncell);
        int side, along;
        if (g < M.ni) { side = 1; along = g; }
        else if (g < M.ni + M.nj) { side = 2; along = g - M.ni; }
        else if (g < 2 * M.ni + M.nj) { side = 3; along = g - M.ni - M.nj; }
        else { side = 4; along = g - 2 * M.ni - M.nj; }
        ghost_state(P, M, q, ncell, side, along, p);
    }
    out[k] = p.u;
    out[ntot + k] = p.v;
    out[2 * ntot + k] = p.t;
    out[3 * ntot + k] = p.p;
}

// ---------------------------------------------------------- post-processing

// POSTPROCESS node averages (solver_state.f90:237-281) of the [4][ncell+nghost] U,V,T,P
// array k_prim_out produced: cells in ascending id order, then the ghosts of the node
// in bc.in order, divided by their count.  Output [4][nnode] as (P, U, V, T).
__global__ void k_node_average(Mesh M, const double* __restrict__ prim, double* __restrict__ out) {
    const size_t ncell = (size_t)M.ni * M.nj, ntot = ncell + M.nghosts();
    const size_t nnode = (size_t)(M.ni + 1) * (M.nj + 1);
    const size_t n = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (n >= nnode) return;
    const int a = (int)(n / (M.nj + 1)), b = (int)(n % (M.nj + 1));
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    int cnt = 0, ng = 0;
    size_t gk[2] = {0, 0};
    int gr[2] = {0, 0};
    for (int k = 0; k < 4; k++) {
        const int pi = a - 1 + (k >> 1), pj = b - 1 + (k & 1);
        int along = 0;
        const int kind = classify(M, pi, pj, along);
        if (kind == 0) {
            const size_t c = (size_t)pi * M.nj + pj;
            s[0] += prim[3 * ntot + c]; s[1] += prim[c]; s[2] += prim[ntot + c]; s[3] += prim[2 * ntot + c];
            cnt++;
        } else if (kind > 0) {
            const int g = M.ghost_index(kind, along);
            gk[ng] = ncell + g;
            gr[ng] = M.grank[g];
            ng++;
        }
    }
    if (ng == 2 && gr[1] < gr[0]) { const size_t t = gk[0]; gk[0] = gk[1]; gk[1] = t; }
    for (int k = 0; k < ng; k++) {
        const size_t c = gk[k];
        s[0] += prim[3 * ntot + c]; s[1] += prim[c]; s[2] += prim[ntot + c]; s[3] += prim[2 * ntot + c];
        cnt++;
    }
    const double d = (double)cnt;
#pragma unroll
    for (int f = 0; f < 4; f++) out[f * nnode + n] = s[f] / d;
}

// Boundary-face sums over the ghosts whose BC type / side match (0 = any), with the face
// state (parent + ghost)/2.  mode 0: [0] sum P*SX, [1] sum P*SY, [2] sum RHO*(U*SX+V*SY),
// [3] sum |S|; mode 1: [0] sum P0*|MDOT|, [1] sum |MDOT| with the face's total pressure
// P0 = P (1 + (GAMA-1)/2 M^2)^(GAMA/(GAMA-1)), M^2 = (U^2+V^2)/(GAMA RR T), and mass flux
// MDOT = RHO (U SX + V SY).  One warp per 32 faces; one atomicAdd per warp and quantity.
__global__ void k_boundary_sums(Params P, Mesh M, const double* __restrict__ prim, int type,
                                int side, int mode, double* __restrict__ out) {
    const size_t ncell = (size_t)M.ni * M.nj, ntot = ncell + M.nghosts();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (g < M.nghosts()) {
        int sd, along;
        if (g < M.ni) { sd = 1; along = g; }
        else if (g < M.ni + M.nj) { sd = 2; along = g - M.ni; }
        else if (g < 2 * M.ni + M.nj) { sd = 3; along = g - M.ni - M.nj; }
        else { sd = 4; along = g - 2 * M.ni - M.nj; }
        if ((type == 0 || M.gtype[g] == type) && (side == 0 || sd == side)) {
            int ip, jp;
            if (sd == 1) { ip = along; jp = 0; }
            else if (sd == 2) { ip = M.ni - 1; jp = along; }
            else if (sd == 3) { ip = along; jp = M.nj - 1; }
            else { ip = 0; jp = along; }
            const size_t cp = (size_t)ip * M.nj + jp, cg = ncell + g;
            const size_t n1 = (size_t)ip * (M.nj + 1) + jp;
            const double X[4] = {M.x[n1], M.x[n1 + M.nj + 1], M.x[n1 + M.nj + 2], M.x[n1 + 1]};
            const double Y[4] = {M.y[n1], M.y[n1 + M.nj + 1], M.y[n1 + M.nj + 2], M.y[n1 + 1]};
            double sx, sy;
            face_vector(P.iaxis, sd, X, Y, sx, sy);
            const double u = 0.5 * (prim[cp] + prim[cg]), vv = 0.5 * (prim[ntot + cp] + prim[ntot + cg]);
            face_sums(P, mode, u, vv, prim[2 * ntot + cp], prim[2 * ntot + cg], prim[3 * ntot + cp],
                      prim[3 * ntot + cg], sx, sy, v);
        }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0 && x != 0.0) atomicAdd(&out[q], x);
    }
}

// Face state (parent + ghost)/2 of every ghost in device order: out [5][nghosts] = U, V,
// P, RHO (the average of P/(RR*T) on both sides), T.
__global__ void k_face_states(Params P, Mesh M, const double* __restrict__ prim, double* __restrict__ out) {
    const size_t ncell = (size_t)M.ni * M.nj, ng = M.nghosts(), ntot = ncell + ng;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (int)ng) return;
    int sd, along;
    if (g < M.ni) { sd = 1; along = g; }
    else if (g < M.ni + M.nj) { sd = 2; along = g - M.ni; }
    else if (g < 2 * M.ni + M.nj) { sd = 3; along = g - M.ni - M.nj; }
    else { sd = 4; along = g - 2 * M.ni - M.nj; }
    int ip, jp;
    if (sd == 1) { ip = along; jp = 0; }
    else if (sd == 2) { ip = M.ni - 1; jp = along; }
    else if (sd == 3) { ip = along; jp = M.nj - 1; }
    else { ip = 0; jp = along; }
    const size_t cp = (size_t)ip * M.nj + jp, cg = ncell + g;
    const double tp = prim[2 * ntot + cp], tgh = prim[2 * ntot + cg];
    const double pp = prim[3 * ntot + cp], pgh = prim[3 * ntot + cg];
    out[g] = 0.5 * (prim[cp] + prim[cg]);
    out[ng + g] = 0.5 * (prim[ntot + cp] + prim[ntot + cg]);
    out[2 * ng + g] = 0.5 * (pp + pgh);
    out[3 * ng + g] = 0.5 * (pp / (P.rr * tp) + pgh / (P.rr * tgh));
    out[4 * ng + g] = 0.5 * (tp + tgh);
}

void launch_face_states(const Params& P, const Mesh& M, const double* prim, double* out, cudaStream_t s) {
    k_face_states<<<(M.nghosts() + 255) / 256, 256, 0, s>>>(P, M, prim, out);
}

// ------------------------------------------------------------ batched kernels

// One launch per kernel advances every active case of a batch; block b works on tile
// tiles[b] = (case, tile j, tile i) with its case's parameters and buffers.
__global__ void __launch_bounds__(NTHREADS) k_dissipation_batch(const BatchCase* __restrict__ cases,
                                                                const int4* __restrict__ tiles,
                                                                const int* __restrict__ active) {
    const int4 t = tiles[blockIdx.x];
    if (!active[t.x]) return;  // whole block: before any barrier
    const BatchCase& c = cases[t.x];
    dissipation_tile<double>(c.P, c.M, c.diss, t.y, t.z);
}

__global__ void __launch_bounds__(VNT, TNS_PER_SM(TNS_VISC_BATCH_MINB)) k_viscous_batch(const BatchCase* __restrict__ cases,
                                                                          const int4* __restrict__ tiles,
                                                                          const int* __restrict__ active) {
    const int4 t = tiles[blockIdx.x];
    if (!active[t.x]) return;
    const BatchCase& c = cases[t.x];
    viscous_tile(c.P, c.M, c.q, c.vis, t.y, t.z);
}

__global__ void __launch_bounds__(NTHREADS, TNS_PER_SM(TNS_STAGE_BATCH_MINB)) k_stage_batch(const BatchCase* __restrict__ cases,
                                                                         const int4* __restrict__ tiles,
                                                                         const int* __restrict__ active,
                                                                         int stage, int monitor) {
    const int4 t = tiles[blockIdx.x];
    if (!active[t.x]) return;
    const BatchCase& c = cases[t.x];
#if TNS_BATCH_SMEM_ARGS
    // the case's arguments copied into shared memory (raw storage, never constructed):
    // loads from constant shared addresses instead of through the descriptor pointer
    __shared__ __align__(16) unsigned char sargs[sizeof(Params) + sizeof(Mesh) + sizeof(StageArgs)];
    Params& sP = *reinterpret_cast<Params*>(sargs);
    Mesh& sM = *reinterpret_cast<Mesh*>(sargs + sizeof(Params));
    StageArgs& sA = *reinterpret_cast<StageArgs*>(sargs + sizeof(Params) + sizeof(Mesh));
    {
        const int tid = threadIdx.y * TJ + threadIdx.x;
        copy_words(&sP, &c.P, sizeof(Params), tid);
        copy_words(&sM, &c.M, sizeof(Mesh), tid);
        copy_words(&sA, &c.stage[monitor][stage], sizeof(StageArgs), tid);
        __syncthreads();
    }
    stage_tile<false>(sP, sM, sA, t.y, t.z);
#else
    stage_tile<false>(c.P, c.M, c.stage[monitor][stage], t.y, t.z);
#endif
}

// Persistent batched iterations (schedule 3): one cooperative launch advances every
// active case by `iters` unmonitored RK4 iterations.  Its blocks walk the tile table
// phase by phase -- dissipation and viscous flux together (both read Q_old only and
// write disjoint arrays), then the four stages -- with a grid barrier between phases
// (bounded waits: a barrier that gives up sets error bit 2 and the kernel returns).  A
// block that finishes a tile synchronises before the next, whose static-block copy
// reuses the tile's shared memory and barrier.  Cases need LOCAL=1 and no type-6 port
// (those add per-case reductions between the phases).
#ifndef TNS_PERSIST_MINB
#define TNS_PERSIST_MINB 3
#endif
__global__ void __launch_bounds__(NTHREADS, TNS_PER_SM(TNS_PERSIST_MINB))
k_batch_persistent(const BatchCase* __restrict__ cases, const int4* __restrict__ tiles,
                   const int* __restrict__ active, int ntiles, int iters, unsigned int* bar,
                   unsigned int* error) {
    for (int it = 0; it < iters; it++) {
        for (int ph = 0; ph < 5; ph++) {
            const int nwork = ph == 0 ? 2 * ntiles : ntiles;
            for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
                const int4 t = tiles[w % ntiles];
                if (active[t.x]) {
                    const BatchCase& c = cases[t.x];
                    if (ph == 0 && w < ntiles) dissipation_tile<double>(c.P, c.M, c.diss, t.y, t.z);
                    else if (ph == 0) viscous_tile(c.P, c.M, c.q, c.vis, t.y, t.z);
                    else stage_tile<false>(c.P, c.M, c.stage[0][ph - 1], t.y, t.z);
                }
                __syncthreads();
            }
            if (!grid_barrier(bar, bar + 1)) {
                if (threadIdx.x == 0 && threadIdx.y == 0) atomicOr(error, 4u);
                return;
            }
        }
    }
}

// ---------------------------------------------------------------- math check

// Evaluates one of the FP64 helpers the kernels use, elementwise, for testing their
// accuracy: fn 0 = pow06(a), 1 = tanh_ratio(a, b), 2 = expm1_nonneg(a).
__global__ void k_debug_math(int fn, long long n, const double* __restrict__ a, const double* __restrict__ b,
                             double* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = fn == 0 ? pow06(a[i]) : (fn == 1 ? tanh_ratio(a[i], b[i]) : expm1_nonneg(a[i]));
}

void launch_debug_math(int fn, long long n, const double* a, const double* b, double* out, cudaStream_t s) {
    const long long blocks = (n + 255) / 256;
    if (blocks > 0) k_debug_math<<<(unsigned)blocks, 256, 0, s>>>(fn, n, a, b, out);
}

// ------------------------------------------------------------------ launchers

static dim3 tile_grid(const Mesh& M) { return dim3((M.nj + TJ - 1) / TJ, (M.ni + TI - 1) / TI); }

#if TNS_STAGE_TMA_ON
// The driver's tensor-map encoder, looked up once through the runtime.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
                cudaSuccess || q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// Tensor map of a state array [5][NI][NJ] for the stage's Q box; false (the caller takes
// the plain-load kernel) where TMA cannot address it: NJ odd (rows not a multiple of 16
// bytes) or the array not 16-byte aligned.
static bool stage_q_map(const Mesh& M, const double* q, CUtensorMap* map) {
    if (M.nj % 2 != 0 || (reinterpret_cast<uintptr_t>(q) & 15) != 0) return false;
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)M.nj, (cuuint64_t)M.ni, 5};
    const cuuint64_t strides[2] = {(cuuint64_t)M.nj * sizeof(double), (cuuint64_t)M.ni * M.nj * sizeof(double)};
    const cuuint32_t box[3] = {(cuuint32_t)QW, (cuuint32_t)QH, 5};
    const cuuint32_t elem[3] = {1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(q), dims, strides, box, elem,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
#endif

cudaError_t configure_kernels() {
    cudaError_t e;
    e = cudaFuncSetAttribute(k_stage<0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)stage_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_stage<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)stage_smem_bytes());
    if (e != cudaSuccess) return e;
#if TNS_STAGE_TMA_ON
    e = cudaFuncSetAttribute(k_stage<0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)stage_tma_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_stage<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)stage_tma_smem_bytes());
    if (e != cudaSuccess) return e;
#endif
    e = cudaFuncSetAttribute(k_viscous, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)visc_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_dissipation<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)diss_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_dissipation<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)diss_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_dissipation_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)diss_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_viscous_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)visc_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_batch_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)persistent_smem_bytes(false));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_stage_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)stage_smem_bytes());
}

size_t persistent_smem_bytes(bool mixed) {
    if (mixed) return std::max(stage_mx_smem_bytes(), std::max(visc_mx_smem_bytes(), diss_mx_smem_bytes()));
    return std::max(stage_smem_bytes(), std::max(visc_smem_bytes(), diss_smem_bytes()));
}

int persistent_grid(bool mixed) {
    int per_sm = 0, dev = 0, sms = 0;
    const void* k = mixed ? persistent_kernel_mx() : (const void*)k_batch_persistent;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NTHREADS, persistent_smem_bytes(mixed)) !=
            cudaSuccess)
        return 0;
    return per_sm * sms;
}

cudaError_t launch_persistent(bool mixed, const BatchCase* cases, const int4* tiles, const int* active,
                              int ntiles, int iters, int parity, int grid, unsigned int* bar,
                              unsigned int* error, cudaStream_t s) {
    if (mixed) return launch_persistent_mx(cases, tiles, active, ntiles, iters, parity, grid, bar, error, s);
    void* args[] = {(void*)&cases, (void*)&tiles, (void*)&active, (void*)&ntiles, (void*)&iters, (void*)&bar,
                    (void*)&error};
    return cudaLaunchCooperativeKernel((const void*)k_batch_persistent, dim3(grid), dim3(TJ, TI), args,
                                       persistent_smem_bytes(false), s);
}

void launch_batch_f64(const BatchCase* cases, const int4* tiles, const int* active, int ntiles,
                      int kernel, int stage, int monitor, cudaStream_t s) {
    const dim3 blk(TJ, TI);
    if (kernel == 0)
        launch_tile(k_dissipation_batch, dim3(ntiles), blk, diss_smem_bytes(), s, cases, tiles, active);
    else if (kernel == 1)
        launch_tile(k_viscous_batch, dim3(ntiles), dim3(TJ, VROWS), visc_smem_bytes(), s, cases, tiles, active);
    else
        launch_tile(k_stage_batch, dim3(ntiles), blk, stage_smem_bytes(), s, cases, tiles, active, stage, monitor);
}

void launch_dissipation(const Params& P, const Mesh& M, const double* q, double* d, double* dt,
                        const double* dtmin, cudaStream_t s) {
    DissArgs<double> A{q, d, dt, dtmin};
    launch_tile(k_dissipation<double>, tile_grid(M), dim3(TJ, TI), diss_smem_bytes(), s, P, M, A);
}

void launch_dissipation_mx(const Params& P, const Mesh& M, const double* q, float* d, float* dt,
                           const double* dtmin, cudaStream_t s) {
    DissArgs<float> A{q, d, dt, dtmin};
    launch_tile(k_dissipation<float>, tile_grid(M), dim3(TJ, TI), diss_smem_bytes(), s, P, M, A);
}

void launch_viscous(const Params& P, const Mesh& M, const double* q, double* vis, cudaStream_t s) {
    launch_tile(k_viscous, tile_grid(M), dim3(TJ, VROWS), visc_smem_bytes(), s, P, M, q, vis);
}

void launch_stage(const Params& P, const Mesh& M, const double* qin, const double* qold,
                  double* qout, const double* d, const double* vis, const double* dt,
                  const double* dtmin, double alpha, unsigned long long* cdiff,
                  unsigned int* status, unsigned int* error, cudaStream_t s) {
    StageArgs A{qin, qold, qout, d, vis, dt, dtmin, alpha, cdiff, status, error};
    CUtensorMap qmap;
#if TNS_STAGE_TMA_ON
    if (stage_q_map(M, qin, &qmap)) {
        launch_tile(cdiff ? k_stage<1, true> : k_stage<0, true>, tile_grid(M), dim3(TJ, TI),
                    stage_tma_smem_bytes(), s, P, M, A, qmap);
        return;
    }
#endif
    memset(&qmap, 0, sizeof(qmap));
    launch_tile(cdiff ? k_stage<1, false> : k_stage<0, false>, tile_grid(M), dim3(TJ, TI), stage_smem_bytes(), s,
                P, M, A, qmap);
}

int dtmin_blocks(const Mesh& M) {
    const long long ncell = (long long)M.ni * M.nj;
    long long b = (ncell + 255) / 256;
    return (int)(b < 1184 ? b : 1184);  // 148 SMs x 8
}

void launch_dtmin(const Params& P, const Mesh& M, const double* q, double* partial,
                  unsigned int* counter, double* dtmin, cudaStream_t s) {
    k_dtmin<<<dtmin_blocks(M), 256, 0, s>>>(P, M, q, nullptr, partial, counter, dtmin);
}

void launch_gport(const Params& P, const Mesh& M, const double* q, const int* ghosts, int nport,
                  double* gport, cudaStream_t s) {
    if (nport <= 0) return;
    k_gport<<<nport, GP_THREADS, 0, s>>>(P, M, q, ghosts, nport, gport);
}

void launch_node_average(const Mesh& M, const double* prim, double* out, cudaStream_t s) {
    const size_t nnode = (size_t)(M.ni + 1) * (M.nj + 1);
    k_node_average<<<(unsigned)((nnode + 255) / 256), 256, 0, s>>>(M, prim, out);
}

void launch_boundary_sums(const Params& P, const Mesh& M, const double* prim, int type, int side,
                          int mode, double* out, cudaStream_t s) {
    k_boundary_sums<<<(M.nghosts() + 255) / 256, 256, 0, s>>>(P, M, prim, type, side, mode, out);
}

void launch_prim_out(const Params& P, const Mesh& M, const double* q, double* out,
                     cudaStream_t s) {
    const size_t ntot = (size_t)M.ni * M.nj + M.nghosts();
    k_prim_out<<<(unsigned)((ntot + 255) / 256), 256, 0, s>>>(P, M, q, out);
}

}  // namespace tns
