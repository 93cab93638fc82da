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
#include "tns_device.cuh"
#include "tns_kernels.h"

namespace tns {

constexpr int TJ = 32;  // tile extent along j (contiguous in memory)
constexpr int TI = 8;   // tile extent along i
constexpr int NTHREADS = TJ * TI;

// ------------------------------------------------------------------ stage kernel

// Halo-1 slot grid (TI+2) x (TJ+2), node grid (TI+3) x (TJ+3) (nodes of every halo cell).
constexpr int SW = TJ + 2;
constexpr int NSLOT = (TI + 2) * SW;
constexpr int NW = TJ + 3;
constexpr int NNODE = (TI + 3) * NW;
constexpr int AW = TJ + 1;  // node-average grid (TI+1) x (TJ+1)
constexpr int NAVG = (TI + 1) * AW;

enum Field {
    FU, FV, FT, FP, FRHO, FRI, FC5, FQM, FF0, FF1, FF2, FF3, FF4, FG0, FG1, FG2, FG3, FG4,
    FXC, FYC, NFIELD
};
enum AvgField { AU, AV, AT, ARHO, AR, NAVGF };

size_t stage_smem_bytes(bool with_viscous) {
    size_t b = sizeof(double) * ((size_t)NFIELD * NSLOT + 2 * NNODE);
    if (with_viscous) b += sizeof(double) * (size_t)NAVGF * NAVG;
    return b;
}

__device__ __forceinline__ void load_prim(const double* sm, int s, Prim& p) {
    p.u = sm[FU * NSLOT + s];
    p.v = sm[FV * NSLOT + s];
    p.t = sm[FT * NSLOT + s];
    p.p = sm[FP * NSLOT + s];
    p.rho = sm[FRHO * NSLOT + s];
    p.ri = sm[FRI * NSLOT + s];
    p.c5 = sm[FC5 * NSLOT + s];
    p.qm = sm[FQM * NSLOT + s];
#pragma unroll
    for (int m = 0; m < 5; m++) {
        p.f[m] = sm[(FF0 + m) * NSLOT + s];
        p.g[m] = sm[(FG0 + m) * NSLOT + s];
    }
}

__device__ __forceinline__ void store_prim(double* sm, int s, const Prim& p) {
    sm[FU * NSLOT + s] = p.u;
    sm[FV * NSLOT + s] = p.v;
    sm[FT * NSLOT + s] = p.t;
    sm[FP * NSLOT + s] = p.p;
    sm[FRHO * NSLOT + s] = p.rho;
    sm[FRI * NSLOT + s] = p.ri;
    sm[FC5 * NSLOT + s] = p.c5;
    sm[FQM * NSLOT + s] = p.qm;
#pragma unroll
    for (int m = 0; m < 5; m++) {
        sm[(FF0 + m) * NSLOT + s] = p.f[m];
        sm[(FG0 + m) * NSLOT + s] = p.g[m];
    }
}

// Loads the halo-1 tile of Q_in, fills primitives / fluxes / centroids of every cell
// and the BC state of every ghost in it.  Shared by the stage kernel and the
// primitive-output kernel.  Ends with a __syncthreads().
__device__ void fill_tile(const Params& P, const Mesh& M, const double* __restrict__ q,
                          size_t ncell, int i0, int j0, double* sm, double* snx,
                          double* sny) {
    const int tid = threadIdx.y * TJ + threadIdx.x;
    // nodes (i0-1 .. i0+TI+1) x (j0-1 .. j0+TJ+1)
    for (int s = tid; s < NNODE; s += NTHREADS) {
        const int a = i0 - 1 + s / NW, b = j0 - 1 + s % NW;
        if (a >= 0 && a <= M.ni && b >= 0 && b <= M.nj) {
            const size_t n = (size_t)a * (M.nj + 1) + b;
            snx[s] = M.x[n];
            sny[s] = M.y[n];
        }
    }
    __syncthreads();
    for (int s = tid; s < NSLOT; s += NTHREADS) {
        const int li = s / SW, lj = s % SW;
        const int i = i0 - 1 + li, j = j0 - 1 + lj;
        if (i >= 0 && i < M.ni && j >= 0 && j < M.nj) {
            const size_t c = (size_t)i * M.nj + j;
            Prim p;
            primitive(P, q[c], q[ncell + c], q[2 * ncell + c], q[3 * ncell + c],
                      q[4 * ncell + c], p);
            store_prim(sm, s, p);
            const int n1 = li * NW + lj;  // node (i, j) in the node grid
            sm[FXC * NSLOT + s] = (snx[n1] + snx[n1 + NW] + snx[n1 + NW + 1] + snx[n1 + 1]) * 0.25;
            sm[FYC * NSLOT + s] = (sny[n1] + sny[n1 + NW] + sny[n1 + NW + 1] + sny[n1 + 1]) * 0.25;
        }
    }
    __syncthreads();
    for (int s = tid; s < NSLOT; s += NTHREADS) {
        const int li = s / SW, lj = s % SW;
        const int i = i0 - 1 + li, j = j0 - 1 + lj;
        const bool in_i = i >= 0 && i < M.ni, in_j = j >= 0 && j < M.nj;
        int side = 0, along = 0, sp = 0, so = 0;
        if (in_i && j == -1) { side = 1; along = i; sp = s + 1; so = s + 2; }
        else if (in_j && i == M.ni) { side = 2; along = j; sp = s - SW; so = s - 2 * SW; }
        else if (in_i && j == M.nj) { side = 3; along = i; sp = s - 1; so = s - 2; }
        else if (in_j && i == -1) { side = 4; along = j; sp = s + SW; so = s + 2 * SW; }
        if (!side) continue;
        const int g = M.ghost_index(side, along);
        Prim par, opp, gh;
        load_prim(sm, sp, par);
        load_prim(sm, so, opp);
        const int type = M.gtype[g];
        double psx = 0.0, psy = 0.0;
        if (type == 6) {
            const int pli = sp / SW, plj = sp % SW;
            const int n1 = pli * NW + plj;
            const double X[4] = {snx[n1], snx[n1 + NW], snx[n1 + NW + 1], snx[n1 + 1]};
            const double Y[4] = {sny[n1], sny[n1 + NW], sny[n1 + NW + 1], sny[n1 + 1]};
            face_vector(P.iaxis, side, X, Y, psx, psy);
        }
        boundary_ghost(P, type, par, opp, psx, psy, M.gyc[g], sm[FYC * NSLOT + sp],
                       type == 6 ? M.gport[g] : 0.0, M.ginj[g], gh);
        store_prim(sm, s, gh);
        sm[FXC * NSLOT + s] = M.gxc[g];
        sm[FYC * NSLOT + s] = M.gyc[g];
    }
    __syncthreads();
}

struct StageArgs {
    const double* qin;   // stage input state [5][ncell]
    const double* qold;  // state at the start of the iteration [5][ncell]
    double* qout;        // stage output [5][ncell] (may alias qold: own-cell reads only)
    const double* d;     // dissipation [5][ncell]
    double* vis;         // viscous flux [4][ncell] (written in stage 1, read otherwise)
    const double* dt;    // per-cell DT (LOCAL=1)
    const double* dtmin; // DTMIN (LOCAL=0)
    double alpha;
    unsigned long long* cdiff;  // 5 slots, ordered bits of max|Q_old-Q_new| (or null)
    unsigned int* status;       // bit 0: non-finite state
};

template <bool VISC>
__global__ void __launch_bounds__(NTHREADS)
k_stage(Params P, Mesh M, StageArgs A) {
    extern __shared__ double smem[];
    double* sm = smem;
    double* snx = sm + NFIELD * NSLOT;
    double* sny = snx + NNODE;
    double* avg = sny + NNODE;
    const size_t ncell = (size_t)M.ni * M.nj;
    const int j0 = blockIdx.x * TJ, i0 = blockIdx.y * TI;
    fill_tile(P, M, A.qin, ncell, i0, j0, sm, snx, sny);

    const int tj = threadIdx.x, ti = threadIdx.y;
    const int i = i0 + ti, j = j0 + tj;

    if (VISC) {
        // nodal averages (viscous.f90:40-59,77-124) of nodes (i0..i0+TI, j0..j0+TJ)
        const int tid = ti * TJ + tj;
        for (int s = tid; s < NAVG; s += NTHREADS) {
            const int la = s / AW, lb = s % AW;
            const int a = i0 + la, b = j0 + lb;
            if (a > M.ni || b > M.nj) continue;
            double un = 0.0, vn = 0.0, tn = 0.0, rhon = 0.0, rn = 0.0;
            int cnt = 0, ng = 0, gs[2], gr[2];
            // surrounding positions in ascending cell-id order
            const int ps[4] = {la * SW + lb, la * SW + lb + 1, (la + 1) * SW + lb,
                               (la + 1) * SW + lb + 1};
            const int pi[4] = {a - 1, a - 1, a, a}, pj[4] = {b - 1, b, b - 1, b};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const bool in_i = pi[k] >= 0 && pi[k] < M.ni, in_j = pj[k] >= 0 && pj[k] < M.nj;
                const int sl = ps[k];
                if (in_i && in_j) {
                    un = un + sm[FU * NSLOT + sl];
                    vn = vn + sm[FV * NSLOT + sl];
                    tn = tn + sm[FT * NSLOT + sl];
                    rhon = rhon + sm[FRHO * NSLOT + sl];
                    rn = rn + sm[FRI * NSLOT + sl];
                    cnt++;
                } else if (in_i || in_j) {
                    int side, along;
                    if (in_i) { side = pj[k] < 0 ? 1 : 3; along = pi[k]; }
                    else { side = pi[k] < 0 ? 4 : 2; along = pj[k]; }
                    const int g = M.ghost_index(side, along);
                    gs[ng] = sl;
                    gr[ng] = g;
                    ng++;
                }
            }
            if (ng == 2 && M.grank[gr[1]] < M.grank[gr[0]]) {
                int t = gs[0]; gs[0] = gs[1]; gs[1] = t;
                t = gr[0]; gr[0] = gr[1]; gr[1] = t;
            }
            for (int k = 0; k < ng; k++) {
                const int sl = gs[k];
                un = un + sm[FU * NSLOT + sl];
                vn = vn + sm[FV * NSLOT + sl];
                tn = tn + sm[FT * NSLOT + sl];
                rhon = rhon + sm[FRHO * NSLOT + sl];
                rn = rn + sm[FRI * NSLOT + sl];
                const int type = M.gtype[gr[k]];
                if (type == 4) {
                    vn = 0.0;
                } else if (type == 5) {
                    un = 0.0;
                    vn = 0.0;
                    rn = P.rtol_rtred;
                }
                cnt++;
            }
            const double df = (double)cnt;
            avg[AU * NAVG + s] = un / df;
            avg[AV * NAVG + s] = vn / df;
            avg[AT * NAVG + s] = tn / df;
            avg[ARHO * NAVG + s] = rhon / df;
            avg[AR * NAVG + s] = dmax1(P.rtol, rn / df);
        }
        __syncthreads();
    }

    const bool valid = i < M.ni && j < M.nj;
    double dv[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (valid) {
    const size_t cell = (size_t)i * M.nj + j;
    const int c = (ti + 1) * SW + (tj + 1);
    const int nb[4] = {c - 1, c + SW, c + 1, c - SW};  // NC1..NC4
    const int n1 = (ti + 1) * NW + (tj + 1);
    const double X[4] = {snx[n1], snx[n1 + NW], snx[n1 + NW + 1], snx[n1 + 1]};
    const double Y[4] = {sny[n1], sny[n1 + NW], sny[n1 + NW + 1], sny[n1 + 1]};
    double SX[4], SY[4];
#pragma unroll
    for (int k = 0; k < 4; k++) face_vector(P.iaxis, k + 1, X, Y, SX[k], SY[k]);
    const double ycc = sm[FYC * NSLOT + c];
    const double VOL = cell_volume(P.iaxis, X, Y, ycc);

    double vis[4];
    if (VISC) {
        const int a1 = ti * AW + tj;  // node (i, j) in the average grid
        const int an[4] = {a1, a1 + AW, a1 + AW + 1, a1 + 1};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int nc = nb[k], B = an[k], D = an[(k + 1) & 3];
            FaceIn f;
            f.sx = SX[k]; f.sy = SY[k];
            f.xa = sm[FXC * NSLOT + c]; f.ya = ycc;
            f.xb = X[k]; f.yb = Y[k];
            f.xc = sm[FXC * NSLOT + nc]; f.yc = sm[FYC * NSLOT + nc];
            f.xd = X[(k + 1) & 3]; f.yd = Y[(k + 1) & 3];
            f.ua = sm[FU * NSLOT + c]; f.va = sm[FV * NSLOT + c]; f.ta = sm[FT * NSLOT + c];
            f.ub = avg[AU * NAVG + B]; f.vb = avg[AV * NAVG + B]; f.tb = avg[AT * NAVG + B];
            f.uc = sm[FU * NSLOT + nc]; f.vc = sm[FV * NSLOT + nc]; f.tc = sm[FT * NSLOT + nc];
            f.ud = avg[AU * NAVG + D]; f.vd = avg[AV * NAVG + D]; f.td = avg[AT * NAVG + D];
            f.rhoa = sm[FRHO * NSLOT + c]; f.rhob = avg[ARHO * NAVG + B];
            f.rhoc = sm[FRHO * NSLOT + nc]; f.rhod = avg[ARHO * NAVG + D];
            f.ra = sm[FRI * NSLOT + c]; f.rb = avg[AR * NAVG + B];
            f.rc = sm[FRI * NSLOT + nc]; f.rd = avg[AR * NAVG + D];
            viscous_face(P, f, k == 0, vis);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) A.vis[k * ncell + cell] = vis[k];
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) vis[k] = A.vis[k * ncell + cell];
    }

    // inviscid residual (residual.f90:23-62)
    double R[5];
#pragma unroll
    for (int m = 0; m < 5; m++) {
        const double* F = sm + (FF0 + m) * NSLOT;
        const double* G = sm + (FG0 + m) * NSLOT;
        const double FI = F[c], GI = G[c];
        R[m] = HALF * ((FI + F[nb[0]]) * SX[0] + (GI + G[nb[0]]) * SY[0] +
                       (FI + F[nb[1]]) * SX[1] + (GI + G[nb[1]]) * SY[1] +
                       (FI + F[nb[2]]) * SX[2] + (GI + G[nb[2]]) * SY[2] +
                       (FI + F[nb[3]]) * SX[3] + (GI + G[nb[3]]) * SY[3]);
    }

    // source terms (source_terms.f90:258-320)
    {
        SrcIn s;
        const int a = nb[0], b = nb[1], cc = nb[2], d = nb[3];
        s.xa = sm[FXC * NSLOT + a]; s.xb = sm[FXC * NSLOT + b];
        s.xc = sm[FXC * NSLOT + cc]; s.xd = sm[FXC * NSLOT + d];
        s.ya = sm[FYC * NSLOT + a]; s.yb = sm[FYC * NSLOT + b];
        s.yc = sm[FYC * NSLOT + cc]; s.yd = sm[FYC * NSLOT + d];
        s.ua = sm[FU * NSLOT + a]; s.ub = sm[FU * NSLOT + b];
        s.uc = sm[FU * NSLOT + cc]; s.ud = sm[FU * NSLOT + d];
        s.va = sm[FV * NSLOT + a]; s.vb = sm[FV * NSLOT + b];
        s.vc = sm[FV * NSLOT + cc]; s.vd = sm[FV * NSLOT + d];
        s.ra = sm[FRI * NSLOT + a]; s.rb = sm[FRI * NSLOT + b];
        s.rc = sm[FRI * NSLOT + cc]; s.rd = sm[FRI * NSLOT + d];
        s.qa = sm[FQM * NSLOT + a]; s.qb = sm[FQM * NSLOT + b];
        s.qc = sm[FQM * NSLOT + cc]; s.qd = sm[FQM * NSLOT + d];
        double src3, src5;
        source_terms(P, s, sm[FRHO * NSLOT + c], sm[FRI * NSLOT + c], sm[FT * NSLOT + c],
                     sm[FP * NSLOT + c], sm[FV * NSLOT + c], ycc, src3, src5);
        R[4] = R[4] - VOL * src5;
        if (P.iaxis == 1) R[2] = R[2] - VOL * src3;
    }

    // update (residual.f90:67-83)
    const double DT = P.local ? A.dt[cell] : *A.dtmin;
    const double DTBYVOL = DT / VOL;
    const double al = A.alpha;
    double Cn[5], Co[5];
#pragma unroll
    for (int m = 0; m < 5; m++) Co[m] = A.qold[m * ncell + cell];
    Cn[0] = Co[0] - al * DTBYVOL * (R[0] - A.d[cell]);
    Cn[1] = Co[1] - al * DTBYVOL * (R[1] - vis[0] - A.d[ncell + cell]);
    Cn[2] = Co[2] - al * DTBYVOL * (R[2] - vis[1] - A.d[2 * ncell + cell]);
    Cn[3] = Co[3] - al * DTBYVOL * (R[3] - vis[2] - A.d[3 * ncell + cell]);
    Cn[4] = Co[4] - al * DTBYVOL * CFLTURB * (R[4] - vis[3] - A.d[4 * ncell + cell]);
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
    }  // valid
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

// --------------------------------------------------------- dissipation kernel

constexpr int DW = TJ + 4;             // halo-2 slot grid (TI+4) x (TJ+4)
constexpr int NDSLOT = (TI + 4) * DW;
constexpr int RW = TJ + 2;             // ring-1 grid (TI+2) x (TJ+2)
constexpr int NRSLOT = (TI + 2) * RW;
enum DField { DC0, DC1, DC2, DC3, DC4, DP, NDF };
enum RField { RVBD, RANU, RANURT, RQ0, RQ1, RQ2, RQ3, RQ4, NRF };

size_t diss_smem_bytes() {
    return sizeof(double) * ((size_t)NDF * NDSLOT + (size_t)NRF * NRSLOT + 2 * NNODE);
}

struct DissArgs {
    const double* q;     // Q_old [5][ncell]
    double* d;           // out: D [5][ncell]
    double* dt;          // out: DT per cell (LOCAL=1)
    const double* dtmin; // DTMIN (LOCAL=0)
};

__device__ __forceinline__ double local_dt(const Params& P, double c1, double c2, double c3,
                                           double c4, double cfldl) {
    // turbnstwod.f90:97-108
    const double RHO = c1;
    const double U = c2 / RHO, V = c3 / RHO;
    const double VEL = sqrt(U * U + V * V);
    const double E = c4 / RHO;
    const double T = (E - 0.5 * (U * U + V * V)) / P.cv;
    return cfldl / (fabs(VEL) + sqrt(P.gamrr * T));
}

__global__ void __launch_bounds__(NTHREADS) k_dissipation(Params P, Mesh M, DissArgs A) {
    extern __shared__ double smem[];
    double* sd = smem;                  // NDF x NDSLOT
    double* sr = sd + NDF * NDSLOT;     // NRF x NRSLOT
    double* snx = sr + NRF * NRSLOT;
    double* sny = snx + NNODE;
    const size_t ncell = (size_t)M.ni * M.nj;
    const int j0 = blockIdx.x * TJ, i0 = blockIdx.y * TI;
    const int tid = threadIdx.y * TJ + threadIdx.x;

    for (int s = tid; s < NNODE; s += NTHREADS) {
        const int a = i0 - 1 + s / NW, b = j0 - 1 + s % NW;
        if (a >= 0 && a <= M.ni && b >= 0 && b <= M.nj) {
            const size_t n = (size_t)a * (M.nj + 1) + b;
            snx[s] = M.x[n];
            sny[s] = M.y[n];
        }
    }
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
            const double U = C[1] / RHO, V = C[2] / RHO;
            const double E = C[3] / RHO;
            const double T = (E - 0.5 * (U * U + V * V)) / P.cv;
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
            if (ri >= 1 && ri <= TI && rj >= 1 && rj <= TJ) A.dt[c] = DT;
        } else {
            DT = *A.dtmin;
        }
        const int n1 = ri * NW + rj;
        const double X[4] = {snx[n1], snx[n1 + NW], snx[n1 + NW + 1], snx[n1 + 1]};
        const double Y[4] = {sny[n1], sny[n1 + NW], sny[n1 + NW + 1], sny[n1 + 1]};
        const double ycc = (Y[0] + Y[1] + Y[2] + Y[3]) * 0.25;
        sr[RVBD * NRSLOT + s] = cell_volume(P.iaxis, X, Y, ycc) / DT;
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
        A.d[m * ncell + cell] = D2 - D4;
    }
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

// ------------------------------------------------------------ port mass flux

// One warp per type-6 ghost: sum of C1*U*DELY(*YCC) along the mesh line through the
// parent, across to the opposite boundary (the repaired GPORT walk).
__global__ void k_gport(Params P, Mesh M, const double* __restrict__ q, const int* ghosts,
                        int nport, double* gport) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= nport) return;
    const size_t ncell = (size_t)M.ni * M.nj;
    const int g = ghosts[w];
    int side, along;
    if (g < M.ni) { side = 1; along = g; }
    else if (g < M.ni + M.nj) { side = 2; along = g - M.ni; }
    else if (g < 2 * M.ni + M.nj) { side = 3; along = g - M.ni - M.nj; }
    else { side = 4; along = g - 2 * M.ni - M.nj; }
    const int len = (side == 1 || side == 3) ? M.nj : M.ni;
    double sum = 0.0;
    for (int k = lane; k < len; k += 32) {
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
    if (lane == 0) gport[g] = sum;
}

// ------------------------------------------------------ primitive output

// U, V, T, P of every cell and ghost computed from q (the last stage's input), the
// arrays COMPUTE_PRIMITIVE_VARS / APPLY_BOUNDARY leave behind.  Output layout:
// [4][ncell + nghost] with ghosts in side-array order.
__global__ void __launch_bounds__(NTHREADS)
k_prim_out(Params P, Mesh M, const double* __restrict__ q, double* out) {
    extern __shared__ double smem[];
    double* sm = smem;
    double* snx = sm + NFIELD * NSLOT;
    double* sny = snx + NNODE;
    const size_t ncell = (size_t)M.ni * M.nj;
    const size_t ntot = ncell + M.nghosts();
    const int j0 = blockIdx.x * TJ, i0 = blockIdx.y * TI;
    fill_tile(P, M, q, ncell, i0, j0, sm, snx, sny);
    const int tid = threadIdx.y * TJ + threadIdx.x;
    for (int s = tid; s < NSLOT; s += NTHREADS) {
        const int li = s / SW, lj = s % SW;
        const int i = i0 - 1 + li, j = j0 - 1 + lj;
        const bool in_i = i >= 0 && i < M.ni, in_j = j >= 0 && j < M.nj;
        size_t o;
        if (in_i && in_j) {
            if (li < 1 || li > TI || lj < 1 || lj > TJ) continue;  // owned by another tile
            o = (size_t)i * M.nj + j;
        } else if (in_i && j == -1) o = ncell + M.ghost_index(1, i);
        else if (in_j && i == M.ni) o = ncell + M.ghost_index(2, j);
        else if (in_i && j == M.nj) o = ncell + M.ghost_index(3, i);
        else if (in_j && i == -1) o = ncell + M.ghost_index(4, j);
        else continue;
        out[o] = sm[FU * NSLOT + s];
        out[ntot + o] = sm[FV * NSLOT + s];
        out[2 * ntot + o] = sm[FT * NSLOT + s];
        out[3 * ntot + o] = sm[FP * NSLOT + s];
    }
}

// ------------------------------------------------------------------ launchers

static dim3 tile_grid(const Mesh& M) { return dim3((M.nj + TJ - 1) / TJ, (M.ni + TI - 1) / TI); }

cudaError_t configure_kernels() {
    cudaError_t e;
    e = cudaFuncSetAttribute(k_stage<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)stage_smem_bytes(true));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_stage<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)stage_smem_bytes(false));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_prim_out, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)stage_smem_bytes(false));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_dissipation, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)diss_smem_bytes());
}

void launch_dissipation(const Params& P, const Mesh& M, const double* q, double* d, double* dt,
                        const double* dtmin, cudaStream_t s) {
    DissArgs A{q, d, dt, dtmin};
    k_dissipation<<<tile_grid(M), dim3(TJ, TI), diss_smem_bytes(), s>>>(P, M, A);
}

void launch_stage(const Params& P, const Mesh& M, bool viscous, const double* qin,
                  const double* qold, double* qout, const double* d, double* vis,
                  const double* dt, const double* dtmin, double alpha,
                  unsigned long long* cdiff, unsigned int* status, cudaStream_t s) {
    StageArgs A{qin, qold, qout, d, vis, dt, dtmin, alpha, cdiff, status};
    if (viscous)
        k_stage<true><<<tile_grid(M), dim3(TJ, TI), stage_smem_bytes(true), s>>>(P, M, A);
    else
        k_stage<false><<<tile_grid(M), dim3(TJ, TI), stage_smem_bytes(false), s>>>(P, M, A);
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
    const int threads = 256, warps_per_block = threads / 32;
    k_gport<<<(nport + warps_per_block - 1) / warps_per_block, threads, 0, s>>>(P, M, q, ghosts,
                                                                               nport, gport);
}

void launch_prim_out(const Params& P, const Mesh& M, const double* q, double* out,
                     cudaStream_t s) {
    k_prim_out<<<tile_grid(M), dim3(TJ, TI), stage_smem_bytes(false), s>>>(P, M, q, out);
}

}  // namespace tns
