// tns_unstructured.cu -- the FP64 RK4 iteration on a general quadrilateral mesh (any
// NOD / NC1..NC4 connectivity), by gather through index arrays.
//
// Per iteration (turbnstwod.f90:95-168), every kernel one thread per cell, slot or node:
//   [dtmin]            global time step (LOCAL=0)
//   k_u_diss1/2        DT, sensors and Laplacians, then the JST blend (solver_state.f90:70-225)
//   [k_u_gport]        type-6 port mass flux of the stage input (boundary.f90:168-223)
//   k_u_prim           primitives and fluxes of every cell and ghost (turbnstwod.f90:204-227,
//                      boundary.f90:24-327) into a slot field set W
//   k_u_node_avg       NODAL_AVERAGE with the bc.in-order resets (viscous.f90:40-124), stage 1
//   k_u_vface/vsum     every face once, then the four faces of every cell in order
//                      (viscous.f90:62-70,130-217), stage 1
//   k_u_stage_chunk    per chunk of 256 cells: primitives and fluxes of its cells and halo
//                      into shared memory, then source, residual and update
//                      (source_terms.f90:24-104, residual.f90:23-83), each RK stage
// The host side lays the mesh out: cells in Hilbert-curve order of their centroids
// (neighbours near in memory, compact chunks), ghosts after them in bc.in order, the
// static geometry computed once with the reference's formulas (geometry.f90:55-149).
#include <algorithm>
#include <cmath>
#include <numeric>
#include <unordered_map>
#include <vector>

#include "tns_handle.h"
#include "tns_umesh.h"
#include "tns_tile.cuh"

namespace tns {


// The state of a general mesh is read through an accessor (tns_tile.cuh): StateF64 (an
// FP64 array [5][ne]) or StateMixed (FP64 COLD plus an FP32 stage increment).
template <class St>
__device__ __forceinline__ void u_cell_prim(const Params& P, const St& st, int c, Prim& p) {
    primitive(P, st.c(0, c), st.c(1, c), st.c(2, c), st.c(3, c), st.c(4, c), p);
}

// Primitives and fluxes of slot s: a cell from the state, a ghost by its BC from the
// parent and (type 3) the parent's opposite neighbour.
template <class St>
__device__ __forceinline__ void u_slot_prim(const Params& P, const UMesh& M, const St& st, int s, Prim& p) {
    if (s < M.ne) {
        u_cell_prim(P, st, s, p);
    } else {
        const int L = s - M.ne;
        const int par = M.gpar[L], type = M.gtype[L];
        Prim pa, op;
        u_cell_prim(P, st, par, pa);
        if (type == 3) u_cell_prim(P, st, M.gopp[L], op);
        else op = pa;
        boundary_ghost(P, type, pa, op, M.gsx[L], M.gsy[L], M.gyc[L], M.cg[UCG_YCC * M.ne + par],
                       type == 6 ? M.gport[L] : 0.0, M.ginj[L], p);
    }
}

// Primitive / flux field set of every slot.
template <class St>
__global__ void __launch_bounds__(UT) k_u_prim(Params P, UMesh M, St st, double* __restrict__ W) {
    const int s = blockIdx.x * UT + threadIdx.x;
    const int ns = M.ne + M.ng;
    if (s >= ns) return;
    Prim p;
    u_slot_prim(P, M, st, s, p);
    const size_t n = (size_t)ns;
#pragma unroll
    for (int m = 0; m < 5; m++) {
        W[(UW_F1 + m) * n + s] = p.f[m];
        W[(UW_G1 + m) * n + s] = p.g[m];
    }
    W[UW_U * n + s] = p.u;
    W[UW_V * n + s] = p.v;
    W[UW_T * n + s] = p.t;
    W[UW_P * n + s] = p.p;
    W[UW_RHO * n + s] = p.rho;
    W[UW_RI * n + s] = p.ri;
    W[UW_QM * n + s] = p.qm;
}

// Port mass flux of each type-6 ghost: the sum of C1*U*DELY (*YCC) along its port line
// in the line's order (the walk of the oracle's repaired COMPUTE_GPORT).
template <class St>
__global__ void __launch_bounds__(UT) k_u_gport(Params P, UMesh M, St st) {
    const int k = blockIdx.x * UT + threadIdx.x;
    if (k >= M.nport) return;
    double sum = 0.0;
    for (int e = M.pptr[k]; e < M.pptr[k + 1]; e++) {
        const int c = M.pcell[e];
        const double c1 = st.c(0, c), u = st.c(1, c) / c1;
        double term = c1 * u * M.pdely[e];
        if (P.iaxis == 1) term = term * M.cg[UCG_YCC * M.ne + c];
        sum = (e == M.pptr[k]) ? term : sum + term;
    }
    M.gport[M.pghost[k]] = sum;
}

__device__ __forceinline__ double u_pressure(const Params& P, const double* __restrict__ q, int ne, int c) {
    const double RHO = q[c];
    const double rr = 1.0 / RHO;
    const double U = q[ne + c] * rr, V = q[2 * ne + c] * rr;
    const double E = q[3 * ne + c] * rr;
    const double T = (E - 0.5 * (U * U + V * V)) * P.inv_cv;
    return RHO * P.rr * T;
}

enum UAux { UA_ANU, UA_ANURT, UA_VBD, UA_D2Q, UA_N = UA_D2Q + 5 };

// DISSIPATION, first pass (solver_state.f90:78-160): DT (turbnstwod.f90:97-108), VOL/DT,
// the pressure and turbulence sensors and the Laplacians; a ghost neighbour holds a
// copy of its parent (this cell).
template <class OutT>
__global__ void __launch_bounds__(UT) k_u_diss1(Params P, UMesh M, const double* __restrict__ q,
                                                double* __restrict__ aux, OutT* __restrict__ dt,
                                                const double* __restrict__ dtmin) {
    const int I = blockIdx.x * UT + threadIdx.x;
    const int ne = M.ne;
    if (I >= ne) return;
    int nb[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int n = M.nc[k * ne + I];
        nb[k] = n < ne ? n : I;
    }
    const double PIE = u_pressure(P, q, ne, I);
    double Pn[4];
#pragma unroll
    for (int k = 0; k < 4; k++) Pn[k] = nb[k] == I ? PIE : u_pressure(P, q, ne, nb[k]);
    const double* C5 = q + 4 * ne;
    const double C1I = q[I], C5I = C5[I];
    double ANUN = fabs(Pn[0] - PIE) + fabs(Pn[1] - PIE) + fabs(Pn[2] - PIE) + fabs(Pn[3] - PIE);
    double ANUD = fabs(Pn[0] + PIE) + fabs(Pn[1] + PIE) + fabs(Pn[2] + PIE) + fabs(Pn[3] + PIE);
    aux[UA_ANU * ne + I] = ANUN / ANUD;
    ANUN = fabs(C5[nb[0]] - C5I) + fabs(C5[nb[1]] - C5I) + fabs(C5[nb[2]] - C5I) + fabs(C5[nb[3]] - C5I);
    ANUD = fabs(C5[nb[0]] + C5I) + fabs(C5[nb[1]] + C5I) + fabs(C5[nb[2]] + C5I) + fabs(C5[nb[3]] + C5I);
    aux[UA_ANURT * ne + I] = ANUN / dmax1(ANUD, 8.0 * C1I * P.rtol);
#pragma unroll
    for (int m = 0; m < 5; m++) {
        const double* Cm = q + m * ne;
        aux[(UA_D2Q + m) * ne + I] = Cm[nb[0]] + Cm[nb[1]] + Cm[nb[2]] + Cm[nb[3]] - 4.0 * Cm[I];
    }
    double DT;
    if (P.local) {
        const double RHO = q[I];
        const double rr = 1.0 / RHO;
        const double U = q[ne + I] * rr, V = q[2 * ne + I] * rr;
        const double VEL = sqrt(U * U + V * V);
        const double E = q[3 * ne + I] * rr;
        const double T = (E - 0.5 * (U * U + V * V)) * P.inv_cv;
        DT = M.cfldl[I] / (fabs(VEL) + sqrt(P.gamrr * T));
        dt[I] = (OutT)DT;
    } else {
        DT = *dtmin;
    }
    aux[UA_VBD * ne + I] = M.cg[UCG_VOL * ne + I] / DT;
}

// DISSIPATION, the blend (solver_state.f90:162-225).  A ghost face contributes exactly
// zero (its state and Laplacian are the cell's own), so it is skipped.
template <class OutT>
__global__ void __launch_bounds__(UT) k_u_diss2(UMesh M, const double* __restrict__ q,
                                                const double* __restrict__ aux, OutT* __restrict__ d) {
    const int I = blockIdx.x * UT + threadIdx.x;
    const int ne = M.ne;
    if (I >= ne) return;
    int nb[4];
    bool has[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        nb[k] = M.nc[k * ne + I];
        has[k] = nb[k] < ne;
        if (!has[k]) nb[k] = I;
    }
    const double VOLBYDT = aux[UA_VBD * ne + I];
    const double ANUI = aux[UA_ANU * ne + I], ANURTI = aux[UA_ANURT * ne + I];
    double D2c[4], D4c[4], D2t[4], D4t[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const double D24N = HALF * (VOLBYDT + aux[UA_VBD * ne + nb[k]]);
        double E2N = C02 * dmax1(ANUI, aux[UA_ANU * ne + nb[k]]);
        double E4N = dmax1(0.0, C04 - E2N);
        D2c[k] = E2N * D24N;
        D4c[k] = E4N * D24N;
        E2N = C02 * dmax1(ANURTI, aux[UA_ANURT * ne + nb[k]]);
        E4N = dmax1(0.0, C04 - E2N);
        D2t[k] = E2N * D24N;
        D4t[k] = E4N * D24N;
    }
#pragma unroll
    for (int m = 0; m < 5; m++) {
        const double* Cm = q + m * ne;
        const double* Qm = aux + (UA_D2Q + m) * ne;
        const double CI = Cm[I], D2I = Qm[I];
        double D2 = 0.0, D4 = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!has[k]) continue;
            const double a2 = (m == 4) ? D2t[k] : D2c[k];
            const double a4 = (m == 4) ? D4t[k] : D4c[k];
            D2 = D2 + a2 * (Cm[nb[k]] - CI);
            D4 = D4 + a4 * (Qm[nb[k]] - D2I);
        }
        d[m * ne + I] = (OutT)(D2 - D4);
    }
}

// NODAL_AVERAGE_ELEMENTS / _GHOSTS / finalize (viscous.f90:40-124): each node sums its
// contributions in the reference's visit order (cells by id, then ghosts in bc.in order),
// with a type-4 ghost zeroing VN and a type-5 ghost zeroing UN, VN and setting RN after
// its contribution; out [5][nnode] = U, V, T, RHO, RI averages.
__global__ void __launch_bounds__(UT) k_u_node_avg(Params P, UMesh M, const double* __restrict__ W,
                                                   double* __restrict__ na) {
    const int n = blockIdx.x * UT + threadIdx.x;
    if (n >= M.nnode) return;
    const size_t ns = (size_t)M.ne + M.ng;
    double un = 0.0, vn = 0.0, tn = 0.0, rhon = 0.0, rn = 0.0;
    const int e0 = M.nptr[n], e1 = M.nptr[n + 1];
    // the first NB contributions' values are loaded together, then summed in order
    constexpr int NB = 4;
    double w[NB][5];
    int rs[NB];
#pragma unroll
    for (int q = 0; q < NB; q++) {
        rs[q] = 0;
        if (e0 + q < e1) {
            const int sl = M.nslot[e0 + q];
            rs[q] = M.nreset[e0 + q];
            w[q][0] = W[UW_U * ns + sl];
            w[q][1] = W[UW_V * ns + sl];
            w[q][2] = W[UW_T * ns + sl];
            w[q][3] = W[UW_RHO * ns + sl];
            w[q][4] = W[UW_RI * ns + sl];
        }
    }
    auto add = [&](const double* v, int r) {
        un = un + v[0];
        vn = vn + v[1];
        tn = tn + v[2];
        rhon = rhon + v[3];
        rn = rn + v[4];
        if (r == 4) {
            vn = 0.0;
        } else if (r == 5) {
            un = 0.0;
            vn = 0.0;
            rn = P.rtol_rtred;
        }
    };
#pragma unroll
    for (int q = 0; q < NB; q++)
        if (e0 + q < e1) add(w[q], rs[q]);
    for (int e = e0 + NB; e < e1; e++) {
        const int sl = M.nslot[e];
        const double v[5] = {W[UW_U * ns + sl], W[UW_V * ns + sl], W[UW_T * ns + sl], W[UW_RHO * ns + sl],
                             W[UW_RI * ns + sl]};
        add(v, M.nreset[e]);
    }
    // one reciprocal of the contribution count (exact for 1, 2 and 4), as the
    // structured kernel
    const int cnt = e1 - e0;
    const double idf = cnt == 4 ? 0.25 : 1.0 / (double)cnt;
    const size_t nn = (size_t)M.nnode;
    na[n] = un * idf;
    na[nn + n] = vn * idf;
    na[2 * nn + n] = tn * idf;
    na[3 * nn + n] = rhon * idf;
    na[4 * nn + n] = dmax1(P.rtol, rn * idf);
}

// COMPUTE_VISCOUS (viscous.f90:62-70, 130-217) in two passes.  k_u_vface evaluates each
// face once, in the orientation of the cell that owns it (A = that cell, C = its
// neighbour across face k, B = node k, D = node k+1); in the neighbour's orientation the
// face has the same gradient and averages and the opposite face vector, so its flux is
// the negative.  k_u_vsum then gives every cell its four faces in order, face 1
// assigning and the others adding, as the reference's loop does.
__global__ void __launch_bounds__(UT) k_u_vface(Params P, UMesh M, const double* __restrict__ W,
                                                const double* __restrict__ na, double* __restrict__ vf) {
    const int e = blockIdx.x * UT + threadIdx.x;
    if (e >= M.nface) return;
    const int ne = M.ne;
    const int I = M.fcell[e] >> 2, k = M.fcell[e] & 3;
    const size_t ns = (size_t)ne + M.ng, nn = (size_t)M.nnode;
    const int nbn = M.nod[k * ne + I], ndn = M.nod[((k + 1) & 3) * ne + I];
    const int cc = M.nc[k * ne + I];
    FaceVals f;
    f.ua = W[UW_U * ns + I]; f.va = W[UW_V * ns + I]; f.ta = W[UW_T * ns + I];
    f.uc = W[UW_U * ns + cc]; f.vc = W[UW_V * ns + cc]; f.tc = W[UW_T * ns + cc];
    f.ub = na[nbn]; f.vb = na[nn + nbn]; f.tb = na[2 * nn + nbn];
    f.ud = na[ndn]; f.vd = na[nn + ndn]; f.td = na[2 * nn + ndn];
    f.rhoa = W[UW_RHO * ns + I]; f.rhoc = W[UW_RHO * ns + cc];
    f.rhob = na[3 * nn + nbn]; f.rhod = na[3 * nn + ndn];
    f.ra = W[UW_RI * ns + I]; f.rc = W[UW_RI * ns + cc];
    f.rb = na[4 * nn + nbn]; f.rd = na[4 * nn + ndn];
    const double* G = M.fg + (size_t)k * ne + I;
    const size_t st = (size_t)4 * ne;
    double out[4];
    viscous_face(P, f, M.cg[(UCG_SX1 + k) * ne + I], M.cg[(UCG_SY1 + k) * ne + I], G[UFG_GA * st],
                 G[UFG_GB * st], G[UFG_GC * st], G[UFG_GD * st], P.iaxis == 1 ? G[UFG_RYAVG * st] : 0.0, out);
    const size_t nf = (size_t)M.nface;
#pragma unroll
    for (int m = 0; m < 4; m++) vf[m * nf + e] = out[m];
}

template <class OutT>
__global__ void __launch_bounds__(UT) k_u_vsum(UMesh M, const double* __restrict__ vf, OutT* __restrict__ vis) {
    const int I = blockIdx.x * UT + threadIdx.x;
    const int ne = M.ne;
    if (I >= ne) return;
    const size_t nf = (size_t)M.nface;
    int r[4];
#pragma unroll
    for (int k = 0; k < 4; k++) r[k] = M.fref[k * ne + I];
    double acc[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int e = r[k] >= 0 ? r[k] : ~r[k];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const double v = r[k] >= 0 ? vf[m * nf + e] : -vf[m * nf + e];
            acc[m] = k == 0 ? v : acc[m] + v;
        }
    }
#pragma unroll
    for (int m = 0; m < 4; m++) vis[m * ne + I] = (OutT)acc[m];
}

// One RK stage of one chunk of UT cells (source_terms.f90:24-104, residual.f90:23-83),
// with the primitives and fluxes of the chunk's cells and halo staged in shared memory
// instead of a field set in global memory: each thread evaluates its own cell (keeping
// its T, P, RHO) and the threads then share the halo slots.  (It gives bitwise the
// results of a slot field set in global memory gathered per cell.)  Shared memory:
// (UT + hmax) slots of (F_m, G_m) x 5, (U, V), (C5/C1, |V|).
#ifndef TNS_U_CHUNK_MINB
// Blocks per SM the register budget is sized for; measured on a renumbered 1024 x 384
// nozzle-plume (B200, one FP64 iteration): 2 -> 0.289 ms, 3 -> 0.294 ms, 4 -> 0.313 ms.
#define TNS_U_CHUNK_MINB 2
#endif
__global__ void __launch_bounds__(UT, TNS_U_CHUNK_MINB) k_u_stage_chunk(Params P, UMesh M, StageArgsU A,
                                                         const double* __restrict__ q) {
    extern __shared__ double2 usm[];
    const int ns = UT + M.hmax;
    double2* fg = usm;
    double2* uv = usm + 5 * ns;
    double2* rq = uv + ns;
    const int ne = M.ne, t = threadIdx.x;
    const int c0 = blockIdx.x * UT, I = c0 + t;
    const int h0 = M.cptr[blockIdx.x], nh = M.cptr[blockIdx.x + 1] - h0;
    auto put = [&](int s, const Prim& p) {
#pragma unroll
        for (int m = 0; m < 5; m++) fg[m * ns + s] = make_double2(p.f[m], p.g[m]);
        uv[s] = make_double2(p.u, p.v);
        rq[s] = make_double2(p.ri, p.qm);
    };
    double own_t = 0.0, own_p = 0.0, own_rho = 0.0;
    if (I < ne) {
        Prim p;
        u_cell_prim(P, StateF64{q, (size_t)ne}, I, p);
        put(t, p);
        own_t = kept(p.t);
        own_p = kept(p.p);
        own_rho = kept(p.rho);
    }
    for (int h = t; h < nh; h += UT) {
        Prim p;
        u_slot_prim(P, M, StateF64{q, (size_t)ne}, M.cslot[h0 + h], p);
        put(UT + h, p);
    }
    __syncthreads();
    double dv[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (I < ne) {
        int nb[4];
#pragma unroll
        for (int k = 0; k < 4; k++) nb[k] = M.lnb[k * ne + I];
        const double* G = M.cg + I;
        double src3, src5;
        {
            SrcIn s;
            s.ga = G[UCG_GA * ne]; s.gb = G[UCG_GB * ne]; s.gc = G[UCG_GC * ne]; s.gd = G[UCG_GD * ne];
            const double2 ua = uv[nb[0]], ub = uv[nb[1]], uc = uv[nb[2]], ud = uv[nb[3]];
            const double2 ra = rq[nb[0]], rb = rq[nb[1]], rc = rq[nb[2]], rd = rq[nb[3]];
            s.ua = ua.x; s.ub = ub.x; s.uc = uc.x; s.ud = ud.x;
            s.va = ua.y; s.vb = ub.y; s.vc = uc.y; s.vd = ud.y;
            s.ra = ra.x; s.rb = rb.x; s.rc = rc.x; s.rd = rd.x;
            s.qa = ra.y; s.qb = rb.y; s.qc = rc.y; s.qd = rd.y;
            source_terms(P, s, own_rho, rq[t].x, own_t, own_p, uv[t].y, G[UCG_YCC * ne], G[UCG_RYCC * ne], src3,
                         src5);
        }
        double R[5];
#pragma unroll
        for (int m = 0; m < 5; m++) {
            const double2* F = fg + m * ns;
            const double2 Fi = F[t], a = F[nb[0]], b = F[nb[1]], e = F[nb[2]], d = F[nb[3]];
            R[m] = HALF * ((Fi.x + a.x) * G[UCG_SX1 * ne] + (Fi.y + a.y) * G[UCG_SY1 * ne] +
                           (Fi.x + b.x) * G[UCG_SX2 * ne] + (Fi.y + b.y) * G[UCG_SY2 * ne] +
                           (Fi.x + e.x) * G[UCG_SX3 * ne] + (Fi.y + e.y) * G[UCG_SY3 * ne] +
                           (Fi.x + d.x) * G[UCG_SX4 * ne] + (Fi.y + d.y) * G[UCG_SY4 * ne]);
        }
        const double VOL = G[UCG_VOL * ne];
        R[4] = R[4] - VOL * src5;
        if (P.iaxis == 1) R[2] = R[2] - VOL * src3;
        const double DT = P.local ? A.dt[I] : *A.dtmin;
        const double DTBYVOL = DT * G[UCG_RVOL * ne];
        const double al = A.alpha;
        double Cn[5], Co[5];
#pragma unroll
        for (int m = 0; m < 5; m++) Co[m] = A.qold[m * ne + I];
        Cn[0] = Co[0] - al * DTBYVOL * (R[0] - A.d[I]);
        Cn[1] = Co[1] - al * DTBYVOL * (R[1] - A.vis[I] - A.d[ne + I]);
        Cn[2] = Co[2] - al * DTBYVOL * (R[2] - A.vis[ne + I] - A.d[2 * ne + I]);
        Cn[3] = Co[3] - al * DTBYVOL * (R[3] - A.vis[2 * ne + I] - A.d[3 * ne + I]);
        Cn[4] = Co[4] - al * DTBYVOL * CFLTURB * (R[4] - A.vis[3 * ne + I] - A.d[4 * ne + I]);
        Cn[4] = Cn[0] * dmax1(P.rtol, Cn[4] / Cn[0]);
#pragma unroll
        for (int m = 0; m < 5; m++) A.qout[m * ne + I] = Cn[m];
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
#pragma unroll
        for (int m = 0; m < 5; m++) {
            double v = dv[m];
            for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
            if ((threadIdx.x & 31) == 0) atomicMax(&A.cdiff[m], (unsigned long long)__double_as_longlong(v));
        }
    }
}

size_t u_chunk_smem_bytes(const UMesh& M) { return sizeof(double2) * 7 * ((size_t)UT + M.hmax); }

// POSTPROCESS node averages (solver_state.f90:237-281): P, U, V, T of the contributions
// in the same visit order, divided by their count; out [4][nnode].
__global__ void __launch_bounds__(UT) k_u_post_avg(UMesh M, const double* __restrict__ W,
                                                   double* __restrict__ out) {
    const int n = blockIdx.x * UT + threadIdx.x;
    if (n >= M.nnode) return;
    const size_t ns = (size_t)M.ne + M.ng, nn = (size_t)M.nnode;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    const int e0 = M.nptr[n], e1 = M.nptr[n + 1];
    for (int e = e0; e < e1; e++) {
        const int sl = M.nslot[e];
        s[0] += W[UW_P * ns + sl];
        s[1] += W[UW_U * ns + sl];
        s[2] += W[UW_V * ns + sl];
        s[3] += W[UW_T * ns + sl];
    }
    const double d = (double)(e1 - e0);
#pragma unroll
    for (int f = 0; f < 4; f++) out[f * nn + n] = s[f] / d;
}

__global__ void __launch_bounds__(UT) k_u_prim_out(UMesh M, const double* __restrict__ W,
                                                   double* __restrict__ out) {
    const int s = blockIdx.x * UT + threadIdx.x;
    const size_t ns = (size_t)M.ne + M.ng;
    if (s >= (int)ns) return;
    out[s] = W[UW_U * ns + s];
    out[ns + s] = W[UW_V * ns + s];
    out[2 * ns + s] = W[UW_T * ns + s];
    out[3 * ns + s] = W[UW_P * ns + s];
}

// Boundary-face sums over the ghosts whose BC type / side match (0 = any), with the face
// state (parent + ghost)/2, as k_boundary_sums.
// Face state (parent + ghost)/2 of every ghost (bc.in order): out [5][ng] = U, V, P, RHO, T.
__global__ void __launch_bounds__(UT) k_u_face_states(Params P, UMesh M, const double* __restrict__ W,
                                                      double* __restrict__ out) {
    const int L = blockIdx.x * UT + threadIdx.x;
    if (L >= M.ng) return;
    const size_t ns = (size_t)M.ne + M.ng, ng = (size_t)M.ng;
    const size_t cp = (size_t)M.gpar[L], cg = (size_t)M.ne + L;
    const double tp = W[UW_T * ns + cp], tgh = W[UW_T * ns + cg];
    const double pp = W[UW_P * ns + cp], pgh = W[UW_P * ns + cg];
    out[L] = 0.5 * (W[UW_U * ns + cp] + W[UW_U * ns + cg]);
    out[ng + L] = 0.5 * (W[UW_V * ns + cp] + W[UW_V * ns + cg]);
    out[2 * ng + L] = 0.5 * (pp + pgh);
    out[3 * ng + L] = 0.5 * (pp / (P.rr * tp) + pgh / (P.rr * tgh));
    out[4 * ng + L] = 0.5 * (tp + tgh);
}

__global__ void __launch_bounds__(UT) k_u_bsums(Params P, UMesh M, const double* __restrict__ W, int type,
                                                int side, int mode, double* __restrict__ out) {
    const int L = blockIdx.x * UT + threadIdx.x;
    const size_t ns = (size_t)M.ne + M.ng;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (L < M.ng && (type == 0 || M.gtype[L] == type) && (side == 0 || M.gside[L] == side)) {
        const size_t cp = (size_t)M.gpar[L], cg = (size_t)M.ne + L;
        const double sx = M.gsx[L], sy = M.gsy[L];
        const double u = 0.5 * (W[UW_U * ns + cp] + W[UW_U * ns + cg]);
        const double vv = 0.5 * (W[UW_V * ns + cp] + W[UW_V * ns + cg]);
        face_sums(P, mode, u, vv, W[UW_T * ns + cp], W[UW_T * ns + cg], W[UW_P * ns + cp], W[UW_P * ns + cg], sx,
                  sy, v);
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0 && x != 0.0) atomicAdd(&out[q], x);
    }
}

static unsigned blocks(long long n) { return (unsigned)((n + UT - 1) / UT); }

void launch_u_prim(const Params& P, const UMesh& M, const double* q, double* W, cudaStream_t s) {
    k_u_prim<<<blocks((long long)M.ne + M.ng), UT, 0, s>>>(P, M, StateF64{q, (size_t)M.ne}, W);
}
void launch_u_prim_mx(const Params& P, const UMesh& M, const double* cold, const float* dq, double* W,
                      cudaStream_t s) {
    k_u_prim<<<blocks((long long)M.ne + M.ng), UT, 0, s>>>(P, M, StateMixed{cold, dq, (size_t)M.ne}, W);
}
void launch_u_gport(const Params& P, const UMesh& M, const double* q, cudaStream_t s) {
    if (M.nport > 0) k_u_gport<<<blocks(M.nport), UT, 0, s>>>(P, M, StateF64{q, (size_t)M.ne});
}
void launch_u_gport_mx(const Params& P, const UMesh& M, const double* cold, const float* dq, cudaStream_t s) {
    if (M.nport > 0) k_u_gport<<<blocks(M.nport), UT, 0, s>>>(P, M, StateMixed{cold, dq, (size_t)M.ne});
}
void launch_u_dissipation(const Params& P, const UMesh& M, const double* q, double* aux, double* d,
                          double* dt, const double* dtmin, cudaStream_t s) {
    k_u_diss1<<<blocks(M.ne), UT, 0, s>>>(P, M, q, aux, dt, dtmin);
    k_u_diss2<<<blocks(M.ne), UT, 0, s>>>(M, q, aux, d);
}
void launch_u_dissipation(const Params& P, const UMesh& M, const double* q, double* aux, float* d, float* dt,
                          const double* dtmin, cudaStream_t s) {
    k_u_diss1<<<blocks(M.ne), UT, 0, s>>>(P, M, q, aux, dt, dtmin);
    k_u_diss2<<<blocks(M.ne), UT, 0, s>>>(M, q, aux, d);
}
void launch_u_viscous(const Params& P, const UMesh& M, const double* W, double* na, double* vf, double* vis,
                      cudaStream_t s) {
    k_u_node_avg<<<blocks(M.nnode), UT, 0, s>>>(P, M, W, na);
    k_u_vface<<<blocks(M.nface), UT, 0, s>>>(P, M, W, na, vf);
    k_u_vsum<<<blocks(M.ne), UT, 0, s>>>(M, vf, vis);
}
void launch_u_viscous(const Params& P, const UMesh& M, const double* W, double* na, double* vf, float* vis,
                      cudaStream_t s) {
    k_u_node_avg<<<blocks(M.nnode), UT, 0, s>>>(P, M, W, na);
    k_u_vface<<<blocks(M.nface), UT, 0, s>>>(P, M, W, na, vf);
    k_u_vsum<<<blocks(M.ne), UT, 0, s>>>(M, vf, vis);
}
void launch_u_stage_chunk(const Params& P, const UMesh& M, const StageArgsU& A, const double* q, cudaStream_t s) {
    k_u_stage_chunk<<<M.nchunk, UT, u_chunk_smem_bytes(M), s>>>(P, M, A, q);
}
cudaError_t configure_u_chunk(const UMesh& M) {
    return cudaFuncSetAttribute(k_u_stage_chunk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)u_chunk_smem_bytes(M));
}
void launch_u_post_average(const UMesh& M, const double* W, double* out, cudaStream_t s) {
    k_u_post_avg<<<blocks(M.nnode), UT, 0, s>>>(M, W, out);
}
void launch_u_prim_out(const UMesh& M, const double* W, double* out, cudaStream_t s) {
    k_u_prim_out<<<blocks((long long)M.ne + M.ng), UT, 0, s>>>(M, W, out);
}
void launch_u_boundary_sums(const Params& P, const UMesh& M, const double* W, int type, int side,
                            int mode, double* out, cudaStream_t s) {
    if (M.ng > 0) k_u_bsums<<<blocks(M.ng), UT, 0, s>>>(P, M, W, type, side, mode, out);
}
void launch_u_face_states(const Params& P, const UMesh& M, const double* W, double* out, cudaStream_t s) {
    if (M.ng > 0) k_u_face_states<<<blocks(M.ng), UT, 0, s>>>(P, M, W, out);
}

}  // namespace tns

// ------------------------------------------------------------------ host runtime

struct tns_umesh_state {
    tns::UMesh M{};
    DevBuf<int> nc, nod, gpar, gopp, gtype, gside, nptr, nslot, nreset, pghost, pptr, pcell, fcell, fref, cptr,
        cslot, lnb;
    DevBuf<double> cg, fg, cfldl, gsx, gsy, gyc, ginj, gport, pdely, W, aux, na, vf;
    // host layout, uploaded by umesh_upload
    std::vector<int> hnc, hnod, hgpar, hgopp, hgtype, hgside, hnptr, hnslot, hnreset, hpghost, hpptr, hpcell,
        hfcell, hfref, hcptr, hcslot, hlnb;
    int hmax = 0;
    std::vector<double> hcg, hfg, hcfldl, hgsx, hgsy, hgyc, hginj, hpdely;
};

namespace tns_rt {

namespace {

// Position along the Hilbert curve of order 20 (2^20 x 2^20 cells) of the point (x, y),
// 0 <= x, y < 2^20: the classical quadrant recursion, with each sub-square rotated or
// reflected so that the curve stays continuous.
unsigned long long hilbert_index(unsigned x, unsigned y) {
    constexpr unsigned N = 1u << 20;
    unsigned long long d = 0;
    for (unsigned s = N / 2; s > 0; s /= 2) {
        const unsigned rx = (x & s) ? 1u : 0u, ry = (y & s) ? 1u : 0u;
        d += (unsigned long long)s * s * ((3u * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) {
                x = N - 1 - x;
                y = N - 1 - y;
            }
            const unsigned t = x;
            x = y;
            y = t;
        }
    }
    return d;
}

// Cells in the order of their centroids along a Hilbert curve over the mesh's bounding
// box (ties by id): consecutive cells form compact patches, so a run of 256 of them has
// a short halo, and neighbours sit nearby in memory.  Returns new index -> cell.
std::vector<int> hilbert_order(const std::vector<double>& xc, const std::vector<double>& yc) {
    const int ne = (int)xc.size();
    double x0 = xc[0], x1 = xc[0], y0 = yc[0], y1 = yc[0];
    for (int c = 1; c < ne; c++) {
        x0 = std::min(x0, xc[c]); x1 = std::max(x1, xc[c]);
        y0 = std::min(y0, yc[c]); y1 = std::max(y1, yc[c]);
    }
    const double sx = x1 > x0 ? 1048575.0 / (x1 - x0) : 0.0, sy = y1 > y0 ? 1048575.0 / (y1 - y0) : 0.0;
    std::vector<unsigned long long> key(ne);
    for (int c = 0; c < ne; c++)
        key[c] = hilbert_index((unsigned)((xc[c] - x0) * sx), (unsigned)((yc[c] - y0) * sy));
    std::vector<int> order(ne);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
    return order;
}

}  // namespace

int umesh_build(tns_handle* h, const tns_mesh* m) {
    using namespace tns;
    const int ne = m->neles, ng = m->nghosts, nn = m->nods;
    const int* ncs[4] = {m->nc1, m->nc2, m->nc3, m->nc4};
    auto NOD = [&](int c, int k) { return m->nod[(size_t)k * m->ld_nod + c] - 1; };
    std::unordered_map<int, int> line_of;
    line_of.reserve((size_t)ng * 2 + 1);
    int maxid = ne;
    for (int L = 0; L < ng; L++) {
        line_of.emplace(m->nghost[L], L);
        maxid = std::max(maxid, m->nghost[L]);
    }
    // every cell face has a cell or a ghost behind it (checked by build_mesh); reject
    // what this layout cannot express
    for (int c = 0; c < ne; c++)
        for (int k = 0; k < 4; k++) {
            const int v = ncs[k][c];
            if (!(v >= 1 && v <= ne) && !line_of.count(v))
                return h->fail(TNS_ERR_MESH, "cell %d face %d: neighbour %d is neither a cell nor a ghost", c + 1,
                               k + 1, v);
        }
    std::vector<double> xc0(ne), yc0(ne);
    for (int c = 0; c < ne; c++) {
        double sx = 0.0, sy = 0.0;
        for (int k = 0; k < 4; k++) {
            const int n = NOD(c, k);
            if (n < 0 || n >= nn) return h->fail(TNS_ERR_MESH, "cell %d: node %d out of range", c + 1, n + 1);
            sx += m->x[n];
            sy += m->y[n];
        }
        xc0[c] = sx * 0.25;
        yc0[c] = sy * 0.25;
        if (!std::isfinite(xc0[c]) || !std::isfinite(yc0[c]))
            return h->fail(TNS_ERR_MESH, "cell %d has a non-finite node coordinate", c + 1);
    }
    std::vector<int> cell_of = hilbert_order(xc0, yc0), new_of(ne);
    for (int k = 0; k < ne; k++) new_of[cell_of[k]] = k;
    // nodes in the order the renumbered cells first reach them, so that a node's
    // contributions and a face's two nodes sit near the cells that read them
    std::vector<int> node_new(nn, -1), node_old;
    node_old.reserve(nn);
    for (int k = 0; k < ne; k++)
        for (int f = 0; f < 4; f++) {
            const int n = NOD(cell_of[k], f);
            if (node_new[n] < 0) {
                node_new[n] = (int)node_old.size();
                node_old.push_back(n);
            }
        }
    for (int n = 0; n < nn; n++)
        if (node_new[n] < 0) return h->fail(TNS_ERR_MESH, "node %d belongs to no cell", n + 1);
    auto NODN = [&](int c, int k) { return node_new[NOD(c, k)]; };  // renumbered node

    tns_umesh_state* u = new tns_umesh_state();
    h->umesh = u;
    auto slot = [&](int v) { return (v >= 1 && v <= ne) ? new_of[v - 1] : ne + line_of.at(v); };
    const int iaxis = h->P.iaxis;
    // geometry of the cells in original numbering (geometry.f90:55-105)
    std::vector<double> xcc(ne), ycc(ne), vol(ne), dl(ne), sx((size_t)4 * ne), sy((size_t)4 * ne);
    for (int c = 0; c < ne; c++) {
        double X[4], Y[4];
        for (int k = 0; k < 4; k++) {
            const int n = NOD(c, k);
            X[k] = m->x[n];
            Y[k] = m->y[n];
            if (!std::isfinite(X[k]) || !std::isfinite(Y[k]))
                return h->fail(TNS_ERR_MESH, "cell %d has a non-finite node coordinate", c + 1);
        }
        xcc[c] = (X[0] + X[1] + X[2] + X[3]) * 0.25;
        ycc[c] = (Y[0] + Y[1] + Y[2] + Y[3]) * 0.25;
        const double DL12 = std::sqrt((X[0] - X[1]) * (X[0] - X[1]) + (Y[0] - Y[1]) * (Y[0] - Y[1]));
        const double DL23 = std::sqrt((X[1] - X[2]) * (X[1] - X[2]) + (Y[1] - Y[2]) * (Y[1] - Y[2]));
        const double DL34 = std::sqrt((X[2] - X[3]) * (X[2] - X[3]) + (Y[2] - Y[3]) * (Y[2] - Y[3]));
        const double DL41 = std::sqrt((X[3] - X[0]) * (X[3] - X[0]) + (Y[3] - Y[0]) * (Y[3] - Y[0]));
        dl[c] = std::min(std::min(std::min(DL12, DL23), DL34), DL41);
        for (int k = 0; k < 4; k++) face_vector(iaxis, k + 1, X, Y, sx[4 * (size_t)c + k], sy[4 * (size_t)c + k]);
        double v = HALF * ((X[2] - X[0]) * (Y[3] - Y[1]) - (X[3] - X[1]) * (Y[2] - Y[0]));
        if (iaxis == 1) v = v * ycc[c];
        if (v == 0.0) return h->fail(TNS_ERR_MESH, "cell %d has zero volume (collapsed or on the axis)", c + 1);
        vol[c] = v < 0.0 ? -v : v;
    }
    // mirrored ghost centroids (geometry.f90:107-149)
    std::vector<double> gxc(ng), gyc(ng);
    for (int L = 0; L < ng; L++) {
        const int p = m->nparent[L] - 1, s = m->nside[L];
        const int na = NOD(p, s - 1), nb = NOD(p, s & 3);
        const double xf = HALF * (m->x[na] + m->x[nb]), yf = HALF * (m->y[na] + m->y[nb]);
        gxc[L] = 2.0 * xf - xcc[p];
        gyc[L] = 2.0 * yf - ycc[p];
    }
    auto centroid = [&](int v, double& x, double& y) {  // a Fortran id: cell or ghost
        if (v >= 1 && v <= ne) { x = xcc[v - 1]; y = ycc[v - 1]; }
        else { const int L = line_of.at(v); x = gxc[L]; y = gyc[L]; }
    };
    auto grad = [](double xa, double ya, double xb, double yb, double xc, double yc, double xd, double yd,
                   double* out, size_t stride) {
        const double ybd = yb - yd, yac = ya - yc, xbd = xb - xd, xac = xa - xc;
        const double iDNR = 1.0 / (xac * ybd - xbd * yac);
        out[0] = ybd * iDNR;
        out[stride] = -yac * iDNR;
        out[2 * stride] = -xbd * iDNR;
        out[3 * stride] = xac * iDNR;
    };
    u->hnc.assign((size_t)4 * ne, 0);
    u->hnod.assign((size_t)4 * ne, 0);
    u->hcg.assign((size_t)UCG_N * ne, 0.0);
    u->hfg.assign((size_t)UFG_N * 4 * ne, 0.0);
    u->hcfldl.assign(ne, 0.0);
    for (int k = 0; k < ne; k++) {
        const int c = cell_of[k];
        for (int f = 0; f < 4; f++) {
            u->hnc[(size_t)f * ne + k] = slot(ncs[f][c]);
            u->hnod[(size_t)f * ne + k] = NODN(c, f);
            u->hcg[(size_t)(UCG_SX1 + f) * ne + k] = sx[4 * (size_t)c + f];
            u->hcg[(size_t)(UCG_SY1 + f) * ne + k] = sy[4 * (size_t)c + f];
        }
        double xa, ya, xb, yb, xc, yc, xd, yd;
        centroid(ncs[0][c], xa, ya);
        centroid(ncs[1][c], xb, yb);
        centroid(ncs[2][c], xc, yc);
        centroid(ncs[3][c], xd, yd);
        grad(xa, ya, xb, yb, xc, yc, xd, yd, &u->hcg[(size_t)UCG_GA * ne + k], ne);
        u->hcg[(size_t)UCG_VOL * ne + k] = vol[c];
        u->hcg[(size_t)UCG_RVOL * ne + k] = 1.0 / vol[c];
        u->hcg[(size_t)UCG_YCC * ne + k] = ycc[c];
        u->hcg[(size_t)UCG_RYCC * ne + k] = 1.0 / ycc[c];
        u->hcfldl[k] = h->P.cfl * dl[c];
        // faces for the viscous flux: A = the cell, C = NC_f, B = N_f, D = N_f+1
        for (int f = 0; f < 4; f++) {
            double xcn, ycn;
            centroid(ncs[f][c], xcn, ycn);
            const int nb = NOD(c, f), nd = NOD(c, (f + 1) & 3);
            const size_t st = (size_t)4 * ne, at = (size_t)f * ne + k;
            grad(xcc[c], ycc[c], m->x[nb], m->y[nb], xcn, ycn, m->x[nd], m->y[nd], &u->hfg[UFG_GA * st + at], st);
            const double yavg = HALF * (m->y[nb] + m->y[nd]);
            u->hfg[UFG_RYAVG * st + at] = (iaxis == 1 && !(yavg < YAXIS_THRESH)) ? 1.0 / yavg : 0.0;
        }
    }
    // viscous faces: a face between two cells is evaluated once, by the lower id, when the
    // other cell meets it with its nodes in the opposite order (both cells oriented alike);
    // otherwise, and for ghost faces, each cell evaluates its own
    u->hfref.assign((size_t)4 * ne, 0);
    u->hfcell.clear();
    u->hfcell.reserve((size_t)2 * ne + ng);
    {
        std::vector<char> done((size_t)4 * ne, 0);
        for (int k = 0; k < ne; k++)
            for (int f = 0; f < 4; f++) {
                if (done[(size_t)f * ne + k]) continue;
                const int e = (int)u->hfcell.size();
                u->hfcell.push_back(4 * k + f);
                u->hfref[(size_t)f * ne + k] = e;
                done[(size_t)f * ne + k] = 1;
                const int v = u->hnc[(size_t)f * ne + k];
                if (v >= ne || v <= k) continue;
                const int nb = u->hnod[(size_t)f * ne + k], nd = u->hnod[(size_t)((f + 1) & 3) * ne + k];
                for (int g = 0; g < 4; g++)
                    if (!done[(size_t)g * ne + v] && u->hnc[(size_t)g * ne + v] == k &&
                        u->hnod[(size_t)g * ne + v] == nd && u->hnod[(size_t)((g + 1) & 3) * ne + v] == nb) {
                        u->hfref[(size_t)g * ne + v] = ~e;
                        done[(size_t)g * ne + v] = 1;
                        break;
                    }
            }
    }
    // stage chunks of UT consecutive cells: each chunk's halo (the slots its cells touch
    // outside it, in first-touch order) and every cell face's local neighbour slot
    {
        const int nch = (ne + UT - 1) / UT;
        u->hcptr.assign(nch + 1, 0);
        u->hcslot.clear();
        u->hlnb.assign((size_t)4 * ne, 0);
        std::vector<int> tag((size_t)ne + ng, -1), loc((size_t)ne + ng, 0);
        int hmax = 0;
        for (int b = 0; b < nch; b++) {
            const int c0 = b * UT, c1 = std::min(ne, c0 + UT);
            for (int k = c0; k < c1; k++)
                for (int f = 0; f < 4; f++) {
                    const int v = u->hnc[(size_t)f * ne + k];
                    int l;
                    if (v >= c0 && v < c1) {
                        l = v - c0;
                    } else {
                        if (tag[v] != b) {
                            tag[v] = b;
                            loc[v] = UT + (int)u->hcslot.size() - u->hcptr[b];
                            u->hcslot.push_back(v);
                        }
                        l = loc[v];
                    }
                    u->hlnb[(size_t)f * ne + k] = l;
                }
            u->hcptr[b + 1] = (int)u->hcslot.size();
            hmax = std::max(hmax, u->hcptr[b + 1] - u->hcptr[b]);
        }
        // at most 4 UT halo slots: (UT + hmax) slots of 112 bytes fit a block's shared memory
        u->hmax = hmax;
    }
    // ghosts in bc.in order
    static const int OPP[5] = {0, 3, 4, 1, 2};  // side -> the opposite face
    u->hgpar.assign(ng, 0); u->hgopp.assign(ng, 0); u->hgtype.assign(ng, 0); u->hgside.assign(ng, 0);
    u->hgsx.assign(ng, 0.0); u->hgsy.assign(ng, 0.0); u->hgyc.assign(ng, 0.0); u->hginj.assign(ng, 1.0);
    for (int L = 0; L < ng; L++) {
        const int p = m->nparent[L] - 1, s = m->nside[L], ty = m->ntype[L];
        u->hgpar[L] = new_of[p];
        u->hgtype[L] = ty;
        u->hgside[L] = s;
        u->hgsx[L] = sx[4 * (size_t)p + s - 1];
        u->hgsy[L] = sy[4 * (size_t)p + s - 1];
        u->hgyc[L] = gyc[L];
        const int o = ncs[OPP[s] - 1][p];
        if (ty == 3 && !(o >= 1 && o <= ne))
            return h->fail(TNS_ERR_UNSUPPORTED,
                           "bc.in line %d: type-3 ghost whose parent %d has no cell across the opposite face", L + 1,
                           p + 1);
        u->hgopp[L] = (o >= 1 && o <= ne) ? new_of[o - 1] : new_of[p];
    }
    // node contributions in the reference's visit order (viscous.f90:77-124,
    // solver_state.f90:237-262): cells by id, then the ghosts in bc.in order
    std::vector<int> cnt(nn, 0);
    for (int c = 0; c < ne; c++)
        for (int k = 0; k < 4; k++) cnt[NODN(c, k)]++;
    for (int L = 0; L < ng; L++) {
        const int p = m->nparent[L] - 1, s = m->nside[L];
        cnt[NODN(p, s - 1)]++;
        cnt[NODN(p, s & 3)]++;
    }
    u->hnptr.assign(nn + 1, 0);
    for (int n = 0; n < nn; n++) u->hnptr[n + 1] = u->hnptr[n] + cnt[n];
    u->hnslot.assign(u->hnptr[nn], 0);
    u->hnreset.assign(u->hnptr[nn], 0);
    std::vector<int> fill(u->hnptr.begin(), u->hnptr.end() - 1);
    for (int c = 0; c < ne; c++)
        for (int k = 0; k < 4; k++) {
            const int n = NODN(c, k);
            u->hnslot[fill[n]++] = new_of[c];
        }
    for (int L = 0; L < ng; L++) {
        const int p = m->nparent[L] - 1, s = m->nside[L], ty = m->ntype[L];
        for (int n : {NODN(p, s - 1), NODN(p, s & 3)}) {
            u->hnreset[fill[n]] = (ty == 4 || ty == 5) ? ty : 0;
            u->hnslot[fill[n]++] = ne + L;
        }
    }
    // port lines of the type-6 ghosts: from the parent straight across the mesh through
    // the face opposite NSIDE until a ghost is reached
    u->hpptr.assign(1, 0);
    for (int L = 0; L < ng; L++) {
        if (m->ntype[L] != 6) continue;
        const int s = m->nside[L];
        int v = m->nparent[L], steps = 0;
        while (v >= 1 && v <= ne && steps <= ne) {
            const int c = v - 1;
            double Y[4];
            for (int k = 0; k < 4; k++) Y[k] = m->y[NOD(c, k)];
            double dely;  // boundary.f90:183-214
            if (s == 1) dely = HALF * ((Y[0] + Y[1]) - (Y[2] + Y[3]));
            else if (s == 2) dely = HALF * ((Y[1] + Y[2]) - (Y[0] + Y[3]));
            else if (s == 3) dely = HALF * ((Y[2] + Y[3]) - (Y[0] + Y[1]));
            else dely = HALF * ((Y[3] + Y[0]) - (Y[1] + Y[2]));
            u->hpcell.push_back(new_of[c]);
            u->hpdely.push_back(dely);
            v = ncs[OPP[s] - 1][c];
            steps++;
        }
        u->hpghost.push_back(L);
        u->hpptr.push_back((int)u->hpcell.size());
    }
    h->ni = ne;
    h->nj = 1;
    h->neles = ne;
    h->nods = nn;
    h->nghosts = ng;
    h->maxid = maxid;
    h->unstructured = true;
    h->identity = true;
    for (int k = 0; k < ne; k++)
        if (cell_of[k] != k) { h->identity = false; break; }
    h->cell_of.swap(cell_of);
    h->ghost_line.resize(ng);
    std::iota(h->ghost_line.begin(), h->ghost_line.end(), 0);
    h->ghost_id.assign(m->nghost, m->nghost + ng);
    h->node_of.resize(nn);
    for (int k = 0; k < nn; k++) h->node_of[k] = node_old[k] + 1;
    h->M = Mesh{};
    h->M.ni = ne;
    h->M.nj = 1;
    return TNS_OK;
}

int umesh_upload(tns_handle* h) {
    tns_umesh_state* u = h->umesh;
    int rc;
    auto upi = [&](DevBuf<int>& b, const std::vector<int>& v) {
        int r = h->cuda(b.alloc(v.size()), "cudaMalloc");
        if (!r && !v.empty()) r = h->cuda(cudaMemcpy(b.p, v.data(), v.size() * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
        return r;
    };
    auto upd = [&](DevBuf<double>& b, const std::vector<double>& v) {
        int r = h->cuda(b.alloc(v.size()), "cudaMalloc");
        if (!r && !v.empty()) r = h->cuda(cudaMemcpy(b.p, v.data(), v.size() * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
        return r;
    };
    const int ne = h->neles, ng = h->nghosts, nn = h->nods;
    if ((rc = upi(u->nc, u->hnc)) || (rc = upi(u->nod, u->hnod)) || (rc = upi(u->gpar, u->hgpar)) ||
        (rc = upi(u->gopp, u->hgopp)) || (rc = upi(u->gtype, u->hgtype)) || (rc = upi(u->gside, u->hgside)) ||
        (rc = upi(u->nptr, u->hnptr)) || (rc = upi(u->nslot, u->hnslot)) || (rc = upi(u->nreset, u->hnreset)) ||
        (rc = upi(u->pghost, u->hpghost)) || (rc = upi(u->pptr, u->hpptr)) || (rc = upi(u->pcell, u->hpcell)) ||
        (rc = upi(u->fcell, u->hfcell)) || (rc = upi(u->fref, u->hfref)) ||
        (rc = upi(u->cptr, u->hcptr)) || (rc = upi(u->cslot, u->hcslot)) || (rc = upi(u->lnb, u->hlnb)) ||
        (rc = upd(u->cg, u->hcg)) || (rc = upd(u->fg, u->hfg)) || (rc = upd(u->cfldl, u->hcfldl)) ||
        (rc = upd(u->gsx, u->hgsx)) || (rc = upd(u->gsy, u->hgsy)) || (rc = upd(u->gyc, u->hgyc)) ||
        (rc = upd(u->ginj, u->hginj)) || (rc = upd(u->pdely, u->hpdely)))
        return rc;
    if ((rc = h->cuda(u->gport.alloc(ng), "cudaMalloc")) ||
        (rc = h->cuda(u->W.alloc((size_t)tns::UW_N * ((size_t)ne + ng)), "cudaMalloc")) ||
        (rc = h->cuda(u->aux.alloc((size_t)tns::UA_N * ne), "cudaMalloc")) ||
        (rc = h->cuda(u->na.alloc((size_t)5 * nn), "cudaMalloc")) ||
        (rc = h->cuda(u->vf.alloc((size_t)4 * std::max<size_t>(u->hfcell.size(), 1)), "cudaMalloc")) ||
        (rc = h->cuda(cudaMemset(u->gport.p, 0, std::max(ng, 1) * 8), "cudaMemset")))
        return rc;
    tns::UMesh& M = u->M;
    M.ne = ne; M.ng = ng; M.nnode = nn; M.nport = (int)u->hpghost.size();
    M.nc = u->nc.p; M.nod = u->nod.p; M.cg = u->cg.p; M.fg = u->fg.p; M.cfldl = u->cfldl.p;
    M.gpar = u->gpar.p; M.gopp = u->gopp.p; M.gtype = u->gtype.p; M.gside = u->gside.p;
    M.gsx = u->gsx.p; M.gsy = u->gsy.p; M.gyc = u->gyc.p; M.ginj = u->ginj.p; M.gport = u->gport.p;
    M.nptr = u->nptr.p; M.nslot = u->nslot.p; M.nreset = u->nreset.p;
    M.pghost = u->pghost.p; M.pptr = u->pptr.p; M.pcell = u->pcell.p; M.pdely = u->pdely.p;
    M.nface = (int)u->hfcell.size(); M.fcell = u->fcell.p; M.fref = u->fref.p;
    M.nchunk = (int)u->hcptr.size() - 1; M.hmax = u->hmax;
    M.cptr = u->cptr.p; M.cslot = u->cslot.p; M.lnb = u->lnb.p;
    if ((rc = h->cuda(tns::configure_u_chunk(M), "cudaFuncSetAttribute")) ||
        (rc = h->cuda(tns::configure_u_chunk_mx(M), "cudaFuncSetAttribute")))
        return rc;
    // the time-step kernels read CFL*DL through the structured view
    h->M.cfldl = u->cfldl.p;
    for (auto* v : {&u->hnc, &u->hnod, &u->hgpar, &u->hgopp, &u->hgside, &u->hnptr, &u->hnslot, &u->hnreset,
                    &u->hpghost, &u->hpptr, &u->hpcell, &u->hfcell, &u->hfref, &u->hcptr, &u->hcslot, &u->hlnb})
        std::vector<int>().swap(*v);
    for (auto* v : {&u->hcg, &u->hfg, &u->hcfldl, &u->hgsx, &u->hgsy, &u->hgyc, &u->hpdely})
        std::vector<double>().swap(*v);
    return TNS_OK;
}

// One FP64 RK4 iteration (turbnstwod.f90:97-168) in the buffers of the structured path:
// A = state, B / C = stage scratch, D, VIS, DT.
void enqueue_iteration_u(tns_handle* h, bool monitor) {
    const tns::Params& P = h->P;
    tns_umesh_state* u = h->umesh;
    const tns::UMesh& M = u->M;
    cudaStream_t s = h->stream;
    double *A = h->qa.p, *B = h->qb.p, *Cq = h->qc.p;
    static const double alpha[4] = {0.25, 1.0 / 3.0, 0.5, 1.0};  // constants.f90:30-33
    const double* in[4] = {A, B, Cq, B};
    double* out[4] = {B, Cq, B, A};
    // the dissipation (with DTMIN before it, LOCAL=0) reads only Q_old and writes D, DT
    // and its own scratch: it runs on the side stream beside stage 1's field set and the
    // viscous flux, joined before stage 1
    const bool fork = !h->profile && h->side;
    cudaStream_t sd = s;
    if (fork) {
        cudaEventRecord(h->fork, s);
        cudaStreamWaitEvent(h->side, h->fork, 0);
        sd = h->side;
    }
    // (with per-kernel profiling everything runs in order on h->stream, each launch timed)
    if (!P.local)
        launch(h, K_DTMIN, [&] {
            tns::launch_time_step_scratch(P, A, M.cfldl, M.ne, h->dt.p, h->partial.p, h->counter.p, h->dtmin.p,
                                          tns::dtmin_blocks(h->M), sd);
        });
    launch(h, K_DISS, [&] { tns::launch_u_dissipation(P, M, A, u->aux.p, h->d.p, h->dt.p, h->dtmin.p, sd); }, 2);
    if (fork) cudaEventRecord(h->join, sd);
    if (monitor) cudaMemsetAsync(h->cdiff.p, 0, 5 * sizeof(unsigned long long), s);
    for (int st = 0; st < 4; st++) {
        if (M.nport) launch(h, K_GPORT, [&] { tns::launch_u_gport(P, M, in[st], s); });
        if (st == 0) {
            // stage 1's field set W feeds the viscous flux (the chunked stages need none)
            launch(h, K_VISC, [&] {
                tns::launch_u_prim(P, M, in[st], u->W.p, s);
                tns::launch_u_viscous(P, M, u->W.p, u->na.p, u->vf.p, h->vis.p, s);
            }, 4);
            if (fork) cudaStreamWaitEvent(s, h->join, 0);
        }
        tns::StageArgsU S{A, out[st], h->d.p, h->vis.p, h->dt.p, h->dtmin.p, alpha[st],
                          (monitor && st == 3) ? h->cdiff.p : nullptr, st == 3 ? h->status.p : nullptr};
        launch(h, K_STAGE, [&] { tns::launch_u_stage_chunk(P, M, S, in[st], s); });
    }
}

void enqueue_iteration_u_mx(tns_handle* h, bool monitor, double* A, double* Aout) {
    const tns::Params& P = h->P;
    tns_umesh_state* u = h->umesh;
    const tns::UMesh& M = u->M;
    cudaStream_t s = h->stream;
    static const double alpha[4] = {0.25, 1.0 / 3.0, 0.5, 1.0};  // constants.f90:30-33
    const float* in[4] = {nullptr, h->dqb.p, h->dqc.p, h->dqb.p};
    float* out[4] = {h->dqb.p, h->dqc.p, h->dqb.p, nullptr};
    // as the FP64 iteration: the dissipation (D, DT in FP32) on the side stream beside
    // stage 1's field set and the viscous flux (VIS in FP32), from the FP64 Q_old
    const bool fork = !h->profile && h->side;
    cudaStream_t sd = s;
    if (fork) {
        cudaEventRecord(h->fork, s);
        cudaStreamWaitEvent(h->side, h->fork, 0);
        sd = h->side;
    }
    if (!P.local)
        launch(h, K_DTMIN, [&] {
            tns::launch_time_step_scratch(P, A, M.cfldl, M.ne, h->dt.p, h->partial.p, h->counter.p, h->dtmin.p,
                                          tns::dtmin_blocks(h->M), sd);
        });
    launch(h, K_DISS, [&] { tns::launch_u_dissipation(P, M, A, u->aux.p, h->df.p, h->dtf.p, h->dtmin.p, sd); }, 2);
    if (fork) cudaEventRecord(h->join, sd);
    if (monitor) cudaMemsetAsync(h->cdiff.p, 0, 5 * sizeof(unsigned long long), s);
    for (int st = 0; st < 4; st++) {
        if (M.nport) launch(h, K_GPORT, [&] { tns::launch_u_gport_mx(P, M, A, in[st], s); });
        if (st == 0) {
            launch(h, K_VISC, [&] {
                tns::launch_u_prim(P, M, A, u->W.p, s);
                tns::launch_u_viscous(P, M, u->W.p, u->na.p, u->vf.p, h->visf.p, s);
            }, 4);
            if (fork) cudaStreamWaitEvent(s, h->join, 0);
        }
        tns::StageArgsMx S{A, in[st], out[st], st == 3 ? Aout : nullptr, h->df.p, h->visf.p, h->dtf.p, h->dtmin.p,
                           (float)alpha[st], (monitor && st == 3) ? h->cdiff.p : nullptr,
                           st == 3 ? h->status.p : nullptr, h->status.p};
        launch(h, K_STAGE, [&] { tns::launch_u_stage_chunk_mx(P, M, S, s); });
    }
}

int umesh_primitives(tns_handle* h) {
    tns_umesh_state* u = h->umesh;
    const size_t nt = (size_t)h->neles + h->nghosts;
    int rc;
    if (!h->primout.p && (rc = h->cuda(h->primout.alloc(4 * nt), "cudaMalloc"))) return rc;
    if (h->precision == 1) {
        // the last stage read the previous state + dQ_B
        tns::launch_u_gport_mx(h->P, u->M, h->other_state(), h->dqb.p, h->stream);
        tns::launch_u_prim_mx(h->P, u->M, h->other_state(), h->dqb.p, u->W.p, h->stream);
    } else {
        // the last stage read B: its primitives and ghosts again from B
        tns::launch_u_gport(h->P, u->M, h->qb.p, h->stream);
        tns::launch_u_prim(h->P, u->M, h->qb.p, u->W.p, h->stream);
    }
    tns::launch_u_prim_out(u->M, u->W.p, h->primout.p, h->stream);
    return h->cuda(cudaGetLastError(), "kernel launch");
}

int umesh_node_averages(tns_handle* h, double* dev_out) {
    tns_umesh_state* u = h->umesh;
    int rc;
    if ((rc = umesh_primitives(h))) return rc;
    tns::launch_u_post_average(u->M, u->W.p, dev_out, h->stream);
    return h->cuda(cudaGetLastError(), "kernel launch");
}

int umesh_boundary_sums(tns_handle* h, int type, int side, int mode, double* dev_out) {
    tns_umesh_state* u = h->umesh;
    int rc;
    if ((rc = umesh_primitives(h))) return rc;
    tns::launch_u_boundary_sums(h->P, u->M, u->W.p, type, side, mode, dev_out, h->stream);
    return h->cuda(cudaGetLastError(), "kernel launch");
}

int umesh_face_states(tns_handle* h, double* dev_out) {
    tns_umesh_state* u = h->umesh;
    int rc;
    if ((rc = umesh_primitives(h))) return rc;
    tns::launch_u_face_states(h->P, u->M, u->W.p, dev_out, h->stream);
    return h->cuda(cudaGetLastError(), "kernel launch");
}

int umesh_set_injection(tns_handle* h, const double* scale) {
    tns_umesh_state* u = h->umesh;
    return h->cuda(cudaMemcpy(u->ginj.p, scale, (size_t)h->nghosts * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
}

void umesh_release(tns_handle* h) {
    tns_umesh_state* u = h->umesh;
    if (!u) return;
    for (auto* b : {&u->nc, &u->nod, &u->gpar, &u->gopp, &u->gtype, &u->gside, &u->nptr, &u->nslot, &u->nreset,
                    &u->pghost, &u->pptr, &u->pcell, &u->fcell, &u->fref, &u->cptr, &u->cslot, &u->lnb})
        b->release();
    for (auto* b : {&u->cg, &u->fg, &u->cfldl, &u->gsx, &u->gsy, &u->gyc, &u->ginj, &u->gport, &u->pdely, &u->W,
                    &u->aux, &u->na, &u->vf})
        b->release();
    delete u;
    h->umesh = nullptr;
}

}  // namespace tns_rt
