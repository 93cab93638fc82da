// tns_kernels_mx.cu -- mixed FP32/FP64 kernels of one RK4 iteration.
//
// What stays FP64: the state Q (and every stage state COLD + dQ), each stage tile's
// reference state with its primitives and fluxes, ghost states, the viscous and
// dissipation kernels' primitives, geometry (node coordinates, surface vectors,
// volumes, centroids), the differences of nearly equal quantities in the viscous and
// dissipation kernels (gradient stencils, node averages), the part of the flux residual
// that cancels (the reference flux times the closed-contour sum of S), the state
// accumulation and the residual monitor.  What is FP32: the stage increments dQ, the
// dissipation D, the viscous flux VIS and DT as stored, the stage slots as deviations
// from the tile reference (primitives, fluxes and the source stencils), and the
// source / viscous arithmetic with its transcendentals (T**0.6, tanh, sqrt).
//
// Working with deviations instead of values keeps the FP32 rounding of the residual
// proportional to the flow's variation inside a tile rather than to the pressure and
// total-enthalpy levels, so the iteration can still converge by RTRED=1e-5 and more.
#include "tns_device.cuh"
#include "tns_kernels.h"
#include "tns_mx.cuh"
#include "tns_tile.cuh"
#include "tns_batch.cuh"

namespace tns {

// ------------------------------------------------------------------ stage kernel

// Slot order: each thread first evaluates its own cell's slot and keeps that cell's T,
// RHO and P - Pref (read for the cell alone) in registers, then the first NRING threads
// evaluate the halo ring (tns_tile.cuh).
struct StageSmemMx {
    double st[STILE];      // the tile's static block (tns_tile.cuh), one bulk copy
    float2 fg[5][NSLOT];   // (F_m - Fref_m, G_m - Gref_m)
    float2 duv[NSLOT];     // (U - Uref, V - Vref)
    float2 drq[NSLOT];     // (C5/C1 - ref, |V| - ref)
    TileRefMx ref;           // the tile's reference state (written by the dissipation kernel)
    unsigned long long bar;  // completion of the static block's copy
};

size_t stage_mx_smem_bytes() { return sizeof(StageSmemMx); }

// Slot of a cell from its state's deviation from the tile reference, dC = C - Cref, all in
// FP32: every quantity the residual and the sources difference is formed as a deviation
// by exact algebra (dU = (dC2 - Uref dC1) / C1, d(C2 U) = dC2 U + C2ref dU, P - Pref =
// R (dC1 T + C1ref dT), |V| - |V|ref = (|V|^2 - |V|ref^2) / (|V| + |V|ref), ...), so its
// FP32 rounding is a fraction of the deviation, as for a FP64 value rounded after the
// subtraction.
__device__ __forceinline__ void put_slot_dev_mx(const Params& P, StageSmemMx& S, int s, float d1, float d2,
                                                float d3, float d4, float d5, float3& own) {
    const TileRefMx& R = S.ref;
    const float rho = R.rho + d1;
    const float rr = 1.0f / rho;
    const float du = (d2 - R.u * d1) * rr;
    const float dv = (d3 - R.v * d1) * rr;
    const float de = (d4 - R.e * d1) * rr;
    const float dri = (d5 - R.ri * d1) * rr;
    const float u = R.u + du, v = R.v + dv;
    const float dq2 = du * (u + R.u) + dv * (v + R.v);  // |V|^2 - |V|ref^2
    const float dt = (de - 0.5f * dq2) * (float)P.inv_cv;
    const float t = R.t + dt;
    const float dp = kept((float)P.rr * (d1 * t + R.rho * dt));
    const float qm = sqrtf(u * u + v * v);
    const float qs = qm + R.qm;
    const float dqm = qs > 0.0f ? dq2 / qs : 0.0f;
    const float f2 = d2 * v + R.c2 * dv;  // d(C2 V) = d(C3 U)
    S.fg[0][s] = make_float2(d2, d3);
    S.fg[1][s] = make_float2(d2 * u + R.c2 * du + dp, f2);
    S.fg[2][s] = make_float2(f2, d3 * v + R.c3 * dv + dp);
    S.fg[3][s] = make_float2((d4 + dp) * u + R.c4p * du, (d4 + dp) * v + R.c4p * dv);
    S.fg[4][s] = make_float2(d5 * u + R.c5 * du, d5 * v + R.c5 * dv);
    S.duv[s] = make_float2(du, dv);
    S.drq[s] = make_float2(dri, dqm);
    own = make_float3(kept(t), kept(rho), kept(dp));
}

// Slot of a ghost: its BC state in FP64, then the deviations.
__device__ __forceinline__ void put_slot_ghost_mx(StageSmemMx& S, int s, const Prim& p, float3& own) {
    const Prim& r = S.ref.q;
#pragma unroll
    for (int m = 0; m < 5; m++) S.fg[m][s] = make_float2((float)(p.f[m] - r.f[m]), (float)(p.g[m] - r.g[m]));
    S.duv[s] = make_float2((float)(p.u - r.u), (float)(p.v - r.v));
    S.drq[s] = make_float2((float)(p.ri - r.ri), (float)(p.qm - r.qm));
    const float dp = (float)(p.p - r.p);
    own = make_float3(kept((float)p.t), kept((float)p.rho), kept(dp));
}

#ifndef TNS_STAGE_MX_MINB
#define TNS_STAGE_MX_MINB 4
#endif
// the batched kernels at 4 blocks/SM as the single-case ones (the stage kernel with its
// arguments in shared memory, TNS_BATCH_SMEM_ARGS)
#ifndef TNS_STAGE_MX_BATCH_MINB
#define TNS_STAGE_MX_BATCH_MINB 4
#endif
#ifndef TNS_VISC_MX_MINB
#define TNS_VISC_MX_MINB 4  // 64 registers with small spills beat 80 registers at 3 blocks/SM
#endif
#ifndef TNS_VISC_MX_BATCH_MINB
#define TNS_VISC_MX_BATCH_MINB 4
#endif
// One stage on tile (bx, by) of a mesh; the single-case and the batched kernels wrap it.
__device__ __forceinline__ void stage_mx_tile(const Params& P, const Mesh& M, const StageArgsMx& A,
                                              int bx, int by) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    StageSmemMx& S = *reinterpret_cast<StageSmemMx*>(smem_raw);
    const size_t ncell = (size_t)M.ni * M.nj;
    const StateMixed st{A.cold, A.dqin, ncell};
    const int j0 = bx * TJ, i0 = by * TI;
    const int tid = threadIdx.y * TJ + threadIdx.x;
    pdl_trigger();
    // the static block is written by nothing: its copy overlaps the previous kernel's tail
    if (tid == 0) {
        bulk_barrier_init(&S.bar);
        const size_t tile = (size_t)by * ((M.nj + TJ - 1) / TJ) + bx;
        bulk_copy_start(S.st, M.stile + tile * STILE, STILE * sizeof(double), &S.bar);
    }
    pdl_wait();
    if (tid < TREF_WORDS) {
        const size_t tile = (size_t)by * ((M.nj + TJ - 1) / TJ) + bx;
        reinterpret_cast<unsigned long long*>(&S.ref)[tid] =
            reinterpret_cast<const unsigned long long*>(M.tref + tile)[tid];
    }
    __syncthreads();
    // the slot at (li, lj) (nothing where the position is neither a cell nor a ghost);
    // own: its T, RHO, P - Pref
    auto slot = [&](int li, int lj, float3& own) {
        int along = 0;
        const int kind = classify(M, i0 - 1 + li, j0 - 1 + lj, along);
        if (kind < 0) return;
        const int s = li * SW + lj;
        if (kind == 0) {
            const size_t cell = (size_t)(i0 - 1 + li) * M.nj + (j0 - 1 + lj);
            float d[5];
#pragma unroll
            for (int m = 0; m < 5; m++) {
                d[m] = (float)(st.cold[m * ncell + cell] - S.ref.c[m]);
                if (st.dq) d[m] += st.dq[m * ncell + cell];
            }
            put_slot_dev_mx(P, S, s, d[0], d[1], d[2], d[3], d[4], own);
        } else {
            Prim p;
            ghost_state(P, M, st, kind, along, p);
            put_slot_ghost_mx(S, s, p, own);
        }
    };
    // own cell first (its T, RHO, P - Pref kept), then the ring
    float3 own = make_float3(0.0f, 0.0f, 0.0f);
    slot(threadIdx.y + 1, threadIdx.x + 1, own);
    if (tid < NRING) {
        int li, lj;
        ring_slot(tid, li, lj);
        float3 o;
        slot(li, lj, o);
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
        const int nb[4] = {c - 1, c + SW, c + 1, c - SW};
        const int n1 = ti * SNW + tj;  // node 1 of the cell in the static block
        const int gc = 2 * SNN + ti * TJ + tj;
        const double* X0 = S.st;
        const double* Y0 = S.st + SNN;
        const double X[4] = {X0[n1], X0[n1 + SNW], X0[n1 + SNW + 1], X0[n1 + 1]};
        const double Y[4] = {Y0[n1], Y0[n1 + SNW], Y0[n1 + SNW + 1], Y0[n1 + 1]};
        double SX[4], SY[4];
#pragma unroll
        for (int k = 0; k < 4; k++) face_vector(P.iaxis, k + 1, X, Y, SX[k], SY[k]);
        const double ycc = (Y[0] + Y[1] + Y[2] + Y[3]) * 0.25;
        const double VOL = M.cvol[cell];
        const double sumx = SX[0] + SX[1] + SX[2] + SX[3], sumy = SY[0] + SY[1] + SY[2] + SY[3];
        float sx[4], sy[4];
#pragma unroll
        for (int k = 0; k < 4; k++) { sx[k] = (float)SX[k]; sy[k] = (float)SY[k]; }

        // residual: FP32 over flux deviations + FP64 reference part (residual.f90:23-62)
        float R[5];
        double R64[5];
#pragma unroll
        for (int m = 0; m < 5; m++) {
            const float2 I = S.fg[m][c], a = S.fg[m][nb[0]], b = S.fg[m][nb[1]], e = S.fg[m][nb[2]],
                         d = S.fg[m][nb[3]];
            R[m] = 0.5f * ((I.x + a.x) * sx[0] + (I.y + a.y) * sy[0] + (I.x + b.x) * sx[1] +
                           (I.y + b.y) * sy[1] + (I.x + e.x) * sx[2] + (I.y + e.y) * sy[2] +
                           (I.x + d.x) * sx[3] + (I.y + d.y) * sy[3]);
            R64[m] = S.ref.q.f[m] * sumx + S.ref.q.g[m] * sumy;
        }

        // source terms (source_terms.f90:24-104): FP64 stencil differences, FP32 rest,
        // the gradient through the tile's stored coefficients
        {
            const int a = nb[0], b = nb[1], cc = nb[2], d = nb[3];
            const float ga = (float)S.st[gc + ST_GA * NTHREADS], gb = (float)S.st[gc + ST_GB * NTHREADS];
            const float gcf = (float)S.st[gc + ST_GC * NTHREADS], gd = (float)S.st[gc + ST_GD * NTHREADS];
            const float2 ua = S.duv[a], ub = S.duv[b], uc = S.duv[cc], ud = S.duv[d];
            const float2 ra = S.drq[a], rb = S.drq[b], rc = S.drq[cc], rd = S.drq[d];
            const float dqac = ra.y - rc.y, dqbd = rb.y - rd.y;
            const float drac = ra.x - rc.x, drbd = rb.x - rd.x;
            const float duac = ua.x - uc.x, dubd = ub.x - ud.x;
            const float dvac = ua.y - uc.y, dvbd = ub.y - ud.y;
            const float DQX = dqac * ga + dqbd * gb, DQY = dqac * gcf + dqbd * gd;
            const float DRX = drac * ga + drbd * gb, DRY = drac * gcf + drbd * gd;
            const float DUX = duac * ga + dubd * gb, DUY = duac * gcf + dubd * gd;
            const float DVX = dvac * ga + dvbd * gb, DVY = dvac * gcf + dvbd * gd;
            const float2 trc = make_float2(own.x, own.y);
            const float RHO = trc.y, RI = S.ref.ri + S.drq[c].x, T = trc.x;
            const float AMU = (float)P.suth_amol * pow06f(T);
            const float CHI = RHO * RI / ((float)CMU * AMU);
            const float chi2 = CHI * CHI;
            const float FMU = tanh_f32((float)ALPHA_T * chi2) / tanh_f32((float)BETA_T * chi2);
            const float FR2 = tanh_f32(sqrtf(CHI)) / tanh_f32(CHI * (float)P.fr2k);
            const float AMUT = FMU * RHO * RI;
            const float PHI = DQX * DRX + DQY * DRY;
            const float DEE = PHI > 0.0f ? DRX * DRX + DRY * DRY : 0.0f;
            const float DIV23 = (float)P.div23;
            float pw = AMUT / fmaxf(AMUT, (float)AMU_THRESH * AMU);
            {
                float r = 1.0f, bb = pw;
                int mm = P.npseudo < 0 ? -P.npseudo : P.npseudo;
                while (mm) {
                    if (mm & 1) r *= bb;
                    mm >>= 1;
                    if (mm) bb *= bb;
                }
                pw = P.npseudo < 0 ? 1.0f / r : r;
            }
            float PK, src5;
            const float volf = (float)VOL;
            if (P.iaxis == 1) {
                const double rycc = S.st[gc + ST_RYCC * NTHREADS];
                const float VBYY = (ycc < YAXIS_THRESH) ? DVY : (S.ref.v + S.duv[c].y) * (float)rycc;
                const float DIVVEL = DUX + DVY + VBYY;
                PK = AMUT / RHO *
                     (DUX * DUX + DVY * DVY + VBYY * VBYY + DUX * DUX + DVY * DVY + VBYY * VBYY +
                      (DUY + DVX) * (DUY + DVX) - DIV23 * DIVVEL * DIVVEL);
                PK = fmaxf(PK, 0.0f);
                src5 = (RHO * ((float)CONST1 - (float)CONST2 * FR2) * sqrtf(RI * PK) -
                        RHO * (float)CONST3 * DEE) * pw;
                const float TTT = (AMU + AMUT) * (VBYY + VBYY - DIV23 * DIVVEL);
                // SOURCE3 = (P - TTT)/YCC: the reference pressure's part cancels the
                // reference flux in FP64
                R64[2] -= VOL * (S.ref.q.p * rycc);
                R[2] += volf * ((TTT - own.z) * (float)rycc);
            } else {
                const float DIVVEL = DUX + DVY;
                PK = AMUT / RHO *
                     (DUX * DUX + DVY * DVY + DUX * DUX + DVY * DVY + (DUY + DVX) * (DUY + DVX) -
                      DIV23 * DIVVEL * DIVVEL);
                PK = fmaxf(PK, 0.0f);
                src5 = (RHO * ((float)CONST1 - (float)CONST2 * FR2) * sqrtf(RI * PK) -
                        RHO * (float)CONST3 * DEE) * pw;
            }
            R[4] -= volf * src5;
        }
#pragma unroll
        for (int m = 0; m < 5; m++) R[m] += (float)R64[m];

        // update (residual.f90:67-83) as an FP32 increment on the FP64 state
        const float DT = P.local ? A.dt[cell] : (float)*A.dtmin;
        const float dtv = -A.alpha * (DT * (float)S.st[gc + ST_RVOL * NTHREADS]);
        float inc[5];
        inc[0] = dtv * (R[0] - A.d[cell]);
        inc[1] = dtv * (R[1] - A.vis[cell] - A.d[ncell + cell]);
        inc[2] = dtv * (R[2] - A.vis[ncell + cell] - A.d[2 * ncell + cell]);
        inc[3] = dtv * (R[3] - A.vis[2 * ncell + cell] - A.d[3 * ncell + cell]);
        inc[4] = dtv * (float)CFLTURB * (R[4] - A.vis[3 * ncell + cell] - A.d[4 * ncell + cell]);
        double Co[5], Cn[5];
#pragma unroll
        for (int m = 0; m < 5; m++) {
            Co[m] = A.cold[m * ncell + cell];
            Cn[m] = Co[m] + (double)inc[m];
        }
        // nu~ floor C5 = C1*max(RTOL, C5/C1), applied only where it binds
        if (Cn[4] < P.rtol * Cn[0]) {
            Cn[4] = P.rtol * Cn[0];
            inc[4] = (float)(Cn[4] - Co[4]);
        }
        if (A.qout) {
#pragma unroll
            for (int m = 0; m < 5; m++) A.qout[m * ncell + cell] = Cn[m];
        } else {
#pragma unroll
            for (int m = 0; m < 5; m++) A.dqout[m * ncell + cell] = inc[m];
        }
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
            if ((threadIdx.x & 31) == 0)
                atomicMax(&A.cdiff[m], (unsigned long long)__double_as_longlong(v));
        }
    }
}

// Specialised on the residual monitor, so the CDIFF reduction is compiled only where it
// runs.  (A local copy of Params to fix IAXIS costs this kernel registers and spills.)
template <int MONITOR>
__global__ void __launch_bounds__(NTHREADS, TNS_PER_SM(TNS_STAGE_MX_MINB)) k_stage_mx(Params P, Mesh M, StageArgsMx A) {
    StageArgsMx Ac = A;
    if (!MONITOR) Ac.cdiff = nullptr;
    stage_mx_tile(P, M, Ac, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------- viscous kernel

constexpr int NIFM = (TI + 1) * TJ;
constexpr int NJFM = TI * (TJ + 1);

struct ViscSmemMx {
    double u[NSLOT], v[NSLOT], t[NSLOT], rho[NSLOT], ri[NSLOT];
    double au[NAVG], av[NAVG], at[NAVG], arho[NAVG], ar[NAVG];
    float fi[4][NIFM], fj[4][NJFM];
};

size_t visc_mx_smem_bytes() { return sizeof(ViscSmemMx); }

// One face of viscous.f90:130-217: FP64 stencil differences, FP32 rest; the face vector
// and diamond-gradient coefficients from the face's stored row fg[k * nf] (FG_*).
__device__ __forceinline__ void face_flux_mx(const Params& P, const ViscSmemMx& S, int sa, int sc,
                                             int ab, int ad, const double* __restrict__ fg, size_t nf,
                                             float out[4]) {
    const float sx = (float)fg[FG_SX * nf], sy = (float)fg[FG_SY * nf];
    const float ga = (float)fg[FG_GA * nf], gb = (float)fg[FG_GB * nf];
    const float gc = (float)fg[FG_GC * nf], gd = (float)fg[FG_GD * nf];
    const double ua = S.u[sa], va = S.v[sa], ta = S.t[sa], uc = S.u[sc], vc = S.v[sc], tc = S.t[sc];
    const double ub = S.au[ab], vb = S.av[ab], tb = S.at[ab], ud = S.au[ad], vd = S.av[ad], td = S.at[ad];
    const double ra = S.ri[sa], rc = S.ri[sc], rb = S.ar[ab], rd = S.ar[ad];
    const float duac = (float)(ua - uc), dubd = (float)(ub - ud);
    const float dvac = (float)(va - vc), dvbd = (float)(vb - vd);
    const float dtac = (float)(ta - tc), dtbd = (float)(tb - td);
    const float drac = (float)(ra - rc), drbd = (float)(rb - rd);
    const float DUX = duac * ga + dubd * gb, DUY = duac * gc + dubd * gd;
    const float DVX = dvac * ga + dvbd * gb, DVY = dvac * gc + dvbd * gd;
    const float DTX = dtac * ga + dtbd * gb, DTY = dtac * gc + dtbd * gd;
    const float DRX = drac * ga + drbd * gb, DRY = drac * gc + drbd * gd;
    const float UAVG = (float)(QUARTER * (ua + ub + uc + ud));
    const float VAVG = (float)(QUARTER * (va + vb + vc + vd));
    const float TAVG = (float)(QUARTER * (ta + tb + tc + td));
    const float RHOAVG = (float)(QUARTER * (S.rho[sa] + S.arho[ab] + S.rho[sc] + S.arho[ad]));
    const float RAVG = (float)(QUARTER * (ra + rb + rc + rd));
    float DIVVEL;
    if (P.iaxis == 1) {
        const double ryavg = fg[FG_RYAVG * nf];
        const float VBYY = (ryavg == 0.0) ? DVY : (float)(QUARTER * (va + vb + vc + vd) * ryavg);
        DIVVEL = DUX + DVY + VBYY;
    } else {
        DIVVEL = DUX + DVY;
    }
    const float AMU = (float)P.suth_amol * pow06f(TAVG);
    const float AK = AMU * (float)P.cp_pr;
    const float CHI = RHOAVG * RAVG / (AMU * (float)CMU);
    const float chi2 = CHI * CHI;
    const float FMU = tanh_f32((float)ALPHA_T * chi2) / tanh_f32((float)BETA_T * chi2);
    const float AMUT = RHOAVG * RAVG * FMU;
    const float AKT = AMUT * (float)P.cp_prt;
    const float AMUEFF = AMU + AMUT;
    const float AKEFF = AK + AKT;
    const float DIV23 = (float)P.div23;
    const float TXX = AMUEFF * (DUX + DUX - DIV23 * DIVVEL);
    const float TYY = AMUEFF * (DVY + DVY - DIV23 * DIVVEL);
    const float TXY = AMUEFF * (DUY + DVX);
    const float QXX = UAVG * TXX + VAVG * TXY + AKEFF * DTX;
    const float QYY = UAVG * TXY + VAVG * TYY + AKEFF * DTY;
    out[0] = TXX * sx + TXY * sy;
    out[1] = TXY * sx + TYY * sy;
    out[2] = QXX * sx + QYY * sy;
    out[3] = AMUEFF * DRX * sx + AMUEFF * DRY * sy;
}

__device__ __forceinline__ void viscous_mx_tile(const Params& P, const Mesh& M, const double* __restrict__ q,
                                                float* __restrict__ vis, int bx, int by) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ViscSmemMx& S = *reinterpret_cast<ViscSmemMx*>(smem_raw);
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
    for (int s = tid; s < NAVG; s += VNT) {
        const int la = s / AW, lb = s % AW;
        const int a = i0 + la, b = j0 + lb;
        if (a > M.ni || b > M.nj) continue;
        double un = 0.0, vn = 0.0, tn = 0.0, rhon = 0.0, rn = 0.0;
        int cnt = 0, ng = 0, gs[2] = {0, 0}, gr[2] = {0, 0};
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
    for (int f = tid; f < NIFM + NJFM; f += VNT) {
        int sa, sc, ab, ad;
        const double* fg;
        size_t nf;
        if (f < NIFM) {
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
            const int g = f - NIFM;
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
        float out[4];
        face_flux_mx(P, S, sa, sc, ab, ad, fg, nf, out);
        if (f < NIFM) {
#pragma unroll
            for (int k = 0; k < 4; k++) S.fi[k][f] = out[k];
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) S.fj[k][f - NIFM] = out[k];
        }
    }
    __syncthreads();
    const int tj = threadIdx.x, ti = threadIdx.y;
    const int i = i0 + ti, j = j0 + tj;
    if (ti >= TI || i >= M.ni || j >= M.nj) return;
    const size_t cell = (size_t)i * M.nj + j;
    const int f1 = ti * AW + tj, f3 = f1 + 1;
    const int f4 = ti * TJ + tj, f2 = f4 + TJ;
    const float s1 = (j == 0) ? 1.0f : -1.0f, s4 = (i == 0) ? 1.0f : -1.0f;
#pragma unroll
    for (int k = 0; k < 4; k++)
        vis[k * ncell + cell] = ((s1 * S.fj[k][f1] + S.fi[k][f2]) + S.fj[k][f3]) + s4 * S.fi[k][f4];
}

__global__ void __launch_bounds__(VNT, TNS_PER_SM(TNS_VISC_MX_MINB)) k_viscous_mx(Params P, Mesh M, const double* __restrict__ q,
                                                         float* __restrict__ vis) {
    viscous_mx_tile(P, M, q, vis, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------ dissipation kernel

// JST dissipation (solver_state.f90:70-225) with FP64 state, pressure and every
// difference of the state, FP32 sensors, Laplacian differences and blend.
constexpr int DWM = TJ + 4;
constexpr int NDSLOTM = (TI + 4) * DWM;
constexpr int RWM = TJ + 2;
constexpr int NRSLOTM = (TI + 2) * RWM;

struct DissSmemMx {
    double c[5][NDSLOTM];
    double p[NDSLOTM];
    float vbd[NRSLOTM], anu[NRSLOTM], anurt[NRSLOTM], d2q[5][NRSLOTM];
};

size_t diss_mx_smem_bytes() { return sizeof(DissSmemMx); }

__device__ __forceinline__ double local_dt_mx(const Params& P, double c1, double c2, double c3,
                                              double c4, double cfldl) {
    const double rr = 1.0 / c1;
    const double U = c2 * rr, V = c3 * rr;
    const double VEL = sqrt(U * U + V * V);
    const double E = c4 * rr;
    const double T = (E - 0.5 * (U * U + V * V)) * P.inv_cv;
    return cfldl / (fabs(VEL) + sqrt(P.gamrr * T));
}

__device__ __forceinline__ void dissipation_mx_tile(const Params& P, const Mesh& M, const double* __restrict__ q,
                                                    float* __restrict__ dout, float* __restrict__ dtout,
                                                    const double* __restrict__ dtmin, int bx, int by) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DissSmemMx& S = *reinterpret_cast<DissSmemMx*>(smem_raw);
    const size_t ncell = (size_t)M.ni * M.nj;
    const int j0 = bx * TJ, i0 = by * TI;
    const int tid = threadIdx.y * TJ + threadIdx.x;
    pdl_trigger();
    pdl_wait();
    for (int s = tid; s < NDSLOTM; s += NTHREADS) {
        const int i = i0 - 2 + s / DWM, j = j0 - 2 + s % DWM;
        if (i >= 0 && i < M.ni && j >= 0 && j < M.nj) {
            const size_t c = (size_t)i * M.nj + j;
            double C[5];
#pragma unroll
            for (int m = 0; m < 5; m++) {
                C[m] = q[m * ncell + c];
                S.c[m][s] = C[m];
            }
            const double rr = 1.0 / C[0];
            const double U = C[1] * rr, V = C[2] * rr;
            const double T = (C[3] * rr - 0.5 * (U * U + V * V)) * P.inv_cv;
            S.p[s] = C[0] * P.rr * T;
        }
    }
    __syncthreads();
    for (int s = tid; s < NRSLOTM; s += NTHREADS) {
        const int ri = s / RWM, rj = s % RWM;
        const int i = i0 - 1 + ri, j = j0 - 1 + rj;
        if (!(i >= 0 && i < M.ni && j >= 0 && j < M.nj)) continue;
        const int d = (ri + 1) * DWM + (rj + 1);
        int nbs[4] = {d - 1, d + DWM, d + 1, d - DWM};
        if (j == 0) nbs[0] = d;
        if (i == M.ni - 1) nbs[1] = d;
        if (j == M.nj - 1) nbs[2] = d;
        if (i == 0) nbs[3] = d;
        const double PIE = S.p[d], C5I = S.c[4][d];
        double an = 0.0, ad = 0.0, rn = 0.0, rd = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            an += fabs(S.p[nbs[k]] - PIE);
            ad += fabs(S.p[nbs[k]] + PIE);
            rn += fabs(S.c[4][nbs[k]] - C5I);
            rd += fabs(S.c[4][nbs[k]] + C5I);
        }
        S.anu[s] = (float)an / (float)ad;
        S.anurt[s] = (float)rn / (float)fmax(rd, 8.0 * S.c[0][d] * P.rtol);
#pragma unroll
        for (int m = 0; m < 5; m++)
            S.d2q[m][s] = (float)(S.c[m][nbs[0]] + S.c[m][nbs[1]] + S.c[m][nbs[2]] + S.c[m][nbs[3]] - 4.0 * S.c[m][d]);
        const size_t c = (size_t)i * M.nj + j;
        double DT;
        if (P.local) {
            DT = local_dt_mx(P, S.c[0][d], S.c[1][d], S.c[2][d], S.c[3][d], M.cfldl[c]);
            if (ri >= 1 && ri <= TI && rj >= 1 && rj <= TJ) dtout[c] = (float)DT;
        } else {
            DT = *dtmin;
        }
        S.vbd[s] = (float)(M.cvol[c] / DT);
    }
    if (tid == NTHREADS - 1) {
        // the tile's reference state for this iteration's stages (its first cell), by the
        // last warp, which has no second ring slot to wait for
        const int d0 = 2 * DWM + 2;
        const double c[5] = {S.c[0][d0], S.c[1][d0], S.c[2][d0], S.c[3][d0], S.c[4][d0]};
        make_tile_ref(P, c, M.tref[(size_t)by * ((M.nj + TJ - 1) / TJ) + bx]);
    }
    __syncthreads();
    const int tj = threadIdx.x, ti = threadIdx.y;
    const int i = i0 + ti, j = j0 + tj;
    if (i >= M.ni || j >= M.nj) return;
    const size_t cell = (size_t)i * M.nj + j;
    const int r = (ti + 1) * RWM + (tj + 1);
    const int d = (ti + 2) * DWM + (tj + 2);
    const int rn[4] = {r - 1, r + RWM, r + 1, r - RWM};
    const int dn[4] = {d - 1, d + DWM, d + 1, d - DWM};
    const bool has[4] = {j > 0, i < M.ni - 1, j < M.nj - 1, i > 0};
    const float VOLBYDT = S.vbd[r];
    float D2c[4], D4c[4], D2t[4], D4t[4];
    const float ANUI = S.anu[r], ANURTI = S.anurt[r];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float D24N = 0.5f * (VOLBYDT + S.vbd[rn[k]]);
        float E2N = (float)C02 * fmaxf(ANUI, S.anu[rn[k]]);
        float E4N = fmaxf(0.0f, (float)C04 - E2N);
        D2c[k] = E2N * D24N;
        D4c[k] = E4N * D24N;
        E2N = (float)C02 * fmaxf(ANURTI, S.anurt[rn[k]]);
        E4N = fmaxf(0.0f, (float)C04 - E2N);
        D2t[k] = E2N * D24N;
        D4t[k] = E4N * D24N;
    }
#pragma unroll
    for (int m = 0; m < 5; m++) {
        const double CI = S.c[m][d];
        const float D2I = S.d2q[m][r];
        float D2 = 0.0f, D4 = 0.0f;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!has[k]) continue;
            const float a2 = (m == 4) ? D2t[k] : D2c[k];
            const float a4 = (m == 4) ? D4t[k] : D4c[k];
            D2 += a2 * (float)(S.c[m][dn[k]] - CI);
            D4 += a4 * (S.d2q[m][rn[k]] - D2I);
        }
        dout[m * ncell + cell] = D2 - D4;
    }
}

__global__ void __launch_bounds__(NTHREADS) k_dissipation_mx(Params P, Mesh M, const double* __restrict__ q,
                                                             float* __restrict__ dout, float* __restrict__ dtout,
                                                             const double* __restrict__ dtmin) {
    dissipation_mx_tile(P, M, q, dout, dtout, dtmin, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------ port mass flux

__global__ void k_gport_mx(Params P, Mesh M, const double* __restrict__ cold,
                           const float* __restrict__ dq, const int* ghosts, int nport,
                           double* gport) {
    const int w = blockIdx.x;  // one block per port ghost
    const int lane = threadIdx.x & 31;
    if (w >= nport) return;  // whole block
    const size_t ncell = (size_t)M.ni * M.nj;
    const StateMixed st{cold, dq, ncell};
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
        const double y1 = M.y[n1], y2 = M.y[n1 + M.nj + 1], y3 = M.y[n1 + M.nj + 2], y4 = M.y[n1 + 1];
        double dely;
        if (side == 1) dely = HALF * ((y1 + y2) - (y3 + y4));
        else if (side == 2) dely = HALF * ((y2 + y3) - (y1 + y4));
        else if (side == 3) dely = HALF * ((y3 + y4) - (y1 + y2));
        else dely = HALF * ((y4 + y1) - (y2 + y3));
        const double c1 = st.c(0, c), u = st.c(1, c) / c1;
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

__global__ void k_prim_out_mx(Params P, Mesh M, const double* __restrict__ cold,
                              const float* __restrict__ dq, double* out) {
    const size_t ncell = (size_t)M.ni * M.nj;
    const size_t ng = M.nghosts(), ntot = ncell + ng;
    const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k >= ntot) return;
    const StateMixed st{cold, dq, ncell};
    Prim p;
    if (k < ncell) {
        cell_prim(P, st, k, p);
    } else {
        const int g = (int)(k - ncell);
        int side, along;
        if (g < M.ni) { side = 1; along = g; }
        else if (g < M.ni + M.nj) { side = 2; along = g - M.ni; }
        else if (g < 2 * M.ni + M.nj) { side = 3; along = g - M.ni - M.nj; }
        else { side = 4; along = g - 2 * M.ni - M.nj; }
        ghost_state(P, M, st, side, along, p);
    }
    out[k] = p.u;
    out[ntot + k] = p.v;
    out[2 * ntot + k] = p.t;
    out[3 * ntot + k] = p.p;
}

// ------------------------------------------------------------ batched kernels

// Mixed-path batch: `parity` selects which of qa / qa2 holds each active case's state
// (all active cases advance together, so they share it).
__global__ void __launch_bounds__(NTHREADS) k_dissipation_mx_batch(const BatchCase* __restrict__ cases,
                                                                   const int4* __restrict__ tiles,
                                                                   const int* __restrict__ active, int parity) {
    const int4 t = tiles[blockIdx.x];
    if (!active[t.x]) return;  // whole block: before any barrier
    const BatchCase& c = cases[t.x];
    dissipation_mx_tile(c.P, c.M, c.qmx[parity], c.df, c.dtf, c.dtmin, t.y, t.z);
}

__global__ void __launch_bounds__(VNT, TNS_PER_SM(TNS_VISC_MX_BATCH_MINB)) k_viscous_mx_batch(const BatchCase* __restrict__ cases,
                                                                                const int4* __restrict__ tiles,
                                                                                const int* __restrict__ active,
                                                                                int parity) {
    const int4 t = tiles[blockIdx.x];
    if (!active[t.x]) return;
    const BatchCase& c = cases[t.x];
    viscous_mx_tile(c.P, c.M, c.qmx[parity], c.visf, t.y, t.z);
}

__global__ void __launch_bounds__(NTHREADS, TNS_PER_SM(TNS_STAGE_MX_BATCH_MINB)) k_stage_mx_batch(const BatchCase* __restrict__ cases,
                                                                               const int4* __restrict__ tiles,
                                                                               const int* __restrict__ active,
                                                                               int parity, int stage, int monitor) {
    const int4 t = tiles[blockIdx.x];
    if (!active[t.x]) return;
    const BatchCase& c = cases[t.x];
#if TNS_BATCH_SMEM_ARGS
    // the case's arguments in shared memory: constant-address loads instead of loads
    // through a descriptor pointer held in registers
    // (raw storage: the structs are copied in, never constructed)
    __shared__ __align__(16) unsigned char sargs[sizeof(Params) + sizeof(Mesh) + sizeof(StageArgsMx)];
    Params& sP = *reinterpret_cast<Params*>(sargs);
    Mesh& sM = *reinterpret_cast<Mesh*>(sargs + sizeof(Params));
    StageArgsMx& sA = *reinterpret_cast<StageArgsMx*>(sargs + sizeof(Params) + sizeof(Mesh));
    {
        const int tid = threadIdx.y * TJ + threadIdx.x;
        copy_words(&sP, &c.P, sizeof(Params), tid);
        copy_words(&sM, &c.M, sizeof(Mesh), tid);
        copy_words(&sA, &c.stage_mx[parity][monitor][stage], sizeof(StageArgsMx), tid);
        __syncthreads();
    }
    stage_mx_tile(sP, sM, sA, t.y, t.z);
#else
    stage_mx_tile(c.P, c.M, c.stage_mx[parity][monitor][stage], t.y, t.z);
#endif
}

// Persistent batched iterations of the mixed path (schedule 3), as k_batch_persistent:
// the state parity alternates from `parity` with every iteration.
#ifndef TNS_PERSIST_MX_MINB
#define TNS_PERSIST_MX_MINB 4
#endif
__global__ void __launch_bounds__(NTHREADS, TNS_PER_SM(TNS_PERSIST_MX_MINB))
k_batch_persistent_mx(const BatchCase* __restrict__ cases, const int4* __restrict__ tiles,
                      const int* __restrict__ active, int ntiles, int iters, int parity0, unsigned int* bar,
                      unsigned int* error) {
    for (int it = 0; it < iters; it++) {
        const int parity = parity0 ^ (it & 1);
        for (int ph = 0; ph < 5; ph++) {
            const int nwork = ph == 0 ? 2 * ntiles : ntiles;
            for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
                const int4 t = tiles[w % ntiles];
                if (active[t.x]) {
                    const BatchCase& c = cases[t.x];
                    if (ph == 0 && w < ntiles)
                        dissipation_mx_tile(c.P, c.M, c.qmx[parity], c.df, c.dtf, c.dtmin, t.y, t.z);
                    else if (ph == 0)
                        viscous_mx_tile(c.P, c.M, c.qmx[parity], c.visf, t.y, t.z);
                    else
                        stage_mx_tile(c.P, c.M, c.stage_mx[parity][0][ph - 1], t.y, t.z);
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

const void* persistent_kernel_mx() { return (const void*)k_batch_persistent_mx; }

cudaError_t launch_persistent_mx(const BatchCase* cases, const int4* tiles, const int* active, int ntiles,
                                 int iters, int parity, int grid, unsigned int* bar, unsigned int* error,
                                 cudaStream_t s) {
    void* args[] = {(void*)&cases, (void*)&tiles, (void*)&active, (void*)&ntiles, (void*)&iters,
                    (void*)&parity, (void*)&bar, (void*)&error};
    return cudaLaunchCooperativeKernel((const void*)k_batch_persistent_mx, dim3(grid), dim3(TJ, TI), args,
                                       persistent_smem_bytes(true), s);
}

// ------------------------------------------------------------------ launchers

static dim3 tile_grid_mx(const Mesh& M) { return dim3((M.nj + TJ - 1) / TJ, (M.ni + TI - 1) / TI); }

cudaError_t configure_kernels_mx() {
    cudaError_t e = cudaFuncSetAttribute(k_stage_mx<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)stage_mx_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_stage_mx<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)stage_mx_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_dissipation_mx, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)diss_mx_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_viscous_mx, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)visc_mx_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_dissipation_mx_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)diss_mx_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_viscous_mx_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)visc_mx_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_batch_persistent_mx, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)persistent_smem_bytes(true));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_stage_mx_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)stage_mx_smem_bytes());
}

void launch_batch_mx(const BatchCase* cases, const int4* tiles, const int* active, int ntiles,
                     int kernel, int parity, int stage, int monitor, cudaStream_t s) {
    const dim3 blk(TJ, TI);
    if (kernel == 0)
        launch_tile(k_dissipation_mx_batch, dim3(ntiles), blk, diss_mx_smem_bytes(), s, cases, tiles, active, parity);
    else if (kernel == 1)
        launch_tile(k_viscous_mx_batch, dim3(ntiles), dim3(TJ, VROWS), visc_mx_smem_bytes(), s, cases, tiles, active,
                    parity);
    else
        launch_tile(k_stage_mx_batch, dim3(ntiles), blk, stage_mx_smem_bytes(), s, cases, tiles, active, parity, stage,
                    monitor);
}

void launch_dissipation_mx2(const Params& P, const Mesh& M, const double* q, float* d, float* dt,
                            const double* dtmin, cudaStream_t s) {
    launch_tile(k_dissipation_mx, tile_grid_mx(M), dim3(TJ, TI), diss_mx_smem_bytes(), s, P, M, q, d, dt, dtmin);
}

void launch_viscous_mx(const Params& P, const Mesh& M, const double* q, float* vis, cudaStream_t s) {
    launch_tile(k_viscous_mx, tile_grid_mx(M), dim3(TJ, VROWS), visc_mx_smem_bytes(), s, P, M, q, vis);
}

void launch_stage_mx(const Params& P, const Mesh& M, const double* cold, const float* dqin,
                     float* dqout, double* qout, const float* d, const float* vis, const float* dt,
                     const double* dtmin, double alpha, unsigned long long* cdiff,
                     unsigned int* status, unsigned int* error, cudaStream_t s) {
    StageArgsMx A{cold, dqin, dqout, qout, d, vis, dt, dtmin, (float)alpha, cdiff, status, error};
    launch_tile(cdiff ? k_stage_mx<1> : k_stage_mx<0>, tile_grid_mx(M), dim3(TJ, TI), stage_mx_smem_bytes(), s,
                P, M, A);
}

void launch_gport_mx(const Params& P, const Mesh& M, const double* cold, const float* dq,
                     const int* ghosts, int nport, double* gport, cudaStream_t s) {
    if (nport <= 0) return;
    k_gport_mx<<<nport, GP_THREADS, 0, s>>>(P, M, cold, dq, ghosts, nport, gport);
}

void launch_prim_out_mx(const Params& P, const Mesh& M, const double* cold, const float* dq,
                        double* out, cudaStream_t s) {
    const size_t ntot = (size_t)M.ni * M.nj + M.nghosts();
    k_prim_out_mx<<<(unsigned)((ntot + 255) / 256), 256, 0, s>>>(P, M, cold, dq, out);
}

}  // namespace tns
