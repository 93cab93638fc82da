// tns_unstructured_mx.cu -- the mixed FP32/FP64 RK stage on a general quadrilateral mesh.
//
// The general path's chunks (tns_unstructured.cu: 256 consecutive cells in Hilbert
// order and their halo) with the mixed path's arithmetic (tns_kernels_mx.cu): FP64 state
// COLD plus FP32 stage increments dQ; each chunk's slots formed in FP32 as deviations
// from a FP64 reference state, the first cell of the chunk's COLD (tns_mx.cuh); the flux
// residual in FP32 over the flux deviations plus the reference flux times the sum of the
// face vectors in FP64; source terms in FP32; D, VIS, DT stored in FP32.  Compiled, like
// tns_kernels_mx.cu, with FP32 division and square root to 2 ulp and FP32 denormals
// flushed.
#include "tns_batch.cuh"
#include "tns_handle.h"
#include "tns_mx.cuh"
#include "tns_tile.cuh"
#include "tns_umesh.h"

namespace tns {

// Chunk slots in shared memory: (UT + hmax) of (F_m - Fref_m, G_m - Gref_m) x 5,
// (U - Uref, V - Vref), (C5/C1 - ref, |V| - ref), after the chunk's reference state.
size_t u_chunk_mx_smem_bytes(const UMesh& M) {
    return sizeof(TileRefMx) + sizeof(float2) * 7 * ((size_t)UT + M.hmax);
}

template <class St>
__device__ __forceinline__ void u_cell_prim_mx(const Params& P, const St& st, int c, Prim& p) {
    primitive(P, st.c(0, c), st.c(1, c), st.c(2, c), st.c(3, c), st.c(4, c), p);
}

// One mixed RK stage of one chunk (source_terms.f90:24-104, residual.f90:23-83): stage
// input COLD + dQin (dQin null in stage 1); stages 1-3 write dQout, stage 4 the state qout.
#ifndef TNS_U_CHUNK_MX_MINB
// Blocks per SM the register budget is sized for; measured on a renumbered 1024 x 384
// nozzle-plume (B200, one mixed iteration): 4 -> 0.248 ms, 3 -> 0.264 ms, 5 -> 0.257 ms.
#define TNS_U_CHUNK_MX_MINB 4
#endif
__global__ void __launch_bounds__(UT, TNS_U_CHUNK_MX_MINB) k_u_stage_chunk_mx(Params P, UMesh M, StageArgsMx A) {
    extern __shared__ __align__(16) unsigned char usm_raw[];
    TileRefMx& R = *reinterpret_cast<TileRefMx*>(usm_raw);
    const int ns = UT + M.hmax;
    float2* fg = reinterpret_cast<float2*>(usm_raw + sizeof(TileRefMx));
    float2* duv = fg + 5 * ns;
    float2* drq = duv + ns;
    const int ne = M.ne, t = threadIdx.x;
    const size_t n = (size_t)ne;
    const StateMixed st{A.cold, A.dqin, n};
    const int c0 = blockIdx.x * UT, I = c0 + t;
    const int h0 = M.cptr[blockIdx.x], nh = M.cptr[blockIdx.x + 1] - h0;
    // the chunk's reference state: its first cell's COLD (the same in all four stages)
    if (t == 0) {
        double c[5];
#pragma unroll
        for (int m = 0; m < 5; m++) c[m] = A.cold[m * n + c0];
        make_tile_ref(P, c, R);
    }
    __syncthreads();
    auto put = [&](int s, const SlotMx& o) {
#pragma unroll
        for (int m = 0; m < 5; m++) fg[m * ns + s] = o.fg[m];
        duv[s] = o.duv;
        drq[s] = o.drq;
    };
    // the slot of a cell or ghost; own: the cell's T, RHO, P - Pref
    auto slot = [&](int s, int local, float3& own) {
        SlotMx o;
        if (s < ne) {
            float d[5];
#pragma unroll
            for (int m = 0; m < 5; m++) {
                d[m] = (float)(A.cold[m * n + s] - R.c[m]);
                if (A.dqin) d[m] += A.dqin[m * n + s];
            }
            slot_dev_mx(P, R, d[0], d[1], d[2], d[3], d[4], o);
        } else {
            const int L = s - ne;
            const int par = M.gpar[L], type = M.gtype[L];
            Prim pa, op, p;
            u_cell_prim_mx(P, st, par, pa);
            if (type == 3) u_cell_prim_mx(P, st, M.gopp[L], op);
            else op = pa;
            boundary_ghost(P, type, pa, op, M.gsx[L], M.gsy[L], M.gyc[L], M.cg[UCG_YCC * ne + par],
                           type == 6 ? M.gport[L] : 0.0, M.ginj[L], p);
            slot_ghost_mx(R, p, o);
        }
        put(local, o);
        own = o.own;
    };
    float3 own = make_float3(0.0f, 0.0f, 0.0f);
    if (I < ne) slot(I, t, own);
    for (int h = t; h < nh; h += UT) {
        float3 o;
        slot(M.cslot[h0 + h], UT + h, o);
    }
    __syncthreads();

    double dv[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (I < ne) {
        int nb[4];
#pragma unroll
        for (int k = 0; k < 4; k++) nb[k] = M.lnb[k * ne + I];
        const double* G = M.cg + I;
        const double SX[4] = {G[UCG_SX1 * n], G[UCG_SX2 * n], G[UCG_SX3 * n], G[UCG_SX4 * n]};
        const double SY[4] = {G[UCG_SY1 * n], G[UCG_SY2 * n], G[UCG_SY3 * n], G[UCG_SY4 * n]};
        const double VOL = G[UCG_VOL * n];
        const double sumx = SX[0] + SX[1] + SX[2] + SX[3], sumy = SY[0] + SY[1] + SY[2] + SY[3];
        float sx[4], sy[4];
#pragma unroll
        for (int k = 0; k < 4; k++) { sx[k] = (float)SX[k]; sy[k] = (float)SY[k]; }

        // residual: FP32 over flux deviations + FP64 reference part (residual.f90:23-62)
        float Rs[5];
        double R64[5];
#pragma unroll
        for (int m = 0; m < 5; m++) {
            const float2* F = fg + m * ns;
            const float2 Fi = F[t], a = F[nb[0]], b = F[nb[1]], e = F[nb[2]], d = F[nb[3]];
            Rs[m] = 0.5f * ((Fi.x + a.x) * sx[0] + (Fi.y + a.y) * sy[0] + (Fi.x + b.x) * sx[1] +
                            (Fi.y + b.y) * sy[1] + (Fi.x + e.x) * sx[2] + (Fi.y + e.y) * sy[2] +
                            (Fi.x + d.x) * sx[3] + (Fi.y + d.y) * sy[3]);
            R64[m] = R.q.f[m] * sumx + R.q.g[m] * sumy;
        }

        // source terms (source_terms.f90:24-104): FP32 over the slot deviations, the
        // gradient through the cell's stored coefficients
        {
            const float ga = (float)G[UCG_GA * n], gb = (float)G[UCG_GB * n];
            const float gcf = (float)G[UCG_GC * n], gd = (float)G[UCG_GD * n];
            const float2 ua = duv[nb[0]], ub = duv[nb[1]], uc = duv[nb[2]], ud = duv[nb[3]];
            const float2 ra = drq[nb[0]], rb = drq[nb[1]], rc = drq[nb[2]], rd = drq[nb[3]];
            const float dqac = ra.y - rc.y, dqbd = rb.y - rd.y;
            const float drac = ra.x - rc.x, drbd = rb.x - rd.x;
            const float duac = ua.x - uc.x, dubd = ub.x - ud.x;
            const float dvac = ua.y - uc.y, dvbd = ub.y - ud.y;
            const float DQX = dqac * ga + dqbd * gb, DQY = dqac * gcf + dqbd * gd;
            const float DRX = drac * ga + drbd * gb, DRY = drac * gcf + drbd * gd;
            const float DUX = duac * ga + dubd * gb, DUY = duac * gcf + dubd * gd;
            const float DVX = dvac * ga + dvbd * gb, DVY = dvac * gcf + dvbd * gd;
            const float RHO = own.y, RI = R.ri + drq[t].x, T = own.x;
            const float AMU = (float)P.suth_amol * pow06f(T);
            const float CHI = RHO * RI / ((float)CMU * AMU);
            const float chi2 = CHI * CHI;
            const float FMU = tanh_f32((float)ALPHA_T * chi2) / tanh_f32((float)BETA_T * chi2);
            const float FR2 = tanh_f32(sqrtf(CHI)) / tanh_f32(CHI * (float)P.fr2k);
            const float AMUT = FMU * RHO * RI;
            const float PHI = DQX * DRX + DQY * DRY;
            const float DEE = PHI > 0.0f ? DRX * DRX + DRY * DRY : 0.0f;
            const float DIV23 = (float)P.div23;
            // (AMUT / max(AMUT, AMU_THRESH AMU))**NPSEUDO by square-and-multiply
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
                const double rycc = G[UCG_RYCC * n];
                const float VBYY = (G[UCG_YCC * n] < YAXIS_THRESH) ? DVY : (R.v + duv[t].y) * (float)rycc;
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
                R64[2] -= VOL * (R.q.p * rycc);
                Rs[2] += volf * ((TTT - own.z) * (float)rycc);
            } else {
                const float DIVVEL = DUX + DVY;
                PK = AMUT / RHO *
                     (DUX * DUX + DVY * DVY + DUX * DUX + DVY * DVY + (DUY + DVX) * (DUY + DVX) -
                      DIV23 * DIVVEL * DIVVEL);
                PK = fmaxf(PK, 0.0f);
                src5 = (RHO * ((float)CONST1 - (float)CONST2 * FR2) * sqrtf(RI * PK) -
                        RHO * (float)CONST3 * DEE) * pw;
            }
            Rs[4] -= volf * src5;
        }
#pragma unroll
        for (int m = 0; m < 5; m++) Rs[m] += (float)R64[m];

        // update (residual.f90:67-83) as an FP32 increment on the FP64 state
        const float DT = P.local ? A.dt[I] : (float)*A.dtmin;
        const float dtv = -A.alpha * (DT * (float)G[UCG_RVOL * n]);
        float inc[5];
        inc[0] = dtv * (Rs[0] - A.d[I]);
        inc[1] = dtv * (Rs[1] - A.vis[I] - A.d[n + I]);
        inc[2] = dtv * (Rs[2] - A.vis[n + I] - A.d[2 * n + I]);
        inc[3] = dtv * (Rs[3] - A.vis[2 * n + I] - A.d[3 * n + I]);
        inc[4] = dtv * (float)CFLTURB * (Rs[4] - A.vis[3 * n + I] - A.d[4 * n + I]);
        double Co[5], Cn[5];
#pragma unroll
        for (int m = 0; m < 5; m++) {
            Co[m] = A.cold[m * n + I];
            Cn[m] = Co[m] + (double)inc[m];
        }
        // nu~ floor C5 = C1*max(RTOL, C5/C1), applied only where it binds
        if (Cn[4] < P.rtol * Cn[0]) {
            Cn[4] = P.rtol * Cn[0];
            inc[4] = (float)(Cn[4] - Co[4]);
        }
        if (A.qout) {
#pragma unroll
            for (int m = 0; m < 5; m++) A.qout[m * n + I] = Cn[m];
        } else {
#pragma unroll
            for (int m = 0; m < 5; m++) A.dqout[m * n + I] = inc[m];
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
            if ((threadIdx.x & 31) == 0) atomicMax(&A.cdiff[m], (unsigned long long)__double_as_longlong(v));
        }
    }
}

void launch_u_stage_chunk_mx(const Params& P, const UMesh& M, const StageArgsMx& A, cudaStream_t s) {
    k_u_stage_chunk_mx<<<M.nchunk, UT, u_chunk_mx_smem_bytes(M), s>>>(P, M, A);
}

cudaError_t configure_u_chunk_mx(const UMesh& M) {
    return cudaFuncSetAttribute(k_u_stage_chunk_mx, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)u_chunk_mx_smem_bytes(M));
}

}  // namespace tns
