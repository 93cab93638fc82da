// tns_mx.cuh -- FP32 helpers of the mixed-precision kernels (structured and general
// meshes): the FP32 transcendentals and the deviation form of a stage slot.
//
// A stage slot is formed as deviations from a reference state of its tile or chunk
// (TileRefMx, tns_device.cuh): dC = C - Cref, and every quantity the residual and the
// sources difference follows by exact algebra (dU = (dC2 - Uref dC1) / C1,
// d(C2 U) = dC2 U + C2ref dU, P - Pref = R (dC1 T + C1ref dT), |V| - |V|ref =
// (|V|^2 - |V|ref^2) / (|V| + |V|ref), ...), so each FP32 rounding is a fraction of a
// deviation, as when a FP64 value is rounded after the subtraction.
#pragma once

#include "tns_device.cuh"

namespace tns {

__device__ __forceinline__ float pow06f(float T) { return __expf(0.6f * __logf(T)); }

// tanh for the FP32 path: the Maclaurin series x - x^3/3 + 2x^5/15 - 17x^7/315 +
// 62x^9/2835 - 1382x^11/155925 + 21844x^13/6081075 for |x| < 1/4 (the first omitted
// term is below 2e-12 relative there), and the identity tanh|x| = 1 - 2/(exp(2|x|)+1)
// above, where its cancellation costs at most ~5e-7 relative.
__device__ __forceinline__ float tanh_f32(float x) {
    const float ax = fabsf(x);
    if (ax < 0.25f) {
        const float x2 = x * x;
        return x * (1.0f + x2 * (-1.0f / 3.0f + x2 * (2.0f / 15.0f + x2 * (-17.0f / 315.0f +
                    x2 * (62.0f / 2835.0f + x2 * (-1382.0f / 155925.0f + x2 * (21844.0f / 6081075.0f)))))));
    }
    const float r = 1.0f - __fdividef(2.0f, __expf(2.0f * ax) + 1.0f);
    return copysignf(r, x);
}

// The FP32 values of one stage slot: flux deviations (F_m - Fref_m, G_m - Gref_m),
// (U - Uref, V - Vref), (C5/C1 - ref, |V| - ref), and for the cell itself its T, RHO and
// P - Pref (each rounded once, kept()).
struct SlotMx {
    float2 fg[5], duv, drq;
    float3 own;
};

// A cell's slot from its state's deviation dC = C - Cref (d1..d5).
__device__ __forceinline__ void slot_dev_mx(const Params& P, const TileRefMx& R, float d1, float d2, float d3,
                                            float d4, float d5, SlotMx& o) {
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
    o.fg[0] = make_float2(d2, d3);
    o.fg[1] = make_float2(d2 * u + R.c2 * du + dp, f2);
    o.fg[2] = make_float2(f2, d3 * v + R.c3 * dv + dp);
    o.fg[3] = make_float2((d4 + dp) * u + R.c4p * du, (d4 + dp) * v + R.c4p * dv);
    o.fg[4] = make_float2(d5 * u + R.c5 * du, d5 * v + R.c5 * dv);
    o.duv = make_float2(du, dv);
    o.drq = make_float2(dri, dqm);
    o.own = make_float3(kept(t), kept(rho), kept(dp));
}

// A ghost's slot: its BC state in FP64, then the deviations.
__device__ __forceinline__ void slot_ghost_mx(const TileRefMx& R, const Prim& p, SlotMx& o) {
    const Prim& r = R.q;
#pragma unroll
    for (int m = 0; m < 5; m++) o.fg[m] = make_float2((float)(p.f[m] - r.f[m]), (float)(p.g[m] - r.g[m]));
    o.duv = make_float2((float)(p.u - r.u), (float)(p.v - r.v));
    o.drq = make_float2((float)(p.ri - r.ri), (float)(p.qm - r.qm));
    o.own = make_float3(kept((float)p.t), kept((float)p.rho), kept((float)(p.p - r.p)));
}

}  // namespace tns
