// tns_params.h -- the device parameter block from the C ABI's tns_params (host only).
#pragma once

#include <cmath>

#include "../../include/tnsgpu.h"
#include "tns_device.cuh"

namespace tns {

// Derived scalars exactly as the Fortran main forms them (turbnstwod.f90:37-42,
// 63/84 for RTOLERANCE), plus constants folded in the Fortran's left-to-right order.
inline Params make_params(const tns_params& p) {
    Params P{};
    P.gama = p.gama; P.amol = p.amol; P.cfl = p.cfl; P.prandtl = p.prandtl;
    P.prandtlt = p.prandtlt; P.p0 = p.p0; P.t0 = p.t0; P.pamb = p.pamb; P.rtred = p.rtred;
    P.rinit = p.rinit; P.tflame = p.tflame; P.ancomb = p.ancomb; P.acomb = p.acomb;
    P.rhoprop = p.rhoprop; P.pinf = p.pinf; P.aminf = p.aminf; P.deltabl = p.deltabl;
    P.local = p.local; P.npseudo = p.npseudo; P.iaxis = p.iaxis;
    P.rr = 8314.0 / p.amol;
    P.cv = P.rr / (p.gama - 1.0);
    P.cp = P.cv * p.gama;
    const double rho0 = p.p0 / (P.rr * p.t0);
    P.s0 = p.p0 / std::pow(rho0, p.gama);
    P.tinf = p.t0 / (1.0 + 0.5 * (p.gama - 1.0) * p.aminf * p.aminf);
    P.rtol = p.rinit * p.rtred;
    P.gamrr = p.gama * P.rr;
    P.suth_amol = 0.00000011848 * std::sqrt(p.amol);
    P.div23 = 2.0 / 3.0;
    P.fr2k = std::sqrt(2.0 * std::sqrt(0.09));
    P.inv1mg = 1.0 / (1.0 - p.gama);
    P.gth08 = std::pow(35.0, 0.8);
    P.rtol_rtred = P.rtol * p.rtred;
    P.bl_u = 2.0 * p.aminf * std::sqrt(P.gamrr * P.tinf);
    P.bl_exp = 1.0 / 7.0;
    P.inv_cv = 1.0 / P.cv;
    P.cp_pr = P.cp / p.prandtl;
    P.cp_prt = P.cp / p.prandtlt;
    return P;
}

}  // namespace tns
