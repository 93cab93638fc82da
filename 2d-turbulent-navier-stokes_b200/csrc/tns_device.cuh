// tns_device.cuh -- device-side constants, parameter block, mesh view and the per-cell
// physics of the RK4 / JST / viscous / source / boundary hot path.
//
// The arithmetic restates the reference solver's Fortran (paths relative to the
// reference project) in its operation order, except where one reciprocal replaces a
// run of divisions by the same value, T**0.6 is computed by a division-free Newton
// refinement, and stored gradient coefficients fold a division by a static determinant
// (each a few ulp).  The memory layout is new: cells live in a structured (i, j) block
// (j fastest), ghosts in four side arrays; face vectors come from the node coordinates
// in each tile, the static gradient coefficients and volumes from per-mesh arrays.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// Host-and-device helpers: the discrete adjoint calls the same arithmetic from its
// point functions, which also compile for the host.
#define TNS_HD __host__ __device__ __forceinline__

namespace tns {

// constants.f90:15-60
constexpr double CMU = 0.09;
constexpr double ALPHA_T = 0.00052;
constexpr double BETA_T = 0.2;
constexpr double CONST1 = 21.479;
constexpr double CONST2 = 21.394;
constexpr double CONST3 = 1.5;
constexpr double C02 = 0.25;
constexpr double C04 = 0.00390625;
constexpr double CFLTURB = 0.5;
constexpr double HALF = 0.5;
constexpr double QUARTER = 0.25;
constexpr double YAXIS_THRESH = 0.001;
constexpr double AMU_THRESH = 0.001;
constexpr double GTH = 35.0;
constexpr double CONVKSC = 1.0 / 98066.5;

// Scalar inputs plus every constant the Fortran folds left to right (computed once on
// the host with the same operation order, so device values equal the reference's).
struct Params {
    double gama, amol, cfl, prandtl, prandtlt, p0, t0, pamb, rtred, rinit;
    double tflame, ancomb, acomb, rhoprop, pinf, aminf, deltabl;
    int local, npseudo, iaxis, pad_;
    double rr, cv, cp, s0, tinf, rtol;  // turbnstwod.f90:37-42, RTOLERANCE
    double gamrr;                        // GAMA*RR
    double suth_amol;                    // SUTH_COEF*DSQRT(AMOL)
    double div23;                        // 2/3
    double fr2k;                         // DSQRT(2*DSQRT(CMU))
    double inv1mg;                       // 1/(1-GAMA)
    double gth08;                        // GTH**0.8
    double rtol_rtred;                   // RTOLERANCE*RTRED
    double bl_u;                         // 2*AMINF*DSQRT(GAMA*RR*TINF)
    double bl_exp;                       // 1/7
    double inv_cv;                       // 1/CV
    double cp_pr, cp_prt;                // CP/PRANDTL, CP/PRANDTLT
};

// Static per-face geometry of the viscous flux (viscous.f90:130-217), [FG_N][nfaces]
// for the i-faces (index i*NJ + j, between cells (i-1, j) and (i, j), i = 0..NI) and the
// j-faces (index i*(NJ+1) + j, between (i, j-1) and (i, j), j = 0..NJ), each in the
// orientation of the cell that evaluates it (that of cell (i-1, j) as its face 2, or of
// (0, j) as its face 4; that of (i, j-1) as its face 3, or of (i, 0) as its face 1):
//   FG_SX, FG_SY  face vector; FG_GA..FG_GD diamond-gradient coefficients (A = the cell,
//   C = the neighbour, B, D = the face's nodes: dF/dx = (F_A - F_C) GA + (F_B - F_D) GB,
//   dF/dy = (F_A - F_C) GC + (F_B - F_D) GD); FG_RYAVG 1/YAVG of the axisymmetric v/y
//   term, or 0 where YAVG is below the axis threshold (then dv/dy).
enum FaceGeo { FG_SX, FG_SY, FG_GA, FG_GB, FG_GC, FG_GD, FG_RYAVG, FG_N };

// Ghost-side numbering: side 1 (j=-1) and 3 (j=NJ) are indexed by i, sides 2 (i=NI)
// and 4 (i=-1) by j; the four runs are stored back to back.
struct TileRefMx;

struct Mesh {
    int ni, nj;             // cells in i and j
    const double* x;        // node x [(ni+1)*(nj+1)], node (i,j) at i*(nj+1)+j
    const double* y;
    const double* cfldl;    // CFL*DL per cell
    const int* gtype;       // BC type per ghost
    const int* grank;       // bc.in line of each ghost (node-average order)
    const double* gxc;      // mirrored ghost centroids (geometry.f90:114-142)
    const double* gyc;
    const double* ginj;     // type-6 burn-rate multiplier
    const double* gport;    // type-6 port mass flux of the current stage
    const double* cvol;     // VOL per cell (geometry.f90:87,98,101)
    const double* stile;    // static data of the stage tiles, one block per tile (tns_tile.cuh)
    const double* fgi;      // [FG_N][(ni+1)*nj] static i-face geometry
    const double* fgj;      // [FG_N][ni*(nj+1)] static j-face geometry
    // (mixed precision) each stage tile's reference state for the current iteration,
    // written by the dissipation kernel from Q_old, read by the four stages
    TileRefMx* tref = nullptr;
    __host__ __device__ int ghost_index(int side, int along) const {
        return side == 1 ? along : side == 2 ? ni + along : side == 3 ? ni + nj + along
                                                                      : 2 * ni + nj + along;
    }
    __host__ __device__ int nghosts() const { return 2 * (ni + nj); }
};

TNS_HD double dmax1(double a, double b) { return a >= b ? a : b; }
TNS_HD double dmin1(double a, double b) { return a <= b ? a : b; }

// Fortran REAL**INTEGER by square-and-multiply.
TNS_HD double powi(double x, int n) {
    double r = 1.0, b = x;
    int m = n < 0 ? -n : n;
    while (m) {
        if (m & 1) r *= b;
        m >>= 1;
        if (m) b *= b;
    }
    return n < 0 ? 1.0 / r : r;
}

// T**0.6 for T > 0, as T * w with w = T^(-2/5) = (T^2)^(-1/5): a single-precision
// estimate exp2(-0.4 log2 T) (about 1e-7 relative) refined by two Newton steps for the
// inverse fifth root of a = T^2, which need no division:
//   w <- w + w (1 - a w^5) / 5,
// whose error goes as e' ~ 3 e^2: 3e-14 after one step, FP64 rounding after two.
// Within a few ulp of pow.
TNS_HD double pow06(double T) {
#ifdef __CUDA_ARCH__
    double w = (double)exp2f(-0.4f * __log2f((float)T));
#else
    double w = (double)exp2f(-0.4f * log2f((float)T));
#endif
    const double a = T * T;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const double w2 = w * w;
        const double t = 1.0 - a * (w2 * w2 * w);
        w = w + 0.2 * w * t;
    }
    return T * w;
}

// expm1(x) for 0 <= x <= 40 (device; libm on the host), by the classical additive
// argument reduction and a truncated series (Cody & Waite; the structure of Tang's
// expm1, ACM TOMS 18(2), 1992, without its table):
//   x = k ln2 + r, k = rint(x / ln2), |r| <= ln2 / 2, with ln2 = LN2_HI + LN2_LO and
//   LN2_HI carrying 32 significant bits, so k LN2_HI is exact and r has no cancellation
//   error;
//   expm1(r) = r + r^2 (1/2! + r/3! + ... + r^11/13!), the Taylor series of e^r - 1 to
//   r^13/13!: the first omitted term, r^14/14!, is below 5e-18 for |r| <= ln2 / 2;
//   expm1(x) = 2^k expm1(r) + (2^k - 1) in one fused multiply-add (2^k - 1 is exact
//   for k <= 53, and k <= 58 here).
// Measured on B200 over 4M points of [0, 40]: within 2.7e-16 relative of libm (the CUDA
// function: 2.2e-16), at 1.4x its throughput.
TNS_HD double expm1_nonneg(double x) {
#ifdef __CUDA_ARCH__
    constexpr double INV_LN2 = 1.4426950408889634;
    constexpr double LN2_HI = 0.6931471804855391;    // ln 2 to 32 significant bits
    constexpr double LN2_LO = 7.440617110012397e-11;  // ln 2 - LN2_HI
    const double k = rint(x * INV_LN2);
    const double r = fma(-k, LN2_LO, fma(-k, LN2_HI, x));
    double q = 1.6059043836821613e-10;  // 1/13!
    q = fma(q, r, 2.08767569878681e-09);   // 1/12!
    q = fma(q, r, 2.505210838544172e-08);  // 1/11!
    q = fma(q, r, 2.755731922398589e-07);  // 1/10!
    q = fma(q, r, 2.7557319223985893e-06); // 1/9!
    q = fma(q, r, 2.48015873015873e-05);   // 1/8!
    q = fma(q, r, 0.0001984126984126984);  // 1/7!
    q = fma(q, r, 0.001388888888888889);   // 1/6!
    q = fma(q, r, 0.008333333333333333);   // 1/5!
    q = fma(q, r, 0.041666666666666664);   // 1/4!
    q = fma(q, r, 0.16666666666666666);    // 1/3!
    q = fma(q, r, 0.5);                    // 1/2!
    const double p = fma(r * r, q, r);
    const double s = __longlong_as_double((long long)((int)k + 1023) << 52);  // 2^k
    return fma(s, p, s - 1.0);
#else
    return expm1(x);
#endif
}

// tanh(a) / tanh(b) for a, b >= 0, from tanh(x) = E / (E + 2) with E = expm1(2x):
// Ea (Eb + 2) / (Eb (Ea + 2)), one division instead of three.  Arguments are capped at
// 20, where tanh is 1 to double precision, so E stays finite.
TNS_HD double tanh_ratio(double a, double b) {
    const double ea = expm1_nonneg(2.0 * fmin(a, 20.0)), eb = expm1_nonneg(2.0 * fmin(b, 20.0));
    return (ea * (eb + 2.0)) / (eb * (ea + 2.0));
}

// Sutherland-type molecular viscosity SUTH_COEF*DSQRT(AMOL)*T**0.6 (viscous.f90:188).
TNS_HD double amu_of(const Params& P, double T) {
    return P.suth_amol * pow06(T);
}

// A value made opaque to the optimizer (device code; the identity on the host).  The
// compiler fuses a multiply into a later add (FMA contraction) or not depending on how
// many uses the product has, so a value whose uses differ between kernels (a slot kept in
// a register for the thread's own cell in one, only stored in another) could round
// differently in each.  Passing it through kept() rounds it once, the same way in every
// kernel and build, which keeps the tile-height builds and the batched kernels
// bit-identical to one another.
TNS_HD double kept(double x) {
#ifdef __CUDA_ARCH__
    double r;
    asm("mov.b64 %0, %1;" : "=d"(r) : "d"(x));
    return r;
#else
    return x;
#endif
}
TNS_HD float kept(float x) {
#ifdef __CUDA_ARCH__
    float r;
    asm("mov.b32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
#else
    return x;
#endif
}

// Primitive variables and fluxes of one interior cell (turbnstwod.f90:204-227).
struct Prim {
    double u, v, t, p, rho, ri, c5, qm;
    double f[5], g[5];
};

TNS_HD void primitive(const Params& P, double c1, double c2, double c3,
                                          double c4, double c5, Prim& s) {
    const double RHO = c1;
    const double rr = 1.0 / RHO;  // one reciprocal instead of four divisions
    s.rho = RHO;
    s.u = c2 * rr;
    s.v = c3 * rr;
    const double E = c4 * rr;
    s.t = (E - 0.5 * (s.u * s.u + s.v * s.v)) * P.inv_cv;
    s.p = kept(RHO * P.rr * s.t);
    s.f[0] = c2;
    s.f[1] = RHO * s.u * s.u + s.p;
    s.f[2] = RHO * s.u * s.v;
    s.f[3] = (c4 + s.p) * s.u;
    s.g[0] = c3;
    s.g[1] = s.f[2];
    s.g[2] = RHO * s.v * s.v + s.p;
    s.g[3] = (c4 + s.p) * s.v;
    const double RT = c5 * rr;
    s.f[4] = RHO * RT * s.u;
    s.g[4] = RHO * RT * s.v;
    s.ri = RT;
    s.c5 = c5;
    s.qm = sqrt(s.u * s.u + s.v * s.v);
}

// The mixed path's reference state of a stage tile: a FP64 state of the tile (its first
// cell's Q_old), its primitives and fluxes, and the primitives in FP32 that the
// deviation formulas multiply by.  Any state of the tile serves: the kernels only form
// differences from it.
struct TileRefMx {
    double c[5];  // conservative state
    Prim q;       // its primitives and fluxes
    float rho, u, v, e, t, ri, qm, c2, c3, c4p, c5;  // (e = C4/C1, c4p = C4 + P)
    float pad;
};
static_assert(sizeof(TileRefMx) % 8 == 0, "a tile reference is copied as 8-byte words");
constexpr int TREF_WORDS = (int)(sizeof(TileRefMx) / 8);

TNS_HD void make_tile_ref(const Params& P, const double c[5], TileRefMx& R) {
    for (int m = 0; m < 5; m++) R.c[m] = c[m];
    primitive(P, c[0], c[1], c[2], c[3], c[4], R.q);
    R.rho = (float)c[0];
    R.u = (float)R.q.u;
    R.v = (float)R.q.v;
    R.e = (float)(c[3] / c[0]);
    R.t = (float)R.q.t;
    R.ri = (float)R.q.ri;
    R.qm = (float)R.q.qm;
    R.c2 = (float)c[1];
    R.c3 = (float)c[2];
    R.c4p = (float)(c[3] + R.q.p);
    R.c5 = (float)c[4];
    R.pad = 0.0f;
}

// Conservative + flux tail shared by BC types 2,3,4,6,7 (e.g. boundary.f90:62-70).
TNS_HD void ghost_tail(const Params& P, double RHO, Prim& g) {
    g.rho = RHO;
    const double C2 = RHO * g.u;
    const double C3 = RHO * g.v;
    const double E = P.cv * g.t + 0.5 * (g.u * g.u + g.v * g.v);
    const double C4 = RHO * E;
    g.f[0] = C2;
    g.f[1] = RHO * g.u * g.u + g.p;
    g.f[2] = RHO * g.u * g.v;
    g.f[3] = (C4 + g.p) * g.u;
    g.g[0] = C3;
    g.g[1] = g.f[2];
    g.g[2] = RHO * g.v * g.v + g.p;
    g.g[3] = (C4 + g.p) * g.v;
}

// Face surface vector (geometry.f90:77-99) for face k (1..4) of a cell with nodes 1..4.
TNS_HD void face_vector(int iaxis, int k, const double X[4],
                                            const double Y[4], double& sx, double& sy) {
    const int a = k - 1, b = k & 3;  // nodes (k, k+1)
    if (iaxis == 1) {
        sx = (Y[b] - Y[a]) * (Y[a] + Y[b]) * HALF;
        sy = -(X[b] - X[a]) * (Y[a] + Y[b]) * HALF;
    } else {
        sx = (Y[b] - Y[a]);
        sy = -(X[b] - X[a]);
    }
}

// Cell volume (geometry.f90:87,98,101).
TNS_HD double cell_volume(int iaxis, const double X[4], const double Y[4],
                                              double ycc) {
    double v = HALF * ((X[2] - X[0]) * (Y[3] - Y[1]) - (X[3] - X[1]) * (Y[2] - Y[0]));
    if (iaxis == 1) v = v * ycc;
    if (v <= 0.0) v = -v;
    return v;
}

// Ghost state from its parent (and the parent's opposite neighbour) for BC types 2..7
// (boundary.f90:53-327; type 6 with the port flux supplied by the caller).
// par: parent cell, opp: parent's neighbour across the face opposite the ghost.
// psx, psy: parent's surface vector on the ghost side; ycc_g, ycc_p: ghost / parent
// centroid y; gport: summed port flux (type 6 only); inj: burn-rate multiplier.
TNS_HD void boundary_ghost(const Params& P, int type, const Prim& par,
                                               const Prim& opp, double psx, double psy,
                                               double ycc_g, double ycc_p, double gport,
                                               double inj, Prim& g) {
    double RHO, AMU, RT, C5;
    switch (type) {
        case 2: {  // subsonic inlet :53-71
            g.u = fabs(par.u);
            g.v = -par.v;
            g.t = P.t0 - 0.5 * (g.u * g.u + g.v * g.v) / P.cp;
            RHO = pow(P.s0 / (P.rr * g.t), P.inv1mg);
            g.p = RHO * P.rr * g.t;
            AMU = amu_of(P, g.t);
            RT = AMU / RHO;
            ghost_tail(P, RHO, g);
            C5 = RHO * RT;
            g.f[4] = C5 * g.u;
            g.g[4] = C5 * g.v;
            break;
        }
        case 3: {  // farfield / extrapolation :76-95
            g.u = fabs(2.0 * par.u - opp.u);
            g.v = 2.0 * par.v - opp.v;
            g.t = 2.0 * par.t - opp.t;
            g.p = 2.0 * par.p - opp.p;
            if (P.pamb >= 0.0) g.p = P.pamb;
            RHO = g.p / (P.rr * g.t);
            ghost_tail(P, RHO, g);
            C5 = par.c5;
            g.f[4] = par.f[4];
            g.g[4] = par.g[4];
            break;
        }
        case 4: {  // symmetry :100-109
            g.u = par.u;
            g.v = -par.v;
            g.t = par.t;
            RHO = par.rho;
            g.p = par.p;
            ghost_tail(P, RHO, g);
            C5 = par.c5;
            g.f[4] = par.f[4];
            g.g[4] = -par.g[4];
            break;
        }
        case 5: {  // no-slip wall / axis :114-122
            g.u = -par.u;
            g.v = -par.v;
            g.t = par.t;
            RHO = par.rho;
            g.p = par.p;
            g.rho = RHO;
            g.f[0] = -par.f[0];
            g.f[1] = 2.0 * par.p - par.f[1];
            g.f[2] = -par.f[2];
            g.f[3] = -par.f[3];
            g.g[0] = -par.g[0];
            g.g[1] = -par.g[1];
            g.g[2] = 2.0 * par.p - par.g[2];
            g.g[3] = -par.g[3];
            C5 = -par.c5;
            g.f[4] = -par.f[4];
            g.g[4] = -par.g[4];
            break;
        }
        case 6: {  // mass injection :128-163
            const double DNR = sqrt(psx * psx + psy * psy);
            const double ENX = -psx / DNR, ENY = -psy / DNR;
            const double DHYD = fabs(ycc_g + ycc_p);
            double GP = (P.iaxis == 1) ? 2.0 * gport / (DHYD * DHYD) : gport / DHYD;
            RHO = par.rho;
            const double RDOT = P.acomb * pow(par.p * CONVKSC, P.ancomb) * inj;
            double RDOTEB = RDOT;
            double VEL = P.rhoprop / RHO * RDOTEB;
            g.p = par.p;
            g.u = VEL * ENX + VEL * ENX - par.u;
            g.v = VEL * ENY + VEL * ENY - par.v;
            g.t = P.tflame - 0.5 * (g.u * g.u + g.v * g.v) / P.cp;
            AMU = amu_of(P, g.t);
            const double GVAL =
                (GP / (P.rhoprop * RDOT)) * pow(P.rhoprop * RDOT * DHYD / AMU, -0.125);
            if (GVAL > GTH) RDOTEB = RDOTEB * (1.0 + 0.023 * (pow(GVAL, 0.8) - P.gth08));
            VEL = P.rhoprop / RHO * RDOTEB;
            g.u = VEL * ENX + VEL * ENX - par.u;
            g.v = VEL * ENY + VEL * ENY - par.v;
            g.t = P.tflame - 0.5 * (g.u * g.u + g.v * g.v) / P.cp;
            RHO = g.p / (P.rr * g.t);
            AMU = amu_of(P, g.t);
            RT = AMU / RHO;
            C5 = RHO * RT;
            ghost_tail(P, RHO, g);
            g.f[4] = C5 * g.u;
            g.g[4] = C5 * g.v;
            break;
        }
        default: {  // 7: boundary-layer inlet :310-327
            g.p = P.pinf;
            g.t = P.tinf;
            g.v = -par.v;
            RHO = g.p / (P.rr * g.t);
            if (ycc_g <= P.deltabl)
                g.u = P.bl_u * pow(ycc_g / P.deltabl, P.bl_exp) - par.u;
            else
                g.u = P.bl_u - par.u;
            AMU = amu_of(P, g.t);
            RT = AMU / RHO;
            ghost_tail(P, RHO, g);
            C5 = RHO * RT;
            g.f[4] = C5 * g.u;
            g.g[4] = C5 * g.v;
            break;
        }
    }
    g.c5 = C5;
    g.ri = C5 / g.rho;
    g.qm = sqrt(g.u * g.u + g.v * g.v);
}

// Turbulence / radial sources of one cell (source_terms.f90:24-104).  Neighbours
// a,b,c,d are NC1..NC4; ga..gd are the cell's stored coefficients of the centroid-
// difference gradient (source_terms.f90:24-60): dF/dx = (F_a - F_c) ga + (F_b - F_d) gb,
// dF/dy = (F_a - F_c) gc + (F_b - F_d) gd, i.e. ga = (y_b - y_d)/DNR, gb = -(y_a - y_c)/DNR,
// gc = -(x_b - x_d)/DNR, gd = (x_a - x_c)/DNR with DNR = (x_a - x_c)(y_b - y_d) -
// (x_b - x_d)(y_a - y_c) over the four neighbour centroids; RYCC is 1/YCC.
struct SrcIn {
    double ga, gb, gc, gd;
    double ua, ub, uc, ud, va, vb, vc, vd, ra, rb, rc, rd, qa, qb, qc, qd;
};

__device__ __forceinline__ void source_terms(const Params& P, const SrcIn& s, double RHO,
                                             double RI, double TI, double PI, double VI,
                                             double YCCI, double RYCC, double& src3,
                                             double& src5) {
    const double dqac = s.qa - s.qc, dqbd = s.qb - s.qd, drac = s.ra - s.rc, drbd = s.rb - s.rd;
    const double duac = s.ua - s.uc, dubd = s.ub - s.ud, dvac = s.va - s.vc, dvbd = s.vb - s.vd;
    const double DQX = dqac * s.ga + dqbd * s.gb, DQY = dqac * s.gc + dqbd * s.gd;
    const double DRX = drac * s.ga + drbd * s.gb, DRY = drac * s.gc + drbd * s.gd;
    const double DUX = duac * s.ga + dubd * s.gb, DUY = duac * s.gc + dubd * s.gd;
    const double DVX = dvac * s.ga + dvbd * s.gb, DVY = dvac * s.gc + dvbd * s.gd;
    const double AMU = amu_of(P, TI);
    const double CHI = RHO * RI / (CMU * AMU);
    const double FMU = tanh_ratio(ALPHA_T * CHI * CHI, BETA_T * CHI * CHI);
    const double FR2 = tanh_ratio(sqrt(CHI), CHI * P.fr2k);
    const double AMUT = FMU * RHO * RI;
    const double PHI = DQX * DRX + DQY * DRY;
    double DEE = 0.0;
    if (PHI > 0.0) DEE = DRX * DRX + DRY * DRY;
    double PK;
    const double DIV23 = P.div23;
    // (AMUT / DMAX1(AMUT, AMU_THRESH*AMU))**NPSEUDO: exactly 1 when AMUT is the larger
    const double thr = AMU_THRESH * AMU;
    const double pw = AMUT >= thr ? 1.0 : powi(AMUT / thr, P.npseudo);
    if (P.iaxis == 1) {
        const double VBYY = (YCCI < YAXIS_THRESH) ? DVY : VI * RYCC;
        const double DIVVEL = DUX + DVY + VBYY;
        PK = AMUT / RHO *
             (DUX * DUX + DVY * DVY + VBYY * VBYY + DUX * DUX + DVY * DVY + VBYY * VBYY +
              (DUY + DVX) * (DUY + DVX) - DIV23 * DIVVEL * DIVVEL);
        PK = dmax1(PK, 0.0);
        src5 = (RHO * (CONST1 - CONST2 * FR2) * sqrt(RI * PK) - RHO * CONST3 * DEE) * pw;
        const double TTT = (AMU + AMUT) * (VBYY + VBYY - DIV23 * DIVVEL);
        src3 = (PI - TTT) * RYCC;
    } else {
        const double DIVVEL = DUX + DVY;
        PK = AMUT / RHO *
             (DUX * DUX + DVY * DVY + DUX * DUX + DVY * DVY + (DUY + DVX) * (DUY + DVX) -
              DIV23 * DIVVEL * DIVVEL);
        PK = dmax1(PK, 0.0);
        src5 = (RHO * (CONST1 - CONST2 * FR2) * sqrt(RI * PK) - RHO * CONST3 * DEE) * pw;
        src3 = 0.0;
    }
}

// One face of the thin-layer viscous flux (viscous.f90:130-217): A = the cell, C = the
// face neighbour, B, D = the face's nodes (node averages).  FaceIn holds the coordinates
// (the discrete adjoint's face reverse reads them).
struct FaceIn {
    double sx, sy, xa, ya, xb, yb, xc, yc, xd, yd;
    double ua, va, ta, ub, vb, tb, uc, vc, tc, ud, vd, td;
    double rhoa, rhob, rhoc, rhod, ra, rb, rc, rd;
};

// Sums of one boundary face with the face state (parent + ghost)/2 (U, V averaged; T, P
// of both sides).  mode 0: v = P*SX, P*SY, RHO*(U*SX+V*SY), |S|; mode 1: v[0] = P0*|MDOT|,
// v[1] = |MDOT| with the face's total pressure P0 = P (1 + (GAMA-1)/2 M^2)^(GAMA/(GAMA-1)),
// M^2 = (U^2+V^2)/(GAMA RR T) and mass flux MDOT = RHO (U SX + V SY); RHO is the average of
// P/(RR*T) on both sides.
__device__ __forceinline__ void face_sums(const Params& P, int mode, double u, double vv, double tp, double tg,
                                          double pp, double pg, double sx, double sy, double v[4]) {
    const double pf = 0.5 * (pp + pg);
    const double rho = 0.5 * (pp / (P.rr * tp) + pg / (P.rr * tg));
    if (mode == 1) {
        const double tf = 0.5 * (tp + tg);
        const double m2 = (u * u + vv * vv) / (P.gama * P.rr * tf);
        const double p0 = pf * pow(1.0 + 0.5 * (P.gama - 1.0) * m2, P.gama / (P.gama - 1.0));
        const double md = fabs(rho * (u * sx + vv * sy));
        v[0] = p0 * md;
        v[1] = md;
        return;
    }
    v[0] = pf * sx;
    v[1] = pf * sy;
    v[2] = rho * (u * sx + vv * sy);
    v[3] = sqrt(sx * sx + sy * sy);
}

// One face from its stored geometry (FG_*): the flux of viscous.f90:130-217 with the
// diamond gradient from the coefficients.  Assigns vis[0..3].
struct FaceVals {
    double ua, va, ta, ub, vb, tb, uc, vc, tc, ud, vd, td;
    double rhoa, rhob, rhoc, rhod, ra, rb, rc, rd;
};

__device__ __forceinline__ void viscous_face(const Params& P, const FaceVals& f, double sx,
                                             double sy, double ga, double gb, double gc,
                                             double gd, double ryavg, double vis[4]) {
    const double duac = f.ua - f.uc, dubd = f.ub - f.ud, dvac = f.va - f.vc, dvbd = f.vb - f.vd;
    const double dtac = f.ta - f.tc, dtbd = f.tb - f.td, drac = f.ra - f.rc, drbd = f.rb - f.rd;
    const double DUX = duac * ga + dubd * gb, DUY = duac * gc + dubd * gd;
    const double DVX = dvac * ga + dvbd * gb, DVY = dvac * gc + dvbd * gd;
    const double DTX = dtac * ga + dtbd * gb, DTY = dtac * gc + dtbd * gd;
    const double DRX = drac * ga + drbd * gb, DRY = drac * gc + drbd * gd;
    const double UAVG = QUARTER * (f.ua + f.ub + f.uc + f.ud);
    const double VAVG = QUARTER * (f.va + f.vb + f.vc + f.vd);
    const double TAVG = QUARTER * (f.ta + f.tb + f.tc + f.td);
    const double RHOAVG = QUARTER * (f.rhoa + f.rhob + f.rhoc + f.rhod);
    const double RAVG = QUARTER * (f.ra + f.rb + f.rc + f.rd);
    double DIVVEL;
    if (P.iaxis == 1) {
        const double VBYY = (ryavg == 0.0) ? DVY : VAVG * ryavg;
        DIVVEL = DUX + DVY + VBYY;
    } else {
        DIVVEL = DUX + DVY;
    }
    const double AMU = amu_of(P, TAVG);
    const double AK = AMU * P.cp_pr;
    const double CHI = RHOAVG * RAVG / (AMU * CMU);
    const double FMU = tanh_ratio(ALPHA_T * CHI * CHI, BETA_T * CHI * CHI);
    const double AMUT = RHOAVG * RAVG * FMU;
    const double AKT = AMUT * P.cp_prt;
    const double AMUEFF = AMU + AMUT;
    const double AKEFF = AK + AKT;
    const double TXX = AMUEFF * (DUX + DUX - P.div23 * DIVVEL);
    const double TYY = AMUEFF * (DVY + DVY - P.div23 * DIVVEL);
    const double TXY = AMUEFF * (DUY + DVX);
    const double QXX = UAVG * TXX + VAVG * TXY + AKEFF * DTX;
    const double QYY = UAVG * TXY + VAVG * TYY + AKEFF * DTY;
    vis[0] = TXX * sx + TXY * sy;
    vis[1] = TXY * sx + TYY * sy;
    vis[2] = QXX * sx + QYY * sy;
    vis[3] = AMUEFF * DRX * sx + AMUEFF * DRY * sy;
}

}  // namespace tns
