// tns_adjoint.cuh -- discrete adjoint of one RK4 iteration (BC types 2-7, FP64).
//
// Given lambda_{n+1} = dJ/dQ_{n+1}, the reverse step returns lambda_n = lambda_{n+1}
// dG/dQ_n for the iteration map Q_{n+1} = G(Q_n) of turbnstwod.f90:95-146, and (on
// request) accumulates lambda_{n+1} dG/dp for the parameters the map reads: the node
// coordinates through every geometric quantity (face vectors, volumes, centroids, DL,
// nodes), RTOLERANCE, and P0/T0 through the type-2 inlet.  Each function below is the
// hand-derived reverse of one piece of the forward scheme:
//
//   stage update + clip        residual.f90:67-83        (s1_point)
//   central flux residual      residual.f90:23-62        (s1_point, s3_point)
//   ghost back-propagation     boundary.f90:53-122       (s3g_point)
//   source terms               source_terms.f90:24-104   (src_forward / src_reverse)
//   primitive variables        turbnstwod.f90:204-227    (prim_adj)
//   ghost states 2..7          boundary.f90:53-327       (ghost_adj)
//   port mass flux GPORT       boundary.f90:168-305      (gport_point, port_point,
//                                                         port_node_point)
//   viscous flux               viscous.f90:29-217        (v0..v3_point, visc_face_adj)
//   JST dissipation            solver_state.f90:70-225   (d0..d2_point)
//   time step (LOCAL 0/1)      turbnstwod.f90:97-114     (ts_adj, dtmin_point)
//
// Non-smooth points take the branch the forward comparison took (DMAX1(a, b) = a >= b ?
// a : b gives its derivative to a on ties; |x| has derivative sign(x), 0 at 0).  Every
// function is a point function (one cell, face, node or halo slot per call) compiled for
// host and device: the CUDA kernels in tns_adjoint.cu call them once per thread.  All
// outputs are owner-written (each point writes only its own entries), so a step is
// deterministic and needs no atomics, except the LOCAL=0 sum of dt adjoints.
#pragma once

#include "tns_device.cuh"

namespace tns {
namespace adj {

// Rows of the per-slot field set of a stage input (cells and the ghost ring):
// U, V, T, P, C1..C5, F1..F5, G1..G5 (COMPUTE_PRIMITIVE_VARS plus APPLY_BOUNDARY).
enum { WU = 0, WV = 1, WT = 2, WP = 3, WC1 = 4, WC5 = 8, WF = 9, WG = 14, NWROW = 19 };
// Dissipation pre-pass per cell: P, VOL/DT, DT, D2Q(5), sensor numerators/denominators.
enum { DP_P = 0, DP_VBD = 1, DP_DT = 2, DP_D2Q = 3, DP_NUMA = 8, DP_DENA = 9, DP_NUMR = 10, DP_DENR = 11,
       NDPRE = 12 };
// Dissipation adjoint per cell: direct C, D2Q, VOL/DT and the two sensors.
enum { DO_C = 0, DO_D2Q = 5, DO_VBD = 10, DO_SA = 11, DO_SR = 12, NDOUT = 13 };
// Viscous face adjoint: cell A, neighbour C, nodes B and D (u v t rho r each), the
// centroids and nodes of the diamond, and dF/dSX, dF/dSY per flux component.
enum { VF_A = 0, VF_C = 5, VF_B = 10, VF_D = 15, VF_XA = 20, VF_YA, VF_XC, VF_YC, VF_XB, VF_YB, VF_XD, VF_YD,
       VF_CX = 28, VF_CY = 32, NVF = 36 };
// Node averages: u v t rho r (after the RTOL floor) and r before it.
enum { NA_R0 = 5, NNA = 6 };
// Node info bits: count (bits 0-2), per surrounding position k the components u, v, r it
// still contributes after the wall / symmetry resets (bit 4 + 3k + {0,1,2}), the wall
// reset of r (bit 16) and the RTOL floor (bit 17).
enum { NI_MASK = 4, NI_RESET = 16, NI_FLOOR = 17 };

struct AdjArgs {
    Params P;
    Mesh M;
    int ni, nj;
    long long ncell, npad, nnode, nif, njf;
    // forward values of the iteration
    const double* qold;   // Q_n [5][ncell]
    const double* qin;    // input of the stage being reversed [5][ncell]
    const double* d;      // dissipation D [5][ncell]
    const double* vis;    // viscous flux VIS [4][ncell]
    const double* dt;     // local time step [ncell] (LOCAL = 1)
    const double* dtmin;  // global time step [1] (LOCAL = 0)
    double alpha;
    double* w;            // field set of the stage input [NWROW][npad]
    double* xcs;          // centroids of the cells and ghosts on the halo grid [npad]
    double* ycs;          //   (fixed geometry: filled once by centroid_point)
    // adjoint state
    const double* lam_in;  // adjoint of the stage output [5][ncell]
    double* lam_out;       // adjoint of the stage input (stages 2-4) [5][ncell]
    double* lam_old;       // adjoint of Q_n, residual / source / viscous parts [5][ncell]
    double* lamg;          // ghost part of the last stage gather, boundary band [5][ncell]
    double* lamd;          // dissipation and time-step part of the adjoint of Q_n [5][ncell]
    double* gbar;          // adjoint of the residual of this stage [5][npad], ghost ring zero
    double* gbar4;         // the four stages' residual adjoints [4][5][npad] (stage k at k)
    double* w4;            // the four stages' field sets [4][NWROW][npad]
    double* srcn;          // source adjoint to neighbour k: u v C1 C5 [4][4][ncell]
    double* srcg;          // source adjoint to neighbour k's centroid x y [4][2][ncell]
    double* wself;         // source adjoint to the cell itself: T P V C1 C5 [5][ncell]
    double* wvisc;         // viscous adjoint per slot: U V T C1 C5 [5][npad]
    double* dbar;          // adjoint of D [5][ncell]
    double* visbar;        // adjoint of VIS [4][ncell]
    double* dtbar;         // adjoint of DT [ncell]
    int first;             // stage 4 (the first reversed): initialise the accumulators
    int stage1;            // stage 1: its input is Q_n, add the viscous adjoint
    double* dpre;          // [NDPRE][ncell]
    double* dout;          // [NDOUT][ncell]
    double* navg;          // [NNA][nnode]
    int* ninfo;            // [nnode]
    double* nbar;          // node adjoint / count [5][nnode]
    double* vfi;           // i-face adjoints [NVF][nif]
    double* vfj;           // j-face adjoints [NVF][njf]
    double* dtsum;         // LOCAL = 0: sum of the dt adjoints [1]
    // type-6 port ghosts
    const double* gport;   // port mass flux of this stage's input [nghost]
    double* gportb;        // its adjoint [nghost] (this stage)
    const double* gportb4; // the four stages' [4][nghost]
    const double* qst[4];  // the four stage inputs (column terms of GPORT)
    double* portacc;       // parent face vector x, y and centroid y adjoints per ghost [3][nghost]
    // parameter sensitivities: sens != 0 accumulates RTOLERANCE, T0 and S0; geo != 0 (which
    // implies sens) also every geometric quantity
    int sens, geo;
    double *sxbar, *sybar;   // [4][ncell] face vectors
    double *volbar, *dlbar;  // [ncell]
    double *xcbar, *ycbar;   // [npad] centroids (ghost ring: mirrored centroids)
    double *xnbar, *ynbar;   // [nnode] node coordinates
    double *rtolc, *rtoln;   // RTOLERANCE per cell / per node
    double *t0bar, *s0bar;   // T0 and S0 per cell (type-2 inlet ghosts of the cell)
};

// ------------------------------------------------------------------ indexing

TNS_HD int di_of(int k) { return k == 1 ? 1 : (k == 3 ? -1 : 0); }   // NC1..NC4: j-1, i+1, j+1, i-1
TNS_HD int dj_of(int k) { return k == 0 ? -1 : (k == 2 ? 1 : 0); }
TNS_HD long long padi(const AdjArgs& a, int i, int j) { return (long long)(i + 1) * (a.nj + 2) + (j + 1); }
TNS_HD bool is_cell(const AdjArgs& a, int i, int j) { return i >= 0 && i < a.ni && j >= 0 && j < a.nj; }
TNS_HD long long cell_of(const AdjArgs& a, int i, int j) { return (long long)i * a.nj + j; }
TNS_HD double wv(const AdjArgs& a, int row, long long ps) { return a.w[row * a.npad + ps]; }
TNS_HD double sgn(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }
// Within two cells of the boundary (a ghost's parent or opposite cell).
TNS_HD bool in_band(const AdjArgs& a, int i, int j) {
    return i < 2 || i >= a.ni - 2 || j < 2 || j >= a.nj - 2;
}

// Ghost side (1..4) of ring position (i, j), or 0 for a cell / corner.
TNS_HD int ghost_side(const AdjArgs& a, int i, int j, int& along) {
    const bool in_i = i >= 0 && i < a.ni, in_j = j >= 0 && j < a.nj;
    if (in_i && j == -1) { along = i; return 1; }
    if (in_j && i == a.ni) { along = j; return 2; }
    if (in_i && j == a.nj) { along = i; return 3; }
    if (in_j && i == -1) { along = j; return 4; }
    return 0;
}

struct CellGeo {
    double X[4], Y[4], sx[4], sy[4], vol, xc, yc;
};

// COMPUTE_GEOMETRY of one cell (geometry.f90:55-101) from its four nodes.
TNS_HD void cell_geo(const AdjArgs& a, int i, int j, CellGeo& g) {
    const long long nw = a.nj + 1, n1 = (long long)i * nw + j;
    g.X[0] = a.M.x[n1]; g.X[1] = a.M.x[n1 + nw]; g.X[2] = a.M.x[n1 + nw + 1]; g.X[3] = a.M.x[n1 + 1];
    g.Y[0] = a.M.y[n1]; g.Y[1] = a.M.y[n1 + nw]; g.Y[2] = a.M.y[n1 + nw + 1]; g.Y[3] = a.M.y[n1 + 1];
    g.xc = (g.X[0] + g.X[1] + g.X[2] + g.X[3]) * 0.25;
    g.yc = (g.Y[0] + g.Y[1] + g.Y[2] + g.Y[3]) * 0.25;
    for (int k = 0; k < 4; k++) face_vector(a.P.iaxis, k + 1, g.X, g.Y, g.sx[k], g.sy[k]);
    g.vol = cell_volume(a.P.iaxis, g.X, g.Y, g.yc);
}

// Centroid of a cell or of a ghost (mirrored, geometry.f90:114-142), from the nodes.
TNS_HD void slot_centroid_nodes(const AdjArgs& a, int i, int j, double& xc, double& yc) {
    if (is_cell(a, i, j)) {
        const long long nw = a.nj + 1, n1 = (long long)i * nw + j;
        xc = (a.M.x[n1] + a.M.x[n1 + nw] + a.M.x[n1 + nw + 1] + a.M.x[n1 + 1]) * 0.25;
        yc = (a.M.y[n1] + a.M.y[n1 + nw] + a.M.y[n1 + nw + 1] + a.M.y[n1 + 1]) * 0.25;
    } else {
        int along = 0;
        const int side = ghost_side(a, i, j, along);
        const int g = a.M.ghost_index(side, along);
        xc = a.M.gxc[g];
        yc = a.M.gyc[g];
    }
}

// Fills the halo-grid centroid table (corners zero); run once per handle.
TNS_HD void centroid_point(const AdjArgs& a, long long ps) {
    const int i = (int)(ps / (a.nj + 2)) - 1, j = (int)(ps % (a.nj + 2)) - 1;
    int along = 0;
    double xc = 0.0, yc = 0.0;
    if (is_cell(a, i, j) || ghost_side(a, i, j, along)) slot_centroid_nodes(a, i, j, xc, yc);
    a.xcs[ps] = xc;
    a.ycs[ps] = yc;
}

// Centroid of a cell or ghost from the table.
TNS_HD void slot_centroid(const AdjArgs& a, int i, int j, double& xc, double& yc) {
    const long long ps = padi(a, i, j);
    xc = a.xcs[ps];
    yc = a.ycs[ps];
}

// ------------------------------------------------------------------ forward field set

// Field set of one halo slot of the stage input: primitives and fluxes of a cell, or the
// APPLY_BOUNDARY state of a ghost.  Ghost rows C2..C4 are never read and stay zero.
TNS_HD void s0_point(const AdjArgs& a, long long ps) {
    const int i = (int)(ps / (a.nj + 2)) - 1, j = (int)(ps % (a.nj + 2)) - 1;
    double row[NWROW];
    for (int r = 0; r < NWROW; r++) row[r] = 0.0;
    int along = 0;
    const int side = is_cell(a, i, j) ? 0 : ghost_side(a, i, j, along);
    if (is_cell(a, i, j) || side) {
        Prim p;
        if (!side) {
            const long long c = cell_of(a, i, j);
            double q[5];
            for (int m = 0; m < 5; m++) q[m] = a.qin[m * a.ncell + c];
            primitive(a.P, q[0], q[1], q[2], q[3], q[4], p);
            for (int m = 0; m < 5; m++) row[WC1 + m] = q[m];
        } else {
            const int k = side - 1;
            const int pi = i - di_of(k), pj = j - dj_of(k);
            const long long pc = cell_of(a, pi, pj), oc = cell_of(a, pi - di_of(k), pj - dj_of(k));
            const int gidx = a.M.ghost_index(side, along);
            const int type = a.M.gtype[gidx];
            Prim par, opp;
            primitive(a.P, a.qin[pc], a.qin[a.ncell + pc], a.qin[2 * a.ncell + pc], a.qin[3 * a.ncell + pc],
                      a.qin[4 * a.ncell + pc], par);
            if (type == 3)
                primitive(a.P, a.qin[oc], a.qin[a.ncell + oc], a.qin[2 * a.ncell + oc], a.qin[3 * a.ncell + oc],
                          a.qin[4 * a.ncell + oc], opp);
            else
                opp = par;
            double psx = 0.0, psy = 0.0, ycp = 0.0, gp = 0.0;
            if (type == 6) {
                CellGeo pg;
                cell_geo(a, pi, pj, pg);
                psx = pg.sx[k];
                psy = pg.sy[k];
                ycp = pg.yc;
                gp = a.gport[gidx];
            }
            boundary_ghost(a.P, type, par, opp, psx, psy, a.M.gyc[gidx], ycp, gp, a.M.ginj[gidx], p);
            row[WC1] = p.rho;
            row[WC5] = p.c5;
        }
        row[WU] = p.u; row[WV] = p.v; row[WT] = p.t; row[WP] = p.p;
        for (int m = 0; m < 5; m++) {
            row[WF + m] = p.f[m];
            row[WG + m] = p.g[m];
        }
    }
    for (int r = 0; r < NWROW; r++) a.w[r * a.npad + ps] = row[r];
}

// ------------------------------------------------------------------ primitives

// Reverse of COMPUTE_PRIMITIVE_VARS (turbnstwod.f90:204-227) for one cell: the adjoint
// of its field-set rows wb -> the adjoint of its conservative state qb (added).
TNS_HD void prim_adj(const Params& P, const double q[5], const double wb[NWROW], double qb[5]) {
    const double irho = 1.0 / q[0];
    const double rho = q[0], u = q[1] * irho, v = q[2] * irho, e = q[3] * irho;
    const double t = (e - 0.5 * (u * u + v * v)) * P.inv_cv;
    const double p = rho * P.rr * t, rt = q[4] * irho;
    double b[5];
    for (int m = 0; m < 5; m++) b[m] = wb[WC1 + m];
    b[1] += wb[WF + 0];
    b[2] += wb[WG + 0];
    const double f2b = wb[WF + 2] + wb[WG + 1];
    double ub = wb[WU] + wb[WF + 1] * 2.0 * rho * u + f2b * rho * v + wb[WF + 3] * (q[3] + p) + wb[WF + 4] * rho * rt;
    double vb = wb[WV] + f2b * rho * u + wb[WG + 2] * 2.0 * rho * v + wb[WG + 3] * (q[3] + p) + wb[WG + 4] * rho * rt;
    const double pb = wb[WP] + wb[WF + 1] + wb[WG + 2] + wb[WF + 3] * u + wb[WG + 3] * v;
    double rhob = wb[WF + 1] * u * u + f2b * u * v + wb[WG + 2] * v * v + wb[WF + 4] * rt * u + wb[WG + 4] * rt * v;
    b[3] += wb[WF + 3] * u + wb[WG + 3] * v;
    const double rtb = wb[WF + 4] * rho * u + wb[WG + 4] * rho * v;
    rhob += pb * P.rr * t;
    const double tb = wb[WT] + pb * rho * P.rr;
    const double eb = tb * P.inv_cv;
    ub -= eb * u;
    vb -= eb * v;
    b[4] += rtb * irho;
    b[3] += eb * irho;
    b[1] += ub * irho;
    b[2] += vb * irho;
    rhob -= (rtb * rt + eb * e + ub * u + vb * v) * irho;
    b[0] += rhob;
    for (int m = 0; m < 5; m++) qb[m] += b[m];
}

// ------------------------------------------------------------------ ghosts

// Reverse of the conservative / flux tail of a ghost (e.g. boundary.f90:62-70): rows
// F1..F4, G1..G4 of gb -> adjoints of the ghost's RHO, U, V, T, P (added).
TNS_HD void tail_adj(const Params& P, double rho, double u, double v, double t, double p, const double* gb,
                     double& rhob, double& ub, double& vb, double& tb, double& pb) {
    const double E = P.cv * t + 0.5 * (u * u + v * v);
    const double C4 = rho * E;
    const double c2b = gb[WF + 0], c3b = gb[WG + 0];
    const double f2b = gb[WF + 2] + gb[WG + 1];
    rhob += gb[WF + 1] * u * u + f2b * u * v + gb[WG + 2] * v * v;
    ub += gb[WF + 1] * 2.0 * rho * u + f2b * rho * v + gb[WF + 3] * (C4 + p);
    vb += f2b * rho * u + gb[WG + 2] * 2.0 * rho * v + gb[WG + 3] * (C4 + p);
    pb += gb[WF + 1] + gb[WG + 2] + gb[WF + 3] * u + gb[WG + 3] * v;
    const double c4b = gb[WF + 3] * u + gb[WG + 3] * v;
    rhob += c4b * E;
    const double Eb = c4b * rho;
    tb += Eb * P.cv;
    ub += Eb * u;
    vb += Eb * v;
    rhob += c2b * u + c3b * v;
    ub += c2b * rho;
    vb += c3b * rho;
}

// Geometry and port inputs of one ghost: its mirrored centroid y, the parent's centroid
// y and face vector on the ghost's side, the port mass flux and burn-rate multiplier.
struct GhostGeo {
    double ycg, ycp, psx, psy, gport, inj;
};
struct GhostGeoBar {
    double ycg, ycp, psx, psy, gport;
};

// Reverse of APPLY_BOUNDARY for one ghost of type 2..7 (boundary.f90:53-327).  gw, pw,
// ow: field-set rows of the ghost, its parent and the parent's opposite neighbour; gb:
// the ghost's row adjoint; gg: its geometry and port inputs.  Adds to the parent's rows
// (pb), the opposite cell's U V T P (ob), the adjoints of T0 and S0 (type-2 inlet; type
// 7 through TINF and the profile velocity, both set by T0) and of the geometry and port
// inputs (gbar: types 6 and 7).
TNS_HD void ghost_adj(const Params& P, int type, const double gw[NWROW], const double pw[NWROW],
                      const double ow[NWROW], const double gb[NWROW], double pb[NWROW], double ob[NWROW],
                      double& t0b, double& s0b, const GhostGeo& gg, GhostGeoBar& gbar) {
    if (type == 5) {
        pb[WU] -= gb[WU];
        pb[WV] -= gb[WV];
        pb[WT] += gb[WT];
        pb[WP] += gb[WP] + 2.0 * gb[WF + 1] + 2.0 * gb[WG + 2];
        pb[WC1] += gb[WC1];
        pb[WC5] -= gb[WC5];
        for (int m = 0; m < 5; m++) {
            pb[WF + m] -= gb[WF + m];
            pb[WG + m] -= gb[WG + m];
        }
        return;
    }
    const double rho = gw[WC1], u = gw[WU], v = gw[WV], t = gw[WT], p = gw[WP];
    double rhob = gb[WC1], ub = gb[WU], vb = gb[WV], tb = gb[WT], ppb = gb[WP];
    tail_adj(P, rho, u, v, t, p, gb, rhob, ub, vb, tb, ppb);
    if (type == 4) {
        pb[WU] += ub;
        pb[WV] -= vb;
        pb[WT] += tb;
        pb[WC1] += rhob;
        pb[WP] += ppb;
        pb[WC5] += gb[WC5];
        pb[WF + 4] += gb[WF + 4];
        pb[WG + 4] -= gb[WG + 4];
    } else if (type == 3) {
        pb[WC5] += gb[WC5];
        pb[WF + 4] += gb[WF + 4];
        pb[WG + 4] += gb[WG + 4];
        // RHO = P / (RR T)
        ppb += rhob / (P.rr * t);
        tb -= rhob * rho / t;
        if (P.pamb < 0.0) {
            pb[WP] += 2.0 * ppb;
            ob[WP] -= ppb;
        }
        pb[WT] += 2.0 * tb;
        ob[WT] -= tb;
        pb[WV] += 2.0 * vb;
        ob[WV] -= vb;
        const double xb = ub * sgn(2.0 * pw[WU] - ow[WU]);
        pb[WU] += 2.0 * xb;
        ob[WU] -= xb;
    } else if (type == 6) {  // mass injection (boundary.f90:128-163)
        // forward, as boundary_ghost evaluates it
        const double DNR = sqrt(gg.psx * gg.psx + gg.psy * gg.psy);
        const double ENX = -gg.psx / DNR, ENY = -gg.psy / DNR;
        const double hs = gg.ycg + gg.ycp;
        const double DHYD = fabs(hs);
        const double GP = (P.iaxis == 1) ? 2.0 * gg.gport / (DHYD * DHYD) : gg.gport / DHYD;
        const double RHO0 = pw[WC1], PP = pw[WP];
        const double RDOT = P.acomb * pow(PP * CONVKSC, P.ancomb) * gg.inj;
        const double VEL1 = P.rhoprop / RHO0 * RDOT;
        const double u1 = VEL1 * ENX + VEL1 * ENX - pw[WU], v1 = VEL1 * ENY + VEL1 * ENY - pw[WV];
        const double t1 = P.tflame - 0.5 * (u1 * u1 + v1 * v1) / P.cp;
        const double AMU1 = amu_of(P, t1);
        const double A = GP / (P.rhoprop * RDOT), B = P.rhoprop * RDOT * DHYD / AMU1;
        const double Bp = pow(B, -0.125);
        const double GVAL = A * Bp;
        const bool ero = GVAL > GTH;
        const double fac = ero ? 1.0 + 0.023 * (pow(GVAL, 0.8) - P.gth08) : 1.0;
        const double RDOTEB = RDOT * fac;
        const double VEL2 = P.rhoprop / RHO0 * RDOTEB;
        // reverse: final state (RHO = P / (RR T), C5 = RHO * (AMU(T) / RHO))
        const double c5 = gw[WC5];
        const double c5b = gb[WC5] + gb[WF + 4] * u + gb[WG + 4] * v;
        ub += gb[WF + 4] * c5;
        vb += gb[WG + 4] * c5;
        tb += c5b * 0.6 * amu_of(P, t) / t;
        ppb += rhob / (P.rr * t);
        tb -= rhob * rho / t;
        // T = TFLAME - (U^2 + V^2) / (2 CP)
        ub -= tb * u / P.cp;
        vb -= tb * v / P.cp;
        // U = 2 VEL2 ENX - U_parent
        double ENXb = 2.0 * ub * VEL2, ENYb = 2.0 * vb * VEL2;
        const double VEL2b = 2.0 * (ub * ENX + vb * ENY);
        pb[WU] -= ub;
        pb[WV] -= vb;
        double RHO0b = -VEL2b * VEL2 / RHO0;
        const double RDOTEBb = VEL2b * P.rhoprop / RHO0;
        double RDOTb = RDOTEBb * fac, GVALb = 0.0;
        if (ero) GVALb = RDOTEBb * RDOT * 0.023 * 0.8 * pow(GVAL, -0.2);
        // GVAL = (GP / (RHOPROP RDOT)) * (RHOPROP RDOT DHYD / AMU1)**(-1/8)
        const double Ab = GVALb * Bp, Bb = GVALb * A * (-0.125) * Bp / B;
        const double GPb = Ab / (P.rhoprop * RDOT);
        RDOTb += -Ab * A / RDOT + Bb * B / RDOT;
        double DHYDb = Bb * B / DHYD;
        const double AMU1b = -Bb * B / AMU1;
        const double t1b = AMU1b * 0.6 * AMU1 / t1;
        const double u1b = -t1b * u1 / P.cp, v1b = -t1b * v1 / P.cp;
        ENXb += 2.0 * u1b * VEL1;
        ENYb += 2.0 * v1b * VEL1;
        const double VEL1b = 2.0 * (u1b * ENX + v1b * ENY);
        pb[WU] -= u1b;
        pb[WV] -= v1b;
        RHO0b -= VEL1b * VEL1 / RHO0;
        RDOTb += VEL1b * P.rhoprop / RHO0;
        // RDOT = ACOMB (P CONVKSC)**ANCOMB INJ; P = P_parent; RHO0 = RHO_parent
        if (P.ancomb != 0.0) ppb += RDOTb * RDOT * P.ancomb / PP;
        pb[WP] += ppb;
        pb[WC1] += RHO0b;
        // GP = GPORT / DHYD (2 GPORT / DHYD^2 for IAXIS=1), DHYD = |YCC_ghost + YCC_parent|
        gbar.gport += GPb * ((P.iaxis == 1) ? 2.0 / (DHYD * DHYD) : 1.0 / DHYD);
        DHYDb -= GPb * GP * ((P.iaxis == 1) ? 2.0 : 1.0) / DHYD;
        gbar.ycg += DHYDb * sgn(hs);
        gbar.ycp += DHYDb * sgn(hs);
        // EN = -PS / |PS|
        const double DNRb = -(ENXb * ENX + ENYb * ENY) / DNR;
        gbar.psx += -ENXb / DNR + DNRb * gg.psx / DNR;
        gbar.psy += -ENYb / DNR + DNRb * gg.psy / DNR;
    } else if (type == 7) {  // boundary-layer inlet: P = PINF, T = TINF, U from the 1/7 profile
        const double c5 = gw[WC5];
        const double c5b = gb[WC5] + gb[WF + 4] * u + gb[WG + 4] * v;
        ub += gb[WF + 4] * c5;
        vb += gb[WG + 4] * c5;
        const double amu = amu_of(P, t);
        tb += c5b * 0.6 * amu / t;  // C5 = RHO * (AMU(T) / RHO)
        tb -= rhob * rho / t;       // RHO = PINF / (RR T)
        // U = BL_U (YCC/DELTABL)**(1/7) - U_parent (BL_U - U_parent above the layer)
        double blub = ub;
        if (gg.ycg <= P.deltabl) {
            const double r = gg.ycg / P.deltabl, f = pow(r, P.bl_exp);
            blub = ub * f;
            if (r > 0.0) gbar.ycg += ub * P.bl_u * P.bl_exp * f / r / P.deltabl;
        }
        pb[WU] -= ub;
        pb[WV] -= vb;
        // TINF = T0 / (1 + (GAMA-1)/2 AMINF^2) and BL_U = 2 AMINF sqrt(GAMA RR TINF)
        t0b += tb * P.tinf / P.t0 + blub * P.bl_u / (2.0 * P.t0);
    } else {  // type 2: subsonic inlet at P0, T0
        const double c5 = gw[WC5];
        double c5b = gb[WC5] + gb[WF + 4] * u + gb[WG + 4] * v;
        ub += gb[WF + 4] * c5;
        vb += gb[WG + 4] * c5;
        // C5 = RHO * (AMU(T) / RHO)
        const double amu = amu_of(P, t);
        tb += c5b * 0.6 * amu / t;
        // P = RHO RR T
        rhob += ppb * P.rr * t;
        tb += ppb * rho * P.rr;
        // RHO = (S0 / (RR T))**(1/(1-GAMA))
        const double B = P.s0 / (P.rr * t);
        const double Bb = rhob * P.inv1mg * rho / B;
        s0b += Bb / (P.rr * t);
        tb -= Bb * B / t;
        // T = T0 - (U^2 + V^2) / (2 CP), U = |U_parent|, V = -V_parent
        t0b += tb;
        ub -= tb * u / P.cp;
        vb -= tb * v / P.cp;
        pb[WU] += ub * sgn(pw[WU]);
        pb[WV] -= vb;
    }
}

// ------------------------------------------------------------------ source terms

struct SrcWork {
    double dnr, yBD, yAC, xBD, xAC;
    double da[4], db[4];  // q r u v: A-C and B-D differences
    double ic1[4];        // 1 / C1 of the neighbours
    double GX[4], GY[4];  // DQX DRX DUX DVX / DQY DRY DUY DVY
    double rho, ri, amu, chi, ta, tb, fmu, sc, t1, t2, fr2, amut, dee, vbyy, divvel, sum, aor, pk, ratio, pw,
        x, sq, A5, s3, s5, ycc, den, T, idnr, irho, ia, itb, it2, iycc;
    bool pos, near, pkpos, selm;
};

// COMPUTE_SOURCE_TERMS (source_terms.f90:24-104) of one cell, keeping the intermediates
// its reverse needs.  nb[k][0..3] = U, V, C1, C5 of neighbour k; nx, ny its centroid.
TNS_HD void src_forward(const Params& P, const double nb[4][4], const double nx[4], const double ny[4], double rho,
                        double c5, double T, double Pc, double Vc, double ycc, SrcWork& s) {
    double f[4][4];  // q r u v per neighbour
    for (int k = 0; k < 4; k++) {
        f[0][k] = sqrt(nb[k][0] * nb[k][0] + nb[k][1] * nb[k][1]);
        s.ic1[k] = 1.0 / nb[k][2];
        f[1][k] = nb[k][3] * s.ic1[k];
        f[2][k] = nb[k][0];
        f[3][k] = nb[k][1];
    }
    s.yBD = ny[1] - ny[3];
    s.yAC = ny[0] - ny[2];
    s.xBD = nx[1] - nx[3];
    s.xAC = nx[0] - nx[2];
    s.dnr = s.xAC * s.yBD - s.xBD * s.yAC;
    s.idnr = 1.0 / s.dnr;
    for (int q = 0; q < 4; q++) {
        s.da[q] = f[q][0] - f[q][2];
        s.db[q] = f[q][1] - f[q][3];
        s.GX[q] = (s.da[q] * s.yBD - s.db[q] * s.yAC) * s.idnr;
        s.GY[q] = (-s.da[q] * s.xBD + s.db[q] * s.xAC) * s.idnr;
    }
    const double DQX = s.GX[0], DRX = s.GX[1], DUX = s.GX[2], DVX = s.GX[3];
    const double DQY = s.GY[0], DRY = s.GY[1], DUY = s.GY[2], DVY = s.GY[3];
    s.rho = rho;
    s.T = T;
    s.irho = 1.0 / rho;
    s.ri = c5 * s.irho;
    s.amu = amu_of(P, T);
    s.ia = 1.0 / (CMU * s.amu);
    s.chi = rho * s.ri * s.ia;
    const double X2 = s.chi * s.chi;
    s.ta = tanh(ALPHA_T * X2);
    s.tb = tanh(BETA_T * X2);
    s.itb = 1.0 / s.tb;
    s.fmu = s.ta * s.itb;
    s.sc = sqrt(s.chi);
    s.t1 = tanh(s.sc);
    s.t2 = tanh(s.chi * P.fr2k);
    s.it2 = 1.0 / s.t2;
    s.fr2 = s.t1 * s.it2;
    s.amut = s.fmu * rho * s.ri;
    const double phi = DQX * DRX + DQY * DRY;
    s.pos = phi > 0.0;
    s.dee = s.pos ? DRX * DRX + DRY * DRY : 0.0;
    s.ycc = ycc;
    s.iycc = 1.0 / ycc;
    s.near = ycc < YAXIS_THRESH;
    const double sxy = DUY + DVX;
    if (P.iaxis == 1) {
        s.vbyy = s.near ? DVY : Vc * s.iycc;
        s.divvel = DUX + DVY + s.vbyy;
        s.sum = DUX * DUX + DVY * DVY + s.vbyy * s.vbyy + DUX * DUX + DVY * DVY + s.vbyy * s.vbyy + sxy * sxy -
                P.div23 * s.divvel * s.divvel;
    } else {
        s.vbyy = 0.0;
        s.divvel = DUX + DVY;
        s.sum = DUX * DUX + DVY * DVY + DUX * DUX + DVY * DVY + sxy * sxy - P.div23 * s.divvel * s.divvel;
    }
    s.aor = s.amut * s.irho;
    const double pk0 = s.aor * s.sum;
    s.pkpos = pk0 >= 0.0;
    s.pk = s.pkpos ? pk0 : 0.0;
    const double thr = AMU_THRESH * s.amu;
    s.selm = s.amut >= thr;
    s.den = s.selm ? s.amut : thr;
    s.ratio = s.selm ? 1.0 : s.amut / s.den;  // x / x = 1 exactly
    s.pw = powi(s.ratio, P.npseudo);
    s.x = s.ri * s.pk;
    s.sq = s.x > 0.0 ? sqrt(s.x) : 0.0;
    s.A5 = rho * (CONST1 - CONST2 * s.fr2) * s.sq - rho * CONST3 * s.dee;
    s.s5 = s.A5 * s.pw;
    s.s3 = 0.0;
    if (P.iaxis == 1) {
        const double ttt = (s.amu + s.amut) * (s.vbyy + s.vbyy - P.div23 * s.divvel);
        s.s3 = (Pc - ttt) * s.iycc;
    }
}

struct SrcBar {
    double c1, c5, t, p, v, ycc;  // the cell itself
    double nb[4][4];              // neighbour k: U, V, C1, C5
    double nx[4], ny[4];          // neighbour k's centroid
};

// Reverse of src_forward for the adjoints s3b, s5b of SOURCE3, SOURCE5.
TNS_HD void src_reverse(const Params& P, const SrcWork& s, const double nb[4][4], double Vc, double s3b, double s5b,
                        SrcBar& b) {
    double rhob = 0.0, rib = 0.0, amub = 0.0, amutb = 0.0, chib = 0.0, divb = 0.0, vbyyb = 0.0;
    double GXb[4] = {0.0, 0.0, 0.0, 0.0}, GYb[4] = {0.0, 0.0, 0.0, 0.0};
    b.p = 0.0; b.v = 0.0; b.ycc = 0.0;
    const double pwb = s5b * s.A5, A5b = s5b * s.pw;
    rhob += A5b * ((CONST1 - CONST2 * s.fr2) * s.sq - CONST3 * s.dee);
    const double fr2b = -A5b * s.rho * CONST2 * s.sq;
    const double sqb = A5b * s.rho * (CONST1 - CONST2 * s.fr2);
    const double deeb = -A5b * s.rho * CONST3;
    const double xb = s.x > 0.0 ? sqb / (2.0 * s.sq) : 0.0;
    rib += xb * s.pk;
    const double pkb = xb * s.ri;
    if (P.iaxis == 1) {
        b.p = s3b * s.iycc;
        const double tttb = -b.p;
        b.ycc -= s3b * s.s3 * s.iycc;
        const double fac = s.vbyy + s.vbyy - P.div23 * s.divvel;
        amub += tttb * fac;
        amutb += tttb * fac;
        vbyyb += 2.0 * tttb * (s.amu + s.amut);
        divb -= P.div23 * tttb * (s.amu + s.amut);
    }
    const double pk0b = s.pkpos ? pkb : 0.0;
    const double aorb = pk0b * s.sum, sumb = pk0b * s.aor;
    amutb += aorb * s.irho;
    rhob -= aorb * s.aor * s.irho;
    const double DUX = s.GX[2], DVX = s.GX[3], DRX = s.GX[1], DUY = s.GY[2], DVY = s.GY[3], DRY = s.GY[1];
    const double sxy = DUY + DVX;
    GXb[2] += sumb * 4.0 * DUX;
    GYb[3] += sumb * 4.0 * DVY;
    GYb[2] += sumb * 2.0 * sxy;
    GXb[3] += sumb * 2.0 * sxy;
    divb -= sumb * 2.0 * P.div23 * s.divvel;
    if (P.iaxis == 1) vbyyb += sumb * 4.0 * s.vbyy;
    GXb[2] += divb;
    GYb[3] += divb;
    if (P.iaxis == 1) {
        vbyyb += divb;
        if (s.near) {
            GYb[3] += vbyyb;
        } else {
            b.v = vbyyb * s.iycc;
            b.ycc -= vbyyb * s.vbyy * s.iycc;
        }
    }
    if (s.pos) {
        GXb[1] += 2.0 * deeb * DRX;
        GYb[1] += 2.0 * deeb * DRY;
    }
    // (mu_t / max(mu_t, 1e-3 mu))**NPSEUDO: the selected branch mu_t / mu_t is constant
    const int np = P.npseudo;
    double ratiob = 0.0;
    if (np > 0) ratiob = pwb * (double)np * powi(s.ratio, np - 1);
    else if (np < 0) ratiob = -pwb * (double)(-np) / powi(s.ratio, 1 - np);
    if (!s.selm) {
        amutb += ratiob / s.den;
        amub -= ratiob * s.amut / (s.den * s.den) * AMU_THRESH;
    }
    const double fmub = amutb * s.rho * s.ri;
    rhob += amutb * s.fmu * s.ri;
    rib += amutb * s.fmu * s.rho;
    chib += fmub * (ALPHA_T * (1.0 - s.ta * s.ta) - s.fmu * BETA_T * (1.0 - s.tb * s.tb)) * s.itb * 2.0 * s.chi;
    chib += fr2b * ((1.0 - s.t1 * s.t1) * 0.5 / s.sc - s.fr2 * (1.0 - s.t2 * s.t2) * P.fr2k) * s.it2;
    rhob += chib * s.ri * s.ia;
    rib += chib * s.rho * s.ia;
    amub -= chib * s.chi * s.ia * CMU;
    b.t = amub * 0.6 * s.amu / s.T;  // AMU = SUTH sqrt(AMOL) T**0.6
    b.c5 = rib * s.irho;
    rhob -= rib * s.ri * s.irho;
    b.c1 = rhob;
    // gradients of q r u v (q only enters the switch PHI > 0: no derivative)
    double dnrb = 0.0, xACb = 0.0, xBDb = 0.0, yACb = 0.0, yBDb = 0.0;
    double fb[4][4];  // [q][k]
    for (int q = 0; q < 4; q++)
        for (int k = 0; k < 4; k++) fb[q][k] = 0.0;
    for (int q = 1; q < 4; q++) {
        const double gx = GXb[q], gy = GYb[q];
        if (gx == 0.0 && gy == 0.0) continue;
        const double dab = (gx * s.yBD - gy * s.xBD) * s.idnr;
        const double dbb = (-gx * s.yAC + gy * s.xAC) * s.idnr;
        fb[q][0] += dab;
        fb[q][2] -= dab;
        fb[q][1] += dbb;
        fb[q][3] -= dbb;
        yBDb += gx * s.da[q] * s.idnr;
        yACb -= gx * s.db[q] * s.idnr;
        xBDb -= gy * s.da[q] * s.idnr;
        xACb += gy * s.db[q] * s.idnr;
        dnrb -= (gx * s.GX[q] + gy * s.GY[q]) * s.idnr;
    }
    xACb += dnrb * s.yBD;
    yBDb += dnrb * s.xAC;
    xBDb -= dnrb * s.yAC;
    yACb -= dnrb * s.xBD;
    b.nx[0] = xACb; b.nx[2] = -xACb; b.nx[1] = xBDb; b.nx[3] = -xBDb;
    b.ny[0] = yACb; b.ny[2] = -yACb; b.ny[1] = yBDb; b.ny[3] = -yBDb;
    for (int k = 0; k < 4; k++) {
        const double r = nb[k][3] * s.ic1[k];
        b.nb[k][0] = fb[2][k];
        b.nb[k][1] = fb[3][k];
        b.nb[k][3] = fb[1][k] * s.ic1[k];
        b.nb[k][2] = -fb[1][k] * r * s.ic1[k];
    }
    (void)Vc;
}

// ------------------------------------------------------------------ stage reverse

// Reverse of UPDATE_SOLUTION(alpha) and COMPUTE_RESIDUAL for one cell (residual.f90:
// 23-83): recomputes R (flux + sources) of the stage input, takes the C5 clip branch of
// the forward, and writes the residual adjoint (gbar), the source adjoints for the
// neighbours (srcn, srcg) and the cell (wself); accumulates the adjoints of Q_n, D, VIS
// and DT.
// TNS_ADJ_SRC_RECOMPUTE: the stage reverse evaluates the source terms twice (values for
// the residual, then intermediates for the reverse) instead of keeping them live across
// the update: spill-free at 166 registers, 414 vs 425 us per 512 x 192 transient step.
#ifndef TNS_ADJ_SRC_RECOMPUTE
#define TNS_ADJ_SRC_RECOMPUTE 1
#endif

TNS_HD void s1_point(const AdjArgs& a, long long cell) {
    const int i = (int)(cell / a.nj), j = (int)(cell % a.nj);
    const Params& P = a.P;
    CellGeo g;
    cell_geo(a, i, j, g);
    const long long ps = padi(a, i, j);
    long long pn[4];
    for (int k = 0; k < 4; k++) pn[k] = padi(a, i + di_of(k), j + dj_of(k));
    // inviscid residual
    double R[5];
    for (int m = 0; m < 5; m++) {
        const double FI = wv(a, WF + m, ps), GI = wv(a, WG + m, ps);
        double acc = (FI + wv(a, WF + m, pn[0])) * g.sx[0] + (GI + wv(a, WG + m, pn[0])) * g.sy[0];
        for (int k = 1; k < 4; k++)
            acc = acc + (FI + wv(a, WF + m, pn[k])) * g.sx[k] + (GI + wv(a, WG + m, pn[k])) * g.sy[k];
        R[m] = 0.5 * acc;
    }
    // sources
    double nb[4][4], nx[4], ny[4];
    for (int k = 0; k < 4; k++) {
        nb[k][0] = wv(a, WU, pn[k]);
        nb[k][1] = wv(a, WV, pn[k]);
        nb[k][2] = wv(a, WC1, pn[k]);
        nb[k][3] = wv(a, WC5, pn[k]);
        slot_centroid(a, i + di_of(k), j + dj_of(k), nx[k], ny[k]);
    }
    const double Vc = wv(a, WV, ps);
    double src5, src3;
#if TNS_ADJ_SRC_RECOMPUTE
    {
        SrcWork s0;  // only SOURCE3/5 here; the reverse recomputes the intermediates
        src_forward(P, nb, nx, ny, wv(a, WC1, ps), wv(a, WC5, ps), wv(a, WT, ps), wv(a, WP, ps), Vc, g.yc, s0);
        src5 = s0.s5;
        src3 = s0.s3;
    }
#else
    SrcWork s;
    src_forward(P, nb, nx, ny, wv(a, WC1, ps), wv(a, WC5, ps), wv(a, WT, ps), wv(a, WP, ps), Vc, g.yc, s);
    src5 = s.s5;
    src3 = s.s3;
#endif
    R[4] = R[4] - g.vol * src5;
    if (P.iaxis == 1) R[2] = R[2] - g.vol * src3;
    // update and clip
    const double DT = P.local ? a.dt[cell] : *a.dtmin;
    const double dtv = a.alpha * (DT / g.vol);
    double qo[5], dd[5], vv[5], res[5], lb[5], lh[5];
    for (int m = 0; m < 5; m++) {
        qo[m] = a.qold[m * a.ncell + cell];
        dd[m] = a.d[m * a.ncell + cell];
        vv[m] = m ? a.vis[(m - 1) * a.ncell + cell] : 0.0;
        res[m] = R[m] - vv[m] - dd[m];
        lb[m] = a.lam_in[m * a.ncell + cell];
        if (!a.first && in_band(a, i, j)) lb[m] += a.lamg[m * a.ncell + cell];
        lh[m] = lb[m];
    }
    const double n0 = qo[0] - dtv * res[0];
    const double n4 = qo[4] - dtv * CFLTURB * res[4];
    double rtolb = 0.0;
    if (P.rtol >= n4 / n0) {  // C5 = C1 * RTOL
        lh[0] += lb[4] * P.rtol;
        rtolb += lb[4] * n0;
        lh[4] = 0.0;
    }
    double coef[5], dtvb = 0.0;
    for (int m = 0; m < 5; m++) {
        coef[m] = m == 4 ? dtv * CFLTURB : dtv;
        dtvb -= (m == 4 ? CFLTURB : 1.0) * res[m] * lh[m];
    }
    double gb[5];
    for (int m = 0; m < 5; m++) {
        gb[m] = -coef[m] * lh[m];
        a.gbar[m * a.npad + ps] = gb[m];
        const double cl = coef[m] * lh[m];
        if (a.first) {
            a.lam_old[m * a.ncell + cell] = lh[m];
            a.dbar[m * a.ncell + cell] = cl;
            if (m) a.visbar[(m - 1) * a.ncell + cell] = cl;
        } else {
            a.lam_old[m * a.ncell + cell] += lh[m];
            a.dbar[m * a.ncell + cell] += cl;
            if (m) a.visbar[(m - 1) * a.ncell + cell] += cl;
        }
    }
    const double dtbyvolb = a.alpha * dtvb;
    const double ivol = 1.0 / g.vol;
    const double dtb = dtbyvolb * ivol;
    double volb = -dtb * DT * ivol;
    if (a.first) a.dtbar[cell] = dtb;
    else a.dtbar[cell] += dtb;
    // source reverse: R5 -= VOL*SOURCE5, R3 -= VOL*SOURCE3
    const double s5b = -g.vol * gb[4];
    const double s3b = P.iaxis == 1 ? -g.vol * gb[2] : 0.0;
    volb -= src5 * gb[4];
    if (P.iaxis == 1) volb -= src3 * gb[2];
#if TNS_ADJ_SRC_RECOMPUTE
    for (int k = 0; k < 4; k++) {
        nb[k][0] = wv(a, WU, pn[k]);
        nb[k][1] = wv(a, WV, pn[k]);
        nb[k][2] = wv(a, WC1, pn[k]);
        nb[k][3] = wv(a, WC5, pn[k]);
        slot_centroid(a, i + di_of(k), j + dj_of(k), nx[k], ny[k]);
    }
    SrcWork s;
    src_forward(P, nb, nx, ny, wv(a, WC1, ps), wv(a, WC5, ps), wv(a, WT, ps), wv(a, WP, ps), Vc, g.yc, s);
#endif
    SrcBar b;
    src_reverse(P, s, nb, Vc, s3b, s5b, b);
    a.wself[0 * a.ncell + cell] = b.t;
    a.wself[1 * a.ncell + cell] = b.p;
    a.wself[2 * a.ncell + cell] = b.v;
    a.wself[3 * a.ncell + cell] = b.c1;
    a.wself[4 * a.ncell + cell] = b.c5;
    for (int k = 0; k < 4; k++) {
        for (int q = 0; q < 4; q++) a.srcn[(k * 4 + q) * a.ncell + cell] = b.nb[k][q];
        a.srcg[(k * 2 + 0) * a.ncell + cell] = b.nx[k];
        a.srcg[(k * 2 + 1) * a.ncell + cell] = b.ny[k];
    }
    if (a.sens) a.rtolc[cell] += rtolb;
    if (a.geo) {  // (the face-vector part of the residual reverse: geo_point)
        a.volbar[cell] += volb;
        a.ycbar[ps] += b.ycc;
    }
}

// Adjoint rows of the ghost on the parent's face k: flux part of the parent's residual,
// the parent's source part, and (stage 1) the viscous part.
TNS_HD void ghost_bar(const AdjArgs& a, long long pcell, long long pps, long long gps, int k, const CellGeo& pg,
                      double gb[NWROW]) {
    for (int r = 0; r < NWROW; r++) gb[r] = 0.0;
    for (int m = 0; m < 5; m++) {
        const double gm = a.gbar[m * a.npad + pps];
        gb[WF + m] = 0.5 * gm * pg.sx[k];
        gb[WG + m] = 0.5 * gm * pg.sy[k];
    }
    gb[WU] += a.srcn[(k * 4 + 0) * a.ncell + pcell];
    gb[WV] += a.srcn[(k * 4 + 1) * a.ncell + pcell];
    gb[WC1] += a.srcn[(k * 4 + 2) * a.ncell + pcell];
    gb[WC5] += a.srcn[(k * 4 + 3) * a.ncell + pcell];
    if (a.stage1) {
        gb[WU] += a.wvisc[0 * a.npad + gps];
        gb[WV] += a.wvisc[1 * a.npad + gps];
        gb[WT] += a.wvisc[2 * a.npad + gps];
        gb[WC1] += a.wvisc[3 * a.npad + gps];
        gb[WC5] += a.wvisc[4 * a.npad + gps];
    }
}

TNS_HD void load_rows(const AdjArgs& a, long long ps, double r[NWROW]) {
    for (int q = 0; q < NWROW; q++) r[q] = wv(a, q, ps);
}

// Gathers the adjoint of one cell's field-set rows from the residual (flux), the
// sources (its own and its neighbours') and, in stage 1, the viscous flux, and pulls it
// back to the cell's conservative state: the adjoint of the stage input (stages 2-4) or
// a part of the adjoint of Q_n (stage 1).  Ghost contributions follow in s3g_point.
TNS_HD void s3_point(const AdjArgs& a, long long cell) {
    const int i = (int)(cell / a.nj), j = (int)(cell % a.nj);
    CellGeo g;
    cell_geo(a, i, j, g);
    const long long ps = padi(a, i, j);
    double wb[NWROW];
    for (int r = 0; r < NWROW; r++) wb[r] = 0.0;
    double xcb = 0.0, ycb = 0.0;
    for (int m = 0; m < 5; m++) {
        const double gc = a.gbar[m * a.npad + ps];
        double fb = 0.0, gg = 0.0;
        for (int k = 0; k < 4; k++) {
            const double gn = a.gbar[m * a.npad + padi(a, i + di_of(k), j + dj_of(k))];
            fb += g.sx[k] * (gc - gn);
            gg += g.sy[k] * (gc - gn);
        }
        wb[WF + m] = 0.5 * fb;
        wb[WG + m] = 0.5 * gg;
    }
    for (int k = 0; k < 4; k++) {
        const int ni_ = i + di_of(k), nj_ = j + dj_of(k);
        if (!is_cell(a, ni_, nj_)) continue;
        const long long nc = cell_of(a, ni_, nj_);
        const int kk = (k + 2) & 3;
        wb[WU] += a.srcn[(kk * 4 + 0) * a.ncell + nc];
        wb[WV] += a.srcn[(kk * 4 + 1) * a.ncell + nc];
        wb[WC1] += a.srcn[(kk * 4 + 2) * a.ncell + nc];
        wb[WC5] += a.srcn[(kk * 4 + 3) * a.ncell + nc];
        xcb += a.srcg[(kk * 2 + 0) * a.ncell + nc];
        ycb += a.srcg[(kk * 2 + 1) * a.ncell + nc];
    }
    wb[WT] += a.wself[0 * a.ncell + cell];
    wb[WP] += a.wself[1 * a.ncell + cell];
    wb[WV] += a.wself[2 * a.ncell + cell];
    wb[WC1] += a.wself[3 * a.ncell + cell];
    wb[WC5] += a.wself[4 * a.ncell + cell];
    if (a.stage1) {
        wb[WU] += a.wvisc[0 * a.npad + ps];
        wb[WV] += a.wvisc[1 * a.npad + ps];
        wb[WT] += a.wvisc[2 * a.npad + ps];
        wb[WC1] += a.wvisc[3 * a.npad + ps];
        wb[WC5] += a.wvisc[4 * a.npad + ps];
    }
    double q[5], qb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int m = 0; m < 5; m++) q[m] = a.qin[m * a.ncell + cell];
    prim_adj(a.P, q, wb, qb);
    for (int m = 0; m < 5; m++) {
        if (a.stage1) a.lam_old[m * a.ncell + cell] += qb[m];
        else a.lam_out[m * a.ncell + cell] = qb[m];
    }
    if (a.geo) {
        a.xcbar[ps] += xcb;
        a.ycbar[ps] += ycb;
    }
}

// Cells within two of the boundary, the ones a ghost can have as parent or opposite cell:
// rows {0, 1, NI-2, NI-1} at every j, then columns {0, 1, NJ-2, NJ-1} of rows 2..NI-3.
TNS_HD long long band_count(const AdjArgs& a) {
    const long long nr = a.ni >= 4 ? 4 : a.ni, nc = a.nj >= 4 ? 4 : a.nj;
    return nr * a.nj + (a.ni >= 5 ? (long long)(a.ni - 4) * nc : 0);
}

TNS_HD void band_cell(const AdjArgs& a, long long idx, int& i, int& j) {
    const int nr = a.ni >= 4 ? 4 : a.ni, nc = a.nj >= 4 ? 4 : a.nj;
    if (idx < (long long)nr * a.nj) {
        const int r = (int)(idx / a.nj);
        i = a.ni >= 4 ? (r < 2 ? r : a.ni - 4 + r) : r;
        j = (int)(idx % a.nj);
    } else {
        const long long t = idx - (long long)nr * a.nj;
        const int c = (int)(t % nc);
        i = 2 + (int)(t / nc);
        j = a.nj >= 4 ? (c < 2 ? c : a.nj - 4 + c) : c;
    }
}

// The ghost part of the stage gather for one boundary-band cell: the adjoint of each
// ghost whose parent this cell is (all types) or whose opposite cell it is (type 3),
// pulled back through APPLY_BOUNDARY and this cell's primitives into lamg (prim_adj is
// linear in the row adjoint, so this part adds to s3_point's; it runs beside it, and the
// next stage -- or final_point -- adds it).
TNS_HD void s3g_point(const AdjArgs& a, long long idx) {
    int i, j;
    band_cell(a, idx, i, j);
    const long long cell = cell_of(a, i, j), ps = padi(a, i, j);
    double wb[NWROW], pw[NWROW], gw[NWROW], ow[NWROW], gb[NWROW];
    for (int r = 0; r < NWROW; r++) wb[r] = 0.0;
    double t0b = 0.0, s0b = 0.0;
    bool any = false;
    CellGeo g;
    cell_geo(a, i, j, g);
    load_rows(a, ps, pw);
    for (int k = 0; k < 4; k++) {
        // the ghost on this cell's face k
        const int gi = i + di_of(k), gj = j + dj_of(k);
        if (is_cell(a, gi, gj)) continue;
        any = true;
        int along = 0;
        const int side = ghost_side(a, gi, gj, along);
        const int type = a.M.gtype[a.M.ghost_index(side, along)];
        const long long gps = padi(a, gi, gj);
        ghost_bar(a, cell, ps, gps, k, g, gb);
        load_rows(a, gps, gw);
        if (type == 3) load_rows(a, padi(a, i - di_of(k), j - dj_of(k)), ow);
        else load_rows(a, ps, ow);
        double dummy[NWROW];
        for (int r = 0; r < NWROW; r++) dummy[r] = 0.0;
        const int gidx = a.M.ghost_index(side, along);
        GhostGeo gg{a.M.gyc[gidx], g.yc, g.sx[k], g.sy[k], type == 6 ? a.gport[gidx] : 0.0, a.M.ginj[gidx]};
        GhostGeoBar gbr{0.0, 0.0, 0.0, 0.0, 0.0};
        ghost_adj(a.P, type, gw, pw, ow, gb, wb, dummy, t0b, s0b, gg, gbr);
        if (type == 6) a.gportb[gidx] = gbr.gport;
        if (a.geo) {
            a.xcbar[gps] += a.srcg[(k * 2 + 0) * a.ncell + cell];
            a.ycbar[gps] += a.srcg[(k * 2 + 1) * a.ncell + cell] + gbr.ycg;
            if (type == 6) {  // parent face vector and centroid: added by geo_point
                a.portacc[0 * a.M.nghosts() + gidx] += gbr.psx;
                a.portacc[1 * a.M.nghosts() + gidx] += gbr.psy;
                a.portacc[2 * a.M.nghosts() + gidx] += gbr.ycp;
            }
        }
    }
    for (int k = 0; k < 4; k++) {
        // a type-3 ghost whose opposite cell this is: parent one step towards side k
        const int pi = i + di_of(k), pj = j + dj_of(k);
        const int gi = pi + di_of(k), gj = pj + dj_of(k);
        if (!is_cell(a, pi, pj) || is_cell(a, gi, gj)) continue;
        int along = 0;
        const int side = ghost_side(a, gi, gj, along);
        if (a.M.gtype[a.M.ghost_index(side, along)] != 3) continue;
        any = true;
        const long long pc = cell_of(a, pi, pj), pps = padi(a, pi, pj), gps = padi(a, gi, gj);
        CellGeo pg;
        cell_geo(a, pi, pj, pg);
        ghost_bar(a, pc, pps, gps, k, pg, gb);
        double par[NWROW], pbd[NWROW], obar[NWROW];
        load_rows(a, pps, par);
        load_rows(a, gps, gw);
        for (int r = 0; r < NWROW; r++) pbd[r] = obar[r] = 0.0;
        double t0d = 0.0, s0d = 0.0;
        const GhostGeo gg{0.0, 0.0, 0.0, 0.0, 0.0, 1.0};
        GhostGeoBar gbd{0.0, 0.0, 0.0, 0.0, 0.0};
        ghost_adj(a.P, 3, gw, par, pw, gb, pbd, obar, t0d, s0d, gg, gbd);
        wb[WU] += obar[WU];
        wb[WV] += obar[WV];
        wb[WT] += obar[WT];
        wb[WP] += obar[WP];
    }
    double qb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (any) {
        double q[5];
        for (int m = 0; m < 5; m++) q[m] = a.qin[m * a.ncell + cell];
        prim_adj(a.P, q, wb, qb);
    }
    for (int m = 0; m < 5; m++) a.lamg[m * a.ncell + cell] = qb[m];
    if (a.sens) {
        a.t0bar[cell] += t0b;
        a.s0bar[cell] += s0b;
    }
}

// ------------------------------------------------------------------ viscous reverse

// Slot values of the viscous flux: u v t rho r (r = C5 / C1).
TNS_HD void visc_vals(const AdjArgs& a, long long ps, double v[5]) {
    v[0] = wv(a, WU, ps);
    v[1] = wv(a, WV, ps);
    v[2] = wv(a, WT, ps);
    v[3] = wv(a, WC1, ps);
    v[4] = wv(a, WC5, ps) / v[3];
}

// NODAL_AVERAGE (viscous.f90:40-124) of node (a_, b_): cells in id order, then the
// adjacent ghosts in bc.in order; a type-4 ghost zeroes VN, a type-5 ghost zeroes UN, VN
// and sets RN = RTOLERANCE*RTRED, each after adding its own values.  Also records which
// positions still contribute to each component.
TNS_HD void v0_point(const AdjArgs& a, long long node) {
    const int na = (int)(node / (a.nj + 1)), nb = (int)(node % (a.nj + 1));
    double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    int cnt = 0, mask = 0, reset_r = 0;
    int gk[2] = {0, 0}, gg[2] = {0, 0}, ng = 0;
    for (int k = 0; k < 4; k++) {
        const int pi = na - 1 + (k >> 1), pj = nb - 1 + (k & 1);
        if (is_cell(a, pi, pj)) {
            double v[5];
            visc_vals(a, padi(a, pi, pj), v);
            for (int c = 0; c < 5; c++) s[c] = s[c] + v[c];
            cnt++;
            mask |= 7 << (3 * k);
        } else {
            int along = 0;
            const int side = ghost_side(a, pi, pj, along);
            if (side) {
                gk[ng] = k;
                gg[ng] = a.M.ghost_index(side, along);
                ng++;
            }
        }
    }
    if (ng == 2 && a.M.grank[gg[1]] < a.M.grank[gg[0]]) {
        int t = gk[0]; gk[0] = gk[1]; gk[1] = t;
        t = gg[0]; gg[0] = gg[1]; gg[1] = t;
    }
    for (int q = 0; q < ng; q++) {
        const int k = gk[q];
        const int pi = na - 1 + (k >> 1), pj = nb - 1 + (k & 1);
        double v[5];
        visc_vals(a, padi(a, pi, pj), v);
        for (int c = 0; c < 5; c++) s[c] = s[c] + v[c];
        cnt++;
        mask |= 7 << (3 * k);
        const int type = a.M.gtype[gg[q]];
        if (type == 4) {
            s[1] = 0.0;
            for (int kk = 0; kk < 4; kk++) mask &= ~(2 << (3 * kk));
        } else if (type == 5) {
            s[0] = 0.0;
            s[1] = 0.0;
            s[4] = a.P.rtol_rtred;
            reset_r = 1;
            for (int kk = 0; kk < 4; kk++) mask &= ~(7 << (3 * kk));
        }
    }
    double avg[NNA];
    for (int c = 0; c < 5; c++) avg[c] = s[c] / (double)cnt;
    avg[NA_R0] = avg[4];
    const int floor_ = a.P.rtol >= avg[4];
    if (floor_) avg[4] = a.P.rtol;
    for (int c = 0; c < NNA; c++) a.navg[c * a.nnode + node] = avg[c];
    a.ninfo[node] = cnt | (mask << NI_MASK) | (reset_r << NI_RESET) | (floor_ << NI_FLOOR);
}

// Reverse of one viscous face (viscous.f90:130-217) weighted by w[0..3] (the adjoint of
// the flux it adds to VISU, VISV, VIST, VISR).  out: NVF values (see VF_*).
TNS_HD void visc_face_adj(const Params& P, const FaceIn& f, const double w[4], double* out, long long stride) {
    const double ybd = f.yb - f.yd, yac = f.ya - f.yc, xbd = f.xb - f.xd, xac = f.xa - f.xc;
    const double dnr = xac * ybd - xbd * yac, idnr = 1.0 / dnr;
    const double A[5] = {f.ua, f.va, f.ta, f.rhoa, f.ra}, B[5] = {f.ub, f.vb, f.tb, f.rhob, f.rb};
    const double C[5] = {f.uc, f.vc, f.tc, f.rhoc, f.rc}, D[5] = {f.ud, f.vd, f.td, f.rhod, f.rd};
    double da[5], db[5], GX[5], GY[5];
    for (int q = 0; q < 5; q++) {
        da[q] = A[q] - C[q];
        db[q] = B[q] - D[q];
        GX[q] = (da[q] * ybd - db[q] * yac) * idnr;
        GY[q] = (-da[q] * xbd + db[q] * xac) * idnr;
    }
    double AV[5];
    for (int q = 0; q < 5; q++) AV[q] = 0.25 * (A[q] + B[q] + C[q] + D[q]);
    const double DUX = GX[0], DVX = GX[1], DTX = GX[2], DRX = GX[4];
    const double DUY = GY[0], DVY = GY[1], DTY = GY[2], DRY = GY[4];
    const double UAVG = AV[0], VAVG = AV[1], TAVG = AV[2], RHOAVG = AV[3], RAVG = AV[4];
    double YAVG = 0.0, VBYY = 0.0, DIVVEL;
    bool near = false;
    if (P.iaxis == 1) {
        YAVG = 0.5 * (f.yb + f.yd);
        near = YAVG < YAXIS_THRESH;
        VBYY = near ? DVY : VAVG / YAVG;
        DIVVEL = DUX + DVY + VBYY;
    } else {
        DIVVEL = DUX + DVY;
    }
    const double AMU = amu_of(P, TAVG);
    const double AK = AMU * P.cp_pr;
    const double iac = 1.0 / (AMU * CMU);
    const double CHI = RHOAVG * RAVG * iac;
    const double X2 = CHI * CHI;
    const double ta = tanh(ALPHA_T * X2), tb = tanh(BETA_T * X2), itb = 1.0 / tb;
    const double FMU = ta * itb;
    const double AMUT = RHOAVG * RAVG * FMU;
    const double AKT = AMUT * P.cp_prt;
    const double AMUEFF = AMU + AMUT, AKEFF = AK + AKT;
    const double TXX = AMUEFF * (DUX + DUX - P.div23 * DIVVEL);
    const double TYY = AMUEFF * (DVY + DVY - P.div23 * DIVVEL);
    const double TXY = AMUEFF * (DUY + DVX);
    const double QXX = UAVG * TXX + VAVG * TXY + AKEFF * DTX;
    const double QYY = UAVG * TXY + VAVG * TYY + AKEFF * DTY;
    // dF/dSX, dF/dSY
    out[(VF_CX + 0) * stride] = TXX; out[(VF_CX + 1) * stride] = TXY;
    out[(VF_CX + 2) * stride] = QXX; out[(VF_CX + 3) * stride] = AMUEFF * DRX;
    out[(VF_CY + 0) * stride] = TXY; out[(VF_CY + 1) * stride] = TYY;
    out[(VF_CY + 2) * stride] = QYY; out[(VF_CY + 3) * stride] = AMUEFF * DRY;
    // reverse
    const double QXXb = w[2] * f.sx, QYYb = w[2] * f.sy;
    const double TXXb = w[0] * f.sx + QXXb * UAVG;
    const double TXYb = w[0] * f.sy + w[1] * f.sx + QXXb * VAVG + QYYb * UAVG;
    const double TYYb = w[1] * f.sy + QYYb * VAVG;
    double AVb[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, GXb[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, GYb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    AVb[0] = QXXb * TXX + QYYb * TXY;
    AVb[1] = QXXb * TXY + QYYb * TYY;
    const double AKEFFb = QXXb * DTX + QYYb * DTY;
    GXb[2] = QXXb * AKEFF;
    GYb[2] = QYYb * AKEFF;
    const double AMUEFFb = w[3] * (DRX * f.sx + DRY * f.sy) + TXXb * (DUX + DUX - P.div23 * DIVVEL) +
                           TYYb * (DVY + DVY - P.div23 * DIVVEL) + TXYb * (DUY + DVX);
    GXb[4] = w[3] * AMUEFF * f.sx;
    GYb[4] = w[3] * AMUEFF * f.sy;
    GXb[0] = 2.0 * TXXb * AMUEFF;
    GYb[1] = 2.0 * TYYb * AMUEFF;
    GYb[0] = TXYb * AMUEFF;
    GXb[1] = TXYb * AMUEFF;
    const double DIVb = -P.div23 * AMUEFF * (TXXb + TYYb);
    GXb[0] += DIVb;
    GYb[1] += DIVb;
    double YAVGb = 0.0;
    if (P.iaxis == 1) {
        if (near) {
            GYb[1] += DIVb;
        } else {
            AVb[1] += DIVb / YAVG;
            YAVGb = -DIVb * VBYY / YAVG;
        }
    }
    double AMUb = AMUEFFb + AKEFFb * P.cp_pr;
    const double AMUTb = AMUEFFb + AKEFFb * P.cp_prt;
    AVb[3] += AMUTb * RAVG * FMU;
    AVb[4] += AMUTb * RHOAVG * FMU;
    const double FMUb = AMUTb * RHOAVG * RAVG;
    const double CHIb = FMUb * (ALPHA_T * (1.0 - ta * ta) - FMU * BETA_T * (1.0 - tb * tb)) * itb * 2.0 * CHI;
    AVb[3] += CHIb * RAVG * iac;
    AVb[4] += CHIb * RHOAVG * iac;
    AMUb -= CHIb * CHI * iac * CMU;
    AVb[2] += AMUb * 0.6 * AMU / TAVG;
    double Ab[5], Bb[5], Cb[5], Db[5];
    for (int q = 0; q < 5; q++) Ab[q] = Bb[q] = Cb[q] = Db[q] = 0.25 * AVb[q];
    double dnrb = 0.0, ybdb = 0.0, yacb = 0.0, xbdb = 0.0, xacb = 0.0;
    for (int q = 0; q < 5; q++) {
        const double gx = GXb[q], gy = GYb[q];
        if (gx == 0.0 && gy == 0.0) continue;
        const double dab = (gx * ybd - gy * xbd) * idnr;
        const double dbb = (-gx * yac + gy * xac) * idnr;
        Ab[q] += dab;
        Cb[q] -= dab;
        Bb[q] += dbb;
        Db[q] -= dbb;
        ybdb += gx * da[q] * idnr;
        yacb -= gx * db[q] * idnr;
        xbdb -= gy * da[q] * idnr;
        xacb += gy * db[q] * idnr;
        dnrb -= (gx * GX[q] + gy * GY[q]) * idnr;
    }
    xacb += dnrb * ybd;
    ybdb += dnrb * xac;
    xbdb -= dnrb * yac;
    yacb -= dnrb * xbd;
    for (int q = 0; q < 5; q++) {
        out[(VF_A + q) * stride] = Ab[q];
        out[(VF_C + q) * stride] = Cb[q];
        out[(VF_B + q) * stride] = Bb[q];
        out[(VF_D + q) * stride] = Db[q];
    }
    out[VF_XA * stride] = xacb;
    out[VF_XC * stride] = -xacb;
    out[VF_YA * stride] = yacb;
    out[VF_YC * stride] = -yacb;
    out[VF_XB * stride] = xbdb;
    out[VF_XD * stride] = -xbdb;
    out[VF_YB * stride] = ybdb + 0.5 * YAVGb;
    out[VF_YD * stride] = -ybdb + 0.5 * YAVGb;
}

// One viscous face, evaluated once in the orientation the primal kernel uses: i-faces
// (f < nif) as face 2 of cell (i-1, j) (face 4 of (0, j) on the boundary), j-faces as
// face 3 of (i, j-1) (face 1 of (i, 0)).  The neighbour's own copy of an interior face is
// the same flux with the opposite sign, so the face's weight is VIS_bar(A) - VIS_bar(C).
TNS_HD void v1_point(const AdjArgs& a, long long f) {
    int ia, ja, ic, jc;           // cell A and neighbour C
    long long nbn, ndn;           // nodes B and D
    double* out;
    long long stride;
    const long long nw = a.nj + 1;
    if (f < a.nif) {
        const int i = (int)(f / a.nj), j = (int)(f % a.nj);
        const long long lo = (long long)i * nw + j, hi = lo + 1;
        if (i == 0) { ia = 0; ja = j; ic = -1; jc = j; nbn = hi; ndn = lo; }
        else { ia = i - 1; ja = j; ic = i; jc = j; nbn = lo; ndn = hi; }
        out = a.vfi + f;
        stride = a.nif;
    } else {
        const long long g = f - a.nif;
        const int i = (int)(g / nw), j = (int)(g % nw);
        const long long L = (long long)i * nw + j, Rn = L + nw;
        if (j == 0) { ia = i; ja = 0; ic = i; jc = -1; nbn = L; ndn = Rn; }
        else { ia = i; ja = j - 1; ic = i; jc = j; nbn = Rn; ndn = L; }
        out = a.vfj + g;
        stride = a.njf;
    }
    FaceIn fi;
    fi.xb = a.M.x[nbn]; fi.yb = a.M.y[nbn];
    fi.xd = a.M.x[ndn]; fi.yd = a.M.y[ndn];
    if (a.P.iaxis == 1) {
        fi.sx = (fi.yd - fi.yb) * (fi.yb + fi.yd) * 0.5;
        fi.sy = -(fi.xd - fi.xb) * (fi.yb + fi.yd) * 0.5;
    } else {
        fi.sx = fi.yd - fi.yb;
        fi.sy = -(fi.xd - fi.xb);
    }
    slot_centroid(a, ia, ja, fi.xa, fi.ya);
    slot_centroid(a, ic, jc, fi.xc, fi.yc);
    double va[5], vc[5];
    visc_vals(a, padi(a, ia, ja), va);
    visc_vals(a, padi(a, ic, jc), vc);
    fi.ua = va[0]; fi.va = va[1]; fi.ta = va[2]; fi.rhoa = va[3]; fi.ra = va[4];
    fi.uc = vc[0]; fi.vc = vc[1]; fi.tc = vc[2]; fi.rhoc = vc[3]; fi.rc = vc[4];
    fi.ub = a.navg[0 * a.nnode + nbn]; fi.vb = a.navg[1 * a.nnode + nbn]; fi.tb = a.navg[2 * a.nnode + nbn];
    fi.rhob = a.navg[3 * a.nnode + nbn]; fi.rb = a.navg[4 * a.nnode + nbn];
    fi.ud = a.navg[0 * a.nnode + ndn]; fi.vd = a.navg[1 * a.nnode + ndn]; fi.td = a.navg[2 * a.nnode + ndn];
    fi.rhod = a.navg[3 * a.nnode + ndn]; fi.rd = a.navg[4 * a.nnode + ndn];
    const long long ca = cell_of(a, ia, ja);
    const bool cc = is_cell(a, ic, jc);
    const long long cn = cc ? cell_of(a, ic, jc) : 0;
    double w[4];
    for (int q = 0; q < 4; q++) {
        w[q] = a.visbar[q * a.ncell + ca];
        if (cc) w[q] -= a.visbar[q * a.ncell + cn];
    }
    visc_face_adj(a.P, fi, w, out, stride);
}

// Node adjoint: the B / D parts of the (up to four) faces at the node, the RTOL floor
// and the wall base of r, divided by the node's count.
TNS_HD void v2_point(const AdjArgs& a, long long node) {
    const int na = (int)(node / (a.nj + 1)), nb = (int)(node % (a.nj + 1));
    double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, xb = 0.0, yb = 0.0;
    auto take = [&](const double* base, long long stride, bool isB) {
        const int off = isB ? VF_B : VF_D;
        for (int c = 0; c < 5; c++) s[c] += base[(off + c) * stride];
        xb += base[(isB ? VF_XB : VF_XD) * stride];
        yb += base[(isB ? VF_YB : VF_YD) * stride];
    };
    // i-faces (i, j) join nodes (i, j) [lo] and (i, j+1) [hi]; B = hi on i == 0, else lo
    if (nb >= 1) take(a.vfi + ((long long)na * a.nj + nb - 1), a.nif, na == 0);
    if (nb < a.nj) take(a.vfi + ((long long)na * a.nj + nb), a.nif, na != 0);
    // j-faces (i, j) join nodes (i, j) [L] and (i+1, j) [R]; B = L on j == 0, else R
    if (na >= 1) take(a.vfj + ((long long)(na - 1) * (a.nj + 1) + nb), a.njf, nb != 0);
    if (na < a.ni) take(a.vfj + ((long long)na * (a.nj + 1) + nb), a.njf, nb == 0);
    const int info = a.ninfo[node];
    const int cnt = info & 7;
    double rtolb = 0.0;
    if ((info >> NI_FLOOR) & 1) {
        rtolb += s[4];
        s[4] = 0.0;
    }
    for (int c = 0; c < 5; c++) {
        s[c] = s[c] / (double)cnt;
        a.nbar[c * a.nnode + node] = s[c];
    }
    if ((info >> NI_RESET) & 1) rtolb += s[4] * a.P.rtred;
    if (a.sens) a.rtoln[node] += rtolb;
    if (a.geo) {
        a.xnbar[node] += xb;
        a.ynbar[node] += yb;
    }
}

// Viscous adjoint of one halo slot (cell or ghost): its face parts and its share of the
// node averages at its corners, as adjoints of its U, V, T, C1, C5 rows.
TNS_HD void v3_point(const AdjArgs& a, long long ps) {
    const int pi = (int)(ps / (a.nj + 2)) - 1, pj = (int)(ps % (a.nj + 2)) - 1;
    int along = 0;
    const bool cell = is_cell(a, pi, pj);
    if (!cell && !ghost_side(a, pi, pj, along)) return;
    double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, xb = 0.0, yb = 0.0;
    auto take = [&](const double* base, long long stride, bool isA) {
        const int off = isA ? VF_A : VF_C;
        for (int c = 0; c < 5; c++) s[c] += base[(off + c) * stride];
        xb += base[(isA ? VF_XA : VF_XC) * stride];
        yb += base[(isA ? VF_YA : VF_YC) * stride];
    };
    const bool jin = pj >= 0 && pj < a.nj, iin = pi >= 0 && pi < a.ni;
    // i-face (pi, pj): this slot is its upper cell; A only on the i == 0 boundary face
    if (jin && pi >= 0 && pi <= a.ni) take(a.vfi + ((long long)pi * a.nj + pj), a.nif, pi == 0);
    // i-face (pi+1, pj): this slot is its lower cell; A unless it is the ghost of i == 0
    if (jin && pi + 1 >= 0 && pi + 1 <= a.ni) take(a.vfi + ((long long)(pi + 1) * a.nj + pj), a.nif, pi + 1 != 0);
    // j-face (pi, pj): upper cell; A only on j == 0
    if (iin && pj >= 0 && pj <= a.nj) take(a.vfj + ((long long)pi * (a.nj + 1) + pj), a.njf, pj == 0);
    // j-face (pi, pj+1): lower cell; A unless it is the ghost of j == 0
    if (iin && pj + 1 >= 0 && pj + 1 <= a.nj) take(a.vfj + ((long long)pi * (a.nj + 1) + pj + 1), a.njf, pj + 1 != 0);
    for (int di = 0; di < 2; di++)
        for (int dj = 0; dj < 2; dj++) {
            const int na = pi + di, nb = pj + dj;
            if (na < 0 || na > a.ni || nb < 0 || nb > a.nj) continue;
            const long long node = (long long)na * (a.nj + 1) + nb;
            const int k = ((1 - di) << 1) | (1 - dj);
            const int m = a.ninfo[node] >> (NI_MASK + 3 * k);
            if (m & 1) s[0] += a.nbar[0 * a.nnode + node];
            if (m & 2) s[1] += a.nbar[1 * a.nnode + node];
            s[2] += a.nbar[2 * a.nnode + node];
            s[3] += a.nbar[3 * a.nnode + node];
            if (m & 4) s[4] += a.nbar[4 * a.nnode + node];
        }
    const double c1 = wv(a, WC1, ps), r = wv(a, WC5, ps) / c1;
    a.wvisc[0 * a.npad + ps] = s[0];
    a.wvisc[1 * a.npad + ps] = s[1];
    a.wvisc[2 * a.npad + ps] = s[2];
    a.wvisc[3 * a.npad + ps] = s[3] - s[4] * r / c1;
    a.wvisc[4 * a.npad + ps] = s[4] / c1;
    if (a.geo) {
        a.xcbar[ps] += xb;
        a.ycbar[ps] += yb;
    }
}

// ------------------------------------------------------------------ dissipation reverse

TNS_HD double ts_pressure(const Params& P, const double* q, long long n, long long c) {
    const double rho = q[c], u = q[n + c] / rho, v = q[2 * n + c] / rho;
    const double t = (q[3 * n + c] / rho - 0.5 * (u * u + v * v)) / P.cv;
    return rho * P.rr * t;
}

// Reverse of the DT loop (turbnstwod.f90:97-108) for one cell: the adjoints pb of its
// pressure and dtb of its local time step -> its conservative state and DL.
TNS_HD void ts_adj(const Params& P, const double q[5], double cfldl, double pb, double dtb, double qb[5],
                   double& dlb) {
    const double rho = q[0], u = q[1] / rho, v = q[2] / rho, e = q[3] / rho;
    const double vel = sqrt(u * u + v * v);
    const double t = (e - 0.5 * (u * u + v * v)) / P.cv;
    const double sq = sqrt(P.gamrr * t);
    const double den = fabs(vel) + sq;
    const double dt = cfldl / den;
    const double denb = -dtb * dt / den;
    dlb += dtb * P.cfl / den;
    double ub = 0.0, vb = 0.0, rhob = 0.0;
    double tb = denb * P.gamrr / (2.0 * sq);
    if (vel > 0.0) {
        const double sb = denb / (2.0 * vel);
        ub += 2.0 * u * sb;
        vb += 2.0 * v * sb;
    }
    rhob += pb * P.rr * t;
    tb += pb * rho * P.rr;
    const double eb = tb / P.cv;
    ub -= tb * u / P.cv;
    vb -= tb * v / P.cv;
    qb[3] += eb / rho;
    rhob -= eb * e / rho;
    qb[1] += ub / rho;
    rhob -= ub * u / rho;
    qb[2] += vb / rho;
    rhob -= vb * v / rho;
    qb[0] += rhob;
}

// DISSIPATION pre-pass of one cell (solver_state.f90:70-130): P, VOL/DT, D2Q and the two
// sensors' numerators and denominators (ghost neighbours read as the cell itself).
TNS_HD void d0_point(const AdjArgs& a, long long cell) {
    const int i = (int)(cell / a.nj), j = (int)(cell % a.nj);
    const Params& P = a.P;
    const long long n = a.ncell;
    CellGeo g;
    cell_geo(a, i, j, g);
    double q[5];
    for (int m = 0; m < 5; m++) q[m] = a.qold[m * n + cell];
    const double p = ts_pressure(P, a.qold, n, cell);
    double dt;
    if (P.local) {
        const double rho = q[0], u = q[1] / rho, v = q[2] / rho;
        const double vel = sqrt(u * u + v * v);
        const double t = (q[3] / rho - 0.5 * (u * u + v * v)) / P.cv;
        dt = a.M.cfldl[cell] / (fabs(vel) + sqrt(P.gamrr * t));
    } else {
        dt = *a.dtmin;
    }
    double d2q[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, numa = 0.0, dena = 0.0, numr = 0.0, denr = 0.0;
    for (int k = 0; k < 4; k++) {
        const int ii = i + di_of(k), jj = j + dj_of(k);
        const long long nc = is_cell(a, ii, jj) ? cell_of(a, ii, jj) : cell;
        for (int m = 0; m < 5; m++) d2q[m] = d2q[m] + a.qold[m * n + nc];
        const double pn = nc == cell ? p : ts_pressure(P, a.qold, n, nc);
        const double c5n = a.qold[4 * n + nc];
        numa = numa + fabs(pn - p);
        dena = dena + fabs(pn + p);
        numr = numr + fabs(c5n - q[4]);
        denr = denr + fabs(c5n + q[4]);
    }
    double* o = a.dpre;
    o[DP_P * n + cell] = p;
    o[DP_VBD * n + cell] = g.vol / dt;
    o[DP_DT * n + cell] = dt;
    for (int m = 0; m < 5; m++) o[(DP_D2Q + m) * n + cell] = d2q[m] - 4.0 * q[m];
    o[DP_NUMA * n + cell] = numa;
    o[DP_DENA * n + cell] = dena;
    o[DP_NUMR * n + cell] = numr;
    o[DP_DENR * n + cell] = denr;
}

TNS_HD double sensor_r(const AdjArgs& a, long long c) {
    const long long n = a.ncell;
    const double den = a.dpre[DP_DENR * n + c], fl = 8.0 * a.qold[c] * a.P.rtol;
    return a.dpre[DP_NUMR * n + c] / (den >= fl ? den : fl);
}

// Reverse of the face blend of DISSIPATION (solver_state.f90:131-225) for the faces of one
// cell, taking this cell's share of each face: the direct C and D2Q adjoints, VOL/DT and
// the sensors (each face's E2 = C02 * DMAX1(s_self, s_nb) gives its derivative to the
// sensor DMAX1 selected, from each side's own evaluation).
TNS_HD void d1_point(const AdjArgs& a, long long cell) {
    const int i = (int)(cell / a.nj), j = (int)(cell % a.nj);
    const long long n = a.ncell;
    const double* o = a.dpre;
    double Cb[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, d2qb[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, vbdb = 0.0, sab = 0.0, srb = 0.0;
    const double sa_c = o[DP_NUMA * n + cell] / o[DP_DENA * n + cell], sr_c = sensor_r(a, cell);
    for (int k = 0; k < 4; k++) {
        const int ii = i + di_of(k), jj = j + dj_of(k);
        if (!is_cell(a, ii, jj)) continue;
        const long long nc = cell_of(a, ii, jj);
        const double sa_n = o[DP_NUMA * n + nc] / o[DP_DENA * n + nc], sr_n = sensor_r(a, nc);
        const double d24 = 0.5 * (o[DP_VBD * n + cell] + o[DP_VBD * n + nc]);
        double e2[2], e4[2], act[2], e2c[2] = {0.0, 0.0}, e2n[2] = {0.0, 0.0};
        const double sc[2] = {sa_c, sr_c}, sn[2] = {sa_n, sr_n};
        for (int s = 0; s < 2; s++) {
            e2[s] = C02 * (sc[s] >= sn[s] ? sc[s] : sn[s]);
            act[s] = (C04 - e2[s] > 0.0) ? 1.0 : 0.0;
            e4[s] = act[s] > 0.0 ? C04 - e2[s] : 0.0;
        }
        double d24b = 0.0;
        for (int m = 0; m < 5; m++) {
            const int s = m < 4 ? 0 : 1;
            const double dC = a.qold[m * n + nc] - a.qold[m * n + cell];
            const double dd = o[(DP_D2Q + m) * n + nc] - o[(DP_D2Q + m) * n + cell];
            const double Dc = a.dbar[m * n + cell], Dn = a.dbar[m * n + nc];
            const double w = Dc - Dn;
            Cb[m] -= e2[s] * d24 * w;
            d2qb[m] += e4[s] * d24 * w;
            d24b += w * (e2[s] * dC - e4[s] * dd);
            e2c[s] += Dc * d24 * (dC + act[s] * dd);
            e2n[s] -= Dn * d24 * (dC + act[s] * dd);
        }
        vbdb += 0.5 * d24b;
        sab += C02 * ((sa_c >= sa_n ? e2c[0] : 0.0) + (sa_c > sa_n ? e2n[0] : 0.0));
        srb += C02 * ((sr_c >= sr_n ? e2c[1] : 0.0) + (sr_c > sr_n ? e2n[1] : 0.0));
    }
    double* out = a.dout;
    for (int m = 0; m < 5; m++) {
        out[(DO_C + m) * n + cell] = Cb[m];
        out[(DO_D2Q + m) * n + cell] = d2qb[m];
    }
    out[DO_VBD * n + cell] = vbdb;
    out[DO_SA * n + cell] = sab;
    out[DO_SR * n + cell] = srb;
}

// Gathers the dissipation adjoint of one cell (direct, Laplacians and sensors of the
// cell and its neighbours), VOL/DT and -- for LOCAL = 1 -- the time step, into the
// adjoint of Q_n.
TNS_HD void d2_point(const AdjArgs& a, long long cell) {
    const int i = (int)(cell / a.nj), j = (int)(cell % a.nj);
    const Params& P = a.P;
    const long long n = a.ncell;
    const double* o = a.dpre;
    const double* dz = a.dout;
    double qb[5], q[5];
    for (int m = 0; m < 5; m++) {
        q[m] = a.qold[m * n + cell];
        qb[m] = dz[(DO_C + m) * n + cell];
    }
    const double p = o[DP_P * n + cell], c5 = q[4];
    int nmiss = 0;
    double pb = 0.0, c5b = 0.0, rtolb = 0.0;
    // this cell's own sensors
    const double sa = dz[DO_SA * n + cell], sr = dz[DO_SR * n + cell];
    const double numa = o[DP_NUMA * n + cell], dena = o[DP_DENA * n + cell];
    const double Na = sa / dena, Da = -sa * numa / (dena * dena);
    const double numr = o[DP_NUMR * n + cell], denr = o[DP_DENR * n + cell], fl = 8.0 * q[0] * P.rtol;
    const double deff = denr >= fl ? denr : fl;
    const double Nr = sr / deff, Deff = -sr * numr / (deff * deff);
    const double Dr = denr >= fl ? Deff : 0.0;
    if (!(denr >= fl)) {
        qb[0] += Deff * 8.0 * P.rtol;
        rtolb += Deff * 8.0 * q[0];
    }
    for (int k = 0; k < 4; k++) {
        const int ii = i + di_of(k), jj = j + dj_of(k);
        if (!is_cell(a, ii, jj)) {
            nmiss++;
            pb += 2.0 * Da * sgn(p);
            c5b += 2.0 * Dr * sgn(c5);
            continue;
        }
        const long long nc = cell_of(a, ii, jj);
        for (int m = 0; m < 5; m++) qb[m] += dz[(DO_D2Q + m) * n + nc];
        const double pn = o[DP_P * n + nc], c5n = a.qold[4 * n + nc];
        pb += -Na * sgn(pn - p) + Da * sgn(pn + p);
        c5b += -Nr * sgn(c5n - c5) + Dr * sgn(c5n + c5);
        // the neighbour's sensors, in which this cell is a neighbour
        const double san = dz[DO_SA * n + nc], srn = dz[DO_SR * n + nc];
        const double numan = o[DP_NUMA * n + nc], denan = o[DP_DENA * n + nc];
        const double Nan = san / denan, Dan = -san * numan / (denan * denan);
        const double numrn = o[DP_NUMR * n + nc], denrn = o[DP_DENR * n + nc];
        const double fln = 8.0 * a.qold[nc] * P.rtol;
        const double deffn = denrn >= fln ? denrn : fln;
        const double Nrn = srn / deffn, Drn = denrn >= fln ? -srn * numrn / (deffn * deffn) : 0.0;
        pb += Nan * sgn(p - pn) + Dan * sgn(p + pn);
        c5b += Nrn * sgn(c5 - c5n) + Drn * sgn(c5 + c5n);
    }
    for (int m = 0; m < 5; m++) qb[m] += (-4.0 + (double)nmiss) * dz[(DO_D2Q + m) * n + cell];
    qb[4] += c5b;
    // VOL/DT
    const double dt = o[DP_DT * n + cell];
    CellGeo g;
    cell_geo(a, i, j, g);
    const double vbdb = dz[DO_VBD * n + cell];
    const double volb = vbdb / dt;
    const double dtb = a.dtbar[cell] - vbdb * g.vol / (dt * dt);
    double dlb = 0.0;
    ts_adj(P, q, a.M.cfldl[cell], pb, P.local ? dtb : 0.0, qb, dlb);
    if (!P.local) a.dtbar[cell] = dtb;
    for (int m = 0; m < 5; m++) a.lamd[m * n + cell] = qb[m];
    if (a.sens) a.rtolc[cell] += rtolb;
    if (a.geo) {
        a.volbar[cell] += volb;
        a.dlbar[cell] += dlb;
    }
}

// LOCAL = 0: the global step DTMIN = min(1e5, min DT) hands the summed dt adjoint to the
// cell(s) whose local step is the minimum.
TNS_HD void dtmin_point(const AdjArgs& a, long long cell) {
    const Params& P = a.P;
    const long long n = a.ncell;
    double q[5];
    for (int m = 0; m < 5; m++) q[m] = a.qold[m * n + cell];
    const double rho = q[0], u = q[1] / rho, v = q[2] / rho;
    const double vel = sqrt(u * u + v * v);
    const double t = (q[3] / rho - 0.5 * (u * u + v * v)) / P.cv;
    const double dtl = a.M.cfldl[cell] / (fabs(vel) + sqrt(P.gamrr * t));
    if (!(dtl == *a.dtmin) || dtl >= 100000.0) return;
    double qb[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, dlb = 0.0;
    ts_adj(P, q, a.M.cfldl[cell], 0.0, *a.dtsum, qb, dlb);
    for (int m = 0; m < 5; m++) a.lamd[m * n + cell] += qb[m];
    if (a.geo) a.dlbar[cell] += dlb;
}


// Face-vector sensitivities of one cell for the step: the residual's (stages 1-4,
// SX_k_bar += 1/2 sum_m R_m_bar (F_m + F_m of neighbour k), likewise G and SY) and the
// viscous flux's (VIS_bar of the cell times dF/dSX, dF/dSY of each face, which both
// sides of a face share).  Runs once per step, beside the rest of the stage-1 reverse.
TNS_HD void geo_point(const AdjArgs& a, long long cell) {
    const int i = (int)(cell / a.nj), j = (int)(cell % a.nj);
    const long long ps = padi(a, i, j);
    double sxb[4] = {0.0, 0.0, 0.0, 0.0}, syb[4] = {0.0, 0.0, 0.0, 0.0};
    for (int st = 0; st < 4; st++) {
        const double* gb = a.gbar4 + (size_t)st * 5 * a.npad;
        const double* w = a.w4 + (size_t)st * NWROW * a.npad;
        for (int m = 0; m < 5; m++) {
            const double g = 0.5 * gb[m * a.npad + ps];
            const double F = w[(WF + m) * a.npad + ps], G = w[(WG + m) * a.npad + ps];
            for (int k = 0; k < 4; k++) {
                const long long pn = padi(a, i + di_of(k), j + dj_of(k));
                sxb[k] += g * (F + w[(WF + m) * a.npad + pn]);
                syb[k] += g * (G + w[(WG + m) * a.npad + pn]);
            }
        }
    }
    // faces 1..4 of the cell: j-face (i, j), i-face (i+1, j), j-face (i, j+1), i-face (i, j)
    const double* fb[4] = {a.vfj + ((long long)i * (a.nj + 1) + j), a.vfi + ((long long)(i + 1) * a.nj + j),
                           a.vfj + ((long long)i * (a.nj + 1) + j + 1), a.vfi + ((long long)i * a.nj + j)};
    const long long stv[4] = {a.njf, a.nif, a.njf, a.nif};
    for (int k = 0; k < 4; k++)
        for (int q = 0; q < 4; q++) {
            const double vb = a.visbar[q * a.ncell + cell];
            sxb[k] += vb * fb[k][(VF_CX + q) * stv[k]];
            syb[k] += vb * fb[k][(VF_CY + q) * stv[k]];
        }
    // a type-6 ghost on one of the cell's faces: its face-vector and centroid adjoints
    // gathered over the step's stages (then cleared for the next step)
    double ycb = 0.0;
    for (int k = 0; k < 4; k++) {
        const int gi = i + di_of(k), gj = j + dj_of(k);
        if (is_cell(a, gi, gj)) continue;
        int along = 0;
        const int side = ghost_side(a, gi, gj, along);
        const int g = a.M.ghost_index(side, along);
        if (a.M.gtype[g] != 6) continue;
        const int ng = a.M.nghosts();
        sxb[k] += a.portacc[0 * ng + g];
        syb[k] += a.portacc[1 * ng + g];
        ycb += a.portacc[2 * ng + g];
        a.portacc[0 * ng + g] = a.portacc[1 * ng + g] = a.portacc[2 * ng + g] = 0.0;
    }
    if (ycb != 0.0) a.ycbar[ps] += ycb;
    for (int k = 0; k < 4; k++) {
        a.sxbar[k * a.ncell + cell] += sxb[k];
        a.sybar[k * a.ncell + cell] += syb[k];
    }
}

// The port ghost of `side` whose line (the cells from the port wall across to the
// opposite side) holds cell (i, j), or -1.
TNS_HD int port_of(const AdjArgs& a, int side, int i, int j) {
    const int along = (side == 1 || side == 3) ? i : j;
    const int g = a.M.ghost_index(side, along);
    return a.M.gtype[g] == 6 ? g : -1;
}

// DELY of the GPORT sum (boundary.f90:230-305 walk) for a cell with node y y[4] seen from
// `side`, and its derivative with respect to each node y.
TNS_HD double port_dely(int side, const double y[4], double d[4]) {
    const double sgn4[4][4] = {{0.5, 0.5, -0.5, -0.5}, {-0.5, 0.5, 0.5, -0.5}, {-0.5, -0.5, 0.5, 0.5},
                               {0.5, -0.5, -0.5, 0.5}};
    for (int n = 0; n < 4; n++) d[n] = sgn4[side - 1][n];
    if (side == 1) return 0.5 * ((y[0] + y[1]) - (y[2] + y[3]));
    if (side == 2) return 0.5 * ((y[1] + y[2]) - (y[0] + y[3]));
    if (side == 3) return 0.5 * ((y[2] + y[3]) - (y[0] + y[1]));
    return 0.5 * ((y[3] + y[0]) - (y[1] + y[2]));
}

TNS_HD void cell_y(const AdjArgs& a, int i, int j, double y[4]) {
    const long long nw = a.nj + 1, n1 = (long long)i * nw + j;
    y[0] = a.M.y[n1];
    y[1] = a.M.y[n1 + nw];
    y[2] = a.M.y[n1 + nw + 1];
    y[3] = a.M.y[n1 + 1];
}

// GPORT of one port ghost: the sum over its line of C1 * U * DELY (* YCC for IAXIS=1)
// (serial; the solver's k_gport sums the same terms in a block reduction).
TNS_HD void gport_point(const AdjArgs& a, long long g, const double* q, double* out) {
    int side, along;
    const int ni = a.ni, nj = a.nj;
    if (g < ni) { side = 1; along = (int)g; }
    else if (g < ni + nj) { side = 2; along = (int)g - ni; }
    else if (g < 2 * ni + nj) { side = 3; along = (int)g - ni - nj; }
    else { side = 4; along = (int)g - 2 * ni - nj; }
    if (a.M.gtype[g] != 6) return;
    const int len = (side == 1 || side == 3) ? nj : ni;
    double sum = 0.0;
    for (int k = 0; k < len; k++) {
        const int i = (side == 1 || side == 3) ? along : k, j = (side == 1 || side == 3) ? k : along;
        const long long c = cell_of(a, i, j);
        double y[4], d[4];
        cell_y(a, i, j, y);
        const double c1 = q[c], u = q[a.ncell + c] / c1;
        double term = c1 * u * port_dely(side, y, d);
        if (a.P.iaxis == 1) term = term * ((y[0] + y[1] + y[2] + y[3]) * 0.25);
        sum += term;
    }
    out[g] = sum;
}

// Reverse of GPORT for one cell of the stage input: the port ghosts whose lines hold the
// cell pass their adjoint to its C2 (C1 * (C2 / C1) * DELY [* YCC]; the C1 dependence
// cancels).
TNS_HD void port_point(const AdjArgs& a, long long cell) {
    const int i = (int)(cell / a.nj), j = (int)(cell % a.nj);
    double y[4], d[4], add = 0.0;
    bool any = false;
    for (int side = 1; side <= 4; side++) {
        const int g = port_of(a, side, i, j);
        if (g < 0) continue;
        if (!any) cell_y(a, i, j, y);
        any = true;
        double f = port_dely(side, y, d);
        if (a.P.iaxis == 1) f *= (y[0] + y[1] + y[2] + y[3]) * 0.25;
        add += a.gportb[g] * f;
    }
    if (!any) return;
    if (a.stage1) a.lam_old[a.ncell + cell] += add;
    else a.lam_out[a.ncell + cell] += add;
}

// Node-y sensitivities of GPORT over the step's four stages, gathered per node from its
// (up to four) cells.
TNS_HD void port_node_point(const AdjArgs& a, long long node) {
    const int na = (int)(node / (a.nj + 1)), nb = (int)(node % (a.nj + 1));
    const int ng = a.M.nghosts();
    double yb = 0.0;
    for (int c4 = 0; c4 < 4; c4++) {
        const int i = na - 1 + (c4 >> 1), j = nb - 1 + (c4 & 1);
        if (!is_cell(a, i, j)) continue;
        const int nn = ((na - i) << 1) | (nb - j);  // 0 (i,j) 2 (i+1,j) 3 (i+1,j+1) 1 (i,j+1)
        const int corner = nn == 0 ? 0 : (nn == 2 ? 1 : (nn == 3 ? 2 : 3));
        double y[4], d[4];
        cell_y(a, i, j, y);
        const double ycc = (y[0] + y[1] + y[2] + y[3]) * 0.25;
        const long long c = cell_of(a, i, j);
        for (int side = 1; side <= 4; side++) {
            const int g = port_of(a, side, i, j);
            if (g < 0) continue;
            const double dely = port_dely(side, y, d);
            for (int st = 0; st < 4; st++) {
                const double* q = a.qst[st];
                const double c1 = q[c];
                const double mom = c1 * (q[a.ncell + c] / c1);
                const double gb = a.gportb4[st * ng + g];
                if (a.P.iaxis == 1) yb += gb * mom * (d[corner] * ycc + dely * 0.25);
                else yb += gb * mom * d[corner];
            }
        }
    }
    a.ynbar[node] += yb;
}

// The adjoint of Q_n: residual / source / viscous part, dissipation / time-step part and
// the ghost part of stage 1's gather.
TNS_HD void final_point(const AdjArgs& a, long long cell) {
    const int i = (int)(cell / a.nj), j = (int)(cell % a.nj);
    const bool band = in_band(a, i, j);
    for (int m = 0; m < 5; m++) {
        double v = a.lam_old[m * a.ncell + cell] + a.lamd[m * a.ncell + cell];
        if (band) v += a.lamg[m * a.ncell + cell];
        a.lam_out[m * a.ncell + cell] = v;
    }
}

}  // namespace adj
}  // namespace tns
