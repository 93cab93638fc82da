/*
 * tns_oracle.c -- TEST INFRASTRUCTURE: line-faithful FP64 C restatement of the
 * reference solver's hot path.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline / reference arm use it.  PARITY UNPINNED (see tns_oracle.h).
 *
 * Every routine cites the Fortran it restates (paths relative to the reference
 * project).  Deliberate deviations from the literal Fortran, all forced by the
 * reference not compiling or leaving values undefined:
 *   - one global IAXIS (the reference's per-module IAXIS copies are never assigned);
 *   - arrays sized from the mesh instead of the NN=60000 PARAMETER;
 *   - FP64 everywhere (the Makefile's -fdefault-real-8 alone would promote
 *     DOUBLE PRECISION to REAL(16)); CDIFF inits 1e-10 / 1e-20 in FP64;
 *   - BC type 6: its inputs (TFLAME, ANCOMB, ACOMB, RHOPROP) are parameters, the burn
 *     rate takes an optional per-ghost multiplier, and the port mass flux GPORT is the
 *     sum of C1*U*DELY(*YCC) over the cells met walking from the parent straight across
 *     the mesh (through the face opposite NSIDE) until a ghost is reached, DELY using
 *     the side-NSIDE formula of boundary.f90:183-214 for every cell;
 *   - BC type 7: PINF, AMINF, DELTABL are parameters.
 */
#include "tns_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* constants.f90:12-60 */
#define RUNIV_VAL 8314.0
#define CMU_VAL 0.09
#define ALPHA_TURB 0.00052
#define BETA_TURB 0.2
#define CONST1_VAL 21.479
#define CONST2_VAL 21.394
#define CONST3_VAL 1.5
#define SUTH_COEF 0.00000011848
#define C02_VAL 0.25
#define C04_VAL 0.00390625
#define CFLTURB_VAL 0.5
#define HALF 0.5
#define QUARTER 0.25
#define CDIFF1_INIT 1.0e-10
#define CDIFF5_INIT 1.0e-20
#define BL_EXPONENT (1.0 / 7.0)
#define CONVKSC_VAL (1.0 / 98066.5)
#define GTH_VAL 35.0
#define YAXIS_THRESH 0.001
#define AMU_THRESH 0.001

static const double ALPHA_RK[4] = {0.25, 1.0 / 3.0, 0.5, 1.0};

struct ora {
    int nods, neles, nghosts, nn; /* nn: highest cell/ghost id */
    ora_params p;
    double rr, cv, cp, s0, tinf, rtolerance, div23;
    /* node arrays 1..nods */
    double *x, *y, *un, *vn, *tn, *rn, *rhon;
    int *itest;
    /* cell arrays 1..nn */
    double *xcc, *ycc, *vol, *dl, *dt, *sc[4][2];
    double *c[5], *cold[5], *f[5], *g[5], *r[5], *d2q[5], *d24[5];
    double *u, *v, *pp, *t, *visu, *visv, *vist, *visr, *source3, *source5, *anu, *anurt;
    int *nod[4], *nc[4];
    int *nparent, *nghost, *ntype, *nside; /* 1..nghosts */
    double *inj;
};

static double dmax1(double a, double b) { return a >= b ? a : b; }
static double dmin1(double a, double b) { return a <= b ? a : b; }

/* x**n for integer n by square-and-multiply (Fortran REAL**INTEGER). */
static double powi(double x, int n) {
    double r = 1.0;
    int m = n < 0 ? -n : n;
    double b = x;
    while (m) {
        if (m & 1) r *= b;
        m >>= 1;
        if (m) b *= b;
    }
    return n < 0 ? 1.0 / r : r;
}

static double *dalloc(int n) { return (double *)calloc((size_t)n + 1, sizeof(double)); }
static int *ialloc(int n) { return (int *)calloc((size_t)n + 1, sizeof(int)); }

/* geometry.f90:22-151 (file reads replaced by the arrays passed in) */
static void compute_geometry(ora *o) {
    int I, NG, NP, NS;
    for (I = 1; I <= o->nods; I++) o->itest[I] = 0;
    for (I = 1; I <= o->neles; I++) {
        int N1 = o->nod[0][I], N2 = o->nod[1][I], N3 = o->nod[2][I], N4 = o->nod[3][I];
        double X1 = o->x[N1], X2 = o->x[N2], X3 = o->x[N3], X4 = o->x[N4];
        double Y1 = o->y[N1], Y2 = o->y[N2], Y3 = o->y[N3], Y4 = o->y[N4];
        o->itest[N1]++; o->itest[N2]++; o->itest[N3]++; o->itest[N4]++;
        o->xcc[I] = (X1 + X2 + X3 + X4) * 0.25;
        o->ycc[I] = (Y1 + Y2 + Y3 + Y4) * 0.25;
        double DL12 = sqrt((X1 - X2) * (X1 - X2) + (Y1 - Y2) * (Y1 - Y2));
        double DL23 = sqrt((X2 - X3) * (X2 - X3) + (Y2 - Y3) * (Y2 - Y3));
        double DL34 = sqrt((X3 - X4) * (X3 - X4) + (Y3 - Y4) * (Y3 - Y4));
        double DL41 = sqrt((X4 - X1) * (X4 - X1) + (Y4 - Y1) * (Y4 - Y1));
        o->dl[I] = dmin1(dmin1(dmin1(DL12, DL23), DL34), DL41);
        if (o->p.iaxis == 1) {
            o->sc[0][0][I] = (Y2 - Y1) * (Y1 + Y2) * HALF;
            o->sc[0][1][I] = -(X2 - X1) * (Y1 + Y2) * HALF;
            o->sc[1][0][I] = (Y3 - Y2) * (Y2 + Y3) * HALF;
            o->sc[1][1][I] = -(X3 - X2) * (Y2 + Y3) * HALF;
            o->sc[2][0][I] = (Y4 - Y3) * (Y3 + Y4) * HALF;
            o->sc[2][1][I] = -(X4 - X3) * (Y3 + Y4) * HALF;
            o->sc[3][0][I] = (Y1 - Y4) * (Y4 + Y1) * HALF;
            o->sc[3][1][I] = -(X1 - X4) * (Y4 + Y1) * HALF;
            o->vol[I] = HALF * ((X3 - X1) * (Y4 - Y2) - (X4 - X2) * (Y3 - Y1)) * o->ycc[I];
        } else {
            o->sc[0][0][I] = (Y2 - Y1);
            o->sc[0][1][I] = -(X2 - X1);
            o->sc[1][0][I] = (Y3 - Y2);
            o->sc[1][1][I] = -(X3 - X2);
            o->sc[2][0][I] = (Y4 - Y3);
            o->sc[2][1][I] = -(X4 - X3);
            o->sc[3][0][I] = (Y1 - Y4);
            o->sc[3][1][I] = -(X1 - X4);
            o->vol[I] = HALF * ((X3 - X1) * (Y4 - Y2) - (X4 - X2) * (Y3 - Y1));
        }
        if (o->vol[I] <= 0.0) o->vol[I] = -o->vol[I];
    }
    for (I = 1; I <= o->nghosts; I++) {
        NP = o->nparent[I]; NG = o->nghost[I]; NS = o->nside[I];
        int N1 = o->nod[0][NP], N2 = o->nod[1][NP], N3 = o->nod[2][NP], N4 = o->nod[3][NP];
        double X1 = o->x[N1], X2 = o->x[N2], X3 = o->x[N3], X4 = o->x[N4];
        double Y1 = o->y[N1], Y2 = o->y[N2], Y3 = o->y[N3], Y4 = o->y[N4];
        double xf = 0, yf = 0;
        if (NS == 1) { xf = HALF * (X1 + X2); yf = HALF * (Y1 + Y2); o->itest[N1]++; o->itest[N2]++; }
        else if (NS == 2) { xf = HALF * (X2 + X3); yf = HALF * (Y2 + Y3); o->itest[N2]++; o->itest[N3]++; }
        else if (NS == 3) { xf = HALF * (X3 + X4); yf = HALF * (Y3 + Y4); o->itest[N3]++; o->itest[N4]++; }
        else if (NS == 4) { xf = HALF * (X4 + X1); yf = HALF * (Y4 + Y1); o->itest[N1]++; o->itest[N4]++; }
        o->xcc[NG] = 2.0 * xf - o->xcc[NP];
        o->ycc[NG] = 2.0 * yf - o->ycc[NP];
        o->vol[NG] = o->vol[NP];
        o->nc[0][NG] = NG; o->nc[1][NG] = NG; o->nc[2][NG] = NG; o->nc[3][NG] = NG;
    }
}

ora *ora_create(int nods, int neles, int nghosts, const double *x, const double *y,
                const int *nod, const int *nc, const int *nparent, const int *nghost,
                const int *ntype, const int *nside, const ora_params *p,
                const double *inj_scale) {
    ora *o = (ora *)calloc(1, sizeof(ora));
    int I, k, nn = neles;
    for (I = 0; I < nghosts; I++)
        if (nghost[I] > nn) nn = nghost[I];
    for (I = 0; I < 4 * neles; I++)
        if (nc[I] > nn) nn = nc[I];
    o->nods = nods; o->neles = neles; o->nghosts = nghosts; o->nn = nn; o->p = *p;
    o->x = dalloc(nods); o->y = dalloc(nods);
    o->un = dalloc(nods); o->vn = dalloc(nods); o->tn = dalloc(nods);
    o->rn = dalloc(nods); o->rhon = dalloc(nods); o->itest = ialloc(nods > nn ? nods : nn);
    o->xcc = dalloc(nn); o->ycc = dalloc(nn); o->vol = dalloc(nn); o->dl = dalloc(nn);
    o->dt = dalloc(nn);
    for (k = 0; k < 4; k++) { o->sc[k][0] = dalloc(nn); o->sc[k][1] = dalloc(nn); }
    for (k = 0; k < 5; k++) {
        o->c[k] = dalloc(nn); o->cold[k] = dalloc(nn); o->f[k] = dalloc(nn);
        o->g[k] = dalloc(nn); o->r[k] = dalloc(nn); o->d2q[k] = dalloc(nn);
        o->d24[k] = dalloc(nn);
    }
    o->u = dalloc(nn); o->v = dalloc(nn); o->pp = dalloc(nn); o->t = dalloc(nn);
    o->visu = dalloc(nn); o->visv = dalloc(nn); o->vist = dalloc(nn); o->visr = dalloc(nn);
    o->source3 = dalloc(nn); o->source5 = dalloc(nn); o->anu = dalloc(nn);
    o->anurt = dalloc(nn);
    for (k = 0; k < 4; k++) { o->nod[k] = ialloc(nn); o->nc[k] = ialloc(nn); }
    o->nparent = ialloc(nghosts); o->nghost = ialloc(nghosts);
    o->ntype = ialloc(nghosts); o->nside = ialloc(nghosts);
    o->inj = dalloc(nghosts);
    for (I = 1; I <= nods; I++) { o->x[I] = x[I - 1]; o->y[I] = y[I - 1]; }
    for (I = 1; I <= neles; I++)
        for (k = 0; k < 4; k++) {
            o->nod[k][I] = nod[(I - 1) * 4 + k];
            o->nc[k][I] = nc[(I - 1) * 4 + k];
        }
    for (I = 1; I <= nghosts; I++) {
        o->nparent[I] = nparent[I - 1]; o->nghost[I] = nghost[I - 1];
        o->ntype[I] = ntype[I - 1]; o->nside[I] = nside[I - 1];
        o->inj[I] = inj_scale ? inj_scale[I - 1] : 1.0;
    }
    /* turbnstwod.f90:37-42 */
    o->rr = RUNIV_VAL / p->amol;
    o->cv = o->rr / (p->gama - 1.0);
    o->cp = o->cv * p->gama;
    {
        double rho0 = p->p0 / (o->rr * p->t0);
        o->s0 = p->p0 / pow(rho0, p->gama);
    }
    o->tinf = p->t0 / (1.0 + 0.5 * (p->gama - 1.0) * p->aminf * p->aminf);
    o->rtolerance = p->rinit * p->rtred;
    o->div23 = 2.0 / 3.0;
    compute_geometry(o);
    return o;
}

void ora_destroy(ora *o) {
    int k;
    if (!o) return;
    free(o->x); free(o->y); free(o->un); free(o->vn); free(o->tn); free(o->rn);
    free(o->rhon); free(o->itest); free(o->xcc); free(o->ycc); free(o->vol); free(o->dl);
    free(o->dt);
    for (k = 0; k < 4; k++) { free(o->sc[k][0]); free(o->sc[k][1]); free(o->nod[k]); free(o->nc[k]); }
    for (k = 0; k < 5; k++) {
        free(o->c[k]); free(o->cold[k]); free(o->f[k]); free(o->g[k]); free(o->r[k]);
        free(o->d2q[k]); free(o->d24[k]);
    }
    free(o->u); free(o->v); free(o->pp); free(o->t); free(o->visu); free(o->visv);
    free(o->vist); free(o->visr); free(o->source3); free(o->source5); free(o->anu);
    free(o->anurt); free(o->nparent); free(o->nghost); free(o->ntype); free(o->nside);
    free(o->inj);
    free(o);
}

/* turbnstwod.f90:53-71 (RINIT / RTOLERANCE come from the parameters so a restart and a
 * cold start are configured the same way). */
void ora_cold_start(ora *o, double amachinit) {
    const ora_params *p = &o->p;
    double DYNRATIO = 1.0 + (p->gama - 1.0) * 0.5 * pow(amachinit, 2.0);
    double TINIT = p->t0 / DYNRATIO;
    double PINIT = p->p0 / pow(DYNRATIO, p->gama / (p->gama - 1.0));
    double UINIT = amachinit * sqrt(p->gama * o->rr * TINIT);
    double VINIT = 0.0;
    double EINIT = o->cv * TINIT + 0.5 * (pow(UINIT, 2.0) + pow(VINIT, 2.0));
    double RHOINIT = PINIT / (o->rr * TINIT);
    int I;
    for (I = 1; I <= o->neles; I++) {
        o->c[0][I] = RHOINIT;
        o->c[1][I] = RHOINIT * UINIT;
        o->c[2][I] = RHOINIT * VINIT;
        o->c[3][I] = RHOINIT * EINIT;
        o->c[4][I] = RHOINIT * p->rinit;
    }
}

void ora_set_state(ora *o, const double *c) {
    int I, k;
    for (k = 0; k < 5; k++)
        for (I = 1; I <= o->neles; I++) o->c[k][I] = c[(size_t)k * o->neles + I - 1];
}

void ora_get_state(const ora *o, double *c) {
    int I, k;
    for (k = 0; k < 5; k++)
        for (I = 1; I <= o->neles; I++) c[(size_t)k * o->neles + I - 1] = o->c[k][I];
}

/* turbnstwod.f90:97-114 -- time step, DTMIN, global step when LOCAL=0 */
void ora_step_dt(ora *o) {
    double DTMIN = 100000.0;
    int I;
    for (I = 1; I <= o->neles; I++) {
        double RHO = o->c[0][I];
        o->u[I] = o->c[1][I] / RHO;
        o->v[I] = o->c[2][I] / RHO;
        double VEL = sqrt(o->u[I] * o->u[I] + o->v[I] * o->v[I]);
        double E = o->c[3][I] / RHO;
        o->t[I] = (E - 0.5 * (o->u[I] * o->u[I] + o->v[I] * o->v[I])) / o->cv;
        o->pp[I] = RHO * o->rr * o->t[I];
        o->dt[I] = o->p.cfl * o->dl[I] / (fabs(VEL) + sqrt(o->p.gama * o->rr * o->t[I]));
        DTMIN = dmin1(DTMIN, o->dt[I]);
    }
    if (o->p.local == 0)
        for (I = 1; I <= o->neles; I++) o->dt[I] = DTMIN;
}

/* solver_state.f90:70-225 -- JST dissipation */
void ora_dissipation(ora *o) {
    const double C02 = C02_VAL, C04 = C04_VAL;
    int I, m, k;
    double *P = o->pp, *DT = o->dt, *VOL = o->vol, *ANU = o->anu, *ANURT = o->anurt;
    for (I = 1; I <= o->nghosts; I++) {
        int NG = o->nghost[I], NP = o->nparent[I];
        P[NG] = P[NP]; DT[NG] = DT[NP];
        for (m = 0; m < 5; m++) o->c[m][NG] = o->c[m][NP];
    }
    for (I = 1; I <= o->neles; I++) {
        int n1 = o->nc[0][I], n2 = o->nc[1][I], n3 = o->nc[2][I], n4 = o->nc[3][I];
        double PIE = P[I], C1I = o->c[0][I], C5I = o->c[4][I];
        double *C5 = o->c[4];
        double ANUN = fabs(P[n1] - PIE) + fabs(P[n2] - PIE) + fabs(P[n3] - PIE) + fabs(P[n4] - PIE);
        double ANUD = fabs(P[n1] + PIE) + fabs(P[n2] + PIE) + fabs(P[n3] + PIE) + fabs(P[n4] + PIE);
        ANU[I] = ANUN / ANUD;
        ANUN = fabs(C5[n1] - C5I) + fabs(C5[n2] - C5I) + fabs(C5[n3] - C5I) + fabs(C5[n4] - C5I);
        ANUD = fabs(C5[n1] + C5I) + fabs(C5[n2] + C5I) + fabs(C5[n3] + C5I) + fabs(C5[n4] + C5I);
        ANURT[I] = ANUN / dmax1(ANUD, 8.0 * C1I * o->rtolerance);
        for (m = 0; m < 5; m++) {
            double *C = o->c[m];
            o->d2q[m][I] = C[n1] + C[n2] + C[n3] + C[n4] - 4.0 * C[I];
        }
    }
    for (I = 1; I <= o->nghosts; I++) {
        int NG = o->nghost[I], NP = o->nparent[I];
        ANU[NG] = ANU[NP];
        for (m = 0; m < 5; m++) o->d2q[m][NG] = o->d2q[m][NP];
    }
    for (I = 1; I <= o->neles; I++) {
        double VOLBYDT = VOL[I] / DT[I];
        for (m = 0; m < 5; m++) {
            const double *SENS = (m == 4) ? ANURT : ANU;
            double SI = SENS[I], CI = o->c[m][I], D2I = o->d2q[m][I];
            double D2 = 0.0, D4 = 0.0;
            for (k = 0; k < 4; k++) {
                int n = o->nc[k][I];
                double E2N = C02 * dmax1(SI, SENS[n]);
                double E4N = dmax1(0.0, C04 - E2N);
                double D24N = HALF * (VOLBYDT + VOL[n] / DT[n]);
                double D2N = E2N * D24N, D4N = E4N * D24N;
                if (k == 0) {
                    D2 = D2N * (o->c[m][n] - CI);
                    D4 = D4N * (o->d2q[m][n] - D2I);
                } else {
                    D2 = D2 + D2N * (o->c[m][n] - CI);
                    D4 = D4 + D4N * (o->d2q[m][n] - D2I);
                }
            }
            o->d24[m][I] = D2 - D4;
        }
    }
}

/* turbnstwod.f90:204-227 -- COMPUTE_PRIMITIVE_VARS */
void ora_primitive(ora *o) {
    int I;
    for (I = 1; I <= o->neles; I++) {
        double RHO = o->c[0][I];
        o->u[I] = o->c[1][I] / RHO;
        o->v[I] = o->c[2][I] / RHO;
        double E = o->c[3][I] / RHO;
        o->t[I] = (E - 0.5 * (o->u[I] * o->u[I] + o->v[I] * o->v[I])) / o->cv;
        o->pp[I] = RHO * o->rr * o->t[I];
        o->f[0][I] = o->c[1][I];
        o->f[1][I] = RHO * o->u[I] * o->u[I] + o->pp[I];
        o->f[2][I] = RHO * o->u[I] * o->v[I];
        o->f[3][I] = (o->c[3][I] + o->pp[I]) * o->u[I];
        o->g[0][I] = o->c[2][I];
        o->g[1][I] = o->f[2][I];
        o->g[2][I] = RHO * o->v[I] * o->v[I] + o->pp[I];
        o->g[3][I] = (o->c[3][I] + o->pp[I]) * o->v[I];
        double RT = o->c[4][I] / RHO;
        o->f[4][I] = RHO * RT * o->u[I];
        o->g[4][I] = RHO * RT * o->v[I];
    }
}

/* ghost conservative + flux tail shared by BC types 2,3,4,6,7 (boundary.f90:62-70 etc.) */
static void ghost_fluxes(ora *o, int NG, double RHO) {
    double *U = o->u, *V = o->v, *T = o->t, *P = o->pp;
    o->c[0][NG] = RHO;
    o->c[1][NG] = RHO * U[NG];
    o->c[2][NG] = RHO * V[NG];
    double E = o->cv * T[NG] + 0.5 * (U[NG] * U[NG] + V[NG] * V[NG]);
    o->c[3][NG] = RHO * E;
    o->f[0][NG] = o->c[1][NG];
    o->f[1][NG] = RHO * U[NG] * U[NG] + P[NG];
    o->f[2][NG] = RHO * U[NG] * V[NG];
    o->f[3][NG] = (o->c[3][NG] + P[NG]) * U[NG];
    o->g[0][NG] = o->c[2][NG];
    o->g[1][NG] = o->f[2][NG];
    o->g[2][NG] = RHO * V[NG] * V[NG] + P[NG];
    o->g[3][NG] = (o->c[3][NG] + P[NG]) * V[NG];
}

static double amu_of(const ora *o, double T) {
    return SUTH_COEF * sqrt(o->p.amol) * pow(T, 0.6);
}

/* DELY of cell N for a port on side SIDE (boundary.f90:183-214, 238-246) */
static double dely_side(const ora *o, int N, int SIDE) {
    int N1 = o->nod[0][N], N2 = o->nod[1][N], N3 = o->nod[2][N], N4 = o->nod[3][N];
    const double *Y = o->y;
    if (SIDE == 1) return HALF * ((Y[N1] + Y[N2]) - (Y[N3] + Y[N4]));
    if (SIDE == 2) return HALF * ((Y[N2] + Y[N3]) - (Y[N1] + Y[N4]));
    if (SIDE == 3) return HALF * ((Y[N3] + Y[N4]) - (Y[N1] + Y[N2]));
    return HALF * ((Y[N4] + Y[N1]) - (Y[N2] + Y[N3]));
}

/* boundary.f90:168-223 with the repaired column walk (see file header) */
static double compute_gport(const ora *o, int NP, int NS) {
    static const int OPP[5] = {0, 3, 4, 1, 2};
    int N = NP, steps = 0;
    double GPORT = 0.0;
    int first = 1;
    while (N >= 1 && N <= o->neles && steps <= o->neles) {
        double term = o->c[0][N] * o->u[N] * dely_side(o, N, NS);
        if (o->p.iaxis == 1) term = term * o->ycc[N];
        GPORT = first ? term : GPORT + term;
        first = 0;
        N = o->nc[OPP[NS] - 1][N];
        steps++;
    }
    return GPORT;
}

/* boundary.f90:24-48 and the BC routines :53-327 */
void ora_boundary(ora *o) {
    const ora_params *p = &o->p;
    double *U = o->u, *V = o->v, *T = o->t, *P = o->pp;
    int I;
    for (I = 1; I <= o->nghosts; I++) {
        int NP = o->nparent[I], NG = o->nghost[I], NT = o->ntype[I], NS = o->nside[I];
        double RHO, AMU, RT;
        if (NT == 2) { /* :53-71 */
            U[NG] = fabs(U[NP]);
            V[NG] = -V[NP];
            T[NG] = p->t0 - 0.5 * (U[NG] * U[NG] + V[NG] * V[NG]) / o->cp;
            RHO = pow(o->s0 / (o->rr * T[NG]), 1.0 / (1.0 - p->gama));
            P[NG] = RHO * o->rr * T[NG];
            AMU = amu_of(o, T[NG]);
            RT = AMU / RHO;
            ghost_fluxes(o, NG, RHO);
            o->c[4][NG] = RHO * RT;
            o->f[4][NG] = o->c[4][NG] * U[NG];
            o->g[4][NG] = o->c[4][NG] * V[NG];
        } else if (NT == 3) { /* :76-95 */
            int NCOPP = NS == 1 ? o->nc[2][NP] : NS == 2 ? o->nc[3][NP] : NS == 3 ? o->nc[0][NP] : o->nc[1][NP];
            U[NG] = fabs(2.0 * U[NP] - U[NCOPP]);
            V[NG] = 2.0 * V[NP] - V[NCOPP];
            T[NG] = 2.0 * T[NP] - T[NCOPP];
            P[NG] = 2.0 * P[NP] - P[NCOPP];
            if (p->pamb >= 0.0) P[NG] = p->pamb;
            RHO = P[NG] / (o->rr * T[NG]);
            ghost_fluxes(o, NG, RHO);
            o->c[4][NG] = o->c[4][NP];
            o->f[4][NG] = o->f[4][NP];
            o->g[4][NG] = o->g[4][NP];
        } else if (NT == 4) { /* :100-109 */
            U[NG] = U[NP]; V[NG] = -V[NP]; T[NG] = T[NP]; RHO = o->c[0][NP]; P[NG] = P[NP];
            ghost_fluxes(o, NG, RHO);
            o->c[4][NG] = o->c[4][NP];
            o->f[4][NG] = o->f[4][NP];
            o->g[4][NG] = -o->g[4][NP];
        } else if (NT == 5) { /* :114-122 */
            U[NG] = -U[NP]; V[NG] = -V[NP]; T[NG] = T[NP]; RHO = o->c[0][NP]; P[NG] = P[NP];
            o->c[0][NG] = RHO;
            o->c[1][NG] = RHO * U[NG];
            o->c[2][NG] = RHO * V[NG];
            {
                double E = o->cv * T[NG] + 0.5 * (U[NG] * U[NG] + V[NG] * V[NG]);
                o->c[3][NG] = RHO * E;
            }
            o->f[0][NG] = -o->f[0][NP];
            o->f[1][NG] = 2.0 * P[NP] - o->f[1][NP];
            o->f[2][NG] = -o->f[2][NP];
            o->f[3][NG] = -o->f[3][NP];
            o->g[0][NG] = -o->g[0][NP];
            o->g[1][NG] = -o->g[1][NP];
            o->g[2][NG] = 2.0 * P[NP] - o->g[2][NP];
            o->g[3][NG] = -o->g[3][NP];
            o->c[4][NG] = -o->c[4][NP];
            o->f[4][NG] = -o->f[4][NP];
            o->g[4][NG] = -o->g[4][NP];
        } else if (NT == 6) { /* :128-163 */
            double SCX = o->sc[NS - 1][0][NP], SCY = o->sc[NS - 1][1][NP];
            double DNR = sqrt(SCX * SCX + SCY * SCY);
            double ENX = -SCX / DNR, ENY = -SCY / DNR;
            double DHYD = fabs(o->ycc[NG] + o->ycc[NP]);
            double GPORT = compute_gport(o, NP, NS);
            if (p->iaxis == 1) GPORT = 2.0 * GPORT / (DHYD * DHYD);
            else GPORT = GPORT / DHYD;
            RHO = o->c[0][NP];
            double RDOT = p->acomb * pow(P[NP] * CONVKSC_VAL, p->ancomb) * o->inj[I];
            double RDOTEB = RDOT;
            double VEL = p->rhoprop / RHO * RDOTEB;
            P[NG] = P[NP];
            U[NG] = VEL * ENX + VEL * ENX - U[NP];
            V[NG] = VEL * ENY + VEL * ENY - V[NP];
            T[NG] = p->tflame - 0.5 * (U[NG] * U[NG] + V[NG] * V[NG]) / o->cp;
            AMU = amu_of(o, T[NG]);
            double GVAL = (GPORT / (p->rhoprop * RDOT)) * pow(p->rhoprop * RDOT * DHYD / AMU, -0.125);
            if (GVAL > GTH_VAL)
                RDOTEB = RDOTEB * (1.0 + 0.023 * (pow(GVAL, 0.8) - pow(GTH_VAL, 0.8)));
            VEL = p->rhoprop / RHO * RDOTEB;
            U[NG] = VEL * ENX + VEL * ENX - U[NP];
            V[NG] = VEL * ENY + VEL * ENY - V[NP];
            T[NG] = p->tflame - 0.5 * (U[NG] * U[NG] + V[NG] * V[NG]) / o->cp;
            RHO = P[NG] / (o->rr * T[NG]);
            AMU = amu_of(o, T[NG]);
            RT = AMU / RHO;
            o->c[4][NG] = RHO * RT;
            ghost_fluxes(o, NG, RHO);
            o->f[4][NG] = o->c[4][NG] * U[NG];
            o->g[4][NG] = o->c[4][NG] * V[NG];
        } else if (NT == 7) { /* :310-327 */
            P[NG] = p->pinf; T[NG] = o->tinf; V[NG] = -V[NP];
            RHO = P[NG] / (o->rr * T[NG]);
            if (o->ycc[NG] <= p->deltabl)
                U[NG] = 2.0 * p->aminf * sqrt(p->gama * o->rr * o->tinf) *
                            pow(o->ycc[NG] / p->deltabl, BL_EXPONENT) - U[NP];
            else
                U[NG] = 2.0 * p->aminf * sqrt(p->gama * o->rr * o->tinf) - U[NP];
            AMU = amu_of(o, T[NG]);
            RT = AMU / RHO;
            ghost_fluxes(o, NG, RHO);
            o->c[4][NG] = RHO * RT;
            o->f[4][NG] = o->c[4][NG] * U[NG];
            o->g[4][NG] = o->c[4][NG] * V[NG];
        }
    }
}

/* viscous.f90:130-217 */
static void viscous_face(ora *o, int I, int FACE, int NN1, int NN2, int NCC) {
    const ora_params *p = &o->p;
    double SX = o->sc[FACE - 1][0][I], SY = o->sc[FACE - 1][1][I];
    double XB = o->x[NN1], YB = o->y[NN1], XD = o->x[NN2], YD = o->y[NN2];
    double XA = o->xcc[I], YA = o->ycc[I], XC = o->xcc[NCC], YC = o->ycc[NCC];
    double UA = o->u[I], VA = o->v[I], TA = o->t[I];
    double UB = o->un[NN1], VB = o->vn[NN1], TB = o->tn[NN1];
    double UC = o->u[NCC], VC = o->v[NCC], TC = o->t[NCC];
    double UD = o->un[NN2], VD = o->vn[NN2], TD = o->tn[NN2];
    double RHOA = o->c[0][I], RHOB = o->rhon[NN1], RHOC = o->c[0][NCC], RHOD = o->rhon[NN2];
    double RA = o->c[4][I] / o->c[0][I], RB = o->rn[NN1], RC = o->c[4][NCC] / o->c[0][NCC],
           RD = o->rn[NN2];
    double DNR = (XA - XC) * (YB - YD) - (XB - XD) * (YA - YC);
    double DUX = ((UA - UC) * (YB - YD) - (UB - UD) * (YA - YC)) / DNR;
    double DVX = ((VA - VC) * (YB - YD) - (VB - VD) * (YA - YC)) / DNR;
    double DTX = ((TA - TC) * (YB - YD) - (TB - TD) * (YA - YC)) / DNR;
    double DRX = ((RA - RC) * (YB - YD) - (RB - RD) * (YA - YC)) / DNR;
    double DUY = (-(UA - UC) * (XB - XD) + (UB - UD) * (XA - XC)) / DNR;
    double DVY = (-(VA - VC) * (XB - XD) + (VB - VD) * (XA - XC)) / DNR;
    double DTY = (-(TA - TC) * (XB - XD) + (TB - TD) * (XA - XC)) / DNR;
    double DRY = (-(RA - RC) * (XB - XD) + (RB - RD) * (XA - XC)) / DNR;
    double UAVG = QUARTER * (UA + UB + UC + UD);
    double VAVG = QUARTER * (VA + VB + VC + VD);
    double TAVG = QUARTER * (TA + TB + TC + TD);
    double RHOAVG = QUARTER * (RHOA + RHOB + RHOC + RHOD);
    double RAVG = QUARTER * (RA + RB + RC + RD);
    double DIVVEL;
    if (p->iaxis == 1) {
        double YAVG = HALF * (YB + YD), VBYY;
        if (YAVG < YAXIS_THRESH) VBYY = DVY;
        else VBYY = VAVG / YAVG;
        DIVVEL = DUX + DVY + VBYY;
    } else {
        DIVVEL = DUX + DVY;
    }
    double AMU = amu_of(o, TAVG);
    double AK = AMU * o->cp / p->prandtl;
    double CHI = RHOAVG * RAVG / (AMU * CMU_VAL);
    double FMU = tanh(ALPHA_TURB * CHI * CHI) / tanh(BETA_TURB * CHI * CHI);
    double AMUT = RHOAVG * RAVG * FMU;
    double AKT = AMUT * o->cp / p->prandtlt;
    double AMUEFF = AMU + AMUT;
    double AKEFF = AK + AKT;
    double TXX = AMUEFF * (DUX + DUX - o->div23 * DIVVEL);
    double TYY = AMUEFF * (DVY + DVY - o->div23 * DIVVEL);
    double TXY = AMUEFF * (DUY + DVX);
    double QXX = UAVG * TXX + VAVG * TXY + AKEFF * DTX;
    double QYY = UAVG * TXY + VAVG * TYY + AKEFF * DTY;
    if (FACE == 1) {
        o->visu[I] = TXX * SX + TXY * SY;
        o->visv[I] = TXY * SX + TYY * SY;
        o->vist[I] = QXX * SX + QYY * SY;
        o->visr[I] = AMUEFF * DRX * SX + AMUEFF * DRY * SY;
    } else {
        o->visu[I] = o->visu[I] + TXX * SX + TXY * SY;
        o->visv[I] = o->visv[I] + TXY * SX + TYY * SY;
        o->vist[I] = o->vist[I] + QXX * SX + QYY * SY;
        o->visr[I] = o->visr[I] + AMUEFF * DRX * SX + AMUEFF * DRY * SY;
    }
}

/* viscous.f90:29-124 */
void ora_viscous(ora *o) {
    int I;
    for (I = 1; I <= o->nods; I++) {
        o->un[I] = 0.0; o->vn[I] = 0.0; o->tn[I] = 0.0; o->rn[I] = 0.0; o->rhon[I] = 0.0;
        o->itest[I] = 0;
    }
    /* NODAL_AVERAGE_ELEMENTS :77-93 */
    for (I = 1; I <= o->neles; I++) {
        double UI = o->u[I], VI = o->v[I], TI = o->t[I], RHOI = o->c[0][I];
        double RI = o->c[4][I] / RHOI;
        int k;
        for (k = 0; k < 4; k++) {
            int N = o->nod[k][I];
            o->un[N] = o->un[N] + UI; o->vn[N] = o->vn[N] + VI; o->tn[N] = o->tn[N] + TI;
            o->rhon[N] = o->rhon[N] + RHOI; o->rn[N] = o->rn[N] + RI;
        }
        for (k = 0; k < 4; k++) o->itest[o->nod[k][I]]++;
    }
    /* NODAL_AVERAGE_GHOSTS :98-124 */
    for (I = 1; I <= o->nghosts; I++) {
        int NP = o->nparent[I], NG = o->nghost[I], NT = o->ntype[I], NS = o->nside[I];
        int N1 = 0, N2 = 0;
        if (NS == 1) { N1 = o->nod[0][NP]; N2 = o->nod[1][NP]; }
        else if (NS == 2) { N1 = o->nod[1][NP]; N2 = o->nod[2][NP]; }
        else if (NS == 3) { N1 = o->nod[2][NP]; N2 = o->nod[3][NP]; }
        else if (NS == 4) { N1 = o->nod[3][NP]; N2 = o->nod[0][NP]; }
        double RG = o->c[4][NG] / o->c[0][NG];
        o->un[N1] = o->un[N1] + o->u[NG]; o->vn[N1] = o->vn[N1] + o->v[NG];
        o->tn[N1] = o->tn[N1] + o->t[NG];
        o->rhon[N1] = o->rhon[N1] + o->c[0][NG]; o->rn[N1] = o->rn[N1] + RG;
        o->un[N2] = o->un[N2] + o->u[NG]; o->vn[N2] = o->vn[N2] + o->v[NG];
        o->tn[N2] = o->tn[N2] + o->t[NG];
        o->rhon[N2] = o->rhon[N2] + o->c[0][NG]; o->rn[N2] = o->rn[N2] + RG;
        if (NT == 4) {
            o->vn[N1] = 0.0; o->vn[N2] = 0.0;
        } else if (NT == 5) {
            o->un[N1] = 0.0; o->un[N2] = 0.0; o->vn[N1] = 0.0; o->vn[N2] = 0.0;
            o->rn[N1] = o->rtolerance * o->p.rtred; o->rn[N2] = o->rtolerance * o->p.rtred;
        }
        o->itest[N1]++; o->itest[N2]++;
    }
    /* finalize :51-59 */
    for (I = 1; I <= o->nods; I++) {
        double DF = (double)o->itest[I];
        o->un[I] = o->un[I] / DF;
        o->vn[I] = o->vn[I] / DF;
        o->tn[I] = o->tn[I] / DF;
        o->rhon[I] = o->rhon[I] / DF;
        o->rn[I] = o->rn[I] / DF;
        o->rn[I] = dmax1(o->rtolerance, o->rn[I]);
    }
    /* face loop :62-70 */
    for (I = 1; I <= o->neles; I++) {
        int N1 = o->nod[0][I], N2 = o->nod[1][I], N3 = o->nod[2][I], N4 = o->nod[3][I];
        viscous_face(o, I, 1, N1, N2, o->nc[0][I]);
        viscous_face(o, I, 2, N2, N3, o->nc[1][I]);
        viscous_face(o, I, 3, N3, N4, o->nc[2][I]);
        viscous_face(o, I, 4, N4, N1, o->nc[3][I]);
    }
}

/* source_terms.f90:24-104 */
void ora_source(ora *o) {
    const ora_params *p = &o->p;
    int I;
    const double DIV23 = o->div23;
    for (I = 1; I <= o->nn; I++) { o->source3[I] = 0.0; o->source5[I] = 0.0; }
    for (I = 1; I <= o->neles; I++) {
        int na = o->nc[0][I], nb = o->nc[1][I], ncc = o->nc[2][I], nd = o->nc[3][I];
        double XA = o->xcc[na], XB = o->xcc[nb], XC = o->xcc[ncc], XD = o->xcc[nd];
        double YA = o->ycc[na], YB = o->ycc[nb], YC = o->ycc[ncc], YD = o->ycc[nd];
        double UA = o->u[na], UB = o->u[nb], UC = o->u[ncc], UD = o->u[nd];
        double VA = o->v[na], VB = o->v[nb], VC = o->v[ncc], VD = o->v[nd];
        double RA = o->c[4][na] / o->c[0][na], RB = o->c[4][nb] / o->c[0][nb];
        double RC = o->c[4][ncc] / o->c[0][ncc], RD = o->c[4][nd] / o->c[0][nd];
        double QA = sqrt(UA * UA + VA * VA), QB = sqrt(UB * UB + VB * VB);
        double QC = sqrt(UC * UC + VC * VC), QD = sqrt(UD * UD + VD * VD);
        double DNR = (XA - XC) * (YB - YD) - (XB - XD) * (YA - YC);
        double DQX = ((QA - QC) * (YB - YD) - (QB - QD) * (YA - YC)) / DNR;
        double DRX = ((RA - RC) * (YB - YD) - (RB - RD) * (YA - YC)) / DNR;
        double DUX = ((UA - UC) * (YB - YD) - (UB - UD) * (YA - YC)) / DNR;
        double DVX = ((VA - VC) * (YB - YD) - (VB - VD) * (YA - YC)) / DNR;
        double DQY = (-(QA - QC) * (XB - XD) + (QB - QD) * (XA - XC)) / DNR;
        double DRY = (-(RA - RC) * (XB - XD) + (RB - RD) * (XA - XC)) / DNR;
        double DUY = (-(UA - UC) * (XB - XD) + (UB - UD) * (XA - XC)) / DNR;
        double DVY = (-(VA - VC) * (XB - XD) + (VB - VD) * (XA - XC)) / DNR;
        double RHO = o->c[0][I];
        double RI = o->c[4][I] / RHO;
        double AMU = amu_of(o, o->t[I]);
        double CHI = RHO * RI / (CMU_VAL * AMU);
        double FMU = tanh(ALPHA_TURB * CHI * CHI) / tanh(BETA_TURB * CHI * CHI);
        double FR2 = tanh(sqrt(CHI)) / tanh(CHI * sqrt(2.0 * sqrt(CMU_VAL)));
        double AMUT = FMU * RHO * RI;
        double PHI = DQX * DRX + DQY * DRY;
        double DEE = 0.0, DIVVEL, PK;
        if (PHI > 0.0) DEE = DRX * DRX + DRY * DRY;
        if (p->iaxis == 1) {
            double VBYY;
            if (o->ycc[I] < YAXIS_THRESH) VBYY = DVY;
            else VBYY = o->v[I] / o->ycc[I];
            DIVVEL = DUX + DVY + VBYY;
            PK = AMUT / RHO * (DUX * DUX + DVY * DVY + VBYY * VBYY + DUX * DUX + DVY * DVY +
                               VBYY * VBYY + (DUY + DVX) * (DUY + DVX) - DIV23 * DIVVEL * DIVVEL);
            PK = dmax1(PK, 0.0);
            o->source5[I] = (RHO * (CONST1_VAL - CONST2_VAL * FR2) * sqrt(RI * PK) -
                             RHO * CONST3_VAL * DEE) *
                            powi(AMUT / dmax1(AMUT, AMU_THRESH * AMU), p->npseudo);
            double TTT = (AMU + AMUT) * (VBYY + VBYY - DIV23 * DIVVEL);
            o->source3[I] = (o->pp[I] - TTT) / o->ycc[I];
        } else {
            DIVVEL = DUX + DVY;
            PK = AMUT / RHO * (DUX * DUX + DVY * DVY + DUX * DUX + DVY * DVY +
                               (DUY + DVX) * (DUY + DVX) - DIV23 * DIVVEL * DIVVEL);
            PK = dmax1(PK, 0.0);
            o->source5[I] = (RHO * (CONST1_VAL - CONST2_VAL * FR2) * sqrt(RI * PK) -
                             RHO * CONST3_VAL * DEE) *
                            powi(AMUT / dmax1(AMUT, AMU_THRESH * AMU), p->npseudo);
        }
    }
}

/* residual.f90:23-62 */
void ora_residual(ora *o) {
    int I, m;
    for (I = 1; I <= o->neles; I++) {
        int n1 = o->nc[0][I], n2 = o->nc[1][I], n3 = o->nc[2][I], n4 = o->nc[3][I];
        double SX1 = o->sc[0][0][I], SX2 = o->sc[1][0][I], SX3 = o->sc[2][0][I], SX4 = o->sc[3][0][I];
        double SY1 = o->sc[0][1][I], SY2 = o->sc[1][1][I], SY3 = o->sc[2][1][I], SY4 = o->sc[3][1][I];
        for (m = 0; m < 5; m++) {
            const double *F = o->f[m], *G = o->g[m];
            double FI = F[I], GI = G[I];
            o->r[m][I] = HALF * ((FI + F[n1]) * SX1 + (GI + G[n1]) * SY1 +
                                 (FI + F[n2]) * SX2 + (GI + G[n2]) * SY2 +
                                 (FI + F[n3]) * SX3 + (GI + G[n3]) * SY3 +
                                 (FI + F[n4]) * SX4 + (GI + G[n4]) * SY4);
        }
        o->r[4][I] = o->r[4][I] - o->vol[I] * o->source5[I];
        if (o->p.iaxis == 1) o->r[2][I] = o->r[2][I] - o->vol[I] * o->source3[I];
    }
}

/* residual.f90:67-83 */
void ora_update(ora *o, double ALPHA) {
    int I;
    const double CFLTURB = CFLTURB_VAL;
    for (I = 1; I <= o->neles; I++) {
        double DTBYVOL = o->dt[I] / o->vol[I];
        o->c[0][I] = o->cold[0][I] - ALPHA * DTBYVOL * (o->r[0][I] - o->d24[0][I]);
        o->c[1][I] = o->cold[1][I] - ALPHA * DTBYVOL * (o->r[1][I] - o->visu[I] - o->d24[1][I]);
        o->c[2][I] = o->cold[2][I] - ALPHA * DTBYVOL * (o->r[2][I] - o->visv[I] - o->d24[2][I]);
        o->c[3][I] = o->cold[3][I] - ALPHA * DTBYVOL * (o->r[3][I] - o->vist[I] - o->d24[3][I]);
        o->c[4][I] = o->cold[4][I] -
                     ALPHA * DTBYVOL * CFLTURB * (o->r[4][I] - o->visr[I] - o->d24[4][I]);
        o->c[4][I] = o->c[0][I] * dmax1(o->rtolerance, o->c[4][I] / o->c[0][I]);
    }
}

/* turbnstwod.f90:87-168 -- the RK4 loop */
int ora_iterate(ora *o, int niter, int monitor_every, double *cdiff_out, int max_records) {
    int ITER, I, m, nrec = 0;
    for (m = 0; m < 5; m++)
        for (I = 1; I <= o->neles; I++) o->cold[m][I] = o->c[m][I];
    for (ITER = 1; ITER <= niter; ITER++) {
        int s;
        ora_step_dt(o);
        ora_dissipation(o);
        for (s = 0; s < 4; s++) {
            ora_primitive(o);
            ora_boundary(o);
            if (s == 0) ora_viscous(o);
            ora_source(o);
            ora_residual(o);
            ora_update(o, ALPHA_RK[s]);
        }
        if (monitor_every > 0 && ITER % monitor_every == 0) {
            double cd[5] = {CDIFF1_INIT, CDIFF1_INIT, CDIFF1_INIT, CDIFF1_INIT, CDIFF5_INIT};
            for (I = 1; I <= o->neles; I++)
                for (m = 0; m < 5; m++) cd[m] = dmax1(fabs(o->cold[m][I] - o->c[m][I]), cd[m]);
            if (cdiff_out && nrec < max_records)
                for (m = 0; m < 5; m++) cdiff_out[nrec * 5 + m] = cd[m];
            nrec++;
        }
        for (m = 0; m < 5; m++)
            for (I = 1; I <= o->neles; I++) o->cold[m][I] = o->c[m][I];
    }
    return nrec;
}

/* solver_state.f90:230-270 (file writing left to the caller) */
void ora_postprocess(ora *o, double *pn, double *un, double *vn, double *tn) {
    int I, J;
    double *s[4];
    int *cnt = (int *)calloc((size_t)o->nods + 1, sizeof(int));
    for (J = 0; J < 4; J++) s[J] = (double *)calloc((size_t)o->nods + 1, sizeof(double));
    for (I = 1; I <= o->neles; I++)
        for (J = 0; J < 4; J++) {
            int K = o->nod[J][I];
            cnt[K]++;
            s[0][K] += o->pp[I]; s[1][K] += o->u[I]; s[2][K] += o->v[I]; s[3][K] += o->t[I];
        }
    for (I = 1; I <= o->nghosts; I++) {
        int NG = o->nghost[I], NP = o->nparent[I], NS = o->nside[I], N1 = 0, N2 = 0;
        if (NS == 1) { N1 = o->nod[0][NP]; N2 = o->nod[1][NP]; }
        else if (NS == 2) { N1 = o->nod[1][NP]; N2 = o->nod[2][NP]; }
        else if (NS == 3) { N1 = o->nod[2][NP]; N2 = o->nod[3][NP]; }
        else if (NS == 4) { N1 = o->nod[3][NP]; N2 = o->nod[0][NP]; }
        s[0][N1] += o->pp[NG]; s[1][N1] += o->u[NG]; s[2][N1] += o->v[NG]; s[3][N1] += o->t[NG];
        s[0][N2] += o->pp[NG]; s[1][N2] += o->u[NG]; s[2][N2] += o->v[NG]; s[3][N2] += o->t[NG];
        cnt[N1]++; cnt[N2]++;
    }
    for (I = 1; I <= o->nods; I++) {
        double d = (double)cnt[I];
        pn[I - 1] = s[0][I] / d; un[I - 1] = s[1][I] / d;
        vn[I - 1] = s[2][I] / d; tn[I - 1] = s[3][I] / d;
    }
    for (J = 0; J < 4; J++) free(s[J]);
    free(cnt);
}

int ora_array_len(const ora *o) { return o->nn; }

int ora_fetch(const ora *o, const char *name, double *out, int maxn) {
    const double *src = 0;
    int n = o->nn, I;
    if (!strcmp(name, "U")) src = o->u;
    else if (!strcmp(name, "V")) src = o->v;
    else if (!strcmp(name, "T")) src = o->t;
    else if (!strcmp(name, "P")) src = o->pp;
    else if (!strcmp(name, "DT")) src = o->dt;
    else if (!strncmp(name, "D24", 3) && name[3] >= '1' && name[3] <= '5') src = o->d24[name[3] - '1'];
    else if (!strncmp(name, "D2Q", 3) && name[3] >= '1' && name[3] <= '5') src = o->d2q[name[3] - '1'];
    else if (!strncmp(name, "C", 1) && name[1] >= '1' && name[1] <= '5' && !name[2]) src = o->c[name[1] - '1'];
    else if (!strncmp(name, "F", 1) && name[1] >= '1' && name[1] <= '5' && !name[2]) src = o->f[name[1] - '1'];
    else if (!strncmp(name, "G", 1) && name[1] >= '1' && name[1] <= '5' && !name[2]) src = o->g[name[1] - '1'];
    else if (!strncmp(name, "R", 1) && name[1] >= '1' && name[1] <= '5' && !name[2]) src = o->r[name[1] - '1'];
    else if (!strcmp(name, "VISU")) src = o->visu;
    else if (!strcmp(name, "VISV")) src = o->visv;
    else if (!strcmp(name, "VIST")) src = o->vist;
    else if (!strcmp(name, "VISR")) src = o->visr;
    else if (!strcmp(name, "SOURCE3")) src = o->source3;
    else if (!strcmp(name, "SOURCE5")) src = o->source5;
    else if (!strcmp(name, "XCC")) src = o->xcc;
    else if (!strcmp(name, "YCC")) src = o->ycc;
    else if (!strcmp(name, "VOL")) src = o->vol;
    else if (!strcmp(name, "DL")) src = o->dl;
    else if (!strcmp(name, "ANU")) src = o->anu;
    else if (!strcmp(name, "ANURT")) src = o->anurt;
    else {
        n = o->nods;
        if (!strcmp(name, "UN")) src = o->un;
        else if (!strcmp(name, "VN")) src = o->vn;
        else if (!strcmp(name, "TN")) src = o->tn;
        else if (!strcmp(name, "RN")) src = o->rn;
        else if (!strcmp(name, "RHON")) src = o->rhon;
        else if (!strcmp(name, "X")) src = o->x;
        else if (!strcmp(name, "Y")) src = o->y;
        else return -1;
    }
    if (n > maxn) n = maxn;
    for (I = 0; I < n; I++) out[I] = src[I + 1];
    return n;
}
