/*
 * tns_oracle.h -- CPU oracle for the RK4 / JST / viscous / source / boundary hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a line-faithful FP64 restatement in C of the
 * reference Fortran solver's per-iteration hot path (the src/solvers Fortran files of
 * Venkatesh-Karuppiah/2D-Turbulent-Navier-Stokes).  It exists to check the CUDA
 * path and to time the CPU baseline; no product code links it.
 *
 * PARITY UNPINNED: the reference is Fortran, no Fortran compiler exists on the build
 * or GPU machines, and the reference ships no golden outputs.  The oracle is pinned
 * only by analytic invariants (free-stream preservation, mirror symmetry, hand-checked
 * single-routine cases) and by an independent literal Python transcription on tiny
 * meshes (tests/test_oracle.py).
 *
 * Arrays inside the oracle are 1-based and sized like the reference's NN-sized module
 * arrays (index 0 unused), so every loop below reads like the Fortran it restates.
 */
#ifndef TNS_ORACLE_H
#define TNS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_params {
    double gama, amol, cfl, prandtl, prandtlt, p0, t0, pamb, rtred, rinit;
    double tflame, ancomb, acomb, rhoprop, pinf, aminf, deltabl;
    int local, npseudo, iaxis, pad_;
} ora_params;

typedef struct ora ora;

/* nod, nc: NELES rows of 4 (row-major, 1-based ids as in grid.in); x,y in metres.
 * ghost arrays: bc.in columns (1-based).  inj_scale: per bc.in line multiplier of the
 * type-6 burn rate (NULL = 1). */
ora *ora_create(int nods, int neles, int nghosts, const double *x, const double *y,
                const int *nod, const int *nc, const int *nparent, const int *nghost,
                const int *ntype, const int *nside, const ora_params *p,
                const double *inj_scale);
void ora_destroy(ora *o);

/* ISTART=0 isentropic cold start (turbnstwod.f90:53-71 restated). */
void ora_cold_start(ora *o, double amachinit);
/* load / fetch conservative state, component-major c[k*neles + (i-1)] */
void ora_set_state(ora *o, const double *c);
void ora_get_state(const ora *o, double *c);

/* run niter full RK4 iterations; every monitor_every-th iteration (local count)
 * appends CDIFF1..5 to cdiff_out (5 doubles per record).  Returns records written. */
int ora_iterate(ora *o, int niter, int monitor_every, double *cdiff_out, int max_records);

/* fetch an internal array (1..n mapped to out[0..n-1]); names:
 * "U","V","T","P","DT","D241".."D245","VISU","VISV","VIST","VISR","SOURCE3","SOURCE5",
 * "XCC","YCC","VOL","DL","C1".."C5","UN","VN","TN","RN","RHON","ANU","ANURT".
 * n = number of entries copied (cells+ghost slots for per-cell arrays, nodes for node
 * arrays).  Returns n or -1 for an unknown name. */
int ora_fetch(const ora *o, const char *name, double *out, int maxn);
int ora_array_len(const ora *o);

/* single routines, for unit tests */
void ora_step_dt(ora *o);
void ora_dissipation(ora *o);
void ora_primitive(ora *o);
void ora_boundary(ora *o);
void ora_viscous(ora *o);
void ora_source(ora *o);
void ora_residual(ora *o);
void ora_update(ora *o, double alpha);

/* nodal P,U,V,T averages of POSTPROCESS (solver_state.f90:237-281), nodes 1..NODS */
void ora_postprocess(ora *o, double *pn, double *un, double *vn, double *tn);

#ifdef __cplusplus
}
#endif
#endif
