/*
 * tnsgpu.h -- C ABI of the B200 RK4 hot path of the 2-D / axisymmetric turbulent
 * Navier-Stokes solver (drop-in for the per-iteration calls of the reference Fortran
 * mains src/solvers/turbnstwod.f90 and turbnsaxis.f90).
 *
 * The reference has no plugin API: its main program calls argument-less subroutines
 * that share module globals.  The entry points below replace exactly that seam
 * (turbnstwod.f90:95-168, the RK4 loop); everything before it (flow.in / grid.in /
 * bc.in reads, geometry.f90:22-52) and after it (restart.in, POSTPROCESS) stays with
 * the caller.  All arguments are plain pointers and sizes; arrays are the caller's
 * Fortran arrays (1-based ids, column-major), borrowed for the duration of a call.
 *
 * Return codes: 0 = success, negative = error (tns_last_error() gives the text).
 * A handle owns one CUDA stream and all device memory; handles are not thread-safe.
 */
#ifndef TNSGPU_H
#define TNSGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define TNS_OK 0
#define TNS_ERR_ARG (-1)          /* null pointer / bad size */
#define TNS_ERR_MESH (-2)         /* inconsistent grid.in / bc.in arrays */
#define TNS_ERR_UNSUPPORTED (-3)  /* a case the layout cannot express (see tns_create) */
#define TNS_ERR_CUDA (-4)         /* CUDA runtime error */
#define TNS_ERR_NONFINITE (-5)    /* state became NaN / Inf */
#define TNS_ERR_STATE (-6)        /* call out of order (e.g. no state uploaded) */
#define TNS_ERR_TOO_LARGE (-7)    /* problem exceeds a fixed-size buffer (tns_time_step_noalloc) */

/* Mesh as COMPUTE_GEOMETRY holds it after reading grid.in and bc.in
 * (geometry.f90:25-52; solver_state.f90:113-125). */
typedef struct tns_mesh {
    int nods, neles, nghosts;
    const double *x, *y;       /* X(1:NODS), Y(1:NODS) in metres (after the 0.001 scaling) */
    const int *nod;            /* NOD(LD,4) column-major: NOD(I,K) = nod[(K-1)*ld_nod + I-1] */
    int ld_nod;                /* leading dimension of NOD (NN in the reference) */
    const int *nc1, *nc2, *nc3, *nc4;             /* NC1..NC4(1:NELES) */
    const int *nparent, *nghost, *ntype, *nside;  /* bc.in columns, (1:NGHOSTS) */
} tns_mesh;

/* The 17 flow.in values that reach the hot path (turbnstwod.f90:20-23) plus RINIT
 * (cold start or restart.in) and the inputs of BC types 6 and 7 that the reference
 * declares but never assigns (solver_state.f90:36-42: TFLAME, ANCOMB, ACOMB, RHOPROP,
 * PINF, AMINF, DELTABL). */
typedef struct tns_params {
    double gama, amol, cfl, prandtl, prandtlt, p0, t0, pamb, rtred, rinit;
    double tflame, ancomb, acomb, rhoprop, pinf, aminf, deltabl;
    int local, npseudo, iaxis;
    int precision; /* 0 = FP64; 1 = mixed: FP64 state, geometry and differences, FP32
                      increments, D, VIS, DT and flux / JST / viscous / source arithmetic */
} tns_params;

typedef struct tns_handle tns_handle;

/* Builds the device mesh: validates the arrays, computes the geometry
 * (geometry.f90:55-149) and uploads everything.  A mesh whose cells form one structured
 * i x j block (any numbering) runs on the tiled kernels; any other quadrilateral mesh
 * (the reference reads any NOD / NC1..NC4) on the gather-indexed kernels, its cells
 * ordered along a Hilbert curve and its nodes renumbered on the device (the ABI's
 * arrays keep the caller's ids); both precisions run there.  TNS_ERR_UNSUPPORTED: a
 * general mesh with a type-3 ghost whose parent has no cell across the opposite face;
 * the adjoint also refuses general meshes, and a batch holding one runs schedules 1
 * and 2 only (tns_batch_set_schedule).
 * Replaces: CALL COMPUTE_GEOMETRY's consumers + the module state setup
 * (turbnstwod.f90:32-48). */
int tns_create(const tns_mesh *mesh, const tns_params *params, tns_handle **out);

/* Burn-rate multiplier per bc.in line for type-6 ghosts (default 1).  No reference
 * counterpart (the reference cannot express an axial variation). */
int tns_set_injection_scale(tns_handle *h, const double *scale /* [NGHOSTS] */);

/* Uploads C1..C5(1:NELES) as the state at the start of the next iteration.
 * Replaces: the COLD <- C copy before the loop (turbnstwod.f90:87-90). */
int tns_upload_state(tns_handle *h, const double *c1, const double *c2, const double *c3,
                     const double *c4, const double *c5);

/* Runs niter full RK4 iterations (turbnstwod.f90:95-168).  Every monitor_every-th
 * iteration (counting from 1 within this call, as MOD(ITER,1000) does) the five CDIFF
 * values max(init, max|COLD-C|) are appended to cdiff_out (5 doubles per record, at
 * most max_records); *n_records receives the count.  monitor_every <= 0 disables it. */
int tns_run(tns_handle *h, int niter, int monitor_every, double *cdiff_out, int max_records,
            int *n_records);

/* Asynchronous form of tns_run without the residual monitor: enqueues niter RK4
 * iterations on the handle's stream and returns at once.  Errors of the iterations
 * (non-finite state) are reported by the next tns_synchronize / tns_run. */
int tns_enqueue(tns_handle *h, int niter);

/* Captures and instantiates, without running anything, every CUDA graph that tns_run
 * and tns_enqueue launch for this handle (the unmonitored and the monitored iteration;
 * in mixed precision one of each per state-buffer parity).  Otherwise each is captured
 * at its first use, inside whichever call first needs it.  Needs an uploaded state;
 * does nothing while per-kernel profiling is on (those iterations are not graphs). */
int tns_prepare(tns_handle *h);

/* Waits for the work enqueued on the handle's stream; TNS_ERR_NONFINITE if the state
 * became NaN / Inf since the last check. */
int tns_synchronize(tns_handle *h);

/* Asynchronous forms of tns_upload_state, tns_run(h, 1, 1, ...) and tns_download_state,
 * for callers that keep several handles in flight (one handle's download overlapping
 * another's upload and iteration).  Each queues its work on the handle's stream and
 * returns at once; the results are there after the next tns_synchronize on the handle,
 * and the host arrays must stay valid (and a download target unread) until then.  Host
 * arrays must be page-locked (cudaHostAlloc / cudaHostRegister; TNS_ERR_ARG otherwise).
 * The transfers need the mesh in its own cell order (a general mesh is renumbered on the
 * device: TNS_ERR_UNSUPPORTED, use the synchronous calls).  tns_enqueue_monitored runs
 * one monitored iteration and queues its five CDIFF values into cdiff[5]; the
 * synchronisation applies the floor tns_run applies.  One record may be pending per
 * handle (TNS_ERR_STATE for a second before the synchronisation). */
int tns_upload_state_async(tns_handle *h, const double *c1, const double *c2, const double *c3,
                           const double *c4, const double *c5);
int tns_enqueue_monitored(tns_handle *h, double *cdiff);
int tns_download_state_async(tns_handle *h, double *c1, double *c2, double *c3, double *c4,
                             double *c5);

/* Downloads C1..C5(1:NELES) (for restart.in, turbnstwod.f90:171-195). */
int tns_download_state(tns_handle *h, double *c1, double *c2, double *c3, double *c4,
                       double *c5);

/* U, V, T, P as the reference leaves them after its last stage (interior cells from the
 * last stage's PRIMITIVE_VARS, ghosts from its APPLY_BOUNDARY), scattered to Fortran
 * ids: u[id-1] for cells 1..NELES and ghosts NGHOST(k).  Arrays must hold the largest
 * id.  Feeds POSTPROCESS (solver_state.f90:230-283). */
int tns_download_primitives(tns_handle *h, double *u, double *v, double *t, double *p);

/* POSTPROCESS on the GPU (solver_state.f90:237-281): node averages of P, U, V, T of the
 * last stage (cells in element order, then ghosts in bc.in order, divided by their
 * count), scattered to node ids: pn[id-1], id = 1..NODS.  tec_plot.dat's P[bar], RHO and
 * MACH follow from these (solver_state.f90:272-278). */
int tns_node_averages(tns_handle *h, double *pn, double *un, double *vn, double *tn);

/* Boundary integrals on the GPU over the faces whose bc.in line has NTYPE == type and
 * NSIDE == side (0 = any), with the face state (parent + ghost)/2 of the last stage and
 * the face vector S of geometry.f90:77-99 (per radian when IAXIS=1):
 * out[0] = sum P*SX, out[1] = sum P*SY (pressure force on those faces), out[2] =
 * sum RHO*(U*SX + V*SY) (mass flow out through them), out[3] = sum |S|.  No reference
 * counterpart (THRUST is declared in solver_state.f90:40 but never computed). */
int tns_boundary_integrals(tns_handle *h, int type, int side, double out[4]);

/* Mass-weighted total pressure over the same faces (NTYPE == type, NSIDE == side, 0 =
 * any), on the GPU: out[0] = sum P0*|MDOT|, out[1] = sum |MDOT| with the face's total
 * pressure P0 = P (1 + (GAMA-1)/2 M^2)^(GAMA/(GAMA-1)), M^2 = (U^2+V^2)/(GAMA RR T) and
 * mass flux MDOT = RHO (U SX + V SY) of the face state above.  The total-pressure loss
 * between an inlet and an outlet face set is 1 - (o[0]/o[1]) / (i[0]/i[1]).  No
 * reference counterpart (an objective of the discrete adjoint). */
int tns_total_pressure_sums(tns_handle *h, int type, int side, double out[2]);

/* The face state of every boundary face, in bc.in order, computed on the GPU: out
 * [5][NGHOSTS] = U, V, P, RHO, T of (parent + ghost)/2 of the last stage (RHO the average
 * of P/(RR*T) on both sides).  The wall pressure distribution is out[2] on the wall
 * lines.  No reference counterpart. */
int tns_boundary_face_states(tns_handle *h, double *out);

/* Frozen terms of the last iteration, for checking: which = 0: D241..D245 (5 arrays),
 * 1: VISU, VISV, VIST, VISR (4), 2: DT (1).  out holds count*NELES doubles, cell order
 * 1..NELES per array. */
int tns_debug_fetch(tns_handle *h, int which, double *out);

/* Accuracy check of the FP64 helpers the kernels use in place of library calls,
 * elementwise on n host values: fn 0 = T**0.6 (viscosity law, viscous.f90:188),
 * fn 1 = tanh(a)/tanh(b) (damping ratios, viscous.f90:191, source_terms.f90:64-67),
 * fn 2 = expm1(a) for 0 <= a <= 40 (the function behind fn 1).
 * For tests; allocates and frees its own device memory. */
int tns_debug_math(int fn, long long n, const double *a, const double *b, double *out);

/* Runs the next tns_run on this CUDA stream (cudaStream_t passed as void*; NULL
 * restores the handle's own stream). */
int tns_set_stream(tns_handle *h, void *stream);

/* Per-kernel device timing of the next tns_run calls (CUDA events around every
 * launch); tns_kernel_times returns, for kernel k, the summed milliseconds and the
 * launch count.  Kernel ids: 0 dissipation, 1 viscous flux, 2 RK stages (all four),
 * 3 dtmin, 4 gport. */
int tns_profile(tns_handle *h, int enable);
int tns_kernel_times(tns_handle *h, int kernel, double *ms, long long *launches);

/* Number of kernel launches issued by this handle so far. */
long long tns_launch_count(tns_handle *h);

const char *tns_last_error(tns_handle *h);

/* Allocation-free time step.  No counterpart in the reference: it serves callers that
 * cannot allocate device memory while they run the solver -- hosts whose device memory
 * all comes from one preallocated pool or arena (an allocation outside it fails or
 * breaks their accounting), and plugin hosts that forbid allocation on their time loop
 * (cudaMalloc synchronises the device and may stall other work).  It computes, for a
 * state already in device memory, the per-cell time step
 * DT = CFL*DL/(|V| + sqrt(GAMA*RR*T)) and DTMIN = min(1e5, min DT) of
 * turbnstwod.f90:97-108, exactly as the handle-based path does, without a handle.
 *
 *   d_q      device, [5][ncell] conservative state, component-major (C1 block, C2, ...)
 *   d_cfldl  device, [ncell] CFL*DL per cell (DL = shortest cell edge, geometry.f90:70-74)
 *   params   gama, amol and cfl are read (the others may be zero)
 *   d_dt     device, [ncell] out: DT per cell (the LOCAL=1 step)
 *   d_dtmin  device, one double out: DTMIN (the LOCAL=0 step)
 *   stream   cudaStream_t as void* (NULL = the legacy default stream)
 *
 * Its reduction scratch is a fixed array inside the library (one partial minimum per
 * block of TNS_NOALLOC_CELLS_PER_THREAD*256 cells, at most TNS_NOALLOC_MAX_BLOCKS
 * blocks: 64 KiB), so ncell is limited to TNS_NOALLOC_MAX_CELLS; larger problems get
 * TNS_ERR_TOO_LARGE.  It calls no cudaMalloc / cudaFree.  The first call on each device
 * looks up the array's device address (cudaGetSymbolAddress), so make that first call
 * before any stream capture starts.  The address is kept until the process exits; after
 * cudaDeviceReset on that device it no longer names the array, so do not call this entry
 * point on a device that has been reset.  All calls share the one array, so calls that
 * may overlap on the GPU (different streams without ordering) race; serialise them.
 * The call is asynchronous on `stream`. */
#define TNS_NOALLOC_MAX_BLOCKS 8192
#define TNS_NOALLOC_CELLS_PER_THREAD 4
#define TNS_NOALLOC_MAX_CELLS (256LL * TNS_NOALLOC_CELLS_PER_THREAD * TNS_NOALLOC_MAX_BLOCKS)
int tns_time_step_noalloc(const double *d_q, const double *d_cfldl, long long ncell,
                          const tns_params *params, double *d_dt, double *d_dtmin, void *stream);
void tns_destroy(tns_handle *h);

/* ---- Discrete adjoint of one FP64 RK4 iteration (no counterpart in the reference,
 * which has no adjoint).  For the iteration map Q_{n+1} = G(Q_n) of
 * turbnstwod.f90:95-146 -- DT, DISSIPATION, and four stages of PRIMITIVE_VARS,
 * APPLY_BOUNDARY (types 2-7, with the type-6 port mass flux), VISCOUS (stage 1), SOURCE_TERMS, RESIDUAL, UPDATE --
 * tns_adjoint_step replaces lambda = dJ/dQ_{n+1} by lambda dG/dQ_n, recomputing the
 * iteration from the checkpoint Q_n on the device.  Non-smooth points (DMAX1 / DMIN1,
 * |x|, the C5 clip, the sensor maxima) take the branch the forward took.  With
 * TNS_ADJ_SENSITIVITIES it also accumulates lambda dG/dp, summed over calls, for:
 *   SX(4), SY(4) per cell (face vectors), VOL, DL per cell, the centroids of the cells
 *   and ghosts on the (NI+2) x (NJ+2) halo grid (x then y), the node coordinates (x then
 *   y), RTOLERANCE (per cell, per node: sum them), T0 and S0 of the type-2 inlet (per
 *   cell: sum them)
 * in that order (tns_adjoint_sensitivity_size values), which a caller maps to node
 * displacements and flow parameters with the derivatives of COMPUTE_GEOMETRY and of its
 * parameter formulas.  Requirements: an FP64 handle, cells numbered in (i, j) order
 * (faces 1..4 = j-, i+, j+, i-), at least 3 x 3 cells.  The type-6 port ghosts' node-y
 * sensitivities (through the port mass flux) are part of the node-coordinate block.  Device arrays are
 * [5][NELES] component-major in that order; calls are asynchronous on the handle's
 * stream (tns_set_stream). */
#define TNS_ADJ_SENSITIVITIES 1
/* TNS_ADJ_FROZEN: Q_n is the state of the previous call (d_q is not read); the forward
 * values kept from that call are reused, which skips the recomputed iteration and every
 * state-only pass -- the fixed-point adjoint at a converged state. */
#define TNS_ADJ_FROZEN 2
/* TNS_ADJ_SCALARS: accumulate only the RTOLERANCE, T0 and S0 sensitivities (enough for
 * gradients with respect to P0, T0 and AMACHINIT); the geometric blocks stay untouched.
 * TNS_ADJ_SENSITIVITIES (everything) takes precedence. */
#define TNS_ADJ_SCALARS 4
int tns_adjoint_enable(tns_handle *h);
int tns_adjoint_step(tns_handle *h, const double *d_q, double *d_lam, int flags);
/* The same step, with the forward values of the next checkpoint d_q_next (the state the
 * following call will reverse, e.g. Q_{n-1}) computed beside this step's reverse on the
 * GPU, on a low-priority branch.  The following call with d_q == d_q_next then skips its
 * recomputation; the memory at d_q_next must not change in between.  d_q_next may be
 * NULL.  Results are bitwise those of tns_adjoint_step; on a B200 at 98k cells the
 * overlapped step measured slower (439 us) than recomputing in sequence (410 us). */
int tns_adjoint_step_next(tns_handle *h, const double *d_q, const double *d_q_next, double *d_lam, int flags);
/* Recorded forward values, for transient sweeps with memory to spare: tns_adjoint_record
 * runs one iteration from d_q (the solver's kernels, the same result as tns_enqueue),
 * writes Q_{n+1} to d_q_next and the iteration's forward values -- stage inputs 1-3, D,
 * VIS, DT, DTMIN, the port mass flux of each stage -- to d_rec
 * (tns_adjoint_record_size doubles).  tns_adjoint_step_recorded(h, Q_n, rec_n, ...)
 * then skips the recomputation (same results as tns_adjoint_step).  d_q_next may equal
 * d_q (the last stage reads only each cell's own old value); d_rec must overlap neither. */
long long tns_adjoint_record_size(tns_handle *h);
int tns_adjoint_record(tns_handle *h, const double *d_q, double *d_q_next, double *d_rec);
int tns_adjoint_step_recorded(tns_handle *h, const double *d_q, const double *d_rec, double *d_lam, int flags);
long long tns_adjoint_sensitivity_size(tns_handle *h);
/* Copies the accumulated sensitivities to host memory `out` (count values, which must
 * equal tns_adjoint_sensitivity_size) and, with reset != 0, zeroes them. */
int tns_adjoint_sensitivities(tns_handle *h, double *out, long long count, int reset);
long long tns_adjoint_launch_count(tns_handle *h);
/* Device-to-device copy of the FP64 state: direction 0 copies it to d_buf, 1 loads it
 * from d_buf ([5][NELES], (i, j) numbering).  For checkpointing on the device. */
int tns_copy_state_device(tns_handle *h, double *d_buf, int direction);

/* ---- Batch of cases (no counterpart in the reference, which solves one case per run).
 * A batch advances several handles made by tns_create together: every kernel phase of
 * an RK4 iteration is one launch over the tiles of all active cases.  The cases may
 * differ in mesh size, geometry and parameters; they share one precision mode.  State
 * moves in and out through each member's tns_upload_state / tns_download_state /
 * tns_download_primitives, before and after tns_batch_run.  The batch borrows the
 * handles: destroy the batch first.  A batch with a general-mesh case (one that is not
 * one structured i x j block) starts in schedule 2 and runs schedules 1 and 2 only. */
typedef struct tns_batch tns_batch;

int tns_batch_create(tns_handle *const *cases, int ncases, tns_batch **out);

/* Runs up to niter RK4 iterations of every active case.  Residual records (the five
 * CDIFF values of tns_run) are taken every monitor_every-th iteration of the call and
 * written to cdiff_out[case][max_records][5]; n_records[case] receives each count.
 * stop_ratio > 0 enables convergence masking: a case stops (becomes inactive) at the
 * first record where max_k CDIFF_k / REF_k <= stop_ratio.  REF is cdiff_ref[case][5]
 * when its entries are positive; otherwise the first iteration of the call is monitored
 * and its CDIFF becomes REF (written back to cdiff_ref when non-NULL, so a later call
 * can continue the criterion).  iterations[case] receives the iterations each case ran.
 * A case whose state becomes non-finite is masked off (case_status[case] =
 * TNS_ERR_NONFINITE) while the others continue; the call then returns TNS_ERR_NONFINITE.
 * Any output pointer may be NULL. */
int tns_batch_run(tns_batch *b, int niter, int monitor_every, double stop_ratio, double *cdiff_ref,
                  double *cdiff_out, int max_records, int *n_records, int *iterations,
                  int *case_status);

/* Per-case active mask (1 = iterate).  Re-activating a case that failed clears its
 * failure: upload a finite state to it first. */
int tns_batch_set_active(tns_batch *b, const int *active);

/* How a batch iteration is scheduled: 0 (default) = one launch per kernel phase over
 * the tiles of all active cases; 1 = every case's own tns_run launches, the cases on
 * parallel branches of one CUDA graph so they run concurrently; 2 = as 1, with 8
 * unmonitored iterations per graph so each case runs ahead without a join between
 * iterations; 3 = one persistent cooperative launch per run of up to 256 unmonitored
 * iterations, its blocks walking the tile table of all active cases phase by phase with
 * grid barriers between the phases (monitored iterations as schedule 0); it needs
 * LOCAL=1 and no type-6 port in every case (TNS_ERR_UNSUPPORTED otherwise), and a grid
 * barrier that does not complete in its bounded wait ends the run with TNS_ERR_CUDA.
 * Schedules 0 and 3 need every case to be one structured i x j block
 * (TNS_ERR_UNSUPPORTED otherwise).  Results are identical; which is fastest depends on
 * the case mix (tnsgpu.autotune measures them). */
int tns_batch_set_schedule(tns_batch *b, int schedule);
int tns_batch_get_schedule(tns_batch *b);

/* Captures and instantiates, without running anything, every CUDA graph that
 * tns_batch_run launches under the current schedule and active mask: the monitored and
 * the unmonitored iteration (schedules 0-2), schedule 2's 8-iteration block, in mixed
 * precision one of each per state-buffer parity.  Otherwise each is captured at its
 * first use inside tns_batch_run.  A change of schedule or of the active mask drops
 * them; call it again after one. */
int tns_batch_prepare(tns_batch *b);
int tns_batch_get_active(tns_batch *b, int *active);
long long tns_batch_launch_count(tns_batch *b);
const char *tns_batch_last_error(tns_batch *b);
void tns_batch_destroy(tns_batch *b);

#ifdef __cplusplus
}
#endif
#endif
