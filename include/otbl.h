/*
 * otbl.h -- C ABI of the B200 RK3 substep of OpenTBL's zero-pressure-gradient
 * boundary-layer DNS.
 *
 * The reference exposes the substep as Fortran external subroutines with
 * implicit interfaces, called from bl_1.F90:98-119 with every coefficient and
 * size held in module globals (mod.F90). Here the globals become an explicit
 * context: the config struct, a packed coefficient buffer (otbl_layout.h) and
 * the device-resident state. Every entry point returns an int status
 * (OTBL_OK = 0) and otbl_last_error() gives the message. Calls on one context
 * are stream-ordered on the context's CUDA stream and are not re-entrant;
 * different contexts may be driven from different host threads. otbl_rhsp
 * forks part of its kernels onto two internal streams of the context and
 * joins them back into the context stream before its work ends, so callers
 * see a single ordered stream (a capture of that stream records the forks).
 *
 * Field arrays use the reference's single-rank plane layout (otbl_layout.h).
 * Plane indices i, rows j and the recycling plane xout are 1-based, as in the
 * Fortran.
 */
#ifndef OTBL_H
#define OTBL_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define OTBL_OK 0
#define OTBL_ERR_ARG 1      /* bad argument (null pointer, bad id, bad size) */
#define OTBL_ERR_CONFIG 2   /* inconsistent configuration                     */
#define OTBL_ERR_OOM 3      /* device allocation failed                       */
#define OTBL_ERR_CUDA 4     /* CUDA runtime error                             */
#define OTBL_ERR_NAN 5      /* non-finite value detected by the dt reduction,
                               or genflu could not profile its rescaled grid
                               (otbl_last_error tells which)                 */
#define OTBL_ERR_NODEV 6    /* no CUDA device / extension not usable          */
#define OTBL_BUSY 7         /* otbl_query / otbl_graph_query: work in flight  */
#define OTBL_ERR_TIMEOUT 8  /* a bounded device-side wait gave up             */

/* transposes (change.f90): round the payload to REAL4 as the reference's
 * MPI_ALLTOALLV(MPI_REAL4) does (change.f90:579,608,641,652,676,686), or
 * keep full FP64 */
#define OTBL_XPOSE_NONE 0
#define OTBL_XPOSE_FP32 1

/* time step: recomputed from the CFL limits at substep 1 of every step
 * (bl_1.F90:91, rhsp.F90:214-262), or held fixed */
#define OTBL_DT_ADAPTIVE 0
#define OTBL_DT_FIXED 1

/* arithmetic of the substep (no counterpart in the reference, which is FP64
 * throughout). OTBL_PREC_FP64: every operator in FP64. OTBL_PREC_MIXED: the
 * velocity (u, v, w), the RK3 combination, implzy, the divergence, the
 * Poisson solve of spanwise modes 0..3, the projection, dt, genflu and the
 * energies stay FP64; the x and y mid-point interpolations, d/dx of
 * difvisxx, the spanwise FFTs, the nonlinear products and the Poisson solve
 * (x-DCTs and y-systems) of spanwise modes >= 4 run in FP32, and the fifteen
 * intermediate fields they exchange, the pressure p and the RHS history
 * rhs*pa are stored in FP32 (their updates computed in FP64). otbl_set_field / otbl_get_field convert those
 * fields from and to the caller's FP64 arrays; otbl_field_device_ptr refuses
 * them (OTBL_ERR_CONFIG). Not combined with OTBL_XPOSE_FP32. */
#define OTBL_PREC_FP64 0
#define OTBL_PREC_MIXED 1

/* options (no counterpart in the reference). OTBL_OPT_YDENSE: on the mixed
 * path, interpyy (lip.f90:359-440) runs as a dense ny x (ny+1) operator on
 * the tensor cores (tcgen05, TF32 in three parts, FP32 accumulation) in
 * place of the banded solve; needs OTBL_PREC_MIXED and ny <= 256. It moves
 * exactly the field bytes but is bound by the shared-memory operand traffic
 * of its three products: on B200 at 1025x193x512 it took 0.98 ms per
 * substep against 0.67 ms for the banded solve, so it is off by default. */
#define OTBL_OPT_YDENSE 1

typedef struct otbl_config {
  int nx, ny, nz;   /* grid (mod.F90:22); nz1 = 2*(nz/3), nz2 = nz1/2-1     */
  int xout;         /* recycling plane, 1-based (mod.F90:23)               */
  int xpose_round;  /* OTBL_XPOSE_*                                        */
  int dt_mode;      /* OTBL_DT_*                                           */
  double re, ax, ay, az, cfl; /* input deck, bl_1.F90:207-210              */
  double y_blend;   /* height that replaces y(119) in genflu.F90:57        */
  double dt_fixed;  /* dt for OTBL_DT_FIXED; <= 0 freezes the first CFL dt */
  int precision;    /* OTBL_PREC_*                                         */
  int options;      /* OTBL_OPT_* bits, 0 for none                         */
} otbl_config;

/* field ids for otbl_set_field / otbl_get_field / otbl_field_device_ptr */
enum {
  OTBL_F_U = 0, OTBL_F_V, OTBL_F_W, OTBL_F_P,
  OTBL_F_RHSUPA, OTBL_F_RHSVPA, OTBL_F_RHSWPA,
  OTBL_F_COUNT
};

/* inflow-recycling state of module genmod (mod.F90:86-93) plus the clock */
typedef struct otbl_inflow {
  double tiempo;    /* simulation time (bl_1.F90:128)                      */
  double timeinit;  /* time origin of the mean-profile filter              */
  double dt;        /* current time step                                   */
  double utauout, rthout, dout, gamma1, gamma2, timec; /* genflu outputs   */
  double umax, wmax, vmax; /* CFL maxima of the last dt reduction          */
} otbl_inflow;

/* ---- setup (host only; coeft.f90 coef, bl_1.F90 inlet_retheta, boun.f90
 *      magicnumber) ---- */
int otbl_config_check(const otbl_config *cfg);
size_t otbl_coef_count(int nx, int ny, int nz);
int otbl_coef_offset(int nx, int ny, int nz, int id, size_t *off);
/* y: y(0:ny+1) (ny+2 values); u0: inlet mean profile u(k=0, 1:ny+1, i=1)
 * (getstartzy-bg.F90:273). Fills coef[otbl_coef_count()] */
int otbl_coef_compute(const otbl_config *cfg, const double *y,
                      const double *u0, double *coef);

/* ---- context ---- */
typedef struct otbl_ctx otbl_ctx;
int otbl_ctx_create(const otbl_config *cfg, const double *coef, int device,
                    otbl_ctx **out);
void otbl_ctx_destroy(otbl_ctx *ctx);
const char *otbl_last_error(const otbl_ctx *ctx);
size_t otbl_device_bytes(const otbl_ctx *ctx);
/* device bytes otbl_ctx_create allocates for cfg (0 if cfg is invalid) */
size_t otbl_ctx_bytes(const otbl_config *cfg);
/* re-binds a context to another box of the same nx, ny, nz and precision:
 * new config values (xout, re, ax, az, cfl, ...) and coefficients, no device
 * allocation; the state is then uploaded with otbl_set_field and
 * otbl_set_inflow. For slot reuse by a serving loop (no counterpart in the
 * reference). Synchronizes. */
int otbl_ctx_rebind(otbl_ctx *ctx, const otbl_config *cfg, const double *coef);

/* host <-> device copies of the state, reference layout */
int otbl_set_field(otbl_ctx *ctx, int id, const double *host);
int otbl_get_field(otbl_ctx *ctx, int id, double *host);
int otbl_field_device_ptr(otbl_ctx *ctx, int id, double **dptr);
/* u0 (ny+1), v0 (ny): inlet profiles (getstartzy-bg.F90:273-276);
 * um (ny+1): filtered mean profile at xout (readheader, getstartzy-bg.F90:578).
 * A restart: also clears the error flag, the frozen dt of OTBL_DT_FIXED with
 * dt_fixed <= 0 and the energies. */
int otbl_set_inflow(otbl_ctx *ctx, const double *u0, const double *v0,
                    const double *um, const otbl_inflow *st);
int otbl_get_inflow(otbl_ctx *ctx, double *um, otbl_inflow *st);
/* ener(1:15) of module statistics (mod.F90:264) as rhsp leaves it: set by
 * energies at substep m = 1 (rhsp.F90:116, rhsp.F90:493-509 with ministats,
 * stotf.F90:395-440) from the state rhsp was called on, ener(13:15) zeroed
 * at the end of rhsp (rhsp.F90:487). One context holds every plane, so the
 * values are those of plane nx/2 (its branch of ministats overwrites the
 * plane-1 branch's ener(1:3)). Zero before the first rhsp(m = 1). */
int otbl_get_energies(otbl_ctx *ctx, double *ener);

/* ---- one-point statistics, statsp (stotf.F90:51-291) ----
 * otbl_statsp adds one sample of the one-point statistics of the context's
 * current state to its accumulators, as rhsp does on its first substep when
 * dostat is set (bl_1.F90:92, rhsp.F90:70-101): the x pre-pass (u
 * interpolated to the half points in x and shifted by one plane, d/dx of it
 * and of v and w; lip.f90:703-765, with the fd_ix/fd_dx operators), then per
 * plane the interpolation onto the wall positions in y (interpy_new, fd_iy
 * and fd_iyp) and the y derivatives (diffy_inplace, fd_dvdy), and the sums
 * over the spanwise modes (cte = 1 for k = 0, 2 otherwise) and over the
 * physical points of the triple products. Call it between substeps, where
 * the reference sets dostat; it uses the context's line scratch and its
 * stream, leaves the state unchanged, and synchronizes nothing. The
 * accumulators (OTBL_NSTATS arrays of the reference's shape (ny, nx), column
 * major: stat(j, i) at s*nx*ny + (i-1)*ny + (j-1)) are allocated on the
 * first call (OTBL_NSTATS*nx*ny doubles, beyond otbl_ctx_bytes; from then
 * on otbl_device_bytes counts them) and start at zero; otbl_get_stats
 * copies them and the number of
 * samples (the reference's totalcal, mod.F90:278) to the host
 * (synchronizes); otbl_reset_stats zeroes them. The spectra, the two-point
 * correlations and the instantaneous enstrophy field of statsp are not
 * computed. On the mixed path the pressure is read from its FP32 storage;
 * everything else is FP64 on both paths. */
enum {
  OTBL_ST_UA = 0, OTBL_ST_VA, OTBL_ST_WA, OTBL_ST_PM,          /* means (k = 0)      */
  OTBL_ST_DUDX0, OTBL_ST_DVDX0, OTBL_ST_DWDX0,                /* mean gradients     */
  OTBL_ST_DUDY0, OTBL_ST_DVDY0, OTBL_ST_DWDY0,
  OTBL_ST_VORTXA, OTBL_ST_VORTYA, OTBL_ST_VORTZA,             /* mean vorticity     */
  OTBL_ST_US, OTBL_ST_VS, OTBL_ST_WS, OTBL_ST_UV, OTBL_ST_UW, OTBL_ST_VW, /* stresses */
  OTBL_ST_PUP, OTBL_ST_PVP, OTBL_ST_PP, OTBL_ST_PDUDX, OTBL_ST_PDUDY, /* pressure     */
  OTBL_ST_PDVDX, OTBL_ST_PDVDY, OTBL_ST_PDWDZ,
  OTBL_ST_VORTX, OTBL_ST_VORTY, OTBL_ST_VORTZ,                /* vorticity squares  */
  OTBL_ST_DISPU, OTBL_ST_DISPV, OTBL_ST_DISPW, OTBL_ST_DISPUV, /* dissipation       */
  OTBL_ST_U3, OTBL_ST_V3, OTBL_ST_U2V, OTBL_ST_V2U, OTBL_ST_W2V, OTBL_ST_W2U, /* triple */
  OTBL_NSTATS
};
int otbl_statsp(otbl_ctx *ctx);                     /* stotf.F90:51       */
int otbl_get_stats(otbl_ctx *ctx, double *stats_host, int *samples);
int otbl_reset_stats(otbl_ctx *ctx);

/* ---- the substep, bl_1.F90:94-125 ----
 * m = RK3 substep 1..3; setstep = 1 recomputes dt (adaptive mode). */
int otbl_rhsp(otbl_ctx *ctx, int m, int setstep);   /* rhsp.F90:22        */
int otbl_outflow_correction(otbl_ctx *ctx);         /* boun.f90:63        */
int otbl_pois(otbl_ctx *ctx, int m);                /* pois.f90:11, with
                                     varstep = 0.5/dt/rkdv(m), bl_1.F90:117 */
int otbl_substep(otbl_ctx *ctx, int m, int setstep);
/* nsteps full RK3 steps, tiempo += dt after each (bl_1.F90:85-128) */
int otbl_advance(otbl_ctx *ctx, int nsteps);
int otbl_sync(otbl_ctx *ctx);

/* ---- pieces of the path, on device buffers owned by the caller ---- */
/* change.f90:224/257, in the reference's argument order chp2x(pen, plan,
 * ...) and chx2p(pen, plan, ...): planes (0:nz2, jee, nx) -> pencils
 * (nx, nz1*jee) and back, rounding to REAL4 when the context's xpose_round
 * is OTBL_XPOSE_FP32 (the reference's buf and communicator arguments have no
 * counterpart: one context holds the whole box) */
int otbl_chp2x(otbl_ctx *ctx, double *pen_dev, const double *plan_dev, int jee);
int otbl_chx2p(otbl_ctx *ctx, const double *pen_dev, double *plan_dev, int jee);
/* ffts.f90:27 fourxz on nlines z-lines: iopt<0 r2c (phys -> fou, x 1/nz,
 * modes 0..nz2 kept); iopt>=0 c2r (fou -> phys, modes > nz2 zeroed).
 * fou: nlines x (nz2+1) complex; phys: nlines x (nz+2) reals */
int otbl_fourxz(otbl_ctx *ctx, double *fou_dev, double *phys_dev, int iopt,
                int nlines);
/* ffts.f90:147 cosftx on nlines x-lines of length nx stored as pencils
 * c(nx, nlines): transforms c(2:nx, :), iopt<0 REDFT10 x 1/(nx-1),
 * iopt>=0 REDFT01 x 0.5 */
int otbl_cosftx(otbl_ctx *ctx, double *c_dev, int nlines, int iopt);
int otbl_boun(otbl_ctx *ctx);                        /* boun.f90:7         */
/* lip.f90:359-440 interpyy of the context's u, w (u-type input) and v
 * (v-type input), as rhsp calls it (rhsp.F90:146,367,393), with the
 * context's operator (banded solve, or the dense tensor-core operator under
 * OTBL_OPT_YDENSE); the three outputs (nx*ny*nz1 each, plane layout) are
 * copied to the host as doubles. Synchronizes. */
int otbl_interpyy(otbl_ctx *ctx, double *uy_host, double *wy_host, double *vy_host);
int otbl_genflu(otbl_ctx *ctx);                      /* genflu.F90:3       */

/* ---- genflu without allocation (no counterpart in the reference, whose
 *      genflu works on module arrays that exist for the whole run) ----
 * genflu.F90:3 as otbl_genflu, on device buffers owned by the caller: u_dev,
 * w_dev (nx, ny+1, nz1) and v_dev (nx, ny, nz1) in the plane layout (plane
 * xout is read, plane 1 written), u0_dev (ny+1), v0_dev (ny), um_dev (ny+1,
 * updated), scal_dev (OTBL_GF_COUNT doubles, slots below), err_dev (one int,
 * may be NULL; set to OTBL_ERR_NAN when the rescaled grid cannot be
 * profiled, never cleared: start it at 0). Only the context's coefficients
 * and stream are used; the launches are ordered on that stream.
 *
 * It is for callers that cannot allocate device memory at call time, e.g. a
 * host that keeps the fields in its own allocations and has given the rest
 * of HBM to its own pool, or one whose time loop must not be stalled by the
 * device-wide synchronisation of cudaMalloc/cudaFree. The scratch that
 * carries genflu's rescaling tables from one launch to the next,
 * 3*(ny+1)+2 doubles, is a static device array of OTBL_GENFLU_SCRATCH_MAX
 * doubles in this library; larger grids are refused with OTBL_ERR_CONFIG.
 * The first call on each device looks up the array's address (and may load
 * the library's device module): make that call before any stream capture.
 * The address is kept for the life of the process and belongs to the
 * device's primary context, the one the CUDA runtime and every context of
 * this library use (the call makes the context's device current with
 * cudaSetDevice). A cudaDeviceReset destroys that context, and with it this
 * address and every otbl_ctx's buffers: after a reset, reload the library
 * before calling it again.
 * The scratch need not start at zero. All calls on one device share the
 * array: calls that can run at the same time (different streams, contexts or
 * host threads without ordering) race. No device or
 * host memory is allocated on the success path. */
enum {
  OTBL_GF_DT = 0, OTBL_GF_TIEMPO, OTBL_GF_TIMEINIT,           /* inputs  */
  OTBL_GF_TIMEC, OTBL_GF_UTAUOUT, OTBL_GF_RTHOUT, OTBL_GF_DOUT,
  OTBL_GF_GAMMA1, OTBL_GF_GAMMA2,                              /* outputs */
  OTBL_GF_COUNT
};
/* doubles (16 KiB) per device. Admitted grids: ny <= 680, where the tables
 * fit and genflu's shared memory stays within 48 KB; larger ny is refused
 * with OTBL_ERR_CONFIG */
#define OTBL_GENFLU_SCRATCH_MAX 2048
int otbl_genflu_noalloc(otbl_ctx *ctx, double *u_dev, double *v_dev,
                        double *w_dev, const double *u0_dev,
                        const double *v0_dev, double *um_dev,
                        double *scal_dev, int *err_dev);

/* ---- the reference's array surface: the state in the caller's device
 *      arrays ----
 * The reference's subroutines take the state as arguments (rhsp.F90:22-27,
 * pois.f90:11, boun.f90:7,63, genflu.F90:3); these entry points take the
 * caller's device arrays of the FP64 path in the plane layout of
 * otbl_layout.h (u, w, rhsupa, rhswpa: nx*(ny+1)*nz1 doubles; v, p, rhsvpa:
 * nx*ny*nz1), 16-byte aligned. The reference's twin arguments (ut and the
 * pencil view of the same memory, res/rest, rhsut/rhsut work arrays, wki*,
 * wkp, wkf, buffers) are one buffer each: a Fortran wrapper passes the
 * state and drops the work arrays, which live in the context.
 *
 * otbl_bind_state points the context's seven state fields at the given
 * arrays (NULL: the context's own array for that field) and keeps them
 * bound for every later call on the context, until the next bind. It
 * re-encodes the TMA descriptors that name the state on the host; it does
 * not synchronize, and launches already issued keep the arrays they were
 * given. A CUDA graph (otbl_graph_create) keeps the arrays bound when it was
 * captured. The caller orders its own writes to the arrays before the call
 * (see the ordering notes of INTEGRATION.md) and keeps them alive while
 * bound. OTBL_ERR_CONFIG on the mixed-precision path, which stores p and the
 * RHS history in FP32.
 *
 * Each *_arrays entry point binds the arrays it is given and runs the
 * context entry point of the same name; with the same arrays bound, the
 * results are bit for bit those of the context API. */
int otbl_bind_state(otbl_ctx *ctx, double *u, double *v, double *w, double *p,
                    double *rhsupa, double *rhsvpa, double *rhswpa);
/* rhsp(ut,vt,wt,pt,rhsupat,rhsvpat,rhswpat, <work arrays>, dt, m, ...),
 * rhsp.F90:22-27; dt and the step counters live in the context */
int otbl_rhsp_arrays(otbl_ctx *ctx, double *u, double *v, double *w, double *p,
                     double *rhsupa, double *rhsvpa, double *rhswpa, int m,
                     int setstep);
/* outflow_correction(ut,vt,rhsupat,communicator), boun.f90:63 */
int otbl_outflow_correction_arrays(otbl_ctx *ctx, double *u, double *v,
                                   double *rhsupa);
/* pois(ut,vt,wt,pt,res,rest,rt,varstep,...), pois.f90:11; res/rest/rt are
 * the context's scratch and varstep = 0.5/dt/rkdv(m) (bl_1.F90:117) */
int otbl_pois_arrays(otbl_ctx *ctx, double *u, double *v, double *w, double *p,
                     int m);
/* boun(ut,vt,wt), boun.f90:7 */
int otbl_boun_arrays(otbl_ctx *ctx, double *u, double *v, double *w);
/* genflu(ut,vt,wt,y,re,dt,tiempo,...), genflu.F90:3; y, re, dt, tiempo and
 * the genmod state live in the context */
int otbl_genflu_arrays(otbl_ctx *ctx, double *u, double *v, double *w);

/* kernel launches issued by this context since creation */
long long otbl_launch_count(const otbl_ctx *ctx);

/* ---- CUDA graphs of RK3 steps, ensembles (no counterpart in the reference,
 *      which advances one box per MPI job) ----
 * otbl_graph_create captures otbl_advance(ctx[k], nsteps) of n contexts on
 * one device into one CUDA graph, each context a branch that runs
 * concurrently with the others. Outstanding work of the members is finished
 * first. Every otbl_graph_launch then advances every member by nsteps RK3
 * steps on the graph's own stream (asynchronous); the members must not be
 * driven through their own entry points while a launch is in flight
 * (otbl_graph_sync or a finished otbl_graph_query orders them again). The
 * graph holds the members' device buffers: destroy it before them.
 * Per-kernel profiling must be off while capturing. */
typedef struct otbl_graph otbl_graph;
int otbl_graph_create(otbl_ctx *const *ctxs, int n, int nsteps, otbl_graph **out);
int otbl_graph_launch(otbl_graph *g);
int otbl_graph_sync(otbl_graph *g);
int otbl_graph_query(otbl_graph *g);           /* OTBL_OK done, OTBL_BUSY */
int otbl_graph_stream(otbl_graph *g, void **stream);
long long otbl_graph_kernels(const otbl_graph *g); /* kernels per launch */
void otbl_graph_destroy(otbl_graph *g);
/* OTBL_OK when every call issued on the context has finished, OTBL_BUSY
 * while work is in flight (never blocks) */
int otbl_query(otbl_ctx *ctx);
/* Autotuner (no counterpart in the reference): times CTA sizes of 32, 64
 * and 128 threads for the x-interpolation, d/dx and y-interpolation line
 * kernels on this context's box and precision and keeps the fastest. Those
 * kernels write only work arrays, so the state is unchanged; the arithmetic
 * does not depend on the CTA size. choice (3 ints, may be NULL) receives the
 * sizes picked. Call before otbl_graph_create. Synchronizes. */
int otbl_autotune(otbl_ctx *ctx, int *choice);
/* sets the three CTA sizes (each 32, 64 or 128) without timing, e.g. those
 * otbl_autotune picked for another context of the same box size */
int otbl_set_tuning(otbl_ctx *ctx, const int *bs);
/* failure detection of the device-side waits (no counterpart in the
 * reference): runs the bounded mbarrier wait of the TMA-fed kernels on a
 * barrier that never completes, with a 1 ms limit; *status receives
 * OTBL_ERR_TIMEOUT when the wait gave up and the kernel returned, as the
 * product kernels do (they record it in the context's error flag, which
 * otbl_sync and otbl_get_inflow report). Synchronizes. */
int otbl_selftest_wait(otbl_ctx *ctx, int *status);

/* ---- instrumentation (no counterpart in the reference, whose timers are
 *      the MPI_WTIME accumulators of module temporal, mod.F90:311-322) ---- */
/* the context's CUDA stream (cudaStream_t), for events recorded by callers */
int otbl_get_stream(otbl_ctx *ctx, void **stream);
/* on != 0: record a CUDA event pair around every kernel launch; clears the
 * records. While on, a substep runs on the context stream alone (none of its
 * kernels overlap), so each class's time is its own kernels' duration.
 * Timing adds events and removes the overlap; leave it off for throughput. */
int otbl_profile_enable(otbl_ctx *ctx, int on);
/* totals per kernel class (kind = 0, 1, ...; OTBL_ERR_ARG past the last):
 * name, summed device milliseconds and number of launches. Synchronizes. */
int otbl_profile_read(otbl_ctx *ctx, int kind, const char **name,
                      double *total_ms, int *count);

#ifdef __cplusplus
}
#endif
#endif
