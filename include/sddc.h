/*
 * sddc.h -- C ABI of the B200 drop-in for SDDC's residual-and-time-step path.
 *
 * The drop-in replaces, on one GPU:
 *   compresid                compresid.f90:1-80   (no arguments; module setup2d state)
 *   compflux and below       compflux.f90:1-157, getrusanov.f90:1-193,
 *                            interfaceflux_all.f90:1-112, cyclocflux_all.f90:1-112,
 *                            bcflux.f90:1-377, AV.f90:1-142
 *   the RK stage updates     iterations.f90:88-213 (FiveStageRk, RK_S5P3)
 *   the monitor sums         iterations.f90:34-46
 * The Fortran host keeps mesh input, connectivity, INIT_SETUP and calcjacob
 * and passes their arrays here once.  The state stays on the device between
 * calls; it crosses only when the host asks for it.
 *
 * Conventions:
 *   - every array is in the reference's Fortran layout (column-major,
 *     variable index fastest) and every index table is 1-based, exactly as
 *     module setup2d holds it (setup2d.f90:39-102);
 *   - the host owns every array it passes and may reuse it after the call;
 *   - every function returns SDDC_OK (0) or a negative SDDC_E* code and
 *     never exits; sddc_last_error() describes the last failure;
 *   - calls on one context are serialised on the context's CUDA stream;
 *     use one context per host thread.
 *
 * A Fortran host binds these through an ISO_C_BINDING interface module
 * (bind(C) interfaces with value arguments for scalars and type(c_ptr) for
 * the context); Python binds them through ctypes (sddc_b200/solver.py).
 */
#ifndef SDDC_H
#define SDDC_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SDDC_OK 0
#define SDDC_EINVAL (-1)      /* bad argument or inconsistent tables          */
#define SDDC_ECUDA (-2)       /* CUDA error (message in sddc_last_error)      */
#define SDDC_ESTATE (-3)      /* call out of order (e.g. no tables yet)       */
#define SDDC_ENUMERIC (-4)    /* non-positive density or non-finite wave speed seen on the device */
#define SDDC_ENOMEM (-5)      /* device allocation failed                     */
#define SDDC_EIO (-6)         /* an output file could not be written          */

/* arithmetic forms of the residual */
#define SDDC_FP64_EXACT 0  /* the reference's FP64 operations, no FMA: bit-exact to the CPU oracle */
#define SDDC_FP64 1        /* FP64 with FMA contraction and reciprocals (fastest FP64) */
#define SDDC_MIXED 2       /* FP32 interpolation, fluxes and derivatives; FP64 state, RK,
                              pressure recovery and reductions */

typedef struct sddc_ctx sddc_ctx;

/* Run parameters: QUAD.INP fields (readinput.f90:6-44) plus the mode. */
typedef struct sddc_params {
    int N;          /* solution points per direction, 2..6                     */
    int ncell;      /* NCELL                                                   */
    int ncellglob;  /* NCELLGLOB (AV epsilon0, AV.f90:126); 0 means ncell      */
    int vismode;    /* 0 or 1                                                  */
    int artiv;      /* ARTIV: 1 computes the AV sensor                         */
    int k_stage;    /* 3: RK_S5P3, 5: FiveStageRk                              */
    int precision;  /* SDDC_FP64_EXACT, SDDC_FP64 or SDDC_MIXED                */
    int cells_per_cta; /* 0: default tile; else 4, 6, 8 or 16 cells per CTA    */
    double mu, eta0;   /* viscosity and resistivity (QUAD.INP), >= 0            */
    double dxcycl, dycycl;
    double rinf, pinf, uinf, vinf, bxinf, byinf; /* free stream (QUAD.INP) */
} sddc_params;

/* Creates a context on the current CUDA device.  With vismode = 1 and mu
   or eta0 nonzero every stage runs the reference's viscous / resistive
   chain (compflux.f90:36-50: nablaQsp, gradient averaging, BCVISFLUX with
   the adiabatic-wall energy gradient, getVfluxvectors) before the stage;
   with both zero that chain adds exactly +0.0 to the residual and is
   skipped.  Batches (sddc_set_cases) and the adjoint need mu = eta0 = 0. */
int sddc_create(sddc_ctx **out, const sddc_params *p);
void sddc_destroy(sddc_ctx *ctx);
const char *sddc_last_error(const sddc_ctx *ctx);

/* Tables from the host set-up, uploaded once (replaces the module arrays
   read by compresid and below):
     Lmat, Mmat (N+1,N)                       initsetup.f90:262-319
     S1 (2,2,N+1,N,NCELL), S2 (2,2,N,N+1,NCELL), Jac (N,N,NCELL)
                                              calcjacob.f90:1-132
     IF2C (NFACE,4)                           connectivity.f90:153-216
     IBFINTER(NINTER)                         connect_bdry.f90:228-244
     IBFINL, IBFOUT, IBFWAL, IBFSYMP, IBFREE  connect_bdry.f90:126-223
     CYC2FPAIR (NPAIR,2)                      map_cyc_loc.f90:9-35
   Every (cell, local face) must be covered by exactly one list entry. */
int sddc_set_tables(sddc_ctx *ctx, const double *Lmat, const double *Mmat, const double *S1,
                    const double *S2, const double *Jac, const int *IF2C, int nface,
                    const int *ibfinter, int ninter, const int *ibfinl, int ninlet,
                    const int *ibfout, int noutlet, const int *ibfwal, int nwall,
                    const int *ibfsymp, int nsymp, const int *ibfree, int nfree,
                    const int *cyc2fpair, int npair);

/* Q (9,N,N,NCELL) from the host, with the running maxima of the wave speed
   and the velocity that set c_h (compflux.f90:6; both 0 at start,
   initsetup.f90:166-167) and the solution time. */
int sddc_set_state(sddc_ctx *ctx, const double *Q, double ctime, double eigvmax, double umax);

/* One residual evaluation of the current state, as compresid: keeps resid,
   nablaQs and the AV sensor on the device and advances the running maxima. */
int sddc_compresid(sddc_ctx *ctx);

/* nsteps time steps of size dt with the scheme of k_stage (RK_S5P3 or
   FiveStageRk), 5 residual evaluations per step.  Launches are captured in a
   CUDA graph after the first step.  Returns SDDC_ENUMERIC if any stage saw a
   non-positive density or a non-finite wave speed (the state is still
   advanced, as the reference would). */
int sddc_rk_step(sddc_ctx *ctx, double dt, int nsteps);

/* Copies device results to the host; any pointer may be NULL.
     Q (9,N,N,NCELL)
     resid (9,N,N,NCELL), nablaQs (9,2,N,N,NCELL): from the last
       sddc_compresid (resid also after the last stage of sddc_rk_step is
       not kept; pass NULL then)
     muAV (2,NCELL): AV.f90:129-140 from the last evaluation's sensor
     sm_ind (2,NCELL): the sensor log10 values (SM_IND) */
int sddc_get_state(sddc_ctx *ctx, double *Q, double *resid, double *nablaQs, double *muAV,
                   double *sm_ind);

/* Monitor sums of the last residual evaluation (iterations.f90:35-46):
   sum of resid^2 over all variables and of divB^2; plus the integrals of
   density and total energy (sum of Jac * w_i * w_j * Q with w the
   quadrature weights of the solution points). */
int sddc_monitor(sddc_ctx *ctx, double *residsum, double *divbsum, double *mass, double *energy);

/* Running maxima after the last evaluation and the c_h used by the next. */
int sddc_get_maxima(sddc_ctx *ctx, double *eigvmax, double *umax, double *c_h, double *ctime);

/* ---- decomposed runs: one partition per rank ---------------------------
   Replace PROCINTFLUX (procintflux_all.f90:1-155), CYCREMFLUX
   (cycremflux_all.f90:1-155) and the MAX allreduce of compflux.f90:10-11.
   A processor face is a face whose other cell lives on another rank
   (IBFPROC; IF2C(K,1) and IF2C(K,3) are the own cell and its local face).
   Each stage this rank evaluates it with its own cell as the left cell,
   the other rank's trace as the right state, as the reference does.

   sddc_set_proc_faces declares them, in exchange-slot order, before
   sddc_set_tables (which then accepts them as covering their (cell, local
   face)).  sddc_set_exchange gives three device buffers the host owns:
     send_dev  [nproc][N][9]: this rank's trace of every processor face,
               nfp ascending (the reference's SBUFC), written by the library;
     recv_dev  [nproc][N][9]: the other ranks' traces, in their point order
               (RBUFC), read by the library;
     maxima_dev [2]: eigvmax, umax of this rank before, and of all ranks
               after, the host's MAX reduction;
   the traces in the form's arithmetic type (float in SDDC_MIXED, else
   double).  After the traces of a new state exist (set_state, every RK
   stage, every residual evaluation) the library fills send_dev and
   maxima_dev on the context's stream and calls fn(user); fn enqueues the
   exchange and the reduction on that stream (sddc_get_stream) and returns
   0, or nonzero to fail the call.  Steps of a decomposed run are launched
   stage by stage (no CUDA graph).  Batches, the viscous chain, the adjoint
   and the AV sensor read back after steps (sddc_get_state muAV / sm_ind
   after sddc_rk_step) are not available in a decomposed run;
   sddc_compresid forms the sensor with the reduced maxima. */
int sddc_set_proc_faces(sddc_ctx *ctx, int nproc, const int *ibfproc);
typedef int (*sddc_exchange_fn)(void *user);
int sddc_set_exchange(sddc_ctx *ctx, sddc_exchange_fn fn, void *user, void *send_dev, void *recv_dev,
                      double *maxima_dev);

/* Device pointer of the state (9,N,N,NCELL), valid until the next call;
   for callers that keep their data on the GPU. */
int sddc_state_device_ptr(sddc_ctx *ctx, double **q_dev);

/* The CUDA stream (cudaStream_t) every launch of the context goes to; for
   callers that order their own work or CUDA events against the drop-in. */
int sddc_get_stream(sddc_ctx *ctx, void **stream);

/* ---- output from the device state ------------------------------------------
   The restart and Tecplot files the reference writes every nwrite
   iterations (iterations.f90:77-80), from the state on the device.  A write
   call snapshots what it needs on the context's stream and returns; a side
   stream copies the snapshot to pinned host memory and a host thread writes
   the file while later calls step on.  A second write of the same kind waits
   until the first file is written.  sddc_output_wait blocks until every
   queued file is written and returns the first failure since the last wait
   (SDDC_EIO with the message in sddc_last_error); sddc_destroy writes what
   is queued before it returns. */

/* The plot mesh of tecplotter2dsetup (tecplotter2dsetup.f90:1-160), as the
   host library's sddc_plotmesh_tables gives it: plotx (2,plotnodes),
   gnumnode (nre+1,nre+1,NCELL), gnode_factor (plotnodes), connec
   (4,plotcells) with plotcells = nre^2 * NCELL, all 1-based.  Copied. */
int sddc_set_plot(sddc_ctx *ctx, int nre, int plotnodes, int plotcells, const double *plotx,
                  const int *gnumnode, const int *gnode_factor, const int *connec);

/* tecplotter2d (tecplotter.f90:1-95) of the current state, synchronous:
   plotq (9,plotnodes) rho u v w p Bx By Bz psi, plotav (2,plotnodes) muAV
   and etaAV averaged over the cells at each node (0 unless vismode = 1 and
   ARTIV = 1: the reference allocates muAV only then, initsetup.f90:36-41).
   The exact FP64 operations of the reference in its order, for every form.
   Either pointer may be NULL.  Not for batches. */
int sddc_plot_nodes(sddc_ctx *ctx, double *plotq, double *plotav);

/* The Tecplot file of tecplotter2d + tecpost_parallel (tecplotter.f90:1-415)
   for the current state and solution time, written in the background.
   path NULL: the reference's name, ./TEC/TEC<int(ctime):7><.fff>.plt. */
int sddc_write_tecplot(sddc_ctx *ctx, const char *path);

/* The restart file of WRITE_ALL_DATA_PARALLEL (write_data.f90:1-83) for the
   current state and solution time, written in the background.  icg (NCELL)
   the global cell numbers IC2ICG, NULL for 1..NCELL.  path NULL: the
   reference's name, restart.<iter:8>.dat in the working directory. */
int sddc_write_restart(sddc_ctx *ctx, const char *path, int iter, const int *icg);

int sddc_output_wait(sddc_ctx *ctx);

/* ---- batches of independent cases ----------------------------------------
   No counterpart in the reference (its runs are one case each).  Several
   cases of the same N and form share one context: their tables are
   concatenated (cells, faces and face lists renumbered so that case k owns
   cells first_cell .. first_cell+ncell-1), and every stage is one launch
   over all of them, tiled so that no CTA straddles two cases.  Each case
   keeps its own free stream, time step and running maxima (c_h). */
typedef struct sddc_case {
    int first_cell;  /* 0-based first cell of the case in the concatenation */
    int ncell;
    double dt;
    double rinf, pinf, uinf, vinf, bxinf, byinf;
} sddc_case;

/* After sddc_set_tables on the concatenated tables; resets the running
   maxima, so sddc_set_state follows. */
int sddc_set_cases(sddc_ctx *ctx, int ncase, const sddc_case *cases);
/* nsteps time steps of every case with its own dt. */
int sddc_rk_step_cases(sddc_ctx *ctx, int nsteps);
/* Running maxima of one case after the last evaluation. */
int sddc_get_case_maxima(sddc_ctx *ctx, int icase, double *eigvmax, double *umax);
/* How a batch's stages launch: on != 0, each stage is one persistent
   launch of as many CTAs as are resident at once, each walking the tile
   table (largest case first) with a grid stride; 0 (the default), one CTA
   per tile.  No counterpart in the reference (it runs one case per job). */
int sddc_set_persistent(sddc_ctx *ctx, int on);

/* ---- residual evaluation without device allocation ----------------------
   No counterpart in the reference.  For callers that cannot call cudaMalloc:
   a host that hands out all device memory from its own pool or budget, or a
   plugin inside a framework that owns the allocator.  The caller passes all inputs
   and outputs as device memory it holds; the working memory (face traces,
   running-maxima slots, AV sensor, fault flags) is one fixed array of
   SDDC_NOALLOC_SCRATCH_BYTES bytes inside the library, which every GPU that
   loads the library keeps until the process exits.  A case whose working
   memory exceeds it (about 11,000 cells at N = 5 in FP64, 14,000 at N = 4)
   is rejected with SDDC_EINVAL.  All calls share the array: calls that
   overlap on the GPU (several host threads, several streams) race; the
   array keeps the last call's contents and each call rewrites what it
   reads.  The first call on a device looks up the array's device address
   (cudaGetSymbolAddress); make it before any stream capture on that device. */
#define SDDC_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)

size_t sddc_noalloc_scratch_bytes(void);
const char *sddc_noalloc_last_error(void);

/* Sizes of the packed tables: met_doubles doubles of metrics and
   face_ints ints of (cell, local face) records. */
int sddc_noalloc_packed_sizes(int N, int ncell, size_t *met_doubles, size_t *face_ints);

/* Packs the reference-layout tables (as for sddc_set_tables) into caller
   host buffers of the sizes above; the caller copies them to the device. */
int sddc_noalloc_pack_tables(int N, int ncell, const double *S1, const double *S2, const double *Jac,
                             const int *IF2C, int nface, const int *ibfinter, int ninter,
                             const int *ibfinl, int ninlet, const int *ibfout, int noutlet,
                             const int *ibfwal, int nwall, const int *ibfsymp, int nsymp,
                             const int *ibfree, int nfree, const int *cyc2fpair, int npair,
                             double *met_out, int *faces_out);

/* One residual evaluation of q_dev (9,N,N,NCELL) on `stream` (NULL: the
   default stream), as sddc_compresid: writes resid_dev (9,N,N,NCELL) and
   nablaqs_dev (9,2,N,N,NCELL), both device memory of the caller.  eigvmax
   and umax are the running maxima before the evaluation (0 at start);
   maxima_out[0..1] receives them after it (pass them to the next call).
   Lmat and Mmat are host arrays (N+1,N).  Synchronises the stream before it
   returns; allocates no device memory.  p->cells_per_cta and p->k_stage
   are ignored. */
int sddc_compresid_noalloc(const sddc_params *p, const double *Lmat, const double *Mmat,
                           const double *q_dev, const double *met_dev, const int *faces_dev,
                           double eigvmax, double umax, double *resid_dev, double *nablaqs_dev,
                           double *maxima_out, void *stream);

/* ---- discrete adjoint -------------------------------------------------------
   The VJP of the FP64 residual and of RK_S5P3 time stepping.  The reference
   has no adjoint; these entries are the "sddc_vjp_resid" and
   "sddc_adjoint_run" that a Fortran or Python caller binds beside
   compresid (compresid.f90:1-80) and RK_S5P3 (iterations.f90:158-213).
   The residual differentiated is the exact FP64 form's (bit-equal to the
   reference's) whatever precision the context runs; the AV sensor enters no
   residual (its coefficients are zero, getrusanov.f90:326,328) and has no
   adjoint.  c_h = sqrt(L (L - U)) depends on the running maxima L, U of the
   wave speed and velocity over all earlier stages; its adjoint goes to the
   points attaining each maximum, split equally among them when several
   attain it bit for bit (a shared face counted once), to the first stage
   that attained it.  |x| has slope +1 at 0 and max() follows the argument
   it returns.  Single case (no batch), mu = eta0 = 0, k_stage = 3. */

/* Qbar = (dR/dQ)^T Rbar at the current state, with R as sddc_compresid
   evaluates it (c_h from the running maxima now held).  Host arrays
   (9,N,N,NCELL).  parbar (nullable) gets 7 values: Rbar . dR/dc_h, then
   Rbar . dR/d(rinf, pinf, uinf, vinf, bxinf, byinf) through the boundary
   states.  The context's state and maxima are unchanged. */
int sddc_vjp_resid(sddc_ctx *ctx, const double *Rbar, double *Qbar, double *parbar);

typedef struct sddc_adjoint_opts {
    double dt;              /* RK_S5P3 time step */
    int nsteps;             /* steps run from the current state */
    int n1, n2;             /* objective window: states after n1..n2 steps, 0 <= n1 <= n2 <= nsteps */
    double w_drag, w_lift;  /* J = mean over the window of w_drag*C_D + w_lift*C_L */
    double diameter;        /* reference length D of C = 2F/(rho_inf |U_inf|^2 D); 0 means 1 */
    int checkpoint_every;   /* steps between stored states (0 means 20) */
} sddc_adjoint_opts;

typedef struct sddc_adjoint_stats {
    double forward_ms;    /* the recorded forward run */
    double reverse_ms;    /* recomputation and reverse sweep */
    double device_bytes;  /* device memory the run allocated (checkpoints, stage states, adjoints) */
    int owner_stages;     /* stages whose wave-speed or velocity maximum raised the running max */
    int tie_stages;       /* of those, stages where several points attained it */
} sddc_adjoint_stats;

/* Drag and lift are not in the reference.  The force on the wall faces is
   F = sum over IBFWAL face points of w * (momentum components of the wall
   face's Rusanov flux out of the fluid), w the solution-point quadrature
   weight along the face; C_D and C_L are its components along the free
   stream (uinf, vinf) and normal to it, times 2/(rho_inf |U_inf|^2 D).
   Runs nsteps exact FP64 RK_S5P3 steps from the current state and running
   maxima, recording a checkpoint every checkpoint_every steps; obj
   (nullable) gets J, mean C_D, mean C_L over the window.  With Qbar0 or
   parbar non-null, then runs the reverse sweep (recomputing each segment
   from its checkpoint): Qbar0 (9,N,N,NCELL) = dJ/dQ(initial state), parbar
   (6) = dJ/d(rinf, pinf, uinf, vinf, bxinf, byinf) through the boundary
   states, the normalisation of C held fixed.  The context ends at the final
   state and maxima, as after sddc_rk_step(ctx, dt, nsteps) in the exact
   form.  The reverse sweep recomputes the next segment on a second stream
   (two stores of 5*checkpoint_every+1 stage states and traces) while it
   reverses the current one; both streams are the call's own and drained
   before it returns.  stats is nullable. */
int sddc_adjoint_run(sddc_ctx *ctx, const sddc_adjoint_opts *opts, double *obj, double *Qbar0, double *parbar,
                     sddc_adjoint_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
