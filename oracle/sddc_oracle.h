/*
 * sddc_oracle.h -- CPU restatement of SDDC's residual-and-time-step path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity oracle: tests/, the smoke
 * check and the cpu_baseline / reference leg of bench.py may load it; the
 * product (libsddc_b200.so and the sddc_b200 package) never does.
 *
 * Parity status: UNPINNED against the reference's own outputs.  The reference
 * (chenkuangxu/SDDC, Fortran 90 + MPI) ships no tests, no golden vectors and
 * no sample decks, and no Fortran compiler exists in this image, so the
 * reference cannot be run to produce fixtures.  The restatement is pinned
 * instead by mathematical known-answer tests (operator exactness, freestream
 * preservation, Rusanov consistency, conservation, RK order) in tests/.
 *
 * Layout: every array uses the reference's Fortran layout (column-major,
 * variable index fastest) and every index table is 1-based, exactly as the
 * module setup2d (setup2d.f90:39-102) holds them.
 */
#ifndef SDDC_ORACLE_H
#define SDDC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

/* State arithmetic: double, or double _Complex in the complex-step tangent
   build (libsddc_oracle_cs.so, -DORC_CSTEP), whose state arrays are
   interleaved (re, im) pairs, or a double that counts its operations in the
   operation-count build (libsddc_oracle_count.so, C++, -DORC_COUNT), whose
   arrays are plain doubles. */
#ifdef ORC_CSTEP
#include <complex.h>
typedef double _Complex orc_real;
#elif defined(ORC_COUNT)
#ifdef __cplusplus
}
#endif
#include "orc_count.hpp"
#ifdef __cplusplus
extern "C" {
#endif
typedef orc_count orc_real;
#else
typedef double orc_real;
#endif

typedef struct orc_params {
    int N;            /* solution points per direction (p+1)          */
    int ncell;        /* NCELL                                        */
    int ncellglob;    /* NCELLGLOB (enters epsilon0, AV.f90:126)      */
    int vismode;      /* 0 inviscid, 1 viscous chain (QUAD.INP)       */
    int artiv;        /* ARTIV                                        */
    int skip_ideal_viscous; /* 1: skip the viscous chain when mu==eta0==0 */
    double mu, eta0;
    double dxcycl, dycycl;
    double rinf, pinf, uinf, vinf, bxinf, byinf;
} orc_params;

/* --- SD operators and metrics (initsetup.f90, mapder.f90, calcjacob.f90) */
void orc_setsandpoints(int np, double *Xs, double *Xf);
void orc_compute_LM(int N, const double *Xs, const double *Xf,
                    double *Lmat, double *Mmat);
/* bilinear metrics from 4-vertex cells (IVCELL(NCELL,4), 1-based) */
void orc_calcjacob_bilinear(int N, int ncell, const int *ivcell,
                            const double *xv, const double *yv,
                            double *S1, double *S2, double *Jac);

/* --- context --------------------------------------------------------- */
orc_ctx *orc_create(const orc_params *p);
void orc_destroy(orc_ctx *c);
void orc_set_threads(int nthreads);
int  orc_get_threads(void);
/* Tables in the reference layout; the oracle copies them. */
int orc_set_tables(orc_ctx *c, const double *Lmat, const double *Mmat,
                   const double *S1, const double *S2, const double *Jac,
                   const int *IF2C, int nface,
                   const int *ibfinter, int ninter,
                   const int *ibfinl, int ninlet,
                   const int *ibfout, int noutlet,
                   const int *ibfwal, int nwall,
                   const int *ibfsymp, int nsymp,
                   const int *ibfree, int nfree,
                   const int *cyc2fpair, int npair);
void orc_set_state(orc_ctx *c, const orc_real *Q, double ctime,
                   double eigvmax, double umax);
void orc_get_state(const orc_ctx *c, orc_real *Q, orc_real *resid,
                   orc_real *nablaQs, double *muAV, double *sm_ind);
/* boundary free stream (rinf, pinf, uinf, vinf, bxinf, byinf); starts as
   the parameters given to orc_create */
void orc_set_freestream(orc_ctx *c, const orc_real *fs);
void orc_get_maxima(const orc_ctx *c, double *eigvmax, double *umax,
                    double *c_h, double *epsilon0, double *ctime);
/* Flux arrays after the last residual (F1, G2 inviscid; Fv1, Gv2 viscous) */
void orc_get_fluxes(const orc_ctx *c, orc_real *F1, orc_real *G2,
                    orc_real *Fv1, orc_real *Gv2);

/* --- the hot path ----------------------------------------------------- */
void orc_compresid(orc_ctx *c);                    /* compresid.f90:1-80 */
void orc_rk_s5p3(orc_ctx *c, double dt, int nsteps); /* iterations.f90:158-213 */
void orc_five_stage_rk(orc_ctx *c, double dt, int nsteps); /* :88-156 */
/* monitor sums of iterations.f90:34-46 (local, before the gather) */
void orc_monitor(const orc_ctx *c, double *residsum, double *divbsum);

/* --- decomposed runs (the reference's MPI partitions) ------------------
   Processor faces (IBFPROC; IF2C(K,1) and IF2C(K,3) name the own cell and
   its local face) take the remote trace from the receive buffer; a stage
   is pack -> exchange -> unpack -> orc_compresid_local -> MAX allreduce of
   orc_get_maxima's eigvmax, umax -> orc_set_global_maxima ->
   orc_compresid_finish. */
int orc_set_proc_faces(orc_ctx *c, int nproc, const int *ibfproc);
void orc_proc_pack(orc_ctx *c, orc_real *sbuf);           /* (9, N, nproc) */
void orc_proc_unpack(orc_ctx *c, const orc_real *rbuf);   /* (9, N, nproc) */
void orc_compresid_local(orc_ctx *c);
void orc_get_local_maxima(const orc_ctx *c, double *eigvmax, double *umax);
void orc_set_global_maxima(orc_ctx *c, double eigvmax_g, double umax_g);
void orc_compresid_finish(orc_ctx *c);
void orc_rk_s5p3_begin_stage(orc_ctx *c, int stage);
void orc_rk_s5p3_end_stage(orc_ctx *c, int stage, double dt);

/* --- point kernels, exposed for consistency tests --------------------- */
void orc_point_iflux(const orc_real *Qi, orc_real c_h, orc_real *umax,
                     orc_real *F, orc_real *G);
void orc_point_rusanov(const orc_real *Qfl, const orc_real *Qfr, orc_real *Fnl,
                       orc_real *Fnr, const orc_real *normf, int sign_l,
                       int sign_r, orc_real c_h, orc_real *eigv,
                       orc_real *eigvmax, orc_real *umax);
/* RK_S5P3 stage combination on plain arrays (for the order test) */
void orc_rk_s5p3_combine(int stage, long n, orc_real dt, orc_real *q,
                         const orc_real *qk0, const orc_real *qka,
                         const orc_real *r);

/* --- drag and lift: not in the reference ------------------------------ */
/* Force on the wall faces (IBFWAL): the x and y momentum components of
   each wall face point's Rusanov flux out of the fluid cell at the current
   state, weighted by w[line] (quadrature weights of the solution points on
   [0,1]) and summed.  The maxima are not updated. */
void orc_wall_force(orc_ctx *c, const double *w, orc_real *fx, orc_real *fy);

/* --- 8-node cells, CURVE_WALL = 1 (sddc_oracle_curved.c; plain build) - */
/* MAPDER_8_NODE + calcjacob (mapder.f90:117-253, calcjacob.f90:1-132) from
   xxf_cell (2,8,NCELL) (readGRIDinfo.f90:86-117) */
void orc_calcjacob_8node(int N, int ncell, const double *xxf_cell, double *S1,
                         double *S2, double *Jac);
/* xyCoor_atGps(8, xxs, xi, eta, xx) with MapBaseFunc8 */
void orc_xycoor8(const double *xxs, double xi, double eta, double *xx);

/* --- output (sddc_oracle_output.c; plain build only) ------------------- */
/* tecplotter2dsetup (tecplotter2dsetup.f90:1-160); xxf_cell (2,8,ncell)
   for 8-node cells (CURVE_WALL = 1), NULL for bilinear ones.  Arrays
   sized for (nre+1)^2*ncell nodes: plotX (2,.), gnode_factor (.),
   gnumnode (nre+1,nre+1,ncell), connec_c2n (4,nre^2*ncell).  Returns 0, -1
   if a vertex is used by no cell, -2 if a face node found no match. */
int orc_plot_setup(int ncell, int nvert, const int *ivcell, const double *xv,
                   const double *yv, const double *xxf_cell, const int *if2c,
                   int nface, int nre, int *plotnodes, int *plotcells,
                   double *plotX, int *gnumnode, int *gnode_factor,
                   int *connec_c2n);
/* tecplotter2d (tecplotter.f90:1-95): plotQ (9,plotnodes) as rho u v w p
   Bx By Bz psi, plotAV (2,plotnodes); muAV (2,ncell) or NULL for zeros. */
void orc_plot_eval(int N, int ncell, const double *Q, const double *muAV,
                   int nre, int plotnodes, const int *gnumnode,
                   const int *gnode_factor, double *plotQ, double *plotAV);

#ifdef __cplusplus
}
#endif
#endif
