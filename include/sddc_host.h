/*
 * sddc_host.h -- host-side set-up that feeds the SDDC residual drop-in.
 *
 * The reference's Fortran host builds these tables before its time loop
 * (main.f90:16-58).  With no Fortran compiler available, this C++ library is
 * the host used by the Python driver, the tests and the benchmark; a Fortran
 * host keeps its own routines and passes their arrays to sddc.h directly.
 *
 * All arrays use the reference's layout: Fortran column-major, 1-based
 * indices.  Every function returns 0 on success and a negative code on
 * failure (never exits); sddc_host_last_error() gives the message.
 */
#ifndef SDDC_HOST_H
#define SDDC_HOST_H

#ifdef __cplusplus
extern "C" {
#endif

/* boundary types of the boundary file (IBOUNTYPE, readGRIDinfo.f90:269-276) */
enum {
    SDDC_BC_INLE = 0,
    SDDC_BC_OUTL = 1,
    SDDC_BC_SYMP = 2,
    SDDC_BC_WALL = 3,
    SDDC_BC_CYCL = 4,
    SDDC_BC_FREE = 5
};

/* indices of sddc_mesh_counts() */
enum {
    SDDC_MC_NFACE = 0,
    SDDC_MC_NINTER,
    SDDC_MC_NINLET,
    SDDC_MC_NOUTLET,
    SDDC_MC_NSYMP,
    SDDC_MC_NWALL,
    SDDC_MC_NCYCL,
    SDDC_MC_NCYCLOC,
    SDDC_MC_NCYCREM,
    SDDC_MC_NPAIR,
    SDDC_MC_NPROCINT,
    SDDC_MC_NFREE,
    SDDC_MC_NREVERSED,
    SDDC_MC_NVERT,
    SDDC_MC_NCELL,
    SDDC_MC_COUNT
};

typedef struct sddc_mesh sddc_mesh;

/* SD points and operators: setsandpoints + computeLandM
   (initsetup.f90:171-319).  Xs[N], Xf[N+1], Lmat and Mmat (N+1,N). */
int sddc_sd_operators(int N, double *Xs, double *Xf, double *Lmat,
                      double *Mmat);

/* Single-rank mesh set-up: CHECK_MESH (connectivity.f90:237-298),
   CONNECTIVITY (:1-234), CONNECT_BDRY (connect_bdry.f90:1-354) and
   MAPCYCLOC (map_cyc_loc.f90:1-42).
   ivcell: IVCELL(ncell,4), 1-based vertex ids.  bnd_v: IVGBOUN(nbound,2).
   bnd_type: SDDC_BC_* per boundary record. */
int sddc_mesh_build(sddc_mesh **out, int ncell, int nvert, const int *ivcell,
                    const double *xv, const double *yv, int nbound,
                    const int *bnd_v, const int *bnd_type, double dxcycl,
                    double dycycl);
void sddc_mesh_destroy(sddc_mesh *m);
/* counts[SDDC_MC_COUNT] */
int sddc_mesh_counts(const sddc_mesh *m, int *counts);
/* Copies the tables out; any pointer may be NULL.  IF2C is (NFACE,4),
   IF2V (NFACE,2), CYC2FPAIR (NPAIR,2), IVCELL (NCELL,4) after CHECK_MESH. */
int sddc_mesh_tables(const sddc_mesh *m, int *if2c, int *if2v, int *ibfinter,
                     int *ibfinl, int *ibfout, int *ibfwal, int *ibfsymp,
                     int *ibfree, int *cyc2fpair, int *ivcell_ccw);
/* calcjacob with bilinear elements (calcjacob.f90:1-132, mapder.f90:1-76):
   S1(2,2,N+1,N,NCELL), S2(2,2,N,N+1,NCELL), Jac(N,N,NCELL); also the
   physical coordinates of the solution points XXsolu(2,N,N,NCELL)
   (initsetup.f90:82-106) when xxsolu is not NULL. */
int sddc_mesh_metrics(const sddc_mesh *m, int N, double *S1, double *S2,
                      double *Jac, double *xxsolu);

const char *sddc_host_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
