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

/* calcjacob with 8-node serendipity cells (CURVE_WALL = 1: MAPDER_8_NODE,
   mapder.f90:117-253; calcjacob.f90:12-132): S1, S2, Jac as
   sddc_mesh_metrics, from xxf_cell (2,8,NCELL), the eight nodes of each cell
   as READ_VRT8_DATA reads them (readGRIDinfo.f90:86-117): corners 1-4
   counter-clockwise, then the mid-side nodes of edges 1-2, 2-3, 3-4, 4-1.
   xxsolu (2,N,N,NCELL), if not NULL, from the same map (MapBaseFunc8). */
int sddc_metrics8(int N, int ncell, const double *xxf_cell, double *S1,
                  double *S2, double *Jac, double *xxsolu);

/* ---- output (iterations.f90:77-80) ---------------------------------------- */

typedef struct sddc_plotmesh sddc_plotmesh;

/* Plot mesh of the Tecplot output: tecplotter2dsetup
   (tecplotter2dsetup.f90:1-160).  Every cell is split
   into nre x nre plot cells; plot nodes 1..NVERT are the mesh vertices,
   then each face's nre-1 inner nodes (made by the first cell that visits
   the face, matched by position within 1e-5 by the second) and each cell's
   (nre-1)^2 interior nodes, in the reference's order.  Fails if a vertex
   is used by no cell or a face node finds no match.  xxf_cell (2,8,NCELL)
   places the face and interior nodes by the 8-node map (CURVE_WALL = 1);
   NULL for bilinear cells. */
int sddc_plotmesh_build(sddc_plotmesh **out, const sddc_mesh *m, int nre,
                        const double *xxf_cell);
void sddc_plotmesh_destroy(sddc_plotmesh *pm);
int sddc_plotmesh_counts(const sddc_plotmesh *pm, int *plotnodes,
                         int *plotcells);
/* plotX(2,plotnodes), gnumnode(nre+1,nre+1,NCELL), gnode_factor(plotnodes),
   connec_c2n(4,plotcells), all 1-based as the reference holds them; any
   pointer may be NULL. */
int sddc_plotmesh_tables(const sddc_plotmesh *pm, double *plotx,
                         int *gnumnode, int *gnode_factor, int *connec);

/* The reference's file names: 'restart.<iter, 8 digits>.dat'
   (write_data.f90:45) and 'TEC<int(ctime), 7 digits><.fff>.plt'
   (tecplotter.f90:176-177).  Return the length, or -1 if buf is short. */
int sddc_restart_filename(int iter, char *buf, int len);
int sddc_tecplot_filename(double ctime, char *buf, int len);

/* Restart file of WRITE_ALL_DATA_PARALLEL (write_data.f90:1-83):
   Q (9,N,N,NCELL); icg (NCELL) the global cell numbers, NULL for 1..NCELL. */
int sddc_restart_write(const char *path, int iter, double ctime, int N,
                       int ncell, const int *icg, const double *Q);
/* READ_ALL_DATA_BINARY (read_data_restart.f90:36-70): reads nrec records
   (NCELLGLOB; 0 means ncell) and stores each whose global number maps to a
   local cell: icg2ic (nglob entries, ICG2IC) or, when NULL, the identity. */
int sddc_restart_read(const char *path, int N, int ncell, int nrec,
                      const int *icg2ic, int nglob, double *Q, int *iter,
                      double *ctime);

/* Tecplot file of tecpost_parallel (tecplotter.f90:99-415) from host
   arrays: plotx (2,plotnodes), plotq (9,plotnodes) as tecplotter2d leaves
   it (rho u v w p Bx By Bz psi), plotav (2,plotnodes) or NULL for zeros,
   connec (4,plotcells) 1-based. */
int sddc_tecplot_write(const char *path, double ctime, int plotnodes,
                       int plotcells, const double *plotx,
                       const double *plotq, const double *plotav,
                       const int *connec);

const char *sddc_host_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
