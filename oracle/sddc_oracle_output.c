/*
 * sddc_oracle_output.c -- CPU restatement of the reference's Tecplot plot
 * mesh and plot-node values.  TEST INFRASTRUCTURE ONLY (see sddc_oracle.h).
 *
 *   orc_plot_setup   tecplotter2dsetup  tecplotter2dsetup.f90:1-160
 *   orc_plot_eval    tecplotter2d       tecplotter.f90:1-95
 *
 * Written as the Fortran reads: 1-based indices through macros, the loops
 * in the reference's order, and the same left-to-right association, so the
 * doubles match the reference's before its conversion to float.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "sddc_oracle.h"

/* bilinear xyCoor_atGps (mapder.f90:79-87, 255-273) */
static void xycoor4(const double xxs[2][4], double xi, double eta, double rx[2])
{
    double func[4];
    func[0] = (1.0 - xi) * (1.0 - eta);
    func[1] = (1.0 - eta) * xi;
    func[2] = xi * eta;
    func[3] = (1.0 - xi) * eta;
    for (int i = 0; i < 2; i++) {
        rx[i] = 0.0;
        for (int nb = 0; nb < 4; nb++) rx[i] = rx[i] + xxs[i][nb] * func[nb];
    }
}

int orc_plot_setup(int ncell, int nvert, const int *ivcell, const double *xv, const double *yv,
                   const double *xxf_cell, const int *if2c, int nface, int nre, int *plotnodes_out,
                   int *plotcells_out, double *plotX, int *gnumnode, int *gnode_factor, int *connec_c2n)
{
    const int Np = nre, NCELL = ncell;
    const double tolplot = 1e-5;
    const long cap = (long)(Np + 1) * (Np + 1) * NCELL;
    int *ic2f = calloc((size_t)NCELL * 4, sizeof(int));
    int *isfacenod = calloc((size_t)nface + 1, sizeof(int));
    int *gfacenode = calloc((size_t)(Np > 1 ? Np - 1 : 1) * (nface + 1), sizeof(int));
#define IVCELL(c, k) ivcell[((c) - 1) + (long)NCELL * ((k) - 1)]
#define IC2F(c, k) ic2f[((c) - 1) + (long)NCELL * ((k) - 1)]
#define IF2C(f, k) if2c[((f) - 1) + (long)nface * ((k) - 1)]
#define PX(i, g) plotX[((i) - 1) + 2L * ((g) - 1)]
#define GN(ii, jj, c) gnumnode[((ii) - 1) + (long)(Np + 1) * (((jj) - 1) + (long)(Np + 1) * ((c) - 1))]
#define GF(g) gnode_factor[(g) - 1]
#define GFN(e, f) gfacenode[((e) - 1) + (long)(Np - 1) * (f)]
    /* IC2F from IF2C (connectivity.f90:101-149 fills both) */
    for (int f = 1; f <= nface; f++) {
        IC2F(IF2C(f, 1), IF2C(f, 3)) = f;
        if (IF2C(f, 2) > 0) IC2F(IF2C(f, 2), IF2C(f, 4)) = f;
    }
    for (long g = 0; g < cap; g++) gnode_factor[g] = 0;
    int plotnodes = 0, plotcells = 0, rc = 0;
    for (int icell = 1; icell <= NCELL; icell++) {
        int IC2V[4];
        for (int k = 1; k <= 4; k++) IC2V[k - 1] = IVCELL(icell, k);
        GN(1, 1, icell) = IC2V[0];
        GN(Np + 1, 1, icell) = IC2V[1];
        GN(Np + 1, Np + 1, icell) = IC2V[2];
        GN(1, Np + 1, icell) = IC2V[3];
        for (int k = 1; k <= 4; k++) {
            int gnid = IC2V[k - 1];
            if (GF(gnid) == 0) {
                plotnodes = plotnodes + 1;
                PX(1, gnid) = xv[gnid - 1];
                PX(2, gnid) = yv[gnid - 1];
            }
            GF(gnid) = GF(gnid) + 1;
        }
    }
    if (plotnodes != nvert) rc = -1;
    for (int icell = 1; icell <= NCELL && rc == 0; icell++) {
        double xxs[2][4];
        for (int j = 1; j <= 4; j++) {
            xxs[0][j - 1] = xv[IVCELL(icell, j) - 1];
            xxs[1][j - 1] = yv[IVCELL(icell, j) - 1];
        }
        /* CURVE_WALL = 1: xyCoor_atGps(8, xxf_cell(:,:,icell), ...) */
        const double *xx8 = xxf_cell ? xxf_cell + 16L * (icell - 1) : NULL;
        for (int k = 1; k <= 4; k++) {
            int iface = IC2F(icell, k);
            for (int enode = 1; enode <= Np - 1; enode++) {
                int ii, jj;
                switch (k) {
                case 1: ii = enode + 1; jj = 1; break;
                case 2: ii = Np + 1; jj = enode + 1; break;
                case 3: ii = Np + 1 - enode; jj = Np + 1; break;
                default: ii = 1; jj = Np + 1 - enode; break;
                }
                double xsi = (double)(ii - 1) / (double)Np, eta = (double)(jj - 1) / (double)Np, rx[2];
                if (xx8) orc_xycoor8(xx8, xsi, eta, rx);
                else xycoor4(xxs, xsi, eta, rx);
                if (isfacenod[iface] == 1) {
                    int checkmatch = 0;
                    for (int existnode = 1; existnode <= Np - 1; existnode++) {
                        int gnid = GFN(existnode, iface);
                        double d = fabs(sqrt((rx[0] - PX(1, gnid)) * (rx[0] - PX(1, gnid)) +
                                             (rx[1] - PX(2, gnid)) * (rx[1] - PX(2, gnid))));
                        if (d <= tolplot) {
                            GN(ii, jj, icell) = gnid;
                            GF(gnid) = GF(gnid) + 1;
                            checkmatch = 1;
                        }
                    }
                    if (checkmatch == 0) rc = -2;
                } else {
                    plotnodes = plotnodes + 1;
                    PX(1, plotnodes) = rx[0];
                    PX(2, plotnodes) = rx[1];
                    GN(ii, jj, icell) = plotnodes;
                    GFN(enode, iface) = plotnodes;
                    GF(plotnodes) = GF(plotnodes) + 1;
                }
            }
            if (isfacenod[iface] == 0) isfacenod[iface] = 1;
        }
        for (int ii = 2; ii <= Np; ii++)
            for (int jj = 2; jj <= Np; jj++) {
                double rx[2];
                if (xx8) orc_xycoor8(xx8, (double)(ii - 1) / (double)Np, (double)(jj - 1) / (double)Np, rx);
                else xycoor4(xxs, (double)(ii - 1) / (double)Np, (double)(jj - 1) / (double)Np, rx);
                plotnodes = plotnodes + 1;
                PX(1, plotnodes) = rx[0];
                PX(2, plotnodes) = rx[1];
                GN(ii, jj, icell) = plotnodes;
                GF(plotnodes) = GF(plotnodes) + 1;
            }
        for (int ii = 1; ii <= Np; ii++)
            for (int jj = 1; jj <= Np; jj++) {
                plotcells = plotcells + 1;
                connec_c2n[4L * (plotcells - 1) + 0] = GN(ii, jj, icell);
                connec_c2n[4L * (plotcells - 1) + 1] = GN(ii + 1, jj, icell);
                connec_c2n[4L * (plotcells - 1) + 2] = GN(ii + 1, jj + 1, icell);
                connec_c2n[4L * (plotcells - 1) + 3] = GN(ii, jj + 1, icell);
            }
    }
    *plotnodes_out = plotnodes;
    *plotcells_out = plotcells;
    free(ic2f);
    free(isfacenod);
    free(gfacenode);
    return rc;
#undef IVCELL
#undef IC2F
#undef IF2C
#undef PX
#undef GF
#undef GFN
}

/* hval: Lagrange basis of the solution points (tecplotter.f90:71-91) */
static double hval(int np, int i, double xval, const double *Xs)
{
    double hvaln = 1.0, hvald = 1.0;
    for (int s = 1; s <= np; s++)
        if (s != i) {
            hvaln = hvaln * (xval - Xs[s - 1]);
            hvald = hvald * (Xs[i - 1] - Xs[s - 1]);
        }
    return hvaln / hvald;
}

void orc_plot_eval(int N, int ncell, const double *Q, const double *muAV, int nre, int plotnodes,
                   const int *gnumnode, const int *gnode_factor, double *plotQ, double *plotAV)
{
    const int Np = nre, numv = 9;
    const double gam = 5.0 / 3;  /* setup2d.f90:67 */
    double Xs[8], Xf[9], Qs[9];
    orc_setsandpoints(N, Xs, Xf);
    for (long i = 0; i < 9L * plotnodes; i++) plotQ[i] = 0.0;
    for (long i = 0; i < 2L * plotnodes; i++) plotAV[i] = 0.0;
#define Q_(k, is, js, c) Q[((k) - 1) + 9L * (((is) - 1) + (long)N * (((js) - 1) + (long)N * ((c) - 1)))]
    for (int icell = 1; icell <= ncell; icell++)
        for (int jj = 1; jj <= Np + 1; jj++)
            for (int ii = 1; ii <= Np + 1; ii++) {
                double xsi = (double)(ii - 1) / (double)Np, eta = (double)(jj - 1) / (double)Np;
                int gnid = GN(ii, jj, icell);
                for (int k = 0; k < numv; k++) Qs[k] = 0.0;
                for (int js = 1; js <= N; js++)
                    for (int is = 1; is <= N; is++)
                        for (int k = 1; k <= numv; k++)
                            Qs[k - 1] = Qs[k - 1] + Q_(k, is, js, icell) * hval(N, is, xsi, Xs) * hval(N, js, eta, Xs);
                for (int k = 0; k < numv; k++) plotQ[k + 9L * (gnid - 1)] = plotQ[k + 9L * (gnid - 1)] + Qs[k];
                double m1 = muAV ? muAV[2L * (icell - 1)] : 0.0, m2 = muAV ? muAV[2L * (icell - 1) + 1] : 0.0;
                plotAV[2L * (gnid - 1)] = plotAV[2L * (gnid - 1)] + m1;
                plotAV[2L * (gnid - 1) + 1] = plotAV[2L * (gnid - 1) + 1] + m2;
            }
    for (int nd = 1; nd <= plotnodes; nd++) {
        double *pq = plotQ + 9L * (nd - 1);
        for (int k = 0; k < numv; k++) Qs[k] = pq[k] / (double)gnode_factor[nd - 1];
        pq[0] = Qs[0];
        pq[1] = Qs[1] / Qs[0];
        pq[2] = Qs[2] / Qs[0];
        pq[3] = Qs[3] / Qs[0];
        for (int k = 5; k < 9; k++) pq[k] = Qs[k];
        double NORM_U = pq[1] * pq[1] + pq[2] * pq[2] + pq[3] * pq[3];
        double NORM_B = pq[5] * pq[5] + pq[6] * pq[6] + pq[7] * pq[7];
        pq[4] = (Qs[4] - 0.5 * Qs[0] * NORM_U - 0.5 * NORM_B) * (gam - 1);
        plotAV[2L * (nd - 1)] = plotAV[2L * (nd - 1)] / (double)gnode_factor[nd - 1];
        plotAV[2L * (nd - 1) + 1] = plotAV[2L * (nd - 1) + 1] / (double)gnode_factor[nd - 1];
    }
#undef Q_
#undef GN
}
