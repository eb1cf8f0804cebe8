/*
 * sddc_oracle_curved.c -- CPU restatement of the reference's 8-node
 * (serendipity) cell geometry, CURVE_WALL = 1.  TEST INFRASTRUCTURE ONLY
 * (see sddc_oracle.h).
 *
 *   mapder8_tables        MAPDER_8_NODE   mapder.f90:117-253
 *   orc_calcjacob_8node   calcjacob       calcjacob.f90:1-132 (CURVE_WALL = 1)
 *   orc_xycoor8           xyCoor_atGps(8) mapder.f90:255-273, MapBaseFunc8 :91-103
 *
 * As the reference: the derivative tables first, then the sums over the
 * eight nodes in order, in the reference's left-to-right association.
 */
#include <stdlib.h>

#include "sddc_oracle.h"

/* dm(k, d) of one point: the eight shape-function derivatives of
   MAPDER_8_NODE (identical expressions for the three point families) */
static void dm8(double psi, double eta, double dm[8][2])
{
    dm[0][0] = (1.0 - eta) * (4.0 * psi + 2.0 * eta - 3.0);
    dm[0][1] = (1.0 - psi) * (4.0 * eta + 2.0 * psi - 3.0);
    dm[1][0] = (1.0 - eta) * (4.0 * psi - 2.0 * eta - 1.0);
    dm[1][1] = psi * (4.0 * eta - 2.0 * psi - 1.0);
    dm[2][0] = eta * (4.0 * psi + 2.0 * eta - 3.0);
    dm[2][1] = psi * (4.0 * eta + 2.0 * psi - 3.0);
    dm[3][0] = eta * (4.0 * psi - 2.0 * eta - 1.0);
    dm[3][1] = (1.0 - psi) * (4.0 * eta - 2.0 * psi - 1.0);
    dm[4][0] = 4.0 * (1.0 - eta) * (1.0 - 2.0 * psi);
    dm[4][1] = 4.0 * psi * (psi - 1.0);
    dm[5][0] = 4.0 * eta * (1.0 - eta);
    dm[5][1] = 4.0 * psi * (1.0 - 2.0 * eta);
    dm[6][0] = 4.0 * eta * (1.0 - 2.0 * psi);
    dm[6][1] = 4.0 * psi * (1.0 - psi);
    dm[7][0] = 4.0 * eta * (eta - 1.0);
    dm[7][1] = 4.0 * (1.0 - psi) * (1.0 - 2.0 * eta);
}

void orc_calcjacob_8node(int N, int ncell, const double *xxf_cell, double *S1, double *S2, double *Jac)
{
    const int N1 = N + 1;
    double Xs[16], Xf[17];
    orc_setsandpoints(N, Xs, Xf);
    /* MAPDER_8_NODE: dmdxs(8,2,N,N), dmdxf1(8,2,N+1,N), dmdxf2(8,2,N,N+1) */
    double(*dmdxs)[8][2] = malloc(sizeof(double[8][2]) * (size_t)N * N);
    double(*dmdxf1)[8][2] = malloc(sizeof(double[8][2]) * (size_t)N1 * N);
    double(*dmdxf2)[8][2] = malloc(sizeof(double[8][2]) * (size_t)N * N1);
    for (int js = 1; js <= N; js++)
        for (int is = 1; is <= N; is++) dm8(Xs[is - 1], Xs[js - 1], dmdxs[(is - 1) + N * (js - 1)]);
    for (int jfp = 1; jfp <= N; jfp++)
        for (int ifp = 1; ifp <= N1; ifp++) dm8(Xf[ifp - 1], Xs[jfp - 1], dmdxf1[(ifp - 1) + N1 * (jfp - 1)]);
    for (int jfp = 1; jfp <= N1; jfp++)
        for (int ifp = 1; ifp <= N; ifp++) dm8(Xs[ifp - 1], Xf[jfp - 1], dmdxf2[(ifp - 1) + N * (jfp - 1)]);
#define XXS(i, k) xxs[((i) - 1) + 2 * ((k) - 1)]
    for (int ic = 1; ic <= ncell; ic++) {
        const double *xxs = xxf_cell + 16L * (ic - 1);
        for (int js = 1; js <= N; js++)
            for (int is = 1; is <= N; is++) {
                double(*d)[2] = dmdxs[(is - 1) + N * (js - 1)];
                double xpsi = 0.0, xeta = 0.0, ypsi = 0.0, yeta = 0.0;
                for (int k = 1; k <= 8; k++) {
                    xpsi = xpsi + d[k - 1][0] * XXS(1, k);
                    ypsi = ypsi + d[k - 1][0] * XXS(2, k);
                    xeta = xeta + d[k - 1][1] * XXS(1, k);
                    yeta = yeta + d[k - 1][1] * XXS(2, k);
                }
                Jac[(is - 1) + N * ((js - 1) + (long)N * (ic - 1))] = xpsi * yeta - xeta * ypsi;
            }
        for (int jfp = 1; jfp <= N; jfp++)
            for (int ifp = 1; ifp <= N1; ifp++) {
                double(*d)[2] = dmdxf1[(ifp - 1) + N1 * (jfp - 1)];
                double xpsi = 0.0, xeta = 0.0, ypsi = 0.0, yeta = 0.0;
                for (int k = 1; k <= 8; k++) {
                    xpsi = xpsi + d[k - 1][0] * XXS(1, k);
                    ypsi = ypsi + d[k - 1][0] * XXS(2, k);
                    xeta = xeta + d[k - 1][1] * XXS(1, k);
                    yeta = yeta + d[k - 1][1] * XXS(2, k);
                }
                long b = 4L * ((ifp - 1) + N1 * ((jfp - 1) + (long)N * (ic - 1)));
                S1[b + 0] = yeta;
                S1[b + 2] = -xeta;
                S1[b + 1] = -ypsi;
                S1[b + 3] = xpsi;
            }
        for (int jfp = 1; jfp <= N1; jfp++)
            for (int ifp = 1; ifp <= N; ifp++) {
                double(*d)[2] = dmdxf2[(ifp - 1) + N * (jfp - 1)];
                double xpsi = 0.0, xeta = 0.0, ypsi = 0.0, yeta = 0.0;
                for (int k = 1; k <= 8; k++) {
                    xpsi = xpsi + d[k - 1][0] * XXS(1, k);
                    ypsi = ypsi + d[k - 1][0] * XXS(2, k);
                    xeta = xeta + d[k - 1][1] * XXS(1, k);
                    yeta = yeta + d[k - 1][1] * XXS(2, k);
                }
                long b = 4L * ((ifp - 1) + N * ((jfp - 1) + (long)N1 * (ic - 1)));
                S2[b + 0] = yeta;
                S2[b + 2] = -xeta;
                S2[b + 1] = -ypsi;
                S2[b + 3] = xpsi;
            }
    }
#undef XXS
    free(dmdxs);
    free(dmdxf1);
    free(dmdxf2);
}

void orc_xycoor8(const double *xxs, double xi, double eta, double *xx)
{
    double func8[8];
    func8[0] = (1.0 - xi) * (1.0 - eta) * (-2.0 * xi - 2.0 * eta + 1.0);
    func8[1] = xi * (1.0 - eta) * (2.0 * xi - 2.0 * eta - 1.0);
    func8[2] = xi * eta * (2.0 * xi + 2.0 * eta - 3.0);
    func8[3] = (1.0 - xi) * eta * (-2.0 * xi + 2.0 * eta - 1.0);
    func8[4] = 4.0 * (1.0 - eta) * (1.0 - xi) * xi;
    func8[5] = 4.0 * eta * (1.0 - eta) * xi;
    func8[6] = 4.0 * (1.0 - xi) * xi * eta;
    func8[7] = 4.0 * (1.0 - eta) * (1.0 - xi) * eta;
    for (int i = 0; i < 2; i++) {
        xx[i] = 0.0;
        for (int nb = 0; nb < 8; nb++) xx[i] = xx[i] + xxs[i + 2 * nb] * func8[nb];
    }
}
