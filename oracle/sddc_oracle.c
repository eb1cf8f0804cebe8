/*
 * sddc_oracle.c -- FP64 CPU restatement of SDDC's residual-and-time-step path.
 *
 * TEST INFRASTRUCTURE ONLY (see sddc_oracle.h).  Parity against the reference
 * itself is UNPINNED: the reference has no tests or golden vectors and cannot
 * be compiled here (no Fortran compiler).  Each routine below follows the
 * reference routine named in its comment, in the same loop order and the same
 * left-to-right evaluation order of every expression, so that, built with
 * -ffp-contract=off (gfortran -O3 without -march emits no FMA on x86-64), it
 * reproduces the reference's rounding.
 *
 * Arrays use the reference's Fortran layout (column-major, 1-based indices,
 * variable index fastest).  The accessor macros take 1-based indices.
 *
 * Where the reference reads memory it never wrote (nablaQs when vismode==0,
 * compresid.f90:58), the oracle reads zeros.
 */
#include "sddc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NV 9

typedef orc_real real;

/* Arithmetic type of every state-dependent quantity.  The plain build uses
 * double.  The tangent build (-DORC_CSTEP) uses double _Complex: a state
 * Q + i*h*V evaluated with h ~ 1e-30 carries Im(f)/h = f'(Q).V to rounding
 * (complex-step differentiation, Squire & Trapp 1998).  Branches, |x| and
 * max() follow the real part, so the tangent is that of the branch the
 * plain build takes. */
#ifdef ORC_CSTEP
#define RV(x) creal(x)
static inline real r_sqrt(real x) { return csqrt(x); }
static inline real r_abs(real x) { return creal(x) < 0.0 ? -x : x; }
static inline real r_max(real a, real b) { return creal(b) > creal(a) ? b : a; }
#elif defined(ORC_COUNT)
/* the operation-count build (C++): |x| and max() select, they count nothing */
orc_tally_t orc_tally;
#define RV(x) ((x).v)
static inline real r_sqrt(real x) { return orc_count_sqrt(x); }
static inline real r_abs(real x) { return x.v < 0.0 ? -x : x; }
static inline real r_max(real a, real b) { return b.v > a.v ? b : a; }
extern "C" void orc_count_read(unsigned long long *out, int reset)
{
    out[0] = orc_tally.add;
    out[1] = orc_tally.mul;
    out[2] = orc_tally.div;
    out[3] = orc_tally.sqrt;
    if (reset) orc_tally = orc_tally_t{0, 0, 0, 0};
}
#else
#define RV(x) (x)
#define r_sqrt sqrt
#define r_abs fabs
#define r_max fmax
#endif

struct orc_ctx {
    orc_params p;
    int N, N1, NC;
    double alpha;
    /* operators */
    double *Xs, *Xf, *Lmat, *Mmat, *Xs_low;
    /* metrics */
    double *S1, *S2, *Jac;
    /* connectivity */
    int nface, ninter, ninlet, noutlet, nwall, nsymp, nfree, npair;
    int *IF2C, *ibfinter, *ibfinl, *ibfout, *ibfwal, *ibfsymp, *ibfree,
        *cyc2fpair;
    int iface2fp[4 * 16], jface2fp[4 * 16]; /* (nfp,lf), N <= 16 */
    /* processor faces of a decomposed run: IBFPROC, the own traces sent
       (Qfl_p) and the remote traces received, in own point order (Qfr_p),
       (9, N, NPROCINT) each (procintflux_all.f90:28-99) */
    int nproc;
    int *ibfproc;
    real *Qfl_p, *Qfr_p;
    /* the RK_S5P3 registers and stage-start time of the staged interface */
    real *Qk0_s, *Qka_s;
    double ctime0_s, ctime_stage_s;
    /* state and work arrays */
    real *Q, *resid, *F1, *G2, *Fv1, *Gv2, *Qvfi, *Qvfj;
    real *nablaQs, *nablaQvfi, *nablaQvfj, *dedxi, *dedeta;
    double *muAV, *SM_IND, *muAVfi, *muAVfj;
    /* free stream of the boundary states (rinf, pinf, uinf, vinf, bxinf,
       byinf), a copy of the parameters that the tangent build can perturb */
    real fs[6];
    /* scalars of module setup2d */
    real eigvmax, eigvmax_g, umax, umax_g, c_h;
    double epsilon0, ctime;
};

/* ---- accessors (1-based, Fortran column-major) ----------------------- */
#define Q_(v, i, j, c) cx->Q[((v)-1) + NV * (((i)-1) + N * (((j)-1) + N * ((c)-1)))]
#define R_(v, i, j, c) cx->resid[((v)-1) + NV * (((i)-1) + N * (((j)-1) + N * ((c)-1)))]
#define FI_(A, v, r, j, c) cx->A[((v)-1) + NV * (((r)-1) + N1 * (((j)-1) + N * ((c)-1)))]
#define FJ_(A, v, i, r, c) cx->A[((v)-1) + NV * (((i)-1) + N * (((r)-1) + N1 * ((c)-1)))]
#define S1_(a, b, r, j, c) cx->S1[((a)-1) + 2 * (((b)-1) + 2 * (((r)-1) + N1 * (((j)-1) + N * ((c)-1))))]
#define S2_(a, b, i, r, c) cx->S2[((a)-1) + 2 * (((b)-1) + 2 * (((i)-1) + N * (((r)-1) + N1 * ((c)-1))))]
#define JAC_(i, j, c) cx->Jac[((i)-1) + N * (((j)-1) + N * ((c)-1))]
#define DEDXI_(i, j, c) cx->dedxi[((i)-1) + N * (((j)-1) + N * ((c)-1))]
#define DEDETA_(i, j, c) cx->dedeta[((i)-1) + N * (((j)-1) + N * ((c)-1))]
#define NQS_(v, d, i, j, c) cx->nablaQs[((v)-1) + NV * (((d)-1) + 2 * (((i)-1) + N * (((j)-1) + N * ((c)-1))))]
#define NQI_(v, d, r, j, c) cx->nablaQvfi[((v)-1) + NV * (((d)-1) + 2 * (((r)-1) + N1 * (((j)-1) + N * ((c)-1))))]
#define NQJ_(v, d, i, r, c) cx->nablaQvfj[((v)-1) + NV * (((d)-1) + 2 * (((i)-1) + N * (((r)-1) + N1 * ((c)-1))))]
#define L_(f, s) cx->Lmat[((f)-1) + N1 * ((s)-1)]
#define M_(f, s) cx->Mmat[((f)-1) + N1 * ((s)-1)]
#define IF2C_(f, k) cx->IF2C[((f)-1) + cx->nface * ((k)-1)]
#define CYC_(q, k) cx->cyc2fpair[((q)-1) + cx->npair * ((k)-1)]
#define IFP_(n, lf) cx->iface2fp[((n)-1) + 16 * ((lf)-1)]
#define JFP_(n, lf) cx->jface2fp[((n)-1) + 16 * ((lf)-1)]
#define MUAV_(v, c) cx->muAV[((v)-1) + 2 * ((c)-1)]
#define SMIND_(v, c) cx->SM_IND[((v)-1) + 2 * ((c)-1)]
#define MUFI_(v, f, c) cx->muAVfi[((v)-1) + 2 * (((f)-1) + 2 * ((c)-1))]
#define MUFJ_(v, f, c) cx->muAVfj[((v)-1) + 2 * (((f)-1) + 2 * ((c)-1))]

static const double PI = 3.141592653589793; /* atan(1.d0)*4.d0, setup2d.f90:66 */
static const double GAM = 5.0 / 3.0;        /* setup2d.f90:67 */
static const double LAMBDA = -2.0 / 3.0;    /* setup2d.f90:69 */
static const double PRANDT = 0.72;          /* setup2d.f90:70 */

static inline real sq(real x) { return x * x; }
static inline void upd_max(real *m, real x) { if (RV(x) > RV(*m)) *m = x; }

/* ===================================================================== */
/* SD points and operators                                               */
/* ===================================================================== */

/* setsandpoints, initsetup.f90:171-259 */
void orc_setsandpoints(int np, double *Xs, double *Xf)
{
    for (int i = 1; i <= np; i++)
        Xs[i - 1] = 0.5 * (1.0 - cos((double)(2 * i - 1) * PI / (2.0 * (double)np)));
    double *X = Xf - 1; /* 1-based view */
    if (np == 1) {
        X[1] = 0.0; X[2] = 1.0;
    } else if (np == 2) {
        X[1] = 0.0; X[2] = 0.5; X[3] = 1.0;
    } else if (np == 3) {
        X[1] = 0.0;
        X[2] = (1.0 - sqrt(3.0) / 3.0) / 2.0;
        X[3] = (1.0 + sqrt(3.0) / 3.0) / 2.0;
        X[4] = 1.0;
    } else if (np == 4) {
        X[1] = 0.0;
        X[2] = (1.0 - sqrt(15.0) / 5.0) / 2.0;
        X[3] = 0.5;
        X[4] = (1.0 + sqrt(15.0) / 5.0) / 2.0;
        X[5] = 1.0;
    } else if (np == 5) {
        X[1] = 0.0;
        X[2] = (1.0 - sqrt(525.0 + 70.0 * sqrt(30.0)) / 35.0) / 2.0;
        X[3] = (1.0 - sqrt(525.0 - 70.0 * sqrt(30.0)) / 35.0) / 2.0;
        X[4] = (1.0 + sqrt(525.0 - 70.0 * sqrt(30.0)) / 35.0) / 2.0;
        X[5] = (1.0 + sqrt(525.0 + 70.0 * sqrt(30.0)) / 35.0) / 2.0;
        X[6] = 1.0;
    } else if (np == 6) {
        X[1] = 0.0;
        X[2] = (1.0 - sqrt(245.0 + 14.0 * sqrt(70.0)) / 21.0) / 2.0;
        X[3] = (1.0 - sqrt(245.0 - 14.0 * sqrt(70.0)) / 21.0) / 2.0;
        X[4] = 0.5;
        X[5] = (1.0 + sqrt(245.0 - 14.0 * sqrt(70.0)) / 21.0) / 2.0;
        X[6] = (1.0 + sqrt(245.0 + 14.0 * sqrt(70.0)) / 21.0) / 2.0;
        X[7] = 1.0;
    } else {
        /* np >= 7 uses 12-digit Gauss abscissae in the reference
           (initsetup.f90:215-256); this build supports np <= 6. */
        for (int i = 1; i <= np + 1; i++) X[i] = NAN;
    }
}

/* hhval, initsetup.f90:322-344 (Lagrange basis on the points X[0..np-1]) */
static double hh(const double *X, int np, int i, double xval)
{
    double hvaln = 1.0, hvald = 1.0;
    for (int s = 1; s <= np; s++) {
        if (s != i) {
            hvaln = hvaln * (xval - X[s - 1]);
            hvald = hvald * (X[i - 1] - X[s - 1]);
        }
    }
    return hvaln / hvald;
}

/* computeLandM, initsetup.f90:262-319 */
void orc_compute_LM(int N, const double *Xs, const double *Xf, double *Lmat,
                    double *Mmat)
{
    int N1 = N + 1;
    for (int ifp = 1; ifp <= N1; ifp++)
        for (int is = 1; is <= N; is++)
            Lmat[(ifp - 1) + N1 * (is - 1)] = hh(Xs, N, is, Xf[ifp - 1]);
    for (int ifp = 1; ifp <= N1; ifp++) {
        for (int is = 1; is <= N; is++) {
            double xval = Xs[is - 1], sum = 0.0;
            for (int k = 1; k <= N1; k++) {
                if (k == ifp) continue;
                double num = 1.0, den = 1.0;
                for (int s = 1; s <= N1; s++) {
                    if (s != ifp && s != k) num = num * (xval - Xf[s - 1]);
                    if (s != ifp) den = den * (Xf[ifp - 1] - Xf[s - 1]);
                }
                sum = sum + num / den;
            }
            Mmat[(ifp - 1) + N1 * (is - 1)] = sum;
        }
    }
}

/* mapder (mapder.f90:1-76) for one point: d(shape_k)/d(psi,eta) */
static void bilinear_dm(double psi, double eta, double dm[4][2])
{
    dm[0][0] = eta - 1.0;  dm[0][1] = psi - 1.0;
    dm[1][0] = 1.0 - eta;  dm[1][1] = -psi;
    dm[2][0] = eta;        dm[2][1] = psi;
    dm[3][0] = -eta;       dm[3][1] = 1.0 - psi;
}

/* calcjacob, calcjacob.f90:1-132, CURVE_WALL = 0 */
void orc_calcjacob_bilinear(int N, int ncell, const int *ivcell,
                            const double *xv, const double *yv, double *S1,
                            double *S2, double *Jac)
{
    int N1 = N + 1;
    double Xs[16], Xf[17];
    orc_setsandpoints(N, Xs, Xf);
    for (int ic = 1; ic <= ncell; ic++) {
        double X[4], Y[4];
        for (int k = 1; k <= 4; k++) {
            int iv = ivcell[(ic - 1) + ncell * (k - 1)];
            X[k - 1] = xv[iv - 1];
            Y[k - 1] = yv[iv - 1];
        }
        double dm[4][2];
        for (int js = 1; js <= N; js++)
            for (int is = 1; is <= N; is++) {
                bilinear_dm(Xs[is - 1], Xs[js - 1], dm);
                double xpsi = 0.0, xeta = 0.0, ypsi = 0.0, yeta = 0.0;
                for (int k = 0; k < 4; k++) {
                    xpsi = xpsi + dm[k][0] * X[k];
                    ypsi = ypsi + dm[k][0] * Y[k];
                    xeta = xeta + dm[k][1] * X[k];
                    yeta = yeta + dm[k][1] * Y[k];
                }
                Jac[(is - 1) + N * ((js - 1) + N * (ic - 1))] = xpsi * yeta - xeta * ypsi;
            }
        for (int jfp = 1; jfp <= N; jfp++)
            for (int ifp = 1; ifp <= N1; ifp++) {
                bilinear_dm(Xf[ifp - 1], Xs[jfp - 1], dm);
                double xpsi = 0.0, xeta = 0.0, ypsi = 0.0, yeta = 0.0;
                for (int k = 0; k < 4; k++) {
                    xpsi = xpsi + dm[k][0] * X[k];
                    ypsi = ypsi + dm[k][0] * Y[k];
                    xeta = xeta + dm[k][1] * X[k];
                    yeta = yeta + dm[k][1] * Y[k];
                }
                long b = 4L * ((ifp - 1) + N1 * ((jfp - 1) + (long)N * (ic - 1)));
                S1[b + 0] = yeta;   /* S1(1,1) */
                S1[b + 2] = -xeta;  /* S1(1,2) */
                S1[b + 1] = -ypsi;  /* S1(2,1) */
                S1[b + 3] = xpsi;   /* S1(2,2) */
            }
        for (int jfp = 1; jfp <= N1; jfp++)
            for (int ifp = 1; ifp <= N; ifp++) {
                bilinear_dm(Xs[ifp - 1], Xf[jfp - 1], dm);
                double xpsi = 0.0, xeta = 0.0, ypsi = 0.0, yeta = 0.0;
                for (int k = 0; k < 4; k++) {
                    xpsi = xpsi + dm[k][0] * X[k];
                    ypsi = ypsi + dm[k][0] * Y[k];
                    xeta = xeta + dm[k][1] * X[k];
                    yeta = yeta + dm[k][1] * Y[k];
                }
                long b = 4L * ((ifp - 1) + N * ((jfp - 1) + (long)N1 * (ic - 1)));
                S2[b + 0] = yeta;
                S2[b + 2] = -xeta;
                S2[b + 1] = -ypsi;
                S2[b + 3] = xpsi;
            }
    }
}

/* ===================================================================== */
/* context                                                               */
/* ===================================================================== */

static int g_threads = 1;

void orc_set_threads(int n)
{
    g_threads = n > 0 ? n : 1;
#ifdef _OPENMP
    omp_set_num_threads(g_threads);
#endif
}

int orc_get_threads(void) { return g_threads; }

#ifdef ORC_COUNT
/* C++ converts void * to a typed pointer only explicitly */
struct orc_anyptr {
    void *p;
    template <class T> operator T *() const { return static_cast<T *>(p); }
};
static orc_anyptr zalloc(size_t n) { return orc_anyptr{calloc(n ? n : 1, 1)}; }
#else
static void *zalloc(size_t n) { return calloc(n ? n : 1, 1); }
#endif

orc_ctx *orc_create(const orc_params *p)
{
    if (p->N < 2 || p->N > 6 || p->ncell < 1) return NULL;
    orc_ctx *cx = (orc_ctx *)zalloc(sizeof(orc_ctx));
    cx->p = *p;
    int N = p->N, N1 = N + 1;
    long NC = p->ncell;
    cx->N = N; cx->N1 = N1; cx->NC = (int)NC;
    cx->alpha = 2.0; /* initsetup.f90:165 */
    cx->fs[0] = p->rinf; cx->fs[1] = p->pinf; cx->fs[2] = p->uinf;
    cx->fs[3] = p->vinf; cx->fs[4] = p->bxinf; cx->fs[5] = p->byinf;
    cx->Xs = zalloc(sizeof(double) * N);
    cx->Xf = zalloc(sizeof(double) * N1);
    cx->Lmat = zalloc(sizeof(double) * N1 * N);
    cx->Mmat = zalloc(sizeof(double) * N1 * N);
    cx->Xs_low = zalloc(sizeof(double) * N);
    orc_setsandpoints(N, cx->Xs, cx->Xf);
    {
        double xfl[17];
        orc_setsandpoints(N - 1, cx->Xs_low, xfl); /* initsetup.f90:43-44 */
    }
    long nsp = (long)N * N * NC, nfi = (long)N1 * N * NC;
    cx->S1 = zalloc(sizeof(double) * 4 * nfi);
    cx->S2 = zalloc(sizeof(double) * 4 * nfi);
    cx->Jac = zalloc(sizeof(double) * nsp);
    cx->Q = zalloc(sizeof(real) * NV * nsp);
    cx->resid = zalloc(sizeof(real) * NV * nsp);
    cx->F1 = zalloc(sizeof(real) * NV * nfi);
    cx->G2 = zalloc(sizeof(real) * NV * nfi);
    cx->Fv1 = zalloc(sizeof(real) * NV * nfi);
    cx->Gv2 = zalloc(sizeof(real) * NV * nfi);
    cx->Qvfi = zalloc(sizeof(real) * NV * nfi);
    cx->Qvfj = zalloc(sizeof(real) * NV * nfi);
    cx->nablaQs = zalloc(sizeof(real) * NV * 2 * nsp);
    cx->nablaQvfi = zalloc(sizeof(real) * NV * 2 * nfi);
    cx->nablaQvfj = zalloc(sizeof(real) * NV * 2 * nfi);
    cx->dedxi = zalloc(sizeof(real) * nsp);
    cx->dedeta = zalloc(sizeof(real) * nsp);
    cx->muAV = zalloc(sizeof(double) * 2 * NC);
    cx->SM_IND = zalloc(sizeof(double) * 2 * NC);
    cx->muAVfi = zalloc(sizeof(double) * 4 * NC);
    cx->muAVfj = zalloc(sizeof(double) * 4 * NC);
    /* face2fpconnec, initsetup.f90:347-383 */
    for (int nfp = 1; nfp <= N; nfp++) {
        IFP_(nfp, 1) = nfp;         JFP_(nfp, 1) = 1;
        IFP_(nfp, 2) = N + 1;       JFP_(nfp, 2) = nfp;
        IFP_(nfp, 3) = N - nfp + 1; JFP_(nfp, 3) = N + 1;
        IFP_(nfp, 4) = 1;           JFP_(nfp, 4) = N - nfp + 1;
    }
    return cx;
}

void orc_destroy(orc_ctx *cx)
{
    if (!cx) return;
    void *ptrs[] = {cx->Xs, cx->Xf, cx->Lmat, cx->Mmat, cx->Xs_low, cx->S1,
                    cx->S2, cx->Jac, cx->IF2C, cx->ibfinter, cx->ibfinl,
                    cx->ibfout, cx->ibfwal, cx->ibfsymp, cx->ibfree,
                    cx->cyc2fpair, cx->Q, cx->resid, cx->F1, cx->G2, cx->Fv1,
                    cx->Gv2, cx->Qvfi, cx->Qvfj, cx->nablaQs, cx->nablaQvfi,
                    cx->nablaQvfj, cx->dedxi, cx->dedeta, cx->muAV,
                    cx->SM_IND, cx->muAVfi, cx->muAVfj, cx->ibfproc,
                    cx->Qfl_p, cx->Qfr_p, cx->Qk0_s, cx->Qka_s};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
    free(cx);
}

static int *dup_ints(const int *a, long n)
{
    int *b = (int *)zalloc(sizeof(int) * (n > 0 ? n : 1));
    if (n > 0 && a) memcpy(b, a, sizeof(int) * n);
    return b;
}

int orc_set_tables(orc_ctx *cx, const double *Lmat, const double *Mmat,
                   const double *S1, const double *S2, const double *Jac,
                   const int *IF2C, int nface, const int *ibfinter, int ninter,
                   const int *ibfinl, int ninlet, const int *ibfout,
                   int noutlet, const int *ibfwal, int nwall,
                   const int *ibfsymp, int nsymp, const int *ibfree, int nfree,
                   const int *cyc2fpair, int npair)
{
    int N = cx->N, N1 = cx->N1;
    long NC = cx->NC;
    if (Lmat) memcpy(cx->Lmat, Lmat, sizeof(double) * N1 * N);
    if (Mmat) memcpy(cx->Mmat, Mmat, sizeof(double) * N1 * N);
    memcpy(cx->S1, S1, sizeof(double) * 4 * N1 * N * NC);
    memcpy(cx->S2, S2, sizeof(double) * 4 * N1 * N * NC);
    memcpy(cx->Jac, Jac, sizeof(double) * N * N * NC);
    free(cx->IF2C); free(cx->ibfinter); free(cx->ibfinl); free(cx->ibfout);
    free(cx->ibfwal); free(cx->ibfsymp); free(cx->ibfree); free(cx->cyc2fpair);
    cx->nface = nface;
    cx->IF2C = dup_ints(IF2C, 4L * nface);
    cx->ninter = ninter;   cx->ibfinter = dup_ints(ibfinter, ninter);
    cx->ninlet = ninlet;   cx->ibfinl = dup_ints(ibfinl, ninlet);
    cx->noutlet = noutlet; cx->ibfout = dup_ints(ibfout, noutlet);
    cx->nwall = nwall;     cx->ibfwal = dup_ints(ibfwal, nwall);
    cx->nsymp = nsymp;     cx->ibfsymp = dup_ints(ibfsymp, nsymp);
    cx->nfree = nfree;     cx->ibfree = dup_ints(ibfree, nfree);
    cx->npair = npair;     cx->cyc2fpair = dup_ints(cyc2fpair, 2L * npair);
    return 0;
}

void orc_set_state(orc_ctx *cx, const real *Q, double ctime,
                   double eigvmax, double umax)
{
    memcpy(cx->Q, Q, sizeof(real) * NV * cx->N * cx->N * (long)cx->NC);
    cx->ctime = ctime;
    /* initsetup.f90:166-167 sets the local maxima; the global copies are
       zero-initialised module scalars until the first allreduce. */
    cx->eigvmax = eigvmax;
    cx->umax = umax;
    cx->eigvmax_g = eigvmax;
    cx->umax_g = umax;
}

void orc_get_state(const orc_ctx *cx, real *Q, real *resid,
                   real *nablaQs, double *muAV, double *sm_ind)
{
    long nsp = (long)cx->N * cx->N * cx->NC;
    if (Q) memcpy(Q, cx->Q, sizeof(real) * NV * nsp);
    if (resid) memcpy(resid, cx->resid, sizeof(real) * NV * nsp);
    if (nablaQs) memcpy(nablaQs, cx->nablaQs, sizeof(real) * NV * 2 * nsp);
    if (muAV) memcpy(muAV, cx->muAV, sizeof(double) * 2 * cx->NC);
    if (sm_ind) memcpy(sm_ind, cx->SM_IND, sizeof(double) * 2 * cx->NC);
}

void orc_get_maxima(const orc_ctx *cx, double *eigvmax, double *umax,
                    double *c_h, double *epsilon0, double *ctime)
{
    if (eigvmax) *eigvmax = RV(cx->eigvmax_g);
    if (umax) *umax = RV(cx->umax_g);
    if (c_h) *c_h = RV(cx->c_h);
    if (epsilon0) *epsilon0 = cx->epsilon0;
    if (ctime) *ctime = cx->ctime;
}

/* this rank's running maxima eigvmax, umax: the operands of the MAX
   allreduce of compflux.f90:10-11 */
void orc_get_local_maxima(const orc_ctx *cx, double *eigvmax, double *umax)
{
    *eigvmax = RV(cx->eigvmax);
    *umax = RV(cx->umax);
}

void orc_get_fluxes(const orc_ctx *cx, real *F1, real *G2, real *Fv1,
                    real *Gv2)
{
    long nfi = (long)cx->N1 * cx->N * cx->NC * NV;
    if (F1) memcpy(F1, cx->F1, sizeof(real) * nfi);
    if (G2) memcpy(G2, cx->G2, sizeof(real) * nfi);
    if (Fv1) memcpy(Fv1, cx->Fv1, sizeof(real) * nfi);
    if (Gv2) memcpy(Gv2, cx->Gv2, sizeof(real) * nfi);
}

void orc_set_freestream(orc_ctx *cx, const real *fs)
{
    for (int k = 0; k < 6; k++) cx->fs[k] = fs[k];
}

/* ===================================================================== */
/* point kernels                                                          */
/* ===================================================================== */

/* getIfluxvectors, getrusanov.f90:127-193 */
static void iflux(const real *Qi, real c_h, real *umax, real *Fi,
                  real *Gi)
{
    real rho = Qi[0], rhou = Qi[1], rhov = Qi[2], rhow = Qi[3],
           rhoE = Qi[4], Bx = Qi[5], By = Qi[6], Bz = Qi[7], psi = Qi[8];
    real NORM_B = (Bx * Bx + By * By) + Bz * Bz;
    real pr = (GAM - 1.0) * (((rhoE - 0.5 * ((rhou * rhou + rhov * rhov) + rhow * rhow) / rho)
                                - 0.5 * NORM_B) - 0.5 * (psi * psi));
    Fi[0] = rhou;
    Fi[1] = ((rhou * rhou) / rho + pr) + (0.5 * NORM_B - Bx * Bx);
    Fi[2] = rhou * rhov / rho - Bx * By;
    Fi[3] = rhou * rhow / rho - Bx * Bz;
    Fi[4] = (rhou / rho) * (((rhoE - 0.5 * (psi * psi)) + pr) + 0.5 * NORM_B)
            - ((rhou / rho * Bx + rhov / rho * By) + rhow / rho * Bz) * Bx;
    Fi[5] = 0.0;
    Fi[6] = rhou / rho * By - rhov / rho * Bx;
    Fi[7] = rhou / rho * Bz - rhow / rho * Bx;

    Gi[0] = rhov;
    Gi[1] = rhou * rhov / rho - Bx * By;
    Gi[2] = ((rhov * rhov) / rho + pr) + (0.5 * NORM_B - By * By);
    Gi[3] = rhow * rhov / rho - By * Bz;
    Gi[4] = (rhov / rho) * (((rhoE - 0.5 * (psi * psi)) + pr) + 0.5 * NORM_B)
            - ((rhou / rho * Bx + rhov / rho * By) + rhow / rho * Bz) * By;
    Gi[5] = rhov / rho * Bx - rhou / rho * By;
    Gi[6] = 0.0;
    Gi[7] = rhov / rho * Bz - rhow / rho * By;

    Fi[4] = Fi[4] + c_h * psi * Bx;
    Gi[4] = Gi[4] + c_h * psi * By;
    Fi[5] = Fi[5] + c_h * psi;
    Gi[6] = Gi[6] + c_h * psi;
    Fi[8] = c_h * Bx;
    Gi[8] = c_h * By;

    real u = rhou / rho, v = rhov / rho, w = rhow / rho;
    real umaxtmp = r_max(r_max(r_abs(u), r_abs(v)), r_abs(w));
    upd_max(umax, umaxtmp);
}

void orc_point_iflux(const real *Qi, real c_h, real *umax, real *F,
                     real *G)
{
    iflux(Qi, c_h, umax, F, G);
}

/* getrusanovflux, getrusanov.f90:1-125 */
static void rusanov(const real *Qfl, const real *Qfr, real *Fnl,
                    real *Fnr, const real *normf, int sign_l, int sign_r,
                    real c_h, real *eigv_out, real *eigvmax,
                    real *umax)
{
    real magnorm = r_sqrt(normf[0] * normf[0] + normf[1] * normf[1]);
    real unit_x = normf[0] / magnorm * (real)sign_l;
    real unit_y = normf[1] / magnorm * (real)sign_l;

    real rhoi = 1.0 / Qfl[0];
    real ul = rhoi * Qfl[1], vl = rhoi * Qfl[2], wl = rhoi * Qfl[3];
    real Bxl = Qfl[5], Byl = Qfl[6], Bzl = Qfl[7], psil = Qfl[8];
    real NORM_Bl = (Bxl * Bxl + Byl * Byl) + Bzl * Bzl;
    real pl = (GAM - 1.0) * (((Qfl[4] - 0.5 * Qfl[0] * ((ul * ul + vl * vl) + wl * wl))
                                - NORM_Bl * 0.5) - 0.5 * (psil * psil));
    pl = pl + 0.5 * NORM_Bl;
    real Vn_l = ul * unit_x + vl * unit_y;
    real Bn_l = Bxl * unit_x + Byl * unit_y;

    rhoi = 1.0 / Qfr[0];
    real ur = rhoi * Qfr[1], vr = rhoi * Qfr[2], wr = rhoi * Qfr[3];
    real Bxr = Qfr[5], Byr = Qfr[6], Bzr = Qfr[7], psir = Qfr[8];
    real NORM_Br = (Bxr * Bxr + Byr * Byr) + Bzr * Bzr;
    real pr = (GAM - 1.0) * (((Qfr[4] - 0.5 * Qfr[0] * ((ur * ur + vr * vr) + wr * wr))
                                - NORM_Br * 0.5) - 0.5 * (psir * psir));
    pr = pr + NORM_Br * 0.5;
    real Vn_r = ur * unit_x + vr * unit_y;
    real Bn_r = Bxr * unit_x + Byr * unit_y;

    Fnl[0] = Qfl[0] * Vn_l;
    Fnl[1] = (Qfl[1] * Vn_l + pl * unit_x) - Bxl * Bn_l;
    Fnl[2] = (Qfl[2] * Vn_l + pl * unit_y) - Byl * Bn_l;
    Fnl[3] = Qfl[3] * Vn_l - Bzl * Bn_l;
    Fnl[4] = ((Qfl[4] - 0.5 * (psil * psil)) + pl) * Vn_l
             - Bn_l * ((ul * Bxl + vl * Byl) + wl * Bzl);
    Fnl[5] = (vl * Bxl - ul * Byl) * unit_y;
    Fnl[6] = (ul * Byl - vl * Bxl) * unit_x;
    Fnl[7] = Bzl * Vn_l - wl * Bn_l;

    Fnr[0] = Qfr[0] * Vn_r;
    Fnr[1] = (Qfr[1] * Vn_r + pr * unit_x) - Bxr * Bn_r;
    Fnr[2] = (Qfr[2] * Vn_r + pr * unit_y) - Byr * Bn_r;
    Fnr[3] = Qfr[3] * Vn_r - Bzr * Bn_r;
    Fnr[4] = ((Qfr[4] - 0.5 * (psir * psir)) + pr) * Vn_r
             - Bn_r * ((ur * Bxr + vr * Byr) + wr * Bzr);
    Fnr[5] = (vr * Bxr - ur * Byr) * unit_y;
    Fnr[6] = (ur * Byr - vr * Bxr) * unit_x;
    Fnr[7] = Bzr * Vn_r - wr * Bn_r;

    Fnl[4] = Fnl[4] + c_h * psil * Bn_l;
    Fnr[4] = Fnr[4] + c_h * psir * Bn_r;
    Fnl[5] = Fnl[5] + c_h * psil * unit_x;
    Fnr[5] = Fnr[5] + c_h * psir * unit_x;
    Fnl[6] = Fnl[6] + c_h * psil * unit_y;
    Fnr[6] = Fnr[6] + c_h * psir * unit_y;
    Fnl[8] = c_h * Bn_l;
    Fnr[8] = c_h * Bn_r;

    pl = pl - 0.5 * NORM_Bl;
    pr = pr - 0.5 * NORM_Br;
    real Bx = 0.5 * (Bxl + Bxr), By = 0.5 * (Byl + Byr), Bz = 0.5 * (Bzl + Bzr);
    real c_a = GAM * (pl + pr) / (Qfl[0] + Qfr[0]);
    real c_d = ((Bx * Bx + By * By) + Bz * Bz) / (0.5 * (Qfl[0] + Qfr[0]));
    real bn = Bx * unit_x + By * unit_y;
    real c_n = bn * bn / (0.5 * (Qfl[0] + Qfr[0]));
    real cad = c_a + c_d;
    real c_tmp = r_sqrt(cad * cad - 4.0 * c_a * c_n);
    real c_f = r_sqrt(0.5 * ((c_a + c_d) + c_tmp));
    real eigv = 0.5 * r_abs(Vn_l + Vn_r) + c_f;

    for (int k = 0; k < NV; k++)
        Fnl[k] = 0.5 * ((Fnl[k] + Fnr[k]) - eigv * (Qfr[k] - Qfl[k]));
    real sl = magnorm * (real)sign_l;
    for (int k = 0; k < NV; k++) Fnl[k] = sl * Fnl[k];
    real slr = (real)(sign_l * sign_r);
    for (int k = 0; k < NV; k++) Fnr[k] = slr * Fnl[k];

    upd_max(eigvmax, eigv);
    real umaxtmp = r_max(r_max(0.5 * r_abs(ul + ur), 0.5 * r_abs(vl + vr)), 0.5 * r_abs(wl + wr));
    upd_max(umax, umaxtmp);
    if (eigv_out) *eigv_out = eigv;
}

void orc_point_rusanov(const real *Qfl, const real *Qfr, real *Fnl,
                       real *Fnr, const real *normf, int sign_l,
                       int sign_r, real c_h, real *eigv,
                       real *eigvmax, real *umax)
{
    rusanov(Qfl, Qfr, Fnl, Fnr, normf, sign_l, sign_r, c_h, eigv, eigvmax, umax);
}

/* getVfluxvectors (getrusanov.f90:197-294) with viscosity mu and
   resistivity eta; getVfluxvectors_AV (:296-413) is the same formula with
   its hard-coded mu_art = eta_art = 0 (:326, :328). */
static void vflux(const real *Qv, const real *nQ /* (9,2) */, real mu,
                  real eta0, real *Fv, real *Gv)
{
    real rho = Qv[0], rhou = Qv[1], rhov = Qv[2], rhow = Qv[3],
           rhoE = Qv[4], Bx = Qv[5], By = Qv[6], Bz = Qv[7], psi = Qv[8];
    real u = rhou / rho, v = rhov / rho, w = rhow / rho;
    real NORM_U = (u * u + v * v) + w * w;
    real NORM_B = (Bx * Bx + By * By) + Bz * Bz;
    real inte = (((rhoE - 0.5 * NORM_U * rho) - 0.5 * NORM_B) - 0.5 * (psi * psi)) / rho;
    real drho[2], du[2], dv[2], dw[2], dBx[2], dBy[2], dBz[2], dpsi[2],
        dKE[2], dpre_B[2], dpsi2[2], de[2];
    for (int d = 0; d < 2; d++) {
        drho[d] = nQ[0 + NV * d];
        du[d] = (nQ[1 + NV * d] - drho[d] * u) / rho;
        dv[d] = (nQ[2 + NV * d] - drho[d] * v) / rho;
        dw[d] = (nQ[3 + NV * d] - drho[d] * w) / rho;
        dBx[d] = nQ[5 + NV * d];
        dBy[d] = nQ[6 + NV * d];
        dBz[d] = nQ[7 + NV * d];
        dpsi[d] = nQ[8 + NV * d];
        dKE[d] = 0.5 * NORM_U * drho[d] + rho * ((u * du[d] + v * dv[d]) + w * dw[d]);
        dpre_B[d] = (Bx * dBx[d] + By * dBy[d]) + Bz * dBz[d];
        dpsi2[d] = psi * dpsi[d];
        de[d] = ((((nQ[4 + NV * d] - dKE[d]) - dpre_B[d]) - drho[d] * inte) - dpsi2[d]) / rho;
    }
    real ux = du[0], uy = du[1], vx = dv[0], vy = dv[1], wx = dw[0],
           wy = dw[1], ex = de[0], ey = de[1];
    real Bxy = dBx[1], Byx = dBy[0], Bzx = dBz[0], Bzy = dBz[1];

    Fv[0] = 0.0;
    Fv[1] = mu * (2.0 * ux + LAMBDA * (ux + vy));
    Fv[2] = mu * (vx + uy);
    Fv[3] = mu * wx;
    Fv[4] = ((u * Fv[1] + v * Fv[2]) + w * Fv[3]) + mu * GAM * ex / PRANDT;
    Gv[0] = 0.0;
    Gv[1] = mu * (vx + uy);
    Gv[2] = mu * (2.0 * vy + LAMBDA * (ux + vy));
    Gv[3] = mu * wy;
    Gv[4] = ((Gv[1] * u + Gv[2] * v) + Gv[3] * w) + mu * GAM * ey / PRANDT;

    real Jx = Bzy - 0.0, Jy = 0.0 - Bzx, Jz = Byx - Bxy;
    Fv[5] = 0.0;
    Fv[6] = eta0 * Jz;
    Fv[7] = -(eta0 * Jy);
    Fv[4] = (Fv[4] + Fv[6] * By) + Fv[7] * Bz;
    Gv[5] = -(eta0 * Jz);
    Gv[6] = 0.0;
    Gv[7] = eta0 * Jx;
    Gv[4] = (Gv[4] + Gv[5] * Bx) + Gv[7] * Bz;
    Fv[8] = 0.0;
    Gv[8] = 0.0;
}

/* ===================================================================== */
/* flux pipeline                                                          */
/* ===================================================================== */

/* Interpolate Q to the flux point of local face lf, face point nfp
   (the left/right blocks of interfaceflux_all.f90:35-77). */
static void face_trace(const orc_ctx *cx, int ic, int lf, int nfp,
                       real *Qf, int *ifp_o, int *jfp_o)
{
    int N = cx->N, N1 = cx->N1;
    int ifp = IFP_(nfp, lf), jfp = JFP_(nfp, lf);
    int fam = (lf % 2) + 1;
    for (int k = 1; k <= NV; k++) Qf[k - 1] = 0.0;
    if (fam == 1) {
        for (int sp = 1; sp <= N; sp++)
            for (int k = 1; k <= NV; k++)
                Qf[k - 1] = Qf[k - 1] + Q_(k, sp, jfp, ic) * L_(ifp, sp);
    } else {
        for (int sp = 1; sp <= N; sp++)
            for (int k = 1; k <= NV; k++)
                Qf[k - 1] = Qf[k - 1] + Q_(k, ifp, sp, ic) * L_(jfp, sp);
    }
    *ifp_o = ifp;
    *jfp_o = jfp;
}

static void face_normal(const orc_ctx *cx, int ic, int lf, int ifp, int jfp,
                        real *normf)
{
    int N = cx->N, N1 = cx->N1;
    if ((lf % 2) + 1 == 1) {
        normf[0] = S1_(1, 1, ifp, jfp, ic);
        normf[1] = S1_(1, 2, ifp, jfp, ic);
    } else {
        normf[0] = S2_(2, 1, ifp, jfp, ic);
        normf[1] = S2_(2, 2, ifp, jfp, ic);
    }
}

static void store_face(orc_ctx *cx, real *Ai, real *Aj, int ic, int lf,
                       int ifp, int jfp, const real *val)
{
    int N = cx->N, N1 = cx->N1;
    if ((lf % 2) + 1 == 1) {
        for (int k = 1; k <= NV; k++)
            Ai[((k)-1) + NV * (((ifp)-1) + N1 * (((jfp)-1) + N * ((ic)-1)))] = val[k - 1];
    } else {
        for (int k = 1; k <= NV; k++)
            Aj[((k)-1) + NV * (((ifp)-1) + N * (((jfp)-1) + N1 * ((ic)-1)))] = val[k - 1];
    }
}

/* inviscid_flux_interior, compflux.f90:53-104 */
static void inviscid_flux_interior(orc_ctx *cx)
{
    int N = cx->N, N1 = cx->N1, NC = cx->NC;
    real umax_all = cx->umax;
    int vis = cx->p.vismode;
    real c_h = cx->c_h;
#pragma omp parallel
    {
        real um = cx->umax;
#pragma omp for schedule(static)
        for (int ic = 1; ic <= NC; ic++) {
            real Qf[NV], F[NV], G[NV];
            for (int jfp = 1; jfp <= N; jfp++)
                for (int ifp = 2; ifp <= N; ifp++) {
                    for (int k = 0; k < NV; k++) Qf[k] = 0.0;
                    for (int sp = 1; sp <= N; sp++)
                        for (int k = 1; k <= NV; k++)
                            Qf[k - 1] = Qf[k - 1] + Q_(k, sp, jfp, ic) * L_(ifp, sp);
                    if (vis == 1)
                        for (int k = 1; k <= NV; k++) FI_(Qvfi, k, ifp, jfp, ic) = Qf[k - 1];
                    iflux(Qf, c_h, &um, F, G);
                    real s11 = S1_(1, 1, ifp, jfp, ic), s12 = S1_(1, 2, ifp, jfp, ic);
                    for (int k = 1; k <= NV; k++)
                        FI_(F1, k, ifp, jfp, ic) = F[k - 1] * s11 + G[k - 1] * s12;
                }
            for (int jfp = 2; jfp <= N; jfp++)
                for (int ifp = 1; ifp <= N; ifp++) {
                    for (int k = 0; k < NV; k++) Qf[k] = 0.0;
                    for (int sp = 1; sp <= N; sp++)
                        for (int k = 1; k <= NV; k++)
                            Qf[k - 1] = Qf[k - 1] + Q_(k, ifp, sp, ic) * L_(jfp, sp);
                    if (vis == 1)
                        for (int k = 1; k <= NV; k++) FJ_(Qvfj, k, ifp, jfp, ic) = Qf[k - 1];
                    iflux(Qf, c_h, &um, F, G);
                    real s21 = S2_(2, 1, ifp, jfp, ic), s22 = S2_(2, 2, ifp, jfp, ic);
                    for (int k = 1; k <= NV; k++)
                        FJ_(G2, k, ifp, jfp, ic) = F[k - 1] * s21 + G[k - 1] * s22;
                }
        }
#pragma omp critical
        upd_max(&umax_all, um);
    }
    cx->umax = umax_all;
}

/* One face shared by two cells: interfaceflux (interfaceflux_all.f90:16-110)
   and CYCLOCFLUX (cyclocflux_all.f90:15-110) run the same body. */
static void pair_flux(orc_ctx *cx, int icleft, int icright, int ifacelc,
                      int ifacerc, real *em, real *um)
{
    int N = cx->N;
    real Qfl[NV], Qfr[NV], Fnl[NV], Fnr[NV], normf[2], avg[NV], eigv;
    for (int nfp = 1; nfp <= N; nfp++) {
        int ifpl, jfpl, ifpr, jfpr;
        face_trace(cx, icleft, ifacelc, nfp, Qfl, &ifpl, &jfpl);
        int faml = (ifacelc % 2) + 1;
        int sign_l = 1;
        if (faml == 1) { if (ifpl == 1) sign_l = -1; }
        else { if (jfpl == 1) sign_l = -1; }
        face_normal(cx, icleft, ifacelc, ifpl, jfpl, normf);
        face_trace(cx, icright, ifacerc, N - nfp + 1, Qfr, &ifpr, &jfpr);
        int famr = (ifacerc % 2) + 1;
        int sign_r = 1;
        if (famr == 1) { if (ifpr == N + 1) sign_r = -1; }
        else { if (jfpr == N + 1) sign_r = -1; }
        if (cx->p.vismode == 1) {
            for (int k = 0; k < NV; k++) avg[k] = 0.5 * Qfl[k] + 0.5 * Qfr[k];
            store_face(cx, cx->Qvfi, cx->Qvfj, icleft, ifacelc, ifpl, jfpl, avg);
            store_face(cx, cx->Qvfi, cx->Qvfj, icright, ifacerc, ifpr, jfpr, avg);
        }
        rusanov(Qfl, Qfr, Fnl, Fnr, normf, sign_l, sign_r, cx->c_h, &eigv, em, um);
        store_face(cx, cx->F1, cx->G2, icleft, ifacelc, ifpl, jfpl, Fnl);
        store_face(cx, cx->F1, cx->G2, icright, ifacerc, ifpr, jfpr, Fnr);
    }
}

static void interface_and_cyclic_flux(orc_ctx *cx)
{
    real em_all = cx->eigvmax, um_all = cx->umax;
#pragma omp parallel
    {
        real em = cx->eigvmax, um = cx->umax;
#pragma omp for schedule(static)
        for (int f = 1; f <= cx->ninter; f++) {
            int iface = cx->ibfinter[f - 1];
            pair_flux(cx, IF2C_(iface, 1), IF2C_(iface, 2), IF2C_(iface, 3),
                      IF2C_(iface, 4), &em, &um);
        }
#pragma omp for schedule(static)
        for (int ip = 1; ip <= cx->npair; ip++) {
            int K1 = CYC_(ip, 1), K2 = CYC_(ip, 2);
            pair_flux(cx, IF2C_(K1, 1), IF2C_(K2, 1), IF2C_(K1, 3),
                      IF2C_(K2, 3), &em, &um);
        }
#pragma omp critical
        {
            upd_max(&em_all, em);
            upd_max(&um_all, um);
        }
    }
    cx->eigvmax = em_all;
    cx->umax = um_all;
}

/* ---- processor faces of a decomposed run ------------------------------
   PROCINTFLUX (procintflux_all.f90:1-155) and CYCREMFLUX
   (cycremflux_all.f90:1-155) evaluate a face whose other cell lives on
   another rank on each side, each with its own cell as the left cell: its
   own trace and normal, sign_r = 1, the received trace as the right state
   (point order reversed), and only Fnl scattered to its own cell. */
int orc_set_proc_faces(orc_ctx *cx, int nproc, const int *ibfproc)
{
    if (nproc < 0 || (nproc > 0 && !ibfproc)) return -1;
    for (int b = 0; b < nproc; b++)
        if (ibfproc[b] < 1 || ibfproc[b] > cx->nface) return -1;
    free(cx->ibfproc); free(cx->Qfl_p); free(cx->Qfr_p);
    cx->nproc = nproc;
    cx->ibfproc = dup_ints(ibfproc, nproc);
    cx->Qfl_p = (real *)zalloc(sizeof(real) * NV * cx->N * (nproc > 0 ? nproc : 1));
    cx->Qfr_p = (real *)zalloc(sizeof(real) * NV * cx->N * (nproc > 0 ? nproc : 1));
    return 0;
}

/* the send buffers SBUFC(9*N, NPROCINT): each processor face's own trace,
   nfp ascending, nine variables per point (procintflux_all.f90:37-76) */
void orc_proc_pack(orc_ctx *cx, real *sbuf)
{
    int N = cx->N;
    for (int b = 1; b <= cx->nproc; b++) {
        int K = cx->ibfproc[b - 1], ic = IF2C_(K, 1), lf = IF2C_(K, 3);
        for (int nfp = 1; nfp <= N; nfp++) {
            int ifp, jfp;
            real *ql = cx->Qfl_p + NV * ((nfp - 1) + N * (b - 1));
            face_trace(cx, ic, lf, nfp, ql, &ifp, &jfp);
            for (int k = 0; k < NV; k++) sbuf[NV * ((nfp - 1) + N * (b - 1)) + k] = ql[k];
        }
    }
}

/* the receive buffers RBUFC(9*N, NPROCINT), remote point nfprm going to
   own point N+1-nfprm (procintflux_all.f90:83-99) */
void orc_proc_unpack(orc_ctx *cx, const real *rbuf)
{
    int N = cx->N;
    for (int b = 1; b <= cx->nproc; b++)
        for (int nfprm = 1; nfprm <= N; nfprm++) {
            int nfp = N + 1 - nfprm;
            for (int k = 0; k < NV; k++)
                cx->Qfr_p[NV * ((nfp - 1) + N * (b - 1)) + k] = rbuf[NV * ((nfprm - 1) + N * (b - 1)) + k];
        }
}

/* procintflux_all.f90:104-151 */
static void proc_flux(orc_ctx *cx)
{
    int N = cx->N;
    real em = cx->eigvmax, um = cx->umax;
    for (int b = 1; b <= cx->nproc; b++) {
        int K = cx->ibfproc[b - 1], ic = IF2C_(K, 1), lf = IF2C_(K, 3);
        int fam = (lf % 2) + 1;
        for (int nfp = 1; nfp <= N; nfp++) {
            int ifpl = IFP_(nfp, lf), jfpl = JFP_(nfp, lf);
            int sign_l = 1;
            real normf[2], Fnl[NV], Fnr[NV], avg[NV], eigv;
            if (fam == 1) { if (ifpl == 1) sign_l = -1; }
            else { if (jfpl == 1) sign_l = -1; }
            face_normal(cx, ic, lf, ifpl, jfpl, normf);
            const real *Qfl = cx->Qfl_p + NV * ((nfp - 1) + N * (b - 1));
            const real *Qfr = cx->Qfr_p + NV * ((nfp - 1) + N * (b - 1));
            rusanov(Qfl, Qfr, Fnl, Fnr, normf, sign_l, 1, cx->c_h, &eigv, &em, &um);
            store_face(cx, cx->F1, cx->G2, ic, lf, ifpl, jfpl, Fnl);
            if (cx->p.vismode == 1) {
                for (int k = 0; k < NV; k++) avg[k] = 0.5 * Qfl[k] + 0.5 * Qfr[k];
                store_face(cx, cx->Qvfi, cx->Qvfj, ic, lf, ifpl, jfpl, avg);
            }
        }
    }
    cx->eigvmax = em;
    cx->umax = um;
}

enum { BC_INLE = 0, BC_OUTL, BC_WALL, BC_SYMP, BC_FREE };

/* Ghost state of one boundary flux point, BCFLUX (bcflux.f90:1-377). */
static void bc_ghost(const orc_ctx *cx, int kind, const real *Qfl,
                     const real *normf, real *Qfr)
{
    const orc_params *p = &cx->p;
    if (kind == BC_INLE) { /* bcflux.f90:51-72 */
        real rhor = cx->fs[0], ur = cx->fs[2], vr = cx->fs[3], wr = 0.0;
        real Bxr = cx->fs[4], Byr = cx->fs[5], Bzr = 0.0;
        Qfr[0] = rhor;
        Qfr[1] = rhor * ur;
        Qfr[2] = rhor * vr;
        Qfr[3] = rhor * wr;
        Qfr[4] = ((cx->fs[1] / (GAM - 1.0) + 0.5 * rhor * ((ur * ur + vr * vr) + wr * wr))
                  + 0.5 * ((Bxr * Bxr + Byr * Byr) + Bzr * Bzr)) + 0.5 * (Qfl[8] * Qfl[8]);
        Qfr[5] = Bxr;
        Qfr[6] = Byr;
        Qfr[7] = Bzr;
        Qfr[8] = Qfl[8];
    } else if (kind == BC_OUTL) { /* :122-143 */
        real rhor = Qfl[0], ur = Qfl[1] / Qfl[0], vr = Qfl[2] / Qfl[0], wr = 0.0;
        real Bxr = cx->fs[4], Byr = cx->fs[5], Bzr = 0.0;
        Qfr[0] = rhor;
        Qfr[1] = rhor * ur;
        Qfr[2] = rhor * vr;
        Qfr[3] = rhor * wr;
        Qfr[4] = ((cx->fs[1] / (GAM - 1.0) + 0.5 * rhor * ((ur * ur + vr * vr) + wr * wr))
                  + 0.5 * ((Bxr * Bxr + Byr * Byr) + Bzr * Bzr)) + 0.5 * (Qfl[8] * Qfl[8]);
        Qfr[5] = Bxr;
        Qfr[6] = Byr;
        Qfr[7] = Bzr;
        Qfr[8] = 0.0;
    } else if (kind == BC_WALL) { /* :196-227 */
        real rhow = Qfl[0];
        real uw = Qfl[1] / rhow, vw = Qfl[2] / rhow, ww = Qfl[3] / rhow;
        Qfr[0] = rhow;
        Qfr[4] = Qfl[4];
        Qfr[5] = -Qfl[5];
        Qfr[6] = -Qfl[6];
        Qfr[7] = -Qfl[7];
        Qfr[8] = Qfl[8];
        if (p->vismode == 0) {
            real magnorm = r_sqrt(normf[0] * normf[0] + normf[1] * normf[1]);
            real VN = uw * normf[0] / magnorm + vw * normf[1] / magnorm;
            Qfr[1] = rhow * (uw - 2.0 * VN * normf[0] / magnorm);
            Qfr[2] = rhow * (vw - 2.0 * VN * normf[1] / magnorm);
            Qfr[3] = -rhow * ww;
        } else {
            Qfr[1] = -rhow * uw;
            Qfr[2] = -rhow * vw;
            Qfr[3] = -rhow * ww;
        }
    } else if (kind == BC_SYMP) { /* :272-299 */
        real rhow = Qfl[0];
        real uw = Qfl[1] / rhow, vw = Qfl[2] / rhow, ww = Qfl[3] / rhow;
        Qfr[0] = cx->fs[0] * 2.0 - Qfl[0];
        real magnorm = r_sqrt(normf[0] * normf[0] + normf[1] * normf[1]);
        real VN = uw * normf[0] / magnorm + vw * normf[1] / magnorm;
        Qfr[1] = Qfr[0] * (uw - 2.0 * VN * normf[0] / magnorm);
        Qfr[2] = Qfr[0] * (vw - 2.0 * VN * normf[1] / magnorm);
        Qfr[3] = -Qfr[0] * ww;
        Qfr[5] = cx->fs[4];
        Qfr[6] = cx->fs[5];
        Qfr[7] = -Qfl[7];
        Qfr[8] = Qfl[8];
        Qfr[4] = (cx->fs[1] / (GAM - 1.0) + 0.5 / Qfr[0] * ((Qfr[1] * Qfr[1] + Qfr[2] * Qfr[2]) + Qfr[3] * Qfr[3]))
                 + 0.5 * (((Qfr[5] * Qfr[5] + Qfr[6] * Qfr[6]) + Qfr[7] * Qfr[7]) + Qfr[8] * Qfr[8]);
    } else { /* FREE, :355 */
        for (int k = 0; k < NV; k++) Qfr[k] = Qfl[k];
    }
}

static void bcflux(orc_ctx *cx)
{
    const int *lists[5] = {cx->ibfinl, cx->ibfout, cx->ibfwal, cx->ibfsymp, cx->ibfree};
    const int counts[5] = {cx->ninlet, cx->noutlet, cx->nwall, cx->nsymp, cx->nfree};
    int N = cx->N;
    real em = cx->eigvmax, um = cx->umax;
    for (int kind = 0; kind < 5; kind++) {
        for (int f = 1; f <= counts[kind]; f++) {
            int iface = lists[kind][f - 1];
            int icleft = IF2C_(iface, 1), ifacelc = IF2C_(iface, 3);
            int faml = (ifacelc % 2) + 1;
            for (int nfp = 1; nfp <= N; nfp++) {
                real Qfl[NV], Qfr[NV], Fnl[NV], Fnr[NV], normf[2], avg[NV], eigv;
                int ifpl, jfpl;
                face_trace(cx, icleft, ifacelc, nfp, Qfl, &ifpl, &jfpl);
                int sign_l = 1;
                if (faml == 1) { if (ifpl == 1) sign_l = -1; }
                else { if (jfpl == 1) sign_l = -1; }
                face_normal(cx, icleft, ifacelc, ifpl, jfpl, normf);
                bc_ghost(cx, kind, Qfl, normf, Qfr);
                if (cx->p.vismode == 1) {
                    for (int k = 0; k < NV; k++) avg[k] = 0.5 * Qfl[k] + 0.5 * Qfr[k];
                    store_face(cx, cx->Qvfi, cx->Qvfj, icleft, ifacelc, ifpl, jfpl, avg);
                }
                rusanov(Qfl, Qfr, Fnl, Fnr, normf, sign_l, 1, cx->c_h, &eigv, &em, &um);
                store_face(cx, cx->F1, cx->G2, icleft, ifacelc, ifpl, jfpl, Fnl);
            }
        }
    }
    cx->eigvmax = em;
    cx->umax = um;
}

/* Drag and lift are not in the reference.  Force on the wall faces: the x
   and y momentum components of each wall face point's Rusanov flux out of
   the fluid cell (the BCFLUX wall state, bcflux.f90:165-240, and
   getrusanovflux), weighted by the quadrature weight of the face point's
   position along the face. */
void orc_wall_force(orc_ctx *cx, const double *w, real *fx, real *fy)
{
    int N = cx->N;
    real sx = 0.0, sy = 0.0, em = 0.0, um = 0.0; /* maxima discarded */
    for (int f = 1; f <= cx->nwall; f++) {
        int iface = cx->ibfwal[f - 1];
        int ic = IF2C_(iface, 1), lf = IF2C_(iface, 3);
        int fam = (lf % 2) + 1;
        for (int nfp = 1; nfp <= N; nfp++) {
            real Qfl[NV], Qfr[NV], Fnl[NV], Fnr[NV], normf[2], eigv;
            int ifp, jfp;
            face_trace(cx, ic, lf, nfp, Qfl, &ifp, &jfp);
            int sign_l = 1;
            if (fam == 1) { if (ifp == 1) sign_l = -1; }
            else { if (jfp == 1) sign_l = -1; }
            face_normal(cx, ic, lf, ifp, jfp, normf);
            bc_ghost(cx, BC_WALL, Qfl, normf, Qfr);
            rusanov(Qfl, Qfr, Fnl, Fnr, normf, sign_l, 1, cx->c_h, &eigv, &em, &um);
            /* Fnl is the flux along +xi (+eta); sign_l turns it into the
               flux out of the fluid cell, the force on the body */
            double wt = w[(fam == 1 ? jfp : ifp) - 1] * (double)sign_l;
            sx = sx + wt * Fnl[1];
            sy = sy + wt * Fnl[2];
        }
    }
    *fx = sx;
    *fy = sy;
}

/* nablaQsp(1,9), compflux.f90:107-157 */
static void nablaQsp(orc_ctx *cx)
{
    int N = cx->N, N1 = cx->N1, NC = cx->NC;
#pragma omp parallel for schedule(static)
    for (int ic = 1; ic <= NC; ic++)
        for (int js = 1; js <= N; js++)
            for (int is = 1; is <= N; is++) {
                real a[NV], b[NV];
                for (int d = 1; d <= 2; d++) {
                    for (int k = 0; k < NV; k++) a[k] = 0.0;
                    for (int rfp = 1; rfp <= N1; rfp++) {
                        real s = S1_(1, d, rfp, js, ic), m = M_(rfp, is);
                        for (int k = 1; k <= NV; k++)
                            a[k - 1] = a[k - 1] + FI_(Qvfi, k, rfp, js, ic) * m * s;
                    }
                    for (int k = 0; k < NV; k++) b[k] = 0.0;
                    for (int rfp = 1; rfp <= N1; rfp++) {
                        real s = S2_(2, d, is, rfp, ic), m = M_(rfp, js);
                        for (int k = 1; k <= NV; k++)
                            b[k - 1] = b[k - 1] + FJ_(Qvfj, k, is, rfp, ic) * m * s;
                    }
                    real J = JAC_(is, js, ic);
                    for (int k = 1; k <= NV; k++) NQS_(k, d, is, js, ic) = (a[k - 1] + b[k - 1]) / J;
                }
            }
}

/* internal energy at a Qvf point, compflux.f90:272-277 */
static real enei_of(const real *q)
{
    return (((q[4] / q[0] - 0.5 * sq(q[1] / q[0])) - 0.5 * sq(q[2] / q[0])) - 0.5 * sq(q[3] / q[0]))
           - 0.5 * (((q[5] * q[5] + q[6] * q[6]) + q[7] * q[7]) + q[8] * q[8]) / q[0];
}

/* comp_grad_internal_energy, compflux.f90:260-298 */
static void comp_grad_internal_energy(orc_ctx *cx)
{
    int N = cx->N, N1 = cx->N1, NC = cx->NC;
#pragma omp parallel for schedule(static)
    for (int ic = 1; ic <= NC; ic++)
        for (int js = 1; js <= N; js++)
            for (int is = 1; is <= N; is++) {
                real t = 0.0;
                for (int rfp = 1; rfp <= N1; rfp++)
                    t = t + enei_of(&FI_(Qvfi, 1, rfp, js, ic)) * M_(rfp, is);
                DEDXI_(is, js, ic) = t;
                t = 0.0;
                for (int rfp = 1; rfp <= N1; rfp++)
                    t = t + enei_of(&FJ_(Qvfj, 1, is, rfp, ic)) * M_(rfp, js);
                DEDETA_(is, js, ic) = t;
            }
}

/* nablaQ_interior_FP, compflux.f90:159-196 */
static void nablaQ_interior_FP(orc_ctx *cx)
{
    int N = cx->N, N1 = cx->N1, NC = cx->NC;
#pragma omp parallel for schedule(static)
    for (int ic = 1; ic <= NC; ic++) {
        real a[NV], b[NV];
        for (int jfp = 1; jfp <= N; jfp++)
            for (int ifp = 2; ifp <= N; ifp++) {
                for (int k = 0; k < NV; k++) { a[k] = 0.0; b[k] = 0.0; }
                for (int sp = 1; sp <= N; sp++)
                    for (int k = 1; k <= NV; k++) {
                        a[k - 1] = a[k - 1] + NQS_(k, 1, sp, jfp, ic) * L_(ifp, sp);
                        b[k - 1] = b[k - 1] + NQS_(k, 2, sp, jfp, ic) * L_(ifp, sp);
                    }
                for (int k = 1; k <= NV; k++) {
                    NQI_(k, 1, ifp, jfp, ic) = a[k - 1];
                    NQI_(k, 2, ifp, jfp, ic) = b[k - 1];
                }
            }
        for (int jfp = 2; jfp <= N; jfp++)
            for (int ifp = 1; ifp <= N; ifp++) {
                for (int k = 0; k < NV; k++) { a[k] = 0.0; b[k] = 0.0; }
                for (int sp = 1; sp <= N; sp++)
                    for (int k = 1; k <= NV; k++) {
                        a[k - 1] = a[k - 1] + NQS_(k, 1, ifp, sp, ic) * L_(jfp, sp);
                        b[k - 1] = b[k - 1] + NQS_(k, 2, ifp, sp, ic) * L_(jfp, sp);
                    }
                for (int k = 1; k <= NV; k++) {
                    NQJ_(k, 1, ifp, jfp, ic) = a[k - 1];
                    NQJ_(k, 2, ifp, jfp, ic) = b[k - 1];
                }
            }
    }
}

/* gradient trace at a face point (the nablaQs analogue of face_trace) */
static void grad_trace(const orc_ctx *cx, int ic, int lf, int nfp,
                       real *g1, real *g2, int *ifp_o, int *jfp_o)
{
    int N = cx->N, N1 = cx->N1;
    int ifp = IFP_(nfp, lf), jfp = JFP_(nfp, lf);
    for (int k = 0; k < NV; k++) { g1[k] = 0.0; g2[k] = 0.0; }
    if ((lf % 2) + 1 == 1) {
        for (int sp = 1; sp <= N; sp++)
            for (int k = 1; k <= NV; k++) {
                g1[k - 1] = g1[k - 1] + NQS_(k, 1, sp, jfp, ic) * L_(ifp, sp);
                g2[k - 1] = g2[k - 1] + NQS_(k, 2, sp, jfp, ic) * L_(ifp, sp);
            }
    } else {
        for (int sp = 1; sp <= N; sp++)
            for (int k = 1; k <= NV; k++) {
                g1[k - 1] = g1[k - 1] + NQS_(k, 1, ifp, sp, ic) * L_(jfp, sp);
                g2[k - 1] = g2[k - 1] + NQS_(k, 2, ifp, sp, ic) * L_(jfp, sp);
            }
    }
    *ifp_o = ifp;
    *jfp_o = jfp;
}

static void store_grad(orc_ctx *cx, int ic, int lf, int ifp, int jfp,
                       const real *g1, const real *g2)
{
    int N = cx->N, N1 = cx->N1;
    if ((lf % 2) + 1 == 1) {
        for (int k = 1; k <= NV; k++) {
            NQI_(k, 1, ifp, jfp, ic) = g1[k - 1];
            NQI_(k, 2, ifp, jfp, ic) = g2[k - 1];
        }
    } else {
        for (int k = 1; k <= NV; k++) {
            NQJ_(k, 1, ifp, jfp, ic) = g1[k - 1];
            NQJ_(k, 2, ifp, jfp, ic) = g2[k - 1];
        }
    }
}

/* interfaceVISflux (interfaceflux_all.f90:114-195), CYCLOCVISFLUX
   (cyclocflux_all.f90:114-204) */
static void pair_visflux(orc_ctx *cx, int icleft, int icright, int ifacelc,
                         int ifacerc)
{
    int N = cx->N;
    real l1[NV], l2[NV], r1[NV], r2[NV], a1[NV], a2[NV];
    for (int nfp = 1; nfp <= N; nfp++) {
        int ifpl, jfpl, ifpr, jfpr;
        grad_trace(cx, icleft, ifacelc, nfp, l1, l2, &ifpl, &jfpl);
        grad_trace(cx, icright, ifacerc, N - nfp + 1, r1, r2, &ifpr, &jfpr);
        for (int k = 0; k < NV; k++) {
            a1[k] = 0.5 * l1[k] + 0.5 * r1[k];
            a2[k] = 0.5 * l2[k] + 0.5 * r2[k];
        }
        store_grad(cx, icleft, ifacelc, ifpl, jfpl, a1, a2);
        store_grad(cx, icright, ifacerc, ifpr, jfpr, a1, a2);
    }
}

/* BCVISFLUX, bcflux.f90:380-666 */
static void bcvisflux(orc_ctx *cx)
{
    int N = cx->N, N1 = cx->N1;
    const int *lists[5] = {cx->ibfinl, cx->ibfout, cx->ibfwal, cx->ibfsymp, cx->ibfree};
    const int counts[5] = {cx->ninlet, cx->noutlet, cx->nwall, cx->nsymp, cx->nfree};
    for (int kind = 0; kind < 5; kind++) {
        for (int f = 1; f <= counts[kind]; f++) {
            int iface = lists[kind][f - 1];
            int ic = IF2C_(iface, 1), lf = IF2C_(iface, 3);
            int faml = (lf % 2) + 1;
            for (int nfp = 1; nfp <= N; nfp++) {
                real g1[NV], g2[NV], r1[NV], r2[NV], a1[NV], a2[NV];
                int ifpl, jfpl;
                grad_trace(cx, ic, lf, nfp, g1, g2, &ifpl, &jfpl);
                for (int k = 0; k < NV; k++) { r1[k] = g1[k]; r2[k] = g2[k]; }
                if (kind == BC_WALL) {
                    real Qfo[NV], dxi = 0.0, deta = 0.0;
                    for (int k = 0; k < NV; k++) Qfo[k] = 0.0;
                    /* the reference accumulates the gradient trace, the
                       state trace and the energy gradients in one sp loop;
                       each accumulator has its own order, so the split
                       loops give the same values */
                    if (faml == 1) {
                        for (int sp = 1; sp <= N; sp++) {
                            for (int k = 1; k <= NV; k++)
                                Qfo[k - 1] = Qfo[k - 1] + Q_(k, sp, jfpl, ic) * L_(ifpl, sp);
                            dxi = dxi + DEDXI_(sp, jfpl, ic) * L_(ifpl, sp);
                            deta = deta + DEDETA_(sp, jfpl, ic) * L_(ifpl, sp);
                        }
                    } else {
                        for (int sp = 1; sp <= N; sp++) {
                            for (int k = 1; k <= NV; k++)
                                Qfo[k - 1] = Qfo[k - 1] + Q_(k, ifpl, sp, ic) * L_(jfpl, sp);
                            dxi = dxi + DEDXI_(ifpl, sp, ic) * L_(jfpl, sp);
                            deta = deta + DEDETA_(ifpl, sp, ic) * L_(jfpl, sp);
                        }
                    }
                    real ur = Qfo[1] / Qfo[0], vr = Qfo[2] / Qfo[0], wr = Qfo[3] / Qfo[0];
                    real inte = (Qfo[4] / Qfo[0] - 0.5 * ((ur * ur + vr * vr) + wr * wr))
                                  - 0.5 * (((Qfo[5] * Qfo[5] + Qfo[6] * Qfo[6]) + Qfo[7] * Qfo[7]) + Qfo[8] * Qfo[8]) / Qfo[0];
                    real dur, dvr, dwr, dKE, dBp;
                    /* first direction */
                    dur = (g1[1] - ur * g1[0]) / Qfo[0];
                    dvr = (g1[2] - vr * g1[0]) / Qfo[0];
                    dwr = (g1[3] - wr * g1[0]) / Qfo[0];
                    dKE = 0.5 * ((ur * ur + vr * vr) + wr * wr) * r1[0]
                          + Qfo[0] * ((ur * dur + vr * dvr) + wr * dwr);
                    dBp = ((Qfo[5] * g1[5] + Qfo[6] * g1[6]) + Qfo[7] * g1[7]) + Qfo[8] * g1[8];
                    if (faml == 1)
                        r1[4] = (((-g1[4] + 2.0 * inte * r1[0]) + 2.0 * dKE) + dBp)
                                + 2.0 * deta * S1_(2, 1, ifpl, jfpl, ic) * Qfo[0];
                    else
                        r1[4] = (((-g1[4] + 2.0 * inte * r1[0]) + 2.0 * dKE) + dBp)
                                + 2.0 * dxi * S2_(1, 1, ifpl, jfpl, ic) * Qfo[0];
                    /* second direction; dBp repeats the first direction's
                       trace (bcflux.f90:563) */
                    dur = (g2[1] - ur * g2[0]) / Qfo[0];
                    dvr = (g2[2] - vr * g2[0]) / Qfo[0];
                    dwr = (g2[3] - wr * g2[0]) / Qfo[0];
                    dKE = 0.5 * ((ur * ur + vr * vr) + wr * wr) * r2[0]
                          + Qfo[0] * ((ur * dur + vr * dvr) + wr * dwr);
                    dBp = ((Qfo[5] * g1[5] + Qfo[6] * g1[6]) + Qfo[7] * g1[7]) + Qfo[8] * g1[8];
                    if (faml == 1)
                        r2[4] = (((-g2[4] + 2.0 * inte * r2[0]) + 2.0 * dKE) + dBp)
                                + 2.0 * deta * S1_(2, 2, ifpl, jfpl, ic) * Qfo[0];
                    else
                        r2[4] = (((-g2[4] + 2.0 * inte * r2[0]) + 2.0 * dKE) + dBp)
                                + 2.0 * dxi * S2_(1, 2, ifpl, jfpl, ic) * Qfo[0];
                }
                for (int k = 0; k < NV; k++) {
                    a1[k] = 0.5 * g1[k] + 0.5 * r1[k];
                    a2[k] = 0.5 * g2[k] + 0.5 * r2[k];
                }
                store_grad(cx, ic, lf, ifpl, jfpl, a1, a2);
            }
        }
    }
}

/* comp_artificial_viscosity, AV.f90:1-142 */
static void comp_artificial_viscosity(orc_ctx *cx)
{
    int N = cx->N, NC = cx->NC, Nl = N - 1;
    /* hhval(is, Xs_low(isl)) and hhval_low(isl, Xs(is)) are pure functions
       of their indices; the reference re-evaluates them inside the loops. */
    double H[16][16], HL[16][16];
    for (int isl = 1; isl <= Nl; isl++)
        for (int is = 1; is <= N; is++) H[isl][is] = hh(cx->Xs, N, is, cx->Xs_low[isl - 1]);
    for (int is = 1; is <= N; is++)
        for (int isl = 1; isl <= Nl; isl++) HL[is][isl] = hh(cx->Xs_low, Nl, isl, cx->Xs[is - 1]);
#pragma omp parallel for schedule(static)
    for (int ic = 1; ic <= NC; ic++) {
        double lo[2][16][16], hi[2][16][16];
        for (int jsl = 1; jsl <= Nl; jsl++)
            for (int isl = 1; isl <= Nl; isl++) {
                lo[0][isl][jsl] = 0.0;
                lo[1][isl][jsl] = 0.0;
                for (int js = 1; js <= N; js++)
                    for (int is = 1; is <= N; is++) {
                        lo[0][isl][jsl] = lo[0][isl][jsl] + RV(Q_(1, is, js, ic)) * H[isl][is] * H[jsl][js];
                        double d = RV(NQS_(7, 1, is, js, ic)) - RV(NQS_(6, 2, is, js, ic));
                        lo[1][isl][jsl] = lo[1][isl][jsl] + d * d * H[isl][is] * H[jsl][js];
                    }
            }
        for (int js = 1; js <= N; js++)
            for (int is = 1; is <= N; is++) {
                hi[0][is][js] = 0.0;
                hi[1][is][js] = 0.0;
                for (int jsl = 1; jsl <= Nl; jsl++)
                    for (int isl = 1; isl <= Nl; isl++)
                        for (int v = 0; v < 2; v++)
                            hi[v][is][js] = hi[v][is][js] + lo[v][isl][jsl] * HL[is][isl] * HL[js][jsl];
            }
        double Se[2] = {0.0, 0.0};
        for (int js = 1; js <= N; js++)
            for (int is = 1; is <= N; is++) {
                double q1 = RV(Q_(1, is, js, ic));
                Se[0] = Se[0] + (hi[0][is][js] - q1) * (hi[0][is][js] - q1) / (q1 * q1);
                double d = RV(NQS_(7, 1, is, js, ic)) - RV(NQS_(6, 2, is, js, ic));
                double Jz = d * d;
                Se[1] = Se[1] + (hi[1][is][js] - Jz) * (hi[1][is][js] - Jz) / (Jz * Jz);
            }
        SMIND_(1, ic) = log10(Se[0]);
        SMIND_(2, ic) = log10(Se[1]);
    }
    /* The global min/max of the sensor (AV.f90:85-104) is never used. */
    const double se_low[2] = {-5.0, -3.0}, se_high[2] = {0.0, 1.0};
    double k_range[2], s0[2];
    for (int v = 0; v < 2; v++) {
        k_range[v] = (se_high[v] - se_low[v]) * 0.5;
        s0[v] = (se_high[v] + se_low[v]) * 0.5;
    }
    double h_msh = sqrt(cx->p.dxcycl * cx->p.dycycl / (double)cx->p.ncellglob);
    cx->epsilon0 = RV(cx->eigvmax_g) * h_msh / (double)(N - 1) * 0.05;
    double e0 = cx->epsilon0;
    for (int ic = 1; ic <= NC; ic++)
        for (int v = 1; v <= 2; v++) {
            double s = SMIND_(v, ic);
            if (s < se_low[v - 1]) MUAV_(v, ic) = 0.0;
            else if (s > se_high[v - 1]) MUAV_(v, ic) = e0;
            else
                MUAV_(v, ic) = e0 / 2.0 * (1.0 + sin(PI * (s - s0[v - 1]) / 2.0 / k_range[v - 1]));
        }
}

/* compAVflux / interfaceAVflux / cyclocAVflux, AV.f90:167-271, 462-532.
   Every (cell, local face) slot belongs to one face, so the averages do not
   depend on the loop order. */
static double *muav_slot(orc_ctx *cx, int ic, int lf)
{
    switch (lf) {
    case 1: return &MUFJ_(1, 1, ic);
    case 2: return &MUFI_(1, 2, ic);
    case 3: return &MUFJ_(1, 2, ic);
    default: return &MUFI_(1, 1, ic);
    }
}

static void comp_av_flux(orc_ctx *cx)
{
    for (int ic = 1; ic <= cx->NC; ic++)
        for (int f = 1; f <= 2; f++)
            for (int v = 1; v <= 2; v++) {
                MUFI_(v, f, ic) = MUAV_(v, ic);
                MUFJ_(v, f, ic) = MUAV_(v, ic);
            }
    for (int pass = 0; pass < 2; pass++) {
        int n = pass == 0 ? cx->ninter : cx->npair;
        for (int f = 1; f <= n; f++) {
            int icl, icr, lfl, lfr;
            if (pass == 0) {
                int iface = cx->ibfinter[f - 1];
                icl = IF2C_(iface, 1); icr = IF2C_(iface, 2);
                lfl = IF2C_(iface, 3); lfr = IF2C_(iface, 4);
            } else {
                int K1 = CYC_(f, 1), K2 = CYC_(f, 2);
                icl = IF2C_(K1, 1); icr = IF2C_(K2, 1);
                lfl = IF2C_(K1, 3); lfr = IF2C_(K2, 3);
            }
            double *L = muav_slot(cx, icl, lfl), *R = muav_slot(cx, icr, lfr);
            double a0 = 0.5 * (L[0] + R[0]), a1 = 0.5 * (L[1] + R[1]);
            L[0] = a0; L[1] = a1;
            R[0] = a0; R[1] = a1;
        }
    }
}

/* comp_viscous_flux, compflux.f90:198-258 */
static void comp_viscous_flux(orc_ctx *cx)
{
    int N = cx->N, N1 = cx->N1, NC = cx->NC;
    real mu = cx->p.mu, eta0 = cx->p.eta0;
    int artiv = cx->p.artiv;
#pragma omp parallel for schedule(static)
    for (int ic = 1; ic <= NC; ic++) {
        real Qs[NV], nQ[2 * NV], Fv[NV], Gv[NV], Fa[NV], Ga[NV];
        for (int jfp = 1; jfp <= N; jfp++)
            for (int ifp = 1; ifp <= N1; ifp++) {
                for (int k = 1; k <= NV; k++) {
                    Qs[k - 1] = FI_(Qvfi, k, ifp, jfp, ic);
                    nQ[k - 1] = NQI_(k, 1, ifp, jfp, ic);
                    nQ[NV + k - 1] = NQI_(k, 2, ifp, jfp, ic);
                }
                vflux(Qs, nQ, mu, eta0, Fv, Gv);
                real s11 = S1_(1, 1, ifp, jfp, ic), s12 = S1_(1, 2, ifp, jfp, ic);
                for (int k = 1; k <= NV; k++)
                    FI_(Fv1, k, ifp, jfp, ic) = Fv[k - 1] * s11 + Gv[k - 1] * s12;
                if (artiv == 1) {
                    vflux(Qs, nQ, 0.0, 0.0, Fa, Ga);
                    for (int k = 1; k <= NV; k++)
                        FI_(Fv1, k, ifp, jfp, ic) = (FI_(Fv1, k, ifp, jfp, ic) + Fa[k - 1] * s11) + Ga[k - 1] * s12;
                }
            }
        for (int jfp = 1; jfp <= N1; jfp++)
            for (int ifp = 1; ifp <= N; ifp++) {
                for (int k = 1; k <= NV; k++) {
                    Qs[k - 1] = FJ_(Qvfj, k, ifp, jfp, ic);
                    nQ[k - 1] = NQJ_(k, 1, ifp, jfp, ic);
                    nQ[NV + k - 1] = NQJ_(k, 2, ifp, jfp, ic);
                }
                vflux(Qs, nQ, mu, eta0, Fv, Gv);
                real s21 = S2_(2, 1, ifp, jfp, ic), s22 = S2_(2, 2, ifp, jfp, ic);
                for (int k = 1; k <= NV; k++)
                    FJ_(Gv2, k, ifp, jfp, ic) = Fv[k - 1] * s21 + Gv[k - 1] * s22;
                if (artiv == 1) {
                    vflux(Qs, nQ, 0.0, 0.0, Fa, Ga);
                    for (int k = 1; k <= NV; k++)
                        FJ_(Gv2, k, ifp, jfp, ic) = (FJ_(Gv2, k, ifp, jfp, ic) + Fa[k - 1] * s21) + Ga[k - 1] * s22;
                }
            }
    }
}

static int viscous_chain_skipped(const orc_ctx *cx)
{
    return cx->p.skip_ideal_viscous && cx->p.mu == 0.0 && cx->p.eta0 == 0.0;
}

/* compflux up to its MAX allreduce, compflux.f90:6-8: c_h from the global
   running maxima, then comp_inviscid_flux in the reference's order
   (compflux.f90:35-51): interior flux points, interfaceflux, PROCINTFLUX
   and CYCREMFLUX (the processor faces), CYCLOCFLUX, BCFLUX */
static void compflux_local(orc_ctx *cx)
{
    cx->c_h = r_sqrt(cx->eigvmax_g * (cx->eigvmax_g - cx->umax_g));
    inviscid_flux_interior(cx);
    interface_and_cyclic_flux(cx);
    proc_flux(cx);
    bcflux(cx);
}

/* compflux after the allreduce (compflux.f90:13-31) */
static void compflux_finish(orc_ctx *cx)
{
    if (cx->p.vismode == 1) {
        nablaQsp(cx);
        int skip = viscous_chain_skipped(cx);
        if (!skip) {
            if (cx->nwall > 0) comp_grad_internal_energy(cx);
            nablaQ_interior_FP(cx);
            for (int f = 1; f <= cx->ninter; f++) {
                int iface = cx->ibfinter[f - 1];
                pair_visflux(cx, IF2C_(iface, 1), IF2C_(iface, 2), IF2C_(iface, 3), IF2C_(iface, 4));
            }
            bcvisflux(cx);
            for (int ip = 1; ip <= cx->npair; ip++) {
                int K1 = CYC_(ip, 1), K2 = CYC_(ip, 2);
                pair_visflux(cx, IF2C_(K1, 1), IF2C_(K2, 1), IF2C_(K1, 3), IF2C_(K2, 3));
            }
        }
        if (cx->p.artiv == 1) {
            comp_artificial_viscosity(cx);
            if (!skip) comp_av_flux(cx);
        }
        if (!skip) comp_viscous_flux(cx);
    }
}

/* compflux, compflux.f90:1-33 */
static void compflux(orc_ctx *cx)
{
    compflux_local(cx);
    /* single rank: MPI_ALLREDUCE(MAX) is the identity (compflux.f90:10-11) */
    cx->eigvmax_g = cx->eigvmax;
    cx->umax_g = cx->umax;
    compflux_finish(cx);
}

static void compresid_divergence(orc_ctx *cx);

/* compresid, compresid.f90:1-80 */
void orc_compresid(orc_ctx *cx)
{
    compflux(cx);
    compresid_divergence(cx);
}

/* A residual of a decomposed run in the two halves around the MAX
   allreduce of compflux.f90:10-11, which the caller performs over the ranks
   between them (orc_get_maxima, then orc_set_global_maxima). */
void orc_compresid_local(orc_ctx *cx) { compflux_local(cx); }

void orc_set_global_maxima(orc_ctx *cx, double eigvmax_g, double umax_g)
{
    cx->eigvmax_g = eigvmax_g;
    cx->umax_g = umax_g;
}

void orc_compresid_finish(orc_ctx *cx)
{
    compflux_finish(cx);
    compresid_divergence(cx);
}

/* compresid.f90:12-78: the flux divergence over Jac and the sources */
static void compresid_divergence(orc_ctx *cx)
{
    int N = cx->N, N1 = cx->N1, NC = cx->NC;
    int vis = cx->p.vismode == 1, skip = viscous_chain_skipped(cx);
    real alpha = cx->alpha;
#pragma omp parallel for schedule(static)
    for (int ic = 1; ic <= NC; ic++)
        for (int js = 1; js <= N; js++)
            for (int is = 1; is <= N; is++) {
                real dF[NV], dG[NV], dFv[NV], dGv[NV];
                for (int k = 0; k < NV; k++) { dF[k] = 0.0; dFv[k] = 0.0; }
                for (int rfp = 1; rfp <= N1; rfp++) {
                    real m = M_(rfp, is);
                    for (int k = 1; k <= NV; k++) {
                        dF[k - 1] = dF[k - 1] + FI_(F1, k, rfp, js, ic) * m;
                        if (vis && !skip) dFv[k - 1] = dFv[k - 1] + FI_(Fv1, k, rfp, js, ic) * m;
                    }
                }
                for (int k = 0; k < NV; k++) { dG[k] = 0.0; dGv[k] = 0.0; }
                for (int rfp = 1; rfp <= N1; rfp++) {
                    real m = M_(rfp, js);
                    for (int k = 1; k <= NV; k++) {
                        dG[k - 1] = dG[k - 1] + FJ_(G2, k, is, rfp, ic) * m;
                        if (vis && !skip) dGv[k - 1] = dGv[k - 1] + FJ_(Gv2, k, is, rfp, ic) * m;
                    }
                }
                for (int k = 1; k <= NV; k++) R_(k, is, js, ic) = -(dF[k - 1] + dG[k - 1]);
                /* with the chain skipped, dFv and dGv are the +0.0 that the
                   full chain produces for mu == eta0 == 0 */
                if (vis)
                    for (int k = 1; k <= NV; k++)
                        R_(k, is, js, ic) = R_(k, is, js, ic) + (dFv[k - 1] + dGv[k - 1]);
            }
#pragma omp parallel for schedule(static)
    for (int ic = 1; ic <= NC; ic++)
        for (int js = 1; js <= N; js++)
            for (int is = 1; is <= N; is++) {
                real J = JAC_(is, js, ic);
                for (int k = 1; k <= NV; k++) R_(k, is, js, ic) = R_(k, is, js, ic) / J;
                real divB = NQS_(6, 1, is, js, ic) + NQS_(7, 2, is, js, ic);
                real Bx = Q_(6, is, js, ic), By = Q_(7, is, js, ic), Bz = Q_(8, is, js, ic);
                real ux = Q_(2, is, js, ic) / Q_(1, is, js, ic);
                real uy = Q_(3, is, js, ic) / Q_(1, is, js, ic);
                real uz = Q_(4, is, js, ic) / Q_(1, is, js, ic);
                real psi = Q_(9, is, js, ic);
                R_(2, is, js, ic) = R_(2, is, js, ic) - divB * Bx;
                R_(3, is, js, ic) = R_(3, is, js, ic) - divB * By;
                R_(4, is, js, ic) = R_(4, is, js, ic) - divB * Bz;
                R_(5, is, js, ic) = R_(5, is, js, ic) - divB * ((ux * Bx + uy * By) + uz * Bz);
                R_(6, is, js, ic) = R_(6, is, js, ic) - divB * ux;
                R_(7, is, js, ic) = R_(7, is, js, ic) - divB * uy;
                R_(8, is, js, ic) = R_(8, is, js, ic) - divB * uz;
                R_(9, is, js, ic) = R_(9, is, js, ic) - alpha * psi;
            }
}

/* ===================================================================== */
/* time integration                                                       */
/* ===================================================================== */

/* RK_S5P3 coefficients, iterations.f90:164-174 */
static const double A30 = 0.355909775063327, A32 = 0.644090224936674,
                    A40 = 0.367933791638137, A43 = 0.632066208361863,
                    A52 = 0.237593836598569, A54 = 0.762406163401431,
                    B10 = 0.377268915331368, B21 = 0.377268915331368,
                    B32 = 0.242995220537396, B43 = 0.238458932846290,
                    B54 = 0.287632146308408;

void orc_rk_s5p3_combine(int stage, long n, real dt, real *q,
                         const real *qk0, const real *qka,
                         const real *r)
{
    long i;
    switch (stage) {
    case 1: { real c = B10 * dt;
#pragma omp parallel for schedule(static)
        for (i = 0; i < n; i++) q[i] = q[i] + c * r[i];
        break; }
    case 2: { real c = B21 * dt;
#pragma omp parallel for schedule(static)
        for (i = 0; i < n; i++) q[i] = q[i] + c * r[i];
        break; }
    case 3: { real c = B32 * dt;
#pragma omp parallel for schedule(static)
        for (i = 0; i < n; i++) q[i] = (A30 * qk0[i] + A32 * q[i]) + c * r[i];
        break; }
    case 4: { real c = B43 * dt;
#pragma omp parallel for schedule(static)
        for (i = 0; i < n; i++) q[i] = (A40 * qk0[i] + A43 * q[i]) + c * r[i];
        break; }
    default: { real c = B54 * dt;
#pragma omp parallel for schedule(static)
        for (i = 0; i < n; i++) q[i] = (A52 * qka[i] + A54 * q[i]) + c * r[i];
        break; }
    }
}

/* RK_S5P3, iterations.f90:158-213 */
void orc_rk_s5p3(orc_ctx *cx, double dt, int nsteps)
{
    long n = (long)NV * cx->N * cx->N * cx->NC;
    real *Qk0 = (real *)malloc(sizeof(real) * n);
    real *Qka = (real *)malloc(sizeof(real) * n);
    for (int s = 0; s < nsteps; s++) {
        memcpy(Qk0, cx->Q, sizeof(real) * n);
        double ctime0 = cx->ctime;
        orc_compresid(cx);
        orc_rk_s5p3_combine(1, n, dt, cx->Q, Qk0, Qka, cx->resid);
        double dt1 = B10 * dt;
        cx->ctime = ctime0 + dt1;
        orc_compresid(cx);
        orc_rk_s5p3_combine(2, n, dt, cx->Q, Qk0, Qka, cx->resid);
        double dt2 = dt1 + B21 * dt;
        cx->ctime = ctime0 + dt2;
        memcpy(Qka, cx->Q, sizeof(real) * n);
        orc_compresid(cx);
        orc_rk_s5p3_combine(3, n, dt, cx->Q, Qk0, Qka, cx->resid);
        double dt3 = A32 * dt2 + B32 * dt;
        cx->ctime = ctime0 + dt3;
        orc_compresid(cx);
        orc_rk_s5p3_combine(4, n, dt, cx->Q, Qk0, Qka, cx->resid);
        double dt4 = A43 * dt3 + B43 * dt;
        cx->ctime = ctime0 + dt4;
        (void)dt4;
        orc_compresid(cx);
        orc_rk_s5p3_combine(5, n, dt, cx->Q, Qk0, Qka, cx->resid);
        cx->ctime = ctime0 + dt;
    }
    free(Qk0);
    free(Qka);
}

/* RK_S5P3 one stage at a time, for a decomposed run whose ranks exchange
   traces and maxima between the stages: orc_rk_s5p3_begin_stage, the
   residual (orc_compresid, or its two halves around the allreduce), then
   orc_rk_s5p3_end_stage.  The same registers and time bookkeeping as
   orc_rk_s5p3 (iterations.f90:175-212). */
void orc_rk_s5p3_begin_stage(orc_ctx *cx, int stage)
{
    long n = (long)NV * cx->N * cx->N * cx->NC;
    if (!cx->Qk0_s) {
        cx->Qk0_s = (real *)zalloc(sizeof(real) * n);
        cx->Qka_s = (real *)zalloc(sizeof(real) * n);
    }
    if (stage == 1) {
        memcpy(cx->Qk0_s, cx->Q, sizeof(real) * n);
        cx->ctime0_s = cx->ctime;
    }
}

void orc_rk_s5p3_end_stage(orc_ctx *cx, int stage, double dt)
{
    long n = (long)NV * cx->N * cx->N * cx->NC;
    orc_rk_s5p3_combine(stage, n, dt, cx->Q, cx->Qk0_s, cx->Qka_s, cx->resid);
    double d;
    switch (stage) {
    case 1: d = B10 * dt; break;
    case 2: d = cx->ctime_stage_s + B21 * dt; break;
    case 3: d = A32 * cx->ctime_stage_s + B32 * dt; break;
    case 4: d = A43 * cx->ctime_stage_s + B43 * dt; break;
    default: d = dt; break;
    }
    cx->ctime_stage_s = d;
    cx->ctime = cx->ctime0_s + d;
    if (stage == 2) memcpy(cx->Qka_s, cx->Q, sizeof(real) * n);
}

/* FiveStageRk, iterations.f90:88-156 */
void orc_five_stage_rk(orc_ctx *cx, double dt, int nsteps)
{
    long n = (long)NV * cx->N * cx->N * cx->NC;
    real *qj0 = (real *)malloc(sizeof(real) * n);
    real *qj2 = (real *)malloc(sizeof(real) * n);
    real *qj3 = (real *)malloc(sizeof(real) * n);
    real *r0 = (real *)malloc(sizeof(real) * n);
    real *Q = cx->Q, *R = cx->resid;
    for (int s = 0; s < nsteps; s++) {
        double old_time = cx->ctime;
        memcpy(qj0, Q, sizeof(real) * n);
        orc_compresid(cx);
        double a11 = 0.39175222700392;
        double rdt = dt * a11;
        for (long i = 0; i < n; i++) Q[i] = qj0[i] + rdt * R[i];
        cx->ctime = old_time + rdt;
        orc_compresid(cx);
        double a21 = 0.44437049406734, a22 = 0.55562950593266, a23 = 0.36841059262959;
        for (long i = 0; i < n; i++) Q[i] = (a21 * qj0[i] + a22 * Q[i]) + a23 * R[i] * dt;
        memcpy(qj2, Q, sizeof(real) * n);
        rdt = rdt * a22 + a23 * dt;
        cx->ctime = old_time + rdt;
        orc_compresid(cx);
        double a31 = 0.6201018513854, a32 = 0.3798981486146, a33 = 0.25189177424738;
        double c3 = a33 * dt;
        for (long i = 0; i < n; i++) Q[i] = (a31 * qj0[i] + a32 * Q[i]) + c3 * R[i];
        memcpy(qj3, Q, sizeof(real) * n);
        rdt = rdt * a32 + a33 * dt;
        cx->ctime = old_time + rdt;
        orc_compresid(cx);
        double a41 = 0.17807995410773, a42 = 0.82192004589227, a43 = 0.54497475021237;
        double c4 = a43 * dt;
        for (long i = 0; i < n; i++) Q[i] = (a41 * qj0[i] + a42 * Q[i]) + c4 * R[i];
        memcpy(r0, R, sizeof(real) * n);
        rdt = rdt * a42 + a43 * dt;
        cx->ctime = old_time + rdt;
        orc_compresid(cx);
        double a51 = 0.00683325884039, a52 = 0.51723167208978, a53 = 0.12759831133288,
               a54 = 0.34833675773694, a55 = 0.08460416338212, a56 = 0.22600748319395;
        double c55 = a55 * dt, c56 = a56 * dt;
        for (long i = 0; i < n; i++)
            Q[i] = ((((a51 * qj0[i] + a52 * qj2[i]) + a53 * qj3[i]) + a54 * Q[i]) + c55 * r0[i]) + c56 * R[i];
        cx->ctime = old_time + dt;
    }
    free(qj0); free(qj2); free(qj3); free(r0);
}

/* residual and divB sums of the monitor, iterations.f90:34-46 */
void orc_monitor(const orc_ctx *cx, double *residsum, double *divbsum)
{
    int N = cx->N, NC = cx->NC;
    real rn = 0.0, db = 0.0;
    for (int ic = 1; ic <= NC; ic++)
        for (int js = 1; js <= N; js++)
            for (int is = 1; is <= N; is++) {
                for (int k = 1; k <= NV; k++) rn = rn + sq(R_(k, is, js, ic));
                db = db + sq(NQS_(6, 1, is, js, ic) + NQS_(7, 2, is, js, ic));
            }
    *residsum = RV(rn);
    *divbsum = RV(db);
}
