// Checks the hand-written adjoint point functions (adjoint_point.cuh)
// against forward-mode dual numbers through the same templated point physics
// (physics.cuh, exact form): for random valid states, directions v and
// output adjoints w, <w, J v> from the duals must equal <J^T w, v> from the
// adjoint functions.  Host code only (test infrastructure); prints the worst
// relative mismatch of each check and exits non-zero above the tolerance.
#include <cmath>
#include <cstdio>
#include <random>

#include "dual.cuh"
#include "adjoint_point.cuh"

using namespace sddc;
using D1 = Dual<1>;

static std::mt19937_64 rng(12345);
static double U(double a, double b) { return std::uniform_real_distribution<double>(a, b)(rng); }

// a random state with positive density and gas pressure
static void rand_state(double *q)
{
    const double rho = U(0.5, 2.0), u = U(-1.5, 1.5), v = U(-1.5, 1.5), w = U(-0.3, 0.3);
    const double Bx = U(-1, 1), By = U(-1, 1), Bz = U(-0.3, 0.3), psi = U(-0.2, 0.2), p = U(0.2, 2.0);
    q[0] = rho; q[1] = rho * u; q[2] = rho * v; q[3] = rho * w;
    q[4] = p / (kGam - 1.0) + 0.5 * rho * (u * u + v * v + w * w) + 0.5 * (Bx * Bx + By * By + Bz * Bz) +
           0.5 * psi * psi;
    q[5] = Bx; q[6] = By; q[7] = Bz; q[8] = psi;
}

static double worst = 0.0;
static void report(const char *what, double a, double b, double scale)
{
    const double e = std::fabs(a - b) / (std::fabs(scale) + 1e-300);
    if (e > worst) worst = e;
    if (e > 1e-11) std::printf("  %s: %.17g vs %.17g (rel %.3g)\n", what, a, b, e);
}

int main()
{
    double m_iflux = 0, m_rus = 0, m_ghost = 0;
    for (int trial = 0; trial < 400; trial++) {
        // ---- interior flux point -------------------------------------------
        {
            double q[9], vdir[9], fb[9];
            rand_state(q);
            for (int k = 0; k < 9; k++) { vdir[k] = U(-1, 1); fb[k] = U(-1, 1); }
            const double c = U(0.0, 3.0), n0 = U(-2, 2), n1 = U(-2, 2);
            D1 Q[9], F[9], G[9];
            for (int k = 0; k < 9; k++) { Q[k] = D1(q[k]); Q[k].d[0] = vdir[k]; }
            D1 um(0.0);
            iflux<D1, true>(Q, D1(c), um, F, G);
            double fwd = 0.0, scale = 0.0;
            for (int k = 0; k < 9; k++) {
                const double t = fb[k] * (n0 * F[k].d[0] + n1 * G[k].d[0]);
                fwd += t;
                scale += std::fabs(t);
            }
            double qb[9] = {0}, umv, umd[9];
            const double cb = iflux_vjp(q, c, n0, n1, fb, qb, umv, umd);
            double rev = 0.0, umdir = 0.0;
            for (int k = 0; k < 9; k++) { rev += qb[k] * vdir[k]; umdir += umd[k] * vdir[k]; }
            report("iflux <w,Jv>", fwd, rev, scale);
            m_iflux = std::fmax(m_iflux, std::fabs(fwd - rev) / scale);
            report("iflux um", um.d[0], umdir, std::fabs(um.d[0]) + 1.0);
            report("iflux um value", um.v, umv, um.v + 1e-300);
            // c derivative
            for (int k = 0; k < 9; k++) Q[k] = D1(q[k]);
            D1 cc(c);
            cc.d[0] = 1.0;
            D1 um2(0.0);
            iflux<D1, true>(Q, cc, um2, F, G);
            double fc = 0.0, d[9];
            iflux_dfdc(q, n0, n1, d);
            double dd = 0.0;
            for (int k = 0; k < 9; k++) { fc += fb[k] * (n0 * F[k].d[0] + n1 * G[k].d[0]); dd += fb[k] * d[k]; }
            report("iflux dc", fc, cb, std::fabs(fc) + 1.0);
            report("iflux dfdc", fc, dd, std::fabs(fc) + 1.0);
        }
        // ---- Rusanov face flux ------------------------------------------------
        {
            double ql[9], qr[9], vl[9], vr[9], fb[9];
            rand_state(ql);
            rand_state(qr);
            for (int k = 0; k < 9; k++) { vl[k] = U(-1, 1); vr[k] = U(-1, 1); fb[k] = U(-1, 1); }
            const double c = U(0.0, 3.0), n0 = U(-2, 2), n1 = U(-2, 2);
            const int sl = trial % 2 ? 1 : -1, sr = (trial / 2) % 2 ? 1 : -1;
            const double eb0 = U(-1, 1), umb0 = U(-1, 1);
            D1 Ql[9], Qr[9], Fl[9], Fr[9], eig, um(0.0);
            for (int k = 0; k < 9; k++) {
                Ql[k] = D1(ql[k]); Ql[k].d[0] = vl[k];
                Qr[k] = D1(qr[k]); Qr[k].d[0] = vr[k];
            }
            rusanov<D1, true>(Ql, Qr, Fl, Fr, D1(n0), D1(n1), sl, sr, D1(c), eig, um);
            double fwd = eb0 * eig.d[0] + umb0 * um.d[0], scale = std::fabs(eb0 * eig.d[0]) + std::fabs(umb0 * um.d[0]);
            for (int k = 0; k < 9; k++) { fwd += fb[k] * Fl[k].d[0]; scale += std::fabs(fb[k] * Fl[k].d[0]); }
            double qlb[9] = {0}, qrb[9] = {0}, eigv, umv, dfdc[9];
            const double wdc = rusanov_vjp(ql, qr, n0, n1, sl, c, fb, eb0, umb0, qlb, qrb, eigv, umv, dfdc, fb);
            double rev = 0.0;
            for (int k = 0; k < 9; k++) rev += qlb[k] * vl[k] + qrb[k] * vr[k];
            report("rusanov <w,Jv>", fwd, rev, scale);
            m_rus = std::fmax(m_rus, std::fabs(fwd - rev) / scale);
            // primal values agree with the exact form to rounding
            double dl[9], dr[9], Fld[9], Frd[9], e2, u2 = 0.0;
            for (int k = 0; k < 9; k++) { dl[k] = ql[k]; dr[k] = qr[k]; }
            rusanov<double, true>(dl, dr, Fld, Frd, n0, n1, sl, sr, c, e2, u2);
            report("rusanov eig", e2, eigv, e2);
            report("rusanov um", u2, umv, u2 + 1e-300);
            // c derivative
            for (int k = 0; k < 9; k++) { Ql[k] = D1(ql[k]); Qr[k] = D1(qr[k]); }
            D1 cc(c);
            cc.d[0] = 1.0;
            D1 um3(0.0);
            rusanov<D1, true>(Ql, Qr, Fl, Fr, D1(n0), D1(n1), sl, sr, cc, eig, um3);
            double wd = 0.0, ws = 0.0;
            for (int k = 0; k < 9; k++) {
                report("rusanov dfdc", Fl[k].d[0], dfdc[k], std::fabs(Fl[k].d[0]) + 1.0);
                wd += fb[k] * Fl[k].d[0];
                ws += std::fabs(fb[k] * Fl[k].d[0]);
            }
            report("rusanov w.dfdc", wd, rusanov_wdfdc(ql, qr, n0, n1, sl, fb), ws + 1.0);
            report("rusanov w.dfdc (returned)", wd, wdc, ws + 1.0);
        }
        // ---- boundary ghost states --------------------------------------------
        {
            const int kinds[6] = {kFaceInle, kFaceOutl, kFaceWall, kFaceWall, kFaceSymp, kFaceFree};
            for (int t = 0; t < 6; t++) {
                const int kind = kinds[t], vismode = t == 2 ? 0 : 1;
                double ql[9], vl[9], qrb[9], fsv[6], pv[6];
                rand_state(ql);
                for (int k = 0; k < 9; k++) { vl[k] = U(-1, 1); qrb[k] = U(-1, 1); }
                fsv[0] = U(0.5, 2); fsv[1] = U(0.2, 2); fsv[2] = U(-1, 1); fsv[3] = U(-1, 1);
                fsv[4] = U(-1, 1); fsv[5] = U(-1, 1);
                for (int k = 0; k < 6; k++) pv[k] = U(-1, 1);
                const double n0 = U(-2, 2), n1 = U(-2, 2);
                // the dual free stream: ghost states read it through (R) casts,
                // so the parameter direction goes in by linearity: two runs
                D1 Ql[9], Gh[9];
                for (int k = 0; k < 9; k++) { Ql[k] = D1(ql[k]); Ql[k].d[0] = vl[k]; }
                Freestream fs{fsv[0], fsv[1], fsv[2], fsv[3], fsv[4], fsv[5]};
                bc_ghost<D1, true>(kind, Ql, D1(n0), D1(n1), vismode, fs, Gh);
                double fwd = 0.0, scale = 0.0;
                for (int k = 0; k < 9; k++) { fwd += qrb[k] * Gh[k].d[0]; scale += std::fabs(qrb[k] * Gh[k].d[0]); }
                // parameter part by central differences of the (polynomial)
                // ghost state
                const double h = 1e-6;
                Freestream fp{fsv[0] + h * pv[0], fsv[1] + h * pv[1], fsv[2] + h * pv[2], fsv[3] + h * pv[3],
                              fsv[4] + h * pv[4], fsv[5] + h * pv[5]};
                Freestream fm{fsv[0] - h * pv[0], fsv[1] - h * pv[1], fsv[2] - h * pv[2], fsv[3] - h * pv[3],
                              fsv[4] - h * pv[4], fsv[5] - h * pv[5]};
                double gp[9], gm[9];
                bc_ghost<double, true>(kind, ql, n0, n1, vismode, fp, gp);
                bc_ghost<double, true>(kind, ql, n0, n1, vismode, fm, gm);
                double fwdp = 0.0;
                for (int k = 0; k < 9; k++) fwdp += qrb[k] * (gp[k] - gm[k]) / (2 * h);
                double qlb[9] = {0}, pb[6] = {0};
                bc_ghost_vjp(kind, ql, n0, n1, vismode, fs, qrb, qlb, pb);
                double rev = 0.0, revp = 0.0;
                for (int k = 0; k < 9; k++) rev += qlb[k] * vl[k];
                for (int k = 0; k < 6; k++) revp += pb[k] * pv[k];
                report("ghost <w,Jv>", fwd, rev, scale + 1e-12);
                m_ghost = std::fmax(m_ghost, std::fabs(fwd - rev) / (scale + 1e-12));
                const double e = std::fabs(fwdp - revp) / (std::fabs(fwdp) + 1.0);
                if (e > 1e-8) { std::printf("  ghost kind %d parameters: %.12g vs %.12g\n", kind, fwdp, revp); worst = 1.0; }
            }
        }
    }
    std::printf("iflux %.3g  rusanov %.3g  ghost %.3g  worst %.3g\n", m_iflux, m_rus, m_ghost, worst);
    return worst < 1e-11 ? 0 : 1;
}
