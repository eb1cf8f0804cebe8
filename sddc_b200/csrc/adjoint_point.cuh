// Reverse-mode (adjoint) point functions of the SDDC residual, by hand.
//
// Each function takes the adjoint of a point function's output and adds the
// adjoint of its inputs (vector-Jacobian product):
//   iflux_vjp     computational flux n0*F + n1*G at an interior flux point
//                 (getIfluxvectors, getrusanov.f90:127-193)
//   rusanov_vjp   Rusanov face flux of the left cell (getrusanovflux,
//                 getrusanov.f90:1-125), with the wave speed and the face
//                 velocity maximum as extra outputs
//   bc_ghost_vjp  boundary ghost states (BCFLUX, bcflux.f90:17-375),
//                 including the free-stream parameters
// They recompute the primal values they need with reciprocals (the argmax of
// a running maximum is located by the forward's own point functions, so
// these need not round as the forward does).  Non-smooth points take the branch the primal takes: |x| has slope +1 at
// x == 0 (as fabs's branch x >= 0), max() the argument it returns, and the
// square root of the fast-speed discriminant has slope 0 where the
// discriminant is 0.
#pragma once

#include "physics.cuh"

namespace sddc {

constexpr double kG1 = kGam - 1.0;

SDDC_HD double sgn1(double x) { return x < 0.0 ? -1.0 : 1.0; }

// 1/sqrt(x): the device's reciprocal square root (within an ulp or so, which
// the adjoint's tolerance allows); the host's sqrt and divide
SDDC_HD double Rsqrt(double x)
{
#ifdef __CUDA_ARCH__
    return rsqrt(x);
#else
    return 1.0 / sqrt(x);
#endif
}

// Adjoint of Fc = n0*F(Q, c) + n1*G(Q, c) at one interior flux point.
// fb: adjoint of Fc; qb += (dFc/dQ)^T fb.  Returns fb . dFc/dc; um gets the
// point's velocity maximum max(|u|, |v|, |w|) and um_d its gradient with
// respect to Q (for the running-max adjoint).
SDDC_HD double iflux_vjp(const double *Q, double c, double n0, double n1, const double *fb, double *qb, double &um,
                         double *um_d)
{
    const double rho = Q[0], mx = Q[1], my = Q[2], mz = Q[3], E = Q[4];
    const double Bx = Q[5], By = Q[6], Bz = Q[7], psi = Q[8];
    const double ri = 1.0 / rho;
    const double u = mx * ri, v = my * ri, w = mz * ri;
    const double au = Abs(u), av = Abs(v), aw = Abs(w);
    const double m1 = Max(au, av);
    um = Max(m1, aw);
    if (um_d) {
        // the selected component: Max(a, b) returns b unless a > b
        const int sel = (m1 > aw) ? (au > av ? 0 : 1) : 2;
        const double comp = sel == 0 ? u : (sel == 1 ? v : w);
        const double s = sgn1(comp) * ri;
        for (int k = 0; k < 9; k++) um_d[k] = 0.0;
        um_d[0] = -s * comp;
        um_d[1 + sel] = s;
    }
    const double NB = (Bx * Bx + By * By) + Bz * Bz;
    const double q2 = (u * u + v * v) + w * w;
    const double pr = kG1 * (((E - 0.5 * rho * q2) - 0.5 * NB) - 0.5 * (psi * psi));
    const double eb = ((E - 0.5 * (psi * psi)) + pr) + 0.5 * NB;
    const double ub = (u * Bx + v * By) + w * Bz;

    double a[9], b[9];
    for (int k = 0; k < 9; k++) {
        a[k] = n0 * fb[k];
        b[k] = n1 * fb[k];
    }
    const double ebb = a[4] * u + b[4] * v;
    const double ubb = -(a[4] * Bx + b[4] * By);
    const double pb = a[1] + b[2] + ebb;
    double ubar = a[0] * rho + 2.0 * a[1] * rho * u + a[2] * rho * v + a[3] * rho * w + a[4] * eb + ubb * Bx +
                  a[6] * By + a[7] * Bz - b[5] * By + b[1] * rho * v;
    double vbar = b[0] * rho + 2.0 * b[2] * rho * v + b[1] * rho * u + b[3] * rho * w + b[4] * eb + ubb * By -
                  a[6] * Bx + b[5] * Bx + b[7] * Bz + a[2] * rho * u;
    double wbar = a[3] * rho * u + b[3] * rho * v + ubb * Bz - a[7] * Bx - b[7] * By;
    double rbar = a[0] * u + b[0] * v + a[1] * u * u + a[2] * u * v + a[3] * u * w + b[1] * u * v + b[2] * v * v +
                  b[3] * v * w;
    double Ebar = ebb;
    double Bxb = -a[1] * Bx - a[2] * By - a[3] * Bz + a[4] * (c * psi - ub) - a[6] * v - a[7] * w + a[8] * c -
                 b[1] * By + b[2] * Bx + b[5] * v + ubb * u + ebb * Bx;
    double Byb = a[1] * By - a[2] * Bx + a[6] * u - b[1] * Bx - b[2] * By - b[3] * Bz + b[4] * (c * psi - ub) -
                 b[5] * u - b[7] * w + b[8] * c + ubb * v + ebb * By;
    double Bzb = a[1] * Bz - a[3] * Bx + a[7] * u + b[2] * Bz - b[3] * By + b[7] * v + ubb * w + ebb * Bz;
    double psib = a[4] * c * Bx + a[5] * c + b[4] * c * By + b[6] * c - ebb * psi;
    // pressure p = (gam-1) (E - rho |u|^2 / 2 - |B|^2 / 2 - psi^2 / 2)
    Ebar += kG1 * pb;
    rbar -= kG1 * 0.5 * q2 * pb;
    ubar -= kG1 * rho * u * pb;
    vbar -= kG1 * rho * v * pb;
    wbar -= kG1 * rho * w * pb;
    Bxb -= kG1 * Bx * pb;
    Byb -= kG1 * By * pb;
    Bzb -= kG1 * Bz * pb;
    psib -= kG1 * psi * pb;
    // primitive -> conserved
    qb[0] += rbar - (ubar * u + vbar * v + wbar * w) * ri;
    qb[1] += ubar * ri;
    qb[2] += vbar * ri;
    qb[3] += wbar * ri;
    qb[4] += Ebar;
    qb[5] += Bxb;
    qb[6] += Byb;
    qb[7] += Bzb;
    qb[8] += psib;
    return a[4] * psi * Bx + a[5] * psi + a[8] * Bx + b[4] * psi * By + b[6] * psi + b[8] * By;
}

// per-side quantities of the Rusanov flux
struct RusSide {
    double rho, mx, my, mz, E, Bx, By, Bz, psi;
    double ri, u, v, w, NB, p, pt, Vn, Bn, ub;
};

SDDC_HD void rus_side(const double *Q, double ux, double uy, RusSide &s)
{
    s.rho = Q[0]; s.mx = Q[1]; s.my = Q[2]; s.mz = Q[3]; s.E = Q[4];
    s.Bx = Q[5]; s.By = Q[6]; s.Bz = Q[7]; s.psi = Q[8];
    s.ri = 1.0 / s.rho;
    s.u = s.ri * s.mx; s.v = s.ri * s.my; s.w = s.ri * s.mz;
    s.NB = (s.Bx * s.Bx + s.By * s.By) + s.Bz * s.Bz;
    s.p = kG1 * (((s.E - 0.5 * s.rho * ((s.u * s.u + s.v * s.v) + s.w * s.w)) - s.NB * 0.5) - 0.5 * (s.psi * s.psi));
    s.pt = s.p + 0.5 * s.NB;
    s.Vn = s.u * ux + s.v * uy;
    s.Bn = s.Bx * ux + s.By * uy;
    s.ub = (s.u * s.Bx + s.v * s.By) + s.w * s.Bz;
}

// adjoint of one side's normal flux Fn (a: adjoint of Fn, 9) plus the
// adjoints that reach the side from the wave speed (Vnb, pgb) and the
// averaged field (Bb) and density (rb), and from the face velocity maximum
// (ubx: adjoint of u, v, w); adds the conserved-variable adjoint to qb
SDDC_HD void rus_side_vjp(const RusSide &s, double c, double ux, double uy, const double *a, double Vnb, double pgb,
                          const double *Bb, double rb, const double *uvwb, double *qb)
{
    Vnb += a[0] * s.rho + a[1] * s.mx + a[2] * s.my + a[3] * s.mz + a[4] * ((s.E - 0.5 * (s.psi * s.psi)) + s.pt) +
           a[7] * s.Bz;
    const double Bnb = -a[1] * s.Bx - a[2] * s.By - a[3] * s.Bz - a[4] * s.ub + a[4] * c * s.psi - a[7] * s.w + a[8] * c;
    const double ptb = a[1] * ux + a[2] * uy + a[4] * s.Vn;
    const double ubb = -a[4] * s.Bn;
    double rhob = a[0] * s.Vn + rb;
    double mxb = a[1] * s.Vn, myb = a[2] * s.Vn, mzb = a[3] * s.Vn;
    double Eb = a[4] * s.Vn;
    double psib = -a[4] * s.psi * s.Vn + a[4] * c * s.Bn + a[5] * c * ux + a[6] * c * uy;
    double Bxb = -a[1] * s.Bn + a[5] * s.v * uy - a[6] * s.v * ux + Bb[0];
    double Byb = -a[2] * s.Bn - a[5] * s.u * uy + a[6] * s.u * ux + Bb[1];
    double Bzb = -a[3] * s.Bn + a[7] * s.Vn + Bb[2];
    double ub = -a[5] * s.By * uy + a[6] * s.By * ux + uvwb[0];
    double vb = a[5] * s.Bx * uy - a[6] * s.Bx * ux + uvwb[1];
    double wb = -a[7] * s.Bn + uvwb[2];
    // Vn = u ux + v uy, Bn = Bx ux + By uy, ub = u.B
    ub += Vnb * ux + ubb * s.Bx;
    vb += Vnb * uy + ubb * s.By;
    wb += ubb * s.Bz;
    Bxb += Bnb * ux + ubb * s.u;
    Byb += Bnb * uy + ubb * s.v;
    Bzb += ubb * s.w;
    // pt = p + |B|^2/2 and pg = pt - |B|^2/2 (= p): the field terms cancel
    // for the wave speed's pg
    const double pb = ptb + pgb;
    Bxb += ptb * s.Bx;
    Byb += ptb * s.By;
    Bzb += ptb * s.Bz;
    // p = (gam-1) (E - rho |u|^2 / 2 - |B|^2 / 2 - psi^2 / 2)
    Eb += kG1 * pb;
    rhob -= kG1 * 0.5 * ((s.u * s.u + s.v * s.v) + s.w * s.w) * pb;
    ub -= kG1 * s.rho * s.u * pb;
    vb -= kG1 * s.rho * s.v * pb;
    wb -= kG1 * s.rho * s.w * pb;
    Bxb -= kG1 * s.Bx * pb;
    Byb -= kG1 * s.By * pb;
    Bzb -= kG1 * s.Bz * pb;
    psib -= kG1 * s.psi * pb;
    // u = mx / rho
    qb[0] += rhob - (ub * s.u + vb * s.v + wb * s.w) * s.ri;
    qb[1] += mxb + ub * s.ri;
    qb[2] += myb + vb * s.ri;
    qb[3] += mzb + wb * s.ri;
    qb[4] += Eb;
    qb[5] += Bxb;
    qb[6] += Byb;
    qb[7] += Bzb;
    qb[8] += psib;
}

// Adjoint of the Rusanov flux f (the left cell's computational flux; the
// right cell's is sign_l*sign_r*f) with respect to the traces.
// fb: adjoint of f; eb0, umb0: extra adjoints of the wave speed and of the
// face velocity maximum.  qlb, qrb accumulate; either may be null (that
// side's adjoint is not formed).  eig and um return the wave speed and
// velocity maximum; dfdc (nullable) gets d f / d c_h.  Returns
// wc . d f / d c_h (0 when wc is null).
SDDC_HD double rusanov_vjp(const double *Ql, const double *Qr, double n0, double n1, int sign_l, double c,
                           const double *fb, double eb0, double umb0, double *qlb, double *qrb, double &eig,
                           double &um, double *dfdc = nullptr, const double *wc = nullptr)
{
    const double n2 = n0 * n0 + n1 * n1, rm = Rsqrt(n2);
    const double magnorm = n2 * rm;
    const double sm = (double)sign_l * rm;
    const double ux = n0 * sm, uy = n1 * sm;
    // the quantities both sides share
    double Vn_s, pg[2], rho[2], Bh[3], uvw[3], Bn[2];
    for (int sd = 0; sd < 2; sd++) {
        RusSide S;
        rus_side(sd == 0 ? Ql : Qr, ux, uy, S);
        pg[sd] = S.p;
        rho[sd] = S.rho;
        Bn[sd] = S.Bn;
        if (sd == 0) {
            Vn_s = S.Vn;
            Bh[0] = S.Bx; Bh[1] = S.By; Bh[2] = S.Bz;
            uvw[0] = S.u; uvw[1] = S.v; uvw[2] = S.w;
        } else {
            Vn_s += S.Vn;
            Bh[0] = 0.5 * (Bh[0] + S.Bx); Bh[1] = 0.5 * (Bh[1] + S.By); Bh[2] = 0.5 * (Bh[2] + S.Bz);
            uvw[0] += S.u; uvw[1] += S.v; uvw[2] += S.w;
        }
    }
    const double K = 0.5 * magnorm * (double)sign_l;
    if (dfdc) {
        const double ps = Ql[8] + Qr[8];
        for (int k = 0; k < 9; k++) dfdc[k] = 0.0;
        dfdc[4] = K * (Ql[8] * Bn[0] + Qr[8] * Bn[1]);
        dfdc[5] = K * ps * ux;
        dfdc[6] = K * ps * uy;
        dfdc[8] = K * (Bn[0] + Bn[1]);
    }
    const double wdc = wc ? K * (wc[4] * (Ql[8] * Bn[0] + Qr[8] * Bn[1]) + (wc[5] * ux + wc[6] * uy) * (Ql[8] + Qr[8]) +
                                 wc[8] * (Bn[0] + Bn[1]))
                          : 0.0;
    const double bn = Bh[0] * ux + Bh[1] * uy;
    const double S = rho[0] + rho[1], iS = 1.0 / S;
    const double ca = kGam * (pg[0] + pg[1]) * iS;
    const double cd = 2.0 * ((Bh[0] * Bh[0] + Bh[1] * Bh[1]) + Bh[2] * Bh[2]) * iS;
    const double cn = 2.0 * bn * bn * iS;
    const double cad = ca + cd;
    // ct = sqrt(disc) and cf = sqrt(xf) through their reciprocal square
    // roots, which the adjoint needs as well (ct's slope is taken as 0 at
    // disc = 0)
    const double disc = cad * cad - 4.0 * ca * cn;
    const double rct = disc > 0.0 ? Rsqrt(disc) : 0.0;
    const double ct = disc > 0.0 ? disc * rct : Sqrt(disc);
    const double xf = 0.5 * (cad + ct), rcf = Rsqrt(xf);
    const double cf = xf * rcf;
    eig = 0.5 * Abs(Vn_s) + cf;
    const double xu = 0.5 * Abs(uvw[0]), xv = 0.5 * Abs(uvw[1]), xw = 0.5 * Abs(uvw[2]);
    const double m1 = Max(xu, xv);
    um = Max(m1, xw);
    const int usel = (m1 > xw) ? (xu > xv ? 0 : 1) : 2;

    // f_k = K ((Fnl_k + Fnr_k) - eig (Qr_k - Ql_k)), K = |n| sign_l / 2
    double ebar = eb0;
    for (int k = 0; k < 9; k++) ebar -= K * fb[k] * (Qr[k] - Ql[k]);
    // eig = |Vnl + Vnr| / 2 + cf
    const double Vnb = 0.5 * sgn1(Vn_s) * ebar;
    const double q4 = 0.25 * ebar * rcf;  // d eig / d cad = d eig / d ct
    const double Db = 0.5 * q4 * rct;
    const double cadb = q4 + 2.0 * cad * Db;
    const double cab = -4.0 * cn * Db + cadb;
    const double cnb = -4.0 * ca * Db;
    const double cdb = cadb;
    const double pgb = cab * kGam * iS;
    const double Sb = -(cab * ca + cdb * cd + cnb * cn) * iS;
    const double bnb = 4.0 * cnb * bn * iS;
    const double c4 = 2.0 * cdb * iS;  // half of d cd / d Bh
    const double Bhalf[3] = {c4 * Bh[0] + 0.5 * bnb * ux, c4 * Bh[1] + 0.5 * bnb * uy, c4 * Bh[2]};
    // face velocity maximum: max over (|ul+ur|, |vl+vr|, |wl+wr|) / 2
    double uvwb[3] = {0.0, 0.0, 0.0};
    uvwb[usel] = 0.5 * sgn1(uvw[usel]) * umb0;
    double g[9];
    for (int k = 0; k < 9; k++) g[k] = K * fb[k];
    for (int sd = 0; sd < 2; sd++) {
        double *qb = sd == 0 ? qlb : qrb;
        if (!qb) continue;
        const double *Q = sd == 0 ? Ql : Qr;
        const double sg = sd == 0 ? eig : -eig;
        for (int k = 0; k < 9; k++) qb[k] += sg * g[k];
        RusSide Sd;
        rus_side(Q, ux, uy, Sd);
        rus_side_vjp(Sd, c, ux, uy, g, Vnb, pgb, Bhalf, Sb, uvwb, qb);
    }
    return wdc;
}

// w . d f / d c_h of the Rusanov flux (f's c_h terms: k = 4, 5, 6, 8)
SDDC_HD double rusanov_wdfdc(const double *Ql, const double *Qr, double n0, double n1, int sign_l, const double *w)
{
    const double magnorm = Sqrt(n0 * n0 + n1 * n1);
    const double sm = (double)sign_l / magnorm;
    const double ux = n0 * sm, uy = n1 * sm;
    const double Bnl = Ql[5] * ux + Ql[6] * uy, Bnr = Qr[5] * ux + Qr[6] * uy;
    const double K = 0.5 * magnorm * (double)sign_l;
    return K * (w[4] * (Ql[8] * Bnl + Qr[8] * Bnr) + (w[5] * ux + w[6] * uy) * (Ql[8] + Qr[8]) + w[8] * (Bnl + Bnr));
}

// d (n0 F_k + n1 G_k) / d c_h at an interior flux point
SDDC_HD void iflux_dfdc(const double *Q, double n0, double n1, double *d)
{
    for (int k = 0; k < 9; k++) d[k] = 0.0;
    d[4] = Q[8] * (Q[5] * n0 + Q[6] * n1);
    d[5] = Q[8] * n0;
    d[6] = Q[8] * n1;
    d[8] = Q[5] * n0 + Q[6] * n1;
}

// Adjoint of the boundary ghost state Qr = ghost(Ql, free stream).
// qrb: adjoint of Qr; qlb += (dQr/dQl)^T qrb; pb (rinf, pinf, uinf, vinf,
// bxinf, byinf) += (dQr/dfs)^T qrb.
SDDC_HD void bc_ghost_vjp(int kind, const double *Ql, double n0, double n1, int vismode, const Freestream &fs,
                          const double *qrb, double *qlb, double *pb)
{
    if (kind == kFaceInle) {
        const double rr = fs.rinf, ur = fs.uinf, vr = fs.vinf;
        qlb[8] += qrb[8] + qrb[4] * Ql[8];
        pb[0] += qrb[0] + qrb[1] * ur + qrb[2] * vr + qrb[4] * 0.5 * (ur * ur + vr * vr);
        pb[2] += qrb[1] * rr + qrb[4] * rr * ur;
        pb[3] += qrb[2] * rr + qrb[4] * rr * vr;
        pb[1] += qrb[4] / kG1;
        pb[4] += qrb[5] + qrb[4] * fs.bxinf;
        pb[5] += qrb[6] + qrb[4] * fs.byinf;
    } else if (kind == kFaceOutl) {
        const double rl = Ql[0], ur = Ql[1] / rl, vr = Ql[2] / rl;
        const double rrb = qrb[0] + qrb[1] * ur + qrb[2] * vr + qrb[4] * 0.5 * (ur * ur + vr * vr);
        const double urb = qrb[1] * rl + qrb[4] * rl * ur;
        const double vrb = qrb[2] * rl + qrb[4] * rl * vr;
        qlb[0] += rrb - (urb * ur + vrb * vr) / rl;
        qlb[1] += urb / rl;
        qlb[2] += vrb / rl;
        qlb[8] += qrb[4] * Ql[8];
        pb[1] += qrb[4] / kG1;
        pb[4] += qrb[5] + qrb[4] * fs.bxinf;
        pb[5] += qrb[6] + qrb[4] * fs.byinf;
    } else if (kind == kFaceWall) {
        qlb[0] += qrb[0];
        qlb[4] += qrb[4];
        qlb[5] -= qrb[5];
        qlb[6] -= qrb[6];
        qlb[7] -= qrb[7];
        qlb[8] += qrb[8];
        qlb[3] -= qrb[3];
        if (vismode == 0) {  // slip: reflected normal momentum
            const double m = Sqrt(n0 * n0 + n1 * n1);
            const double h0 = n0 / m, h1 = n1 / m;
            qlb[1] += qrb[1] * (1.0 - 2.0 * h0 * h0) - 2.0 * h0 * h1 * qrb[2];
            qlb[2] += -2.0 * h0 * h1 * qrb[1] + (1.0 - 2.0 * h1 * h1) * qrb[2];
        } else {  // no-slip: momentum negated
            qlb[1] -= qrb[1];
            qlb[2] -= qrb[2];
        }
    } else if (kind == kFaceSymp) {
        const double rl = Ql[0];
        const double uw = Ql[1] / rl, vw = Ql[2] / rl, ww = Ql[3] / rl;
        const double rr = fs.rinf * 2.0 - rl;
        const double m = Sqrt(n0 * n0 + n1 * n1);
        const double h0 = n0 / m, h1 = n1 / m;
        const double VN = uw * h0 + vw * h1;
        const double uh = uw - 2.0 * VN * h0, vh = vw - 2.0 * VN * h1, wh = -ww;
        const double Q1 = rr * uh, Q2 = rr * vh, Q3 = rr * wh;
        const double Q1b = qrb[1] + qrb[4] * Q1 / rr;
        const double Q2b = qrb[2] + qrb[4] * Q2 / rr;
        const double Q3b = qrb[3] + qrb[4] * Q3 / rr;
        const double rrb = qrb[0] - qrb[4] * 0.5 * ((Q1 * Q1 + Q2 * Q2) + Q3 * Q3) / (rr * rr) + Q1b * uh + Q2b * vh +
                           Q3b * wh;
        const double uhb = rr * Q1b, vhb = rr * Q2b, whb = rr * Q3b;
        const double VNb = -2.0 * (uhb * h0 + vhb * h1);
        const double uwb = uhb + VNb * h0, vwb = vhb + VNb * h1, wwb = -whb;
        qlb[1] += uwb / rl;
        qlb[2] += vwb / rl;
        qlb[3] += wwb / rl;
        qlb[0] += -(uwb * uw + vwb * vw + wwb * ww) / rl - rrb;
        qlb[7] += -qrb[7] + qrb[4] * Ql[7];
        qlb[8] += qrb[8] + qrb[4] * Ql[8];
        pb[0] += 2.0 * rrb;
        pb[1] += qrb[4] / kG1;
        pb[4] += qrb[5] + qrb[4] * fs.bxinf;
        pb[5] += qrb[6] + qrb[4] * fs.byinf;
    } else {  // FREE: copy
        for (int k = 0; k < 9; k++) qlb[k] += qrb[k];
    }
}

}  // namespace sddc
