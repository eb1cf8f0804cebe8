// Point physics of the SDDC residual on the device: physical MHD flux with
// GLM terms, the Rusanov face flux and the boundary ghost states.
//
// Template parameter R is the arithmetic type of the flux work (double for
// the FP64 forms, float for the mixed form).  EX selects the exact form: the
// reference's own expressions, operation by operation and in the same
// left-to-right order, to be compiled without FMA contraction (-fmad=false)
// so the results round exactly as the reference's FP64 code does.  The
// non-exact forms use reciprocals and contraction; in the mixed form the
// pressure is still recovered from the total energy in FP64.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sddc {

constexpr double kGam = 5.0 / 3.0;  // gam, setup2d.f90:67

#define SDDC_HD __host__ __device__ __forceinline__

// overloads per arithmetic type (a test's dual-number type adds its own)
SDDC_HD double Sqrt(double x) { return sqrt(x); }
SDDC_HD float Sqrt(float x) { return sqrtf(x); }
SDDC_HD double Abs(double x) { return fabs(x); }
SDDC_HD float Abs(float x) { return fabsf(x); }
template <typename R> SDDC_HD R Max(R a, R b) { return a > b ? a : b; }

struct Freestream {
    double rinf, pinf, uinf, vinf, bxinf, byinf;
};

// gas pressure from a conserved state; in the mixed form the subtraction is
// done in FP64, where the cancellation of E against the kinetic, magnetic and
// psi energies (low plasma beta) costs no digits beyond the inputs'.
template <typename R>
SDDC_HD R pressure_fast(const R *q, R rinv)
{
    const double rho_i = (double)rinv;
    const double m2 = (double)q[1] * q[1] + (double)q[2] * q[2] + (double)q[3] * q[3];
    const double b2 = (double)q[5] * q[5] + (double)q[6] * q[6] + (double)q[7] * q[7];
    const double ps = (double)q[8] * q[8];
    return (R)((kGam - 1.0) * ((double)q[4] - 0.5 * m2 * rho_i - 0.5 * b2 - 0.5 * ps));
}

// getIfluxvectors, getrusanov.f90:127-193: F and G at one flux point,
// and the running max of |u|,|v|,|w|.
template <typename R, bool EX>
SDDC_HD void iflux(const R *Q, R c_h, R &umax, R *F, R *G)
{
    const R rho = Q[0], rhou = Q[1], rhov = Q[2], rhow = Q[3], rhoE = Q[4];
    const R Bx = Q[5], By = Q[6], Bz = Q[7], psi = Q[8];
    const R NORM_B = (Bx * Bx + By * By) + Bz * Bz;
    if constexpr (EX) {
        const R pr = (R)(kGam - 1.0) *
                     (((rhoE - (R)0.5 * ((rhou * rhou + rhov * rhov) + rhow * rhow) / rho) - (R)0.5 * NORM_B) -
                      (R)0.5 * (psi * psi));
        F[0] = rhou;
        F[1] = ((rhou * rhou) / rho + pr) + ((R)0.5 * NORM_B - Bx * Bx);
        F[2] = rhou * rhov / rho - Bx * By;
        F[3] = rhou * rhow / rho - Bx * Bz;
        const R ub = (rhou / rho * Bx + rhov / rho * By) + rhow / rho * Bz;
        const R eb = ((rhoE - (R)0.5 * (psi * psi)) + pr) + (R)0.5 * NORM_B;
        F[4] = (rhou / rho) * eb - ub * Bx;
        F[5] = (R)0;
        F[6] = rhou / rho * By - rhov / rho * Bx;
        F[7] = rhou / rho * Bz - rhow / rho * Bx;
        G[0] = rhov;
        G[1] = rhou * rhov / rho - Bx * By;
        G[2] = ((rhov * rhov) / rho + pr) + ((R)0.5 * NORM_B - By * By);
        G[3] = rhow * rhov / rho - By * Bz;
        G[4] = (rhov / rho) * eb - ub * By;
        G[5] = rhov / rho * Bx - rhou / rho * By;
        G[6] = (R)0;
        G[7] = rhov / rho * Bz - rhow / rho * By;
        F[4] = F[4] + c_h * psi * Bx;
        G[4] = G[4] + c_h * psi * By;
        F[5] = F[5] + c_h * psi;
        G[6] = G[6] + c_h * psi;
        F[8] = c_h * Bx;
        G[8] = c_h * By;
        const R u = rhou / rho, v = rhov / rho, w = rhow / rho;
        const R um = Max(Max(Abs(u), Abs(v)), Abs(w));
        if (um > umax) umax = um;
    } else {
        const R ri = (R)1 / rho;
        const R u = rhou * ri, v = rhov * ri, w = rhow * ri;
        const R pr = pressure_fast<R>(Q, ri);
        const R ub = u * Bx + v * By + w * Bz;
        const R eb = rhoE - (R)0.5 * psi * psi + pr + (R)0.5 * NORM_B;
        const R cp = c_h * psi;
        F[0] = rhou;
        F[1] = rhou * u + pr + ((R)0.5 * NORM_B - Bx * Bx);
        F[2] = rhou * v - Bx * By;
        F[3] = rhou * w - Bx * Bz;
        F[4] = u * eb - ub * Bx + cp * Bx;
        F[5] = cp;
        F[6] = u * By - v * Bx;
        F[7] = u * Bz - w * Bx;
        F[8] = c_h * Bx;
        G[0] = rhov;
        G[1] = F[2];
        G[2] = rhov * v + pr + ((R)0.5 * NORM_B - By * By);
        G[3] = rhov * w - By * Bz;
        G[4] = v * eb - ub * By + cp * By;
        G[5] = -F[6];
        G[6] = cp;
        G[7] = v * Bz - w * By;
        G[8] = c_h * By;
        const R um = Max(Max(Abs(u), Abs(v)), Abs(w));
        if (um > umax) umax = um;
    }
}

// F n0 + G n1 at one flux point, formed directly along (n0, n1) (the FP64
// and mixed forms; the exact form projects iflux's F and G as the reference
// does): the same flux, associated differently; updates the running max of
// |u|,|v|,|w|
template <typename R>
SDDC_HD void iflux_n(const R *Q, R c_h, R n0, R n1, R &umax, R *Fn)
{
    const R rho = Q[0], rhou = Q[1], rhov = Q[2], rhow = Q[3], rhoE = Q[4];
    const R Bx = Q[5], By = Q[6], Bz = Q[7], psi = Q[8];
    const R ri = (R)1 / rho;
    const R u = rhou * ri, v = rhov * ri, w = rhow * ri;
    const R pr = pressure_fast<R>(Q, ri);
    const R NORM_B = Bx * Bx + By * By + Bz * Bz;
    const R un = u * n0 + v * n1, bn = Bx * n0 + By * n1;
    const R pt = pr + (R)0.5 * NORM_B;
    const R ub = u * Bx + v * By + w * Bz;
    const R eb = rhoE - (R)0.5 * psi * psi + pt;
    const R cp = c_h * psi;
    Fn[0] = rhou * n0 + rhov * n1;
    Fn[1] = rhou * un + pt * n0 - Bx * bn;
    Fn[2] = rhov * un + pt * n1 - By * bn;
    Fn[3] = rhow * un - Bz * bn;
    Fn[4] = un * eb - (ub - cp) * bn;
    Fn[5] = Bx * un - u * bn + cp * n0;
    Fn[6] = By * un - v * bn + cp * n1;
    Fn[7] = Bz * un - w * bn;
    Fn[8] = c_h * bn;
    const R um = Max(Max(Abs(u), Abs(v)), Abs(w));
    if (um > umax) umax = um;
}

// getrusanovflux, getrusanov.f90:1-125.  Returns the left cell's
// computational flux in Fnl, the right cell's in Fnr and the wave speed in
// eigv; updates the running max of the face-averaged velocity.
template <typename R, bool EX>
SDDC_HD void rusanov(const R *Qfl, const R *Qfr, R *Fnl, R *Fnr, R n0, R n1, int sign_l,
                                        int sign_r, R c_h, R &eigv_out, R &umax)
{
    const R magnorm = Sqrt(n0 * n0 + n1 * n1);
    R unit_x, unit_y, ul, vl, wl, ur, vr, wr, pl, pr;
    const R Bxl = Qfl[5], Byl = Qfl[6], Bzl = Qfl[7], psil = Qfl[8];
    const R Bxr = Qfr[5], Byr = Qfr[6], Bzr = Qfr[7], psir = Qfr[8];
    const R NORM_Bl = (Bxl * Bxl + Byl * Byl) + Bzl * Bzl;
    const R NORM_Br = (Bxr * Bxr + Byr * Byr) + Bzr * Bzr;
    if constexpr (EX) {
        unit_x = n0 / magnorm * (R)sign_l;
        unit_y = n1 / magnorm * (R)sign_l;
        R rhoi = (R)1 / Qfl[0];
        ul = rhoi * Qfl[1]; vl = rhoi * Qfl[2]; wl = rhoi * Qfl[3];
        pl = (R)(kGam - 1.0) * (((Qfl[4] - (R)0.5 * Qfl[0] * ((ul * ul + vl * vl) + wl * wl)) - NORM_Bl * (R)0.5) -
                                (R)0.5 * (psil * psil));
        pl = pl + (R)0.5 * NORM_Bl;
        rhoi = (R)1 / Qfr[0];
        ur = rhoi * Qfr[1]; vr = rhoi * Qfr[2]; wr = rhoi * Qfr[3];
        pr = (R)(kGam - 1.0) * (((Qfr[4] - (R)0.5 * Qfr[0] * ((ur * ur + vr * vr) + wr * wr)) - NORM_Br * (R)0.5) -
                                (R)0.5 * (psir * psir));
        pr = pr + NORM_Br * (R)0.5;
    } else {
        const R rm = (R)sign_l / magnorm;
        unit_x = n0 * rm;
        unit_y = n1 * rm;
        const R ril = (R)1 / Qfl[0], rir = (R)1 / Qfr[0];
        ul = ril * Qfl[1]; vl = ril * Qfl[2]; wl = ril * Qfl[3];
        ur = rir * Qfr[1]; vr = rir * Qfr[2]; wr = rir * Qfr[3];
        pl = pressure_fast<R>(Qfl, ril) + (R)0.5 * NORM_Bl;
        pr = pressure_fast<R>(Qfr, rir) + (R)0.5 * NORM_Br;
    }
    const R Vn_l = ul * unit_x + vl * unit_y, Bn_l = Bxl * unit_x + Byl * unit_y;
    const R Vn_r = ur * unit_x + vr * unit_y, Bn_r = Bxr * unit_x + Byr * unit_y;
    // fast magnetosonic speed of the averaged state first, so that each
    // flux component is formed and combined in turn (fewer values live at
    // once); every component's arithmetic is the reference's
    const R pgl = pl - (R)0.5 * NORM_Bl, pgr = pr - (R)0.5 * NORM_Br;
    const R Bx = (R)0.5 * (Bxl + Bxr), By = (R)0.5 * (Byl + Byr), Bz = (R)0.5 * (Bzl + Bzr);
    const R bn = Bx * unit_x + By * unit_y;
    R c_a, c_d, c_n;
    if constexpr (EX) {
        c_a = (R)kGam * (pgl + pgr) / (Qfl[0] + Qfr[0]);
        c_d = ((Bx * Bx + By * By) + Bz * Bz) / ((R)0.5 * (Qfl[0] + Qfr[0]));
        c_n = bn * bn / ((R)0.5 * (Qfl[0] + Qfr[0]));
    } else {
        const R rs = (R)1 / (Qfl[0] + Qfr[0]);
        c_a = (R)kGam * (pgl + pgr) * rs;
        c_d = (R)2 * ((Bx * Bx + By * By) + Bz * Bz) * rs;
        c_n = (R)2 * bn * bn * rs;
    }
    const R cad = c_a + c_d;
    const R c_tmp = Sqrt(cad * cad - (R)4 * c_a * c_n);
    const R c_f = Sqrt((R)0.5 * ((c_a + c_d) + c_tmp));
    const R eigv = (R)0.5 * Abs(Vn_l + Vn_r) + c_f;
    const R sl = magnorm * (R)sign_l;
    const R slr = (R)(sign_l * sign_r);
    auto put = [&](int k, R fl, R fr) {
        R f = (R)0.5 * ((fl + fr) - eigv * (Qfr[k] - Qfl[k]));
        f = sl * f;
        Fnl[k] = f;
        Fnr[k] = slr * f;
    };
    put(0, Qfl[0] * Vn_l, Qfr[0] * Vn_r);
    put(1, (Qfl[1] * Vn_l + pl * unit_x) - Bxl * Bn_l, (Qfr[1] * Vn_r + pr * unit_x) - Bxr * Bn_r);
    put(2, (Qfl[2] * Vn_l + pl * unit_y) - Byl * Bn_l, (Qfr[2] * Vn_r + pr * unit_y) - Byr * Bn_r);
    put(3, Qfl[3] * Vn_l - Bzl * Bn_l, Qfr[3] * Vn_r - Bzr * Bn_r);
    // with the GLM terms (getrusanov.f90:77-89)
    put(4, (((Qfl[4] - (R)0.5 * (psil * psil)) + pl) * Vn_l - Bn_l * ((ul * Bxl + vl * Byl) + wl * Bzl)) +
               c_h * psil * Bn_l,
        (((Qfr[4] - (R)0.5 * (psir * psir)) + pr) * Vn_r - Bn_r * ((ur * Bxr + vr * Byr) + wr * Bzr)) +
            c_h * psir * Bn_r);
    put(5, (vl * Bxl - ul * Byl) * unit_y + c_h * psil * unit_x, (vr * Bxr - ur * Byr) * unit_y + c_h * psir * unit_x);
    put(6, (ul * Byl - vl * Bxl) * unit_x + c_h * psil * unit_y, (ur * Byr - vr * Bxr) * unit_x + c_h * psir * unit_y);
    put(7, Bzl * Vn_l - wl * Bn_l, Bzr * Vn_r - wr * Bn_r);
    put(8, c_h * Bn_l, c_h * Bn_r);
    eigv_out = eigv;
    const R um = Max(Max((R)0.5 * Abs(ul + ur), (R)0.5 * Abs(vl + vr)), (R)0.5 * Abs(wl + wr));
    if (um > umax) umax = um;
}

// face kinds of the per-(cell, local face) connectivity records
enum FaceKind : int {
    kFaceNone = 0,
    kFaceLeft = 1,   // shared face, this cell is the left cell
    kFaceRight = 2,  // shared face, this cell is the right cell
    kFaceInle = 3,
    kFaceOutl = 4,
    kFaceWall = 5,
    kFaceSymp = 6,
    kFaceFree = 7,
    // processor face of a decomposed run (PROCINTFLUX / CYCREMFLUX): the
    // other cell is on another rank; the record's partner field is the
    // face's slot in the exchange buffers
    kFaceProc = 8
};

// Boundary ghost states of BCFLUX (bcflux.f90:17-375).
template <typename R, bool EX>
SDDC_HD void bc_ghost(int kind, const R *Qfl, R n0, R n1, int vismode, const Freestream &fs,
                                         R *Qfr)
{
    const R gm1 = (R)(kGam - 1.0);
    if (kind == kFaceInle || kind == kFaceOutl) {
        R rhor, ur, vr;
        if (kind == kFaceInle) {
            rhor = (R)fs.rinf; ur = (R)fs.uinf; vr = (R)fs.vinf;
        } else {
            rhor = Qfl[0]; ur = Qfl[1] / Qfl[0]; vr = Qfl[2] / Qfl[0];
        }
        const R wr = (R)0, Bxr = (R)fs.bxinf, Byr = (R)fs.byinf, Bzr = (R)0;
        Qfr[0] = rhor;
        Qfr[1] = rhor * ur;
        Qfr[2] = rhor * vr;
        Qfr[3] = rhor * wr;
        Qfr[4] = (((R)fs.pinf / gm1 + (R)0.5 * rhor * ((ur * ur + vr * vr) + wr * wr)) +
                  (R)0.5 * ((Bxr * Bxr + Byr * Byr) + Bzr * Bzr)) +
                 (R)0.5 * (Qfl[8] * Qfl[8]);
        Qfr[5] = Bxr;
        Qfr[6] = Byr;
        Qfr[7] = Bzr;
        Qfr[8] = kind == kFaceInle ? Qfl[8] : (R)0;
    } else if (kind == kFaceWall) {
        const R rhow = Qfl[0];
        const R uw = Qfl[1] / rhow, vw = Qfl[2] / rhow, ww = Qfl[3] / rhow;
        Qfr[0] = rhow;
        Qfr[4] = Qfl[4];
        Qfr[5] = -Qfl[5];
        Qfr[6] = -Qfl[6];
        Qfr[7] = -Qfl[7];
        Qfr[8] = Qfl[8];
        if (vismode == 0) {
            const R magnorm = Sqrt(n0 * n0 + n1 * n1);
            const R VN = uw * n0 / magnorm + vw * n1 / magnorm;
            Qfr[1] = rhow * (uw - (R)2 * VN * n0 / magnorm);
            Qfr[2] = rhow * (vw - (R)2 * VN * n1 / magnorm);
            Qfr[3] = -rhow * ww;
        } else {
            Qfr[1] = -rhow * uw;
            Qfr[2] = -rhow * vw;
            Qfr[3] = -rhow * ww;
        }
    } else if (kind == kFaceSymp) {
        const R rhow = Qfl[0];
        const R uw = Qfl[1] / rhow, vw = Qfl[2] / rhow, ww = Qfl[3] / rhow;
        Qfr[0] = (R)fs.rinf * (R)2 - Qfl[0];
        const R magnorm = Sqrt(n0 * n0 + n1 * n1);
        const R VN = uw * n0 / magnorm + vw * n1 / magnorm;
        Qfr[1] = Qfr[0] * (uw - (R)2 * VN * n0 / magnorm);
        Qfr[2] = Qfr[0] * (vw - (R)2 * VN * n1 / magnorm);
        Qfr[3] = -Qfr[0] * ww;
        Qfr[5] = (R)fs.bxinf;
        Qfr[6] = (R)fs.byinf;
        Qfr[7] = -Qfl[7];
        Qfr[8] = Qfl[8];
        Qfr[4] = ((R)fs.pinf / gm1 + (R)0.5 / Qfr[0] * ((Qfr[1] * Qfr[1] + Qfr[2] * Qfr[2]) + Qfr[3] * Qfr[3])) +
                 (R)0.5 * (((Qfr[5] * Qfr[5] + Qfr[6] * Qfr[6]) + Qfr[7] * Qfr[7]) + Qfr[8] * Qfr[8]);
    } else {  // FREE
#pragma unroll
        for (int k = 0; k < 9; k++) Qfr[k] = Qfl[k];
    }
}

// running max of a non-negative double through its bit pattern (the order
// of non-negative IEEE doubles is the order of their bit patterns); NaN and
// non-positive values never raise a running max (as `x > max` in the
// reference).
__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v)
{
    if (v > 0.0) atomicMax(reinterpret_cast<unsigned long long *>(addr), (unsigned long long)__double_as_longlong(v));
}

}  // namespace sddc
