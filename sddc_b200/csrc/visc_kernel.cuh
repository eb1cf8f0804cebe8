// The viscous / resistive chain of the SDDC residual (vismode = 1 with
// mu or eta0 nonzero): compflux.f90:36-50 and what it calls.
//
// Two launches before each stage launch, both per tile of cells staged in
// shared memory:
//   visc_grad_kernel  face-averaged states at every flux point (interior:
//                     the interpolated state; faces: (left + right)/2 with
//                     the neighbour's trace or the boundary ghost state, as
//                     interfaceflux/BCFLUX store Qvfi/Qvfj), the gradient of
//                     all nine variables at the solution points (nablaQsp,
//                     compflux.f90:107-157), and its trace at the 4N face
//                     points, published for the neighbours;
//   visc_flux_kernel  the gradient at every flux point (interior:
//                     nablaQ_interior_FP, compflux.f90:159-196; faces: the
//                     average of both cells' traces, interfaceVISflux /
//                     CYCLOCVISFLUX, or the boundary state of BCVISFLUX with
//                     the adiabatic-wall energy gradient, bcflux.f90:380-666,
//                     which needs the internal-energy gradient of
//                     comp_grad_internal_energy, compflux.f90:260-298), the
//                     viscous flux there (getVfluxvectors, getrusanov.f90:
//                     197-294; comp_viscous_flux, compflux.f90:198-258) and
//                     its divergence dFv + dGv (compresid.f90:14-32), which
//                     the stage kernel adds to the inviscid residual.
// The AV viscous flux (getVfluxvectors_AV) has its coefficients hard-coded
// to zero (getrusanov.f90:326,328); it is not formed (it could only change
// the sign of a zero).  Every expression keeps the reference's order; the
// exact instantiation is compiled without FMA.
#pragma once

#include "stage_kernel.cuh"

namespace sddc {

constexpr double kLambdaVisc = -2.0 / 3.0;  // LAMBDA, setup2d.f90:69
constexpr double kPrandtl = 0.72;           // PRANDT, setup2d.f90:70

struct ViscArgs {
    int ncell, vismode;
    double mu, eta0;
    Freestream fs;
    const double *__restrict__ q;     // stage input state
    const void *t_in;                 // its face traces (layout trace_at), in the form's type
    const double *__restrict__ met;   // packed metrics
    const double *__restrict__ met2;  // [cell][lf][nfp][2]: S1(2,1:2) or S2(1,1:2) at the face point
    const int2 *__restrict__ faces;
    double *grad;  // nablaQs (9,2,N,N,NCELL)
    double *gt;    // gradient traces [cell][lf][nfp][18]: (9 x-derivatives, 9 y-derivatives)
    double *rv;    // dFv + dGv (9,N,N,NCELL)
};

constexpr int kViscCpb = 4;
constexpr int kViscThreads = 128;

// getVfluxvectors (getrusanov.f90:197-294) with viscosity mu and resistivity
// eta0; nQ = (9 x-derivatives, 9 y-derivatives)
__device__ __forceinline__ void vflux(const double *Qv, const double *nQ, double mu, double eta0, double *Fv,
                                      double *Gv)
{
    const double rho = Qv[0], rhou = Qv[1], rhov = Qv[2], rhow = Qv[3], rhoE = Qv[4];
    const double Bx = Qv[5], By = Qv[6], Bz = Qv[7], psi = Qv[8];
    const double u = rhou / rho, v = rhov / rho, w = rhow / rho;
    const double NORM_U = (u * u + v * v) + w * w;
    const double NORM_B = (Bx * Bx + By * By) + Bz * Bz;
    const double inte = (((rhoE - 0.5 * NORM_U * rho) - 0.5 * NORM_B) - 0.5 * (psi * psi)) / rho;
    double du[2], dv[2], dw[2], de[2], dBx[2], dBy[2], dBz[2];
#pragma unroll
    for (int d = 0; d < 2; d++) {
        const double *g = nQ + 9 * d;
        const double drho = g[0];
        du[d] = (g[1] - drho * u) / rho;
        dv[d] = (g[2] - drho * v) / rho;
        dw[d] = (g[3] - drho * w) / rho;
        dBx[d] = g[5];
        dBy[d] = g[6];
        dBz[d] = g[7];
        const double dpsi = g[8];
        const double dKE = 0.5 * NORM_U * drho + rho * ((u * du[d] + v * dv[d]) + w * dw[d]);
        const double dpre_B = (Bx * dBx[d] + By * dBy[d]) + Bz * dBz[d];
        const double dpsi2 = psi * dpsi;
        de[d] = ((((g[4] - dKE) - dpre_B) - drho * inte) - dpsi2) / rho;
    }
    const double ux = du[0], uy = du[1], vx = dv[0], vy = dv[1], wx = dw[0], wy = dw[1], ex = de[0], ey = de[1];
    const double Bxy = dBx[1], Byx = dBy[0], Bzx = dBz[0], Bzy = dBz[1];
    Fv[0] = 0.0;
    Fv[1] = mu * (2.0 * ux + kLambdaVisc * (ux + vy));
    Fv[2] = mu * (vx + uy);
    Fv[3] = mu * wx;
    Fv[4] = ((u * Fv[1] + v * Fv[2]) + w * Fv[3]) + mu * kGam * ex / kPrandtl;
    Gv[0] = 0.0;
    Gv[1] = mu * (vx + uy);
    Gv[2] = mu * (2.0 * vy + kLambdaVisc * (ux + vy));
    Gv[3] = mu * wy;
    Gv[4] = ((Gv[1] * u + Gv[2] * v) + Gv[3] * w) + mu * kGam * ey / kPrandtl;
    const double Jx = Bzy - 0.0, Jy = 0.0 - Bzx, Jz = Byx - Bxy;
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

// internal energy at a face-averaged state (compflux.f90:272-277)
__device__ __forceinline__ double enei_of(const double *q)
{
    const double a = q[1] / q[0], b = q[2] / q[0], c = q[3] / q[0];
    return (((q[4] / q[0] - 0.5 * (a * a)) - 0.5 * (b * b)) - 0.5 * (c * c)) -
           0.5 * (((q[5] * q[5] + q[6] * q[6]) + q[7] * q[7]) + q[8] * q[8]) / q[0];
}

template <int N> struct ViscSmem {
    static constexpr int NQ = 9 * N * N, NP = N + 1, NN = N * N;
    static constexpr int kF = 2 * N * NP * 9;   // a state or flux at every flux point
    static constexpr int kG = 2 * N * NP * 18;  // a gradient at every flux point
    static constexpr int NM = 2 * MetLayout<N>::kFam;
};

// the staging both kernels share: the state, Jac, the normals, the
// operators, and the face-averaged state at every flux point (in sV)
template <int N, typename T>
__device__ __forceinline__ void visc_stage_states(const ViscArgs &a, const Ops &ops, int c0, int ncl, double *sQ,
                                                  double *sJac, double *sNrm, double *sL, double *sM, double *sV)
{
    using ML = MetLayout<N>;
    using S = ViscSmem<N>;
    constexpr int NQ = S::NQ, NP = S::NP, NN = S::NN, NM = S::NM, kF = S::kF;
    const int tid = threadIdx.x;
    for (int k = tid; k < NP * N; k += kViscThreads) {
        sL[k] = ops.L[k];
        sM[k] = ops.M[k];
    }
    for (int k = tid; k < ncl * NQ; k += kViscThreads) sQ[k] = __ldg(a.q + (size_t)c0 * NQ + k);
    for (int k = tid; k < ncl * ML::kSize; k += kViscThreads) {
        const int c = k / ML::kSize, o = k - c * ML::kSize;
        const double v = __ldg(a.met + (size_t)c0 * ML::kSize + k);
        if (o < NM) sNrm[c * NM + o] = v;
        else if (o < NM + NN) sJac[c * NN + (o - NM)] = v;
    }
    __syncthreads();
    // interpolation to every flux point (inviscid_flux_interior's Qf)
    for (int t = tid; t < ncl * 2 * N * 9; t += kViscThreads) {
        const int v = t % 9, l = (t / 9) % N, f = (t / (9 * N)) % 2, c = t / (18 * N);
        const double *q = sQ + c * NQ;
        double qs[N];
#pragma unroll
        for (int s = 0; s < N; s++) qs[s] = f == 0 ? q[v + 9 * (s + N * l)] : q[v + 9 * (l + N * s)];
        double *o = sV + c * kF + (f * N + l) * NP * 9 + v;
#pragma unroll
        for (int r = 0; r < NP; r++) {
            double acc = 0.0;
#pragma unroll
            for (int s = 0; s < N; s++) acc = acc + qs[s] * sL[r * N + s];
            o[r * 9] = acc;
        }
    }
    __syncthreads();
    // face points: (left + right)/2 with the neighbour's trace or the ghost
    for (int t = tid; t < ncl * 4 * N; t += kViscThreads) {
        const int nfp = 1 + t % N, lf = 1 + (t / N) % 4, c = t / (4 * N);
        int fam, line, r;
        face_point<N>(lf, nfp, fam, line, r);
        double *slot = sV + c * kF + ((fam * N + line) * NP + r) * 9;
        double own[9], oth[9];
#pragma unroll
        for (int k = 0; k < 9; k++) own[k] = slot[k];
        const int2 rec = a.faces[(size_t)(c0 + c) * 4 + (lf - 1)];
        const int kind = rec.y & 0xff;
        const bool own_right = kind == kFaceRight;
        if (kind == kFaceLeft || own_right) {
            const int pc = rec.x, plf = (rec.y >> 8) & 0xff;
            const T *tp = reinterpret_cast<const T *>(a.t_in);
#pragma unroll
            for (int k = 0; k < 9; k++) oth[k] = (double)tp[trace_at<N>(pc, plf, N - nfp, k)];
        } else {
            const double *nrm = sNrm + c * NM + ML::normal(fam, line, r);
            bc_ghost<double, true>(kind, own, nrm[0], nrm[1], a.vismode, a.fs, oth);
        }
#pragma unroll
        for (int k = 0; k < 9; k++) slot[k] = own_right ? 0.5 * oth[k] + 0.5 * own[k] : 0.5 * own[k] + 0.5 * oth[k];
    }
    __syncthreads();
}

// ---- gradients at the solution points and their face traces ------------------------
// T: the trace type of the form (EX and T keep the instantiations of the
// translation units apart)
template <int N, bool EX, typename T>
__global__ void __launch_bounds__(kViscThreads) visc_grad_kernel(const ViscArgs a, const Ops ops)
{
    using ML = MetLayout<N>;
    using S = ViscSmem<N>;
    constexpr int NQ = S::NQ, NP = S::NP, NN = S::NN, NM = S::NM, kF = S::kF, CPB = kViscCpb;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sQ = reinterpret_cast<double *>(smem_raw);  // [CPB][NQ]
    double *sV = sQ + CPB * NQ;                         // [CPB][kF] face-averaged states
    double *sG = sV + CPB * kF;                         // [CPB][NN][18] gradients
    double *sJac = sG + CPB * NN * 18;                  // [CPB][NN]
    double *sNrm = sJac + CPB * NN;                     // [CPB][NM]
    double *sL = sNrm + CPB * NM;
    double *sM = sL + NP * N;
    const int tid = threadIdx.x, c0 = blockIdx.x * CPB, ncl = min(CPB, a.ncell - c0);
    visc_stage_states<N, T>(a, ops, c0, ncl, sQ, sJac, sNrm, sL, sM, sV);
    // nablaQsp (compflux.f90:107-157), one thread per (cell, point, variable)
    for (int t = tid; t < ncl * NN * 9; t += kViscThreads) {
        const int v = t % 9, i = (t / 9) % N, j = (t / (9 * N)) % N, c = t / (9 * NN);
        const double *met = sNrm + c * NM;
        const double J = sJac[c * NN + i + N * j];
        const double *Vx = sV + c * kF + (0 * N + j) * NP * 9;
        const double *Vy = sV + c * kF + (1 * N + i) * NP * 9;
        double g[2];
#pragma unroll
        for (int d = 0; d < 2; d++) {
            double aa = 0.0, bb = 0.0;
#pragma unroll
            for (int r = 0; r < NP; r++) aa = aa + Vx[r * 9 + v] * sM[r * N + i] * met[ML::normal(0, j, r) + d];
#pragma unroll
            for (int r = 0; r < NP; r++) bb = bb + Vy[r * 9 + v] * sM[r * N + j] * met[ML::normal(1, i, r) + d];
            g[d] = (aa + bb) / J;
        }
        sG[(c * NN + i + N * j) * 18 + v] = g[0];
        sG[(c * NN + i + N * j) * 18 + 9 + v] = g[1];
        double *go = a.grad + ((size_t)(c0 + c) * NN + i + N * j) * 18;
        go[v] = g[0];
        go[9 + v] = g[1];
    }
    __syncthreads();
    // gradient traces at the face points (grad_trace: the same interpolation)
    for (int t = tid; t < ncl * 4 * N * 18; t += kViscThreads) {
        const int k = t % 18, fpt = (t / 18) % (4 * N), c = t / (72 * N);
        const int nfp = 1 + fpt % N, lf = 1 + fpt / N;
        int fam, line, r;
        face_point<N>(lf, nfp, fam, line, r);
        double acc = 0.0;
#pragma unroll
        for (int s = 0; s < N; s++) {
            const int sp = fam == 0 ? s + N * line : line + N * s;
            acc = acc + sG[(c * NN + sp) * 18 + k] * sL[r * N + s];
        }
        a.gt[((size_t)(c0 + c) * 4 * N + fpt) * 18 + k] = acc;
    }
}

// ---- the viscous flux and its divergence ---------------------------------------------
template <int N, bool EX, typename T>
__global__ void __launch_bounds__(kViscThreads) visc_flux_kernel(const ViscArgs a, const Ops ops)
{
    using ML = MetLayout<N>;
    using S = ViscSmem<N>;
    constexpr int NQ = S::NQ, NP = S::NP, NN = S::NN, NM = S::NM, kF = S::kF, kG = S::kG, CPB = kViscCpb;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sQ = reinterpret_cast<double *>(smem_raw);  // [CPB][NQ]
    double *sV = sQ + CPB * NQ;                         // [CPB][kF] face-averaged states
    double *sFv = sV + CPB * kF;                        // [CPB][kF] viscous flux
    double *sGf = sFv + CPB * kF;                       // [CPB][kG] gradient at the flux points
    double *sG = sGf + CPB * kG;                        // [CPB][NN][18] gradients at the solution points
    double *sDE = sG + CPB * NN * 18;                   // [CPB][NN][2] internal-energy gradient
    double *sJac = sDE + CPB * NN * 2;                  // [CPB][NN]
    double *sNrm = sJac + CPB * NN;                     // [CPB][NM]
    double *sL = sNrm + CPB * NM;
    double *sM = sL + NP * N;
    __shared__ int sWall[CPB];
    const int tid = threadIdx.x, c0 = blockIdx.x * CPB, ncl = min(CPB, a.ncell - c0);
    if (tid < CPB) {
        int w = 0;
        if (tid < ncl)
            for (int lf = 0; lf < 4; lf++) w |= (a.faces[(size_t)(c0 + tid) * 4 + lf].y & 0xff) == kFaceWall;
        sWall[tid] = w;
    }
    for (int k = tid; k < ncl * NN * 18; k += kViscThreads) sG[k] = __ldg(a.grad + (size_t)c0 * NN * 18 + k);
    visc_stage_states<N, T>(a, ops, c0, ncl, sQ, sJac, sNrm, sL, sM, sV);
    // comp_grad_internal_energy (compflux.f90:260-298) for cells with a wall
    // face (the only ones whose values are read)
    for (int t = tid; t < ncl * NN; t += kViscThreads) {
        const int i = t % N, j = (t / N) % N, c = t / NN;
        if (!sWall[c]) continue;
        double x = 0.0, y = 0.0;
#pragma unroll
        for (int r = 0; r < NP; r++) x = x + enei_of(sV + c * kF + ((0 * N + j) * NP + r) * 9) * sM[r * N + i];
#pragma unroll
        for (int r = 0; r < NP; r++) y = y + enei_of(sV + c * kF + ((1 * N + i) * NP + r) * 9) * sM[r * N + j];
        sDE[(c * NN + i + N * j) * 2] = x;
        sDE[(c * NN + i + N * j) * 2 + 1] = y;
    }
    __syncthreads();
    // the gradient at the interior flux points (nablaQ_interior_FP)
    for (int t = tid; t < ncl * 2 * N * (N - 1) * 18; t += kViscThreads) {
        const int k = t % 18, r = 1 + (t / 18) % (N - 1), l = (t / (18 * (N - 1))) % N,
                  f = (t / (18 * (N - 1) * N)) % 2, c = t / (36 * (N - 1) * N);
        double acc = 0.0;
#pragma unroll
        for (int s = 0; s < N; s++) {
            const int sp = f == 0 ? s + N * l : l + N * s;
            acc = acc + sG[(c * NN + sp) * 18 + k] * sL[r * N + s];
        }
        sGf[c * kG + ((f * N + l) * NP + r) * 18 + k] = acc;
    }
    // the gradient at the face points: the average of both sides' traces
    // (interfaceVISflux, CYCLOCVISFLUX) or of the trace and the boundary
    // state (BCVISFLUX)
    for (int t = tid; t < ncl * 4 * N; t += kViscThreads) {
        const int nfp = 1 + t % N, lf = 1 + (t / N) % 4, c = t / (4 * N);
        int fam, line, r;
        face_point<N>(lf, nfp, fam, line, r);
        double g[18], o[18];
#pragma unroll
        for (int k = 0; k < 18; k++) {
            double acc = 0.0;
#pragma unroll
            for (int s = 0; s < N; s++) {
                const int sp = fam == 0 ? s + N * line : line + N * s;
                acc = acc + sG[(c * NN + sp) * 18 + k] * sL[r * N + s];
            }
            g[k] = acc;
        }
        const int2 rec = a.faces[(size_t)(c0 + c) * 4 + (lf - 1)];
        const int kind = rec.y & 0xff;
        const bool own_right = kind == kFaceRight;
        double *dst = sGf + c * kG + ((fam * N + line) * NP + r) * 18;
        if (kind == kFaceLeft || own_right) {
            const int pc = rec.x, plf = (rec.y >> 8) & 0xff;
            const double *tp = a.gt + (((size_t)pc * 4 + (plf - 1)) * N + (N - nfp)) * 18;
#pragma unroll
            for (int k = 0; k < 18; k++) {
                const double p = tp[k];
                dst[k] = own_right ? 0.5 * p + 0.5 * g[k] : 0.5 * g[k] + 0.5 * p;
            }
            continue;
        }
#pragma unroll
        for (int k = 0; k < 18; k++) o[k] = g[k];
        if (kind == kFaceWall) {
            // adiabatic wall: the boundary energy gradient (bcflux.f90:469-583)
            const double *q = sQ + c * NQ;
            double Qfo[9], dxi = 0.0, deta = 0.0;
#pragma unroll
            for (int k = 0; k < 9; k++) Qfo[k] = 0.0;
#pragma unroll
            for (int s = 0; s < N; s++) {
                const int sp = fam == 0 ? s + N * line : line + N * s;
                const double l = sL[r * N + s];
#pragma unroll
                for (int k = 0; k < 9; k++) Qfo[k] = Qfo[k] + q[9 * sp + k] * l;
                dxi = dxi + sDE[(c * NN + sp) * 2] * l;
                deta = deta + sDE[(c * NN + sp) * 2 + 1] * l;
            }
            const double *m2 = a.met2 + (((size_t)(c0 + c) * 4 + (lf - 1)) * N + (nfp - 1)) * 2;
            const double ur = Qfo[1] / Qfo[0], vr = Qfo[2] / Qfo[0], wr = Qfo[3] / Qfo[0];
            const double inte = (Qfo[4] / Qfo[0] - 0.5 * ((ur * ur + vr * vr) + wr * wr)) -
                                0.5 * (((Qfo[5] * Qfo[5] + Qfo[6] * Qfo[6]) + Qfo[7] * Qfo[7]) + Qfo[8] * Qfo[8]) /
                                    Qfo[0];
            // dBp of both directions is the first direction's (bcflux.f90:563)
            const double dBp = ((Qfo[5] * g[5] + Qfo[6] * g[6]) + Qfo[7] * g[7]) + Qfo[8] * g[8];
#pragma unroll
            for (int d = 0; d < 2; d++) {
                const double *gd = g + 9 * d;
                const double dur = (gd[1] - ur * gd[0]) / Qfo[0];
                const double dvr = (gd[2] - vr * gd[0]) / Qfo[0];
                const double dwr = (gd[3] - wr * gd[0]) / Qfo[0];
                const double dKE =
                    0.5 * ((ur * ur + vr * vr) + wr * wr) * o[9 * d] + Qfo[0] * ((ur * dur + vr * dvr) + wr * dwr);
                // the ghost family's other normal row: S1(2,d) on xi faces,
                // S2(1,d) on eta faces; the energy gradient along it
                const double tw = fam == 0 ? 2.0 * deta * m2[d] * Qfo[0] : 2.0 * dxi * m2[d] * Qfo[0];
                o[9 * d + 4] = (((-gd[4] + 2.0 * inte * o[9 * d]) + 2.0 * dKE) + dBp) + tw;
            }
        }
#pragma unroll
        for (int k = 0; k < 18; k++) dst[k] = 0.5 * g[k] + 0.5 * o[k];
    }
    __syncthreads();
    // the viscous flux at every flux point (comp_viscous_flux)
    for (int t = tid; t < ncl * 2 * N * NP; t += kViscThreads) {
        const int r = t % NP, l = (t / NP) % N, f = (t / (NP * N)) % 2, c = t / (2 * N * NP);
        const int slot = (f * N + l) * NP + r;
        double Fv[9], Gv[9];
        vflux(sV + c * kF + slot * 9, sGf + c * kG + slot * 18, a.mu, a.eta0, Fv, Gv);
        const double *nr = sNrm + c * NM + ML::normal(f, l, r);
        double *o = sFv + c * kF + slot * 9;
#pragma unroll
        for (int k = 0; k < 9; k++) o[k] = Fv[k] * nr[0] + Gv[k] * nr[1];
    }
    __syncthreads();
    // dFv + dGv at the solution points (compresid.f90:14-32)
    for (int t = tid; t < ncl * NQ; t += kViscThreads) {
        const int k = t % 9, i = (t / 9) % N, j = (t / (9 * N)) % N, c = t / NQ;
        const double *Fx = sFv + c * kF + (0 * N + j) * NP * 9 + k;
        const double *Fy = sFv + c * kF + (1 * N + i) * NP * 9 + k;
        double dF = 0.0, dG = 0.0;
#pragma unroll
        for (int r = 0; r < NP; r++) dF = dF + Fx[r * 9] * sM[r * N + i];
#pragma unroll
        for (int r = 0; r < NP; r++) dG = dG + Fy[r * 9] * sM[r * N + j];
        a.rv[(size_t)c0 * NQ + t] = dF + dG;
    }
}

template <int N> constexpr size_t visc_grad_smem()
{
    using S = ViscSmem<N>;
    return sizeof(double) * ((size_t)kViscCpb * (S::NQ + S::kF + 18 * S::NN + S::NN + S::NM) + 2 * S::NP * N);
}
template <int N> constexpr size_t visc_flux_smem()
{
    using S = ViscSmem<N>;
    return sizeof(double) *
           ((size_t)kViscCpb * (S::NQ + 2 * S::kF + S::kG + 18 * S::NN + 2 * S::NN + S::NN + S::NM) + 2 * S::NP * N);
}

}  // namespace sddc
