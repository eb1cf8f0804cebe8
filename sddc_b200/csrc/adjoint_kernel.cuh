// Kernels of the discrete adjoint (VJP) of the SDDC residual and RK stage.
//
// For one RK stage out = ... + c R(q) the reverse stage needs
// qbar = (dR/dq)^T lambda with lambda = c * xbar (xbar: adjoint of the stage
// output).  R is the compresid chain (compresid.f90:1-80, compflux.f90,
// interfaceflux_all.f90, cyclocflux_all.f90, bcflux.f90); its linear parts
// (interpolation, flux derivative, metric gradient of B, sources) are
// transposed here by hand, its point functions go through
// adjoint_point.cuh.  The AV sensor enters no residual (its coefficients are
// zero, getrusanov.f90:326,328) and so has no adjoint.
//
// Per reverse stage:
//   adjoint traces    per (cell, face point): the adjoint of the flux value
//                     and of the face-averaged Bx, By that this cell's
//                     residual sees at the face point (its neighbour needs
//                     them: a shared face's flux and average enter both
//                     cells' residuals).  They depend on the cell's own
//                     output adjoint only, which is the previous reverse
//                     stage's out: that stage's vjp_kernel forms them in its
//                     epilogue when it knows this stage's input state, else
//                     adj_trace_kernel does;
//   vjp_kernel        per tile of cells, staged in shared memory: primal
//                     recomputation (traces, divB), the transposed
//                     divergence and gradient, the point adjoints, the
//                     transposed interpolation, the RK reverse update as an
//                     element-wise epilogue, and the next stage's adjoint
//                     traces.
// c_h = sqrt(L (L - U)) is a function of the running maxima L, U of the wave
// speed and velocity over all earlier stages; its adjoint is carried by
// adj_reduce_kernel to the stage and points where the maximum was attained
// (argmax records written by vjp_kernel).
#pragma once

#include "adjoint_point.cuh"
#include "stage_kernel.cuh"

namespace sddc {

enum : unsigned { kErrAdjointMaxLost = 4u, kErrAdjointRecords = 8u };

// a point where a running maximum was attained: the gradient of the wave
// speed (kind 0) or velocity maximum (kind 1) there with respect to the
// cell's own flux-point state (slot: (fam*N + line)*(N+1) + r) and to the
// free stream (boundary faces)
struct AdjRec {
    int cell, slot, kind, counted;
    double d[9];
    double p[6];
};

// device-side scalars carried across reverse stages
struct AdjScalars {
    double lam_eig, lam_um;  // adjoints of the running maxima not yet given to their argmax
    double pbar[6];          // adjoint of (rinf, pinf, uinf, vinf, bxinf, byinf)
    double cbar;             // sum over stages of lambda . dR/dc_h
    double ties;             // stages whose raised maximum several points attained
};

struct VjpArgs {
    int ncell, vismode;
    double alpha, c_h;
    Freestream fs;
    const double *__restrict__ q;     // stage input state (9,N,N,NCELL)
    const double *__restrict__ t_in;  // its face traces, layout trace_at
    const double *xbar;               // adjoint of the stage output; null: objective seeds only
    double lam_scale;                 // lambda = lam_scale * xbar
    const double *__restrict__ at;    // adjoint traces, layout adj_trace_at
    const double *__restrict__ met;
    // the split metrics of an exact context (double normals [NCELL][4N(N+1)],
    // Jac [NCELL][MetLayout::kJacPad]), staged directly; null: the packed record
    const double *__restrict__ nrm, *__restrict__ jac;
    const int2 *__restrict__ faces;
    // epilogue: out = (wa*ra + wb*rb) + qbar;  out2 = wc*rc + wd*xbar
    const double *ra, *rb;
    double wa, wb;
    double *out;
    const double *rc;
    double wc, wd;
    double *out2;
    // objective: adjoint of the wall force (Fx, Fy) at this state
    double sx, sy;
    double wq[kMaxN];
    double *part;  // [8][CTAs]: cbar, pbar[6], 0
    unsigned *err;
    // the next reverse stage's adjoint traces, formed from out (the adjoint of
    // that stage's output) in the epilogue: its input state and lam_scale, and
    // the trace buffer (null: its own trace launch forms them)
    const double *q_next;
    double scale_next;
    double *at_next;
};

constexpr int kAdjCpb = 4;
__host__ __device__ constexpr int adj_threads(int n, int cpb) { return (4 * n * cpb > 128 ? (4 * n * cpb + 31) / 32 * 32 : 128); }

// Warps of vjp_kernel given to the face points (the rest take the interior
// flux points): the count that minimises the slower side's rounds, with a
// face point's Rusanov adjoint costing about kFaceCost interior points' flux
// adjoints (measured on the B200 at N = 4); ties go to fewer face warps.
constexpr int kFaceCost = 7;
__host__ __device__ constexpr int adj_face_warps(int n, int cpb)
{
    const int nw = adj_threads(n, cpb) / 32, nf = cpb * 4 * n, ni = cpb * 2 * n * (n - 1);
    int best = 1, cost = 1 << 30;
    for (int w = 1; w < nw; w++) {
        const int cf = (nf + 32 * w - 1) / (32 * w) * kFaceCost, ci = (ni + 32 * (nw - w) - 1) / (32 * (nw - w));
        const int c = cf > ci ? cf : ci;
        if (c < cost) {
            cost = c;
            best = w;
        }
    }
    return best;
}

template <int N, int CPB> constexpr size_t vjp_smem_doubles()
{
    constexpr int NQ = 9 * N * N, NP = N + 1, NN = N * N;
    constexpr int kF = 2 * N * NP * 9, kV = 2 * N * NP * 2, kO = 4 * N * 9, kP = 4 * N * 13;
    constexpr int NM = 2 * MetLayout<N>::kFam;
    return (size_t)CPB * (2 * NQ + 2 * kF + kV + kO + kP + MetLayout<N>::kJacPad + NN + NM) + 2 * NP * N + 8 * 32;
}

// the tile fits a CTA's shared memory (227 KB) at every N; at N = 4 four
// CTAs fit an SM (228 KB, 1 KB reserved per CTA), which the 128-register cap
// of vjp_kernel's launch bounds assumes
static_assert(vjp_smem_doubles<6, kAdjCpb>() * sizeof(double) <= 227 * 1024, "VJP tile exceeds shared memory");
static_assert(4 * (vjp_smem_doubles<4, kAdjCpb>() * sizeof(double) + 1024) <= 228 * 1024,
              "VJP tile at N = 4 no longer fits four CTAs per SM");

// ---- adjoint traces ----------------------------------------------------------
// at(cell, lf, nfp) = (Fbar(9), Vbar_Bx, Vbar_By, 0): the adjoint of this
// cell's flux value at the face point (from the divergence, compresid.f90:
// 12-51) and of the face-averaged Bx, By (from divB in the Powell source,
// compresid.f90:58, through nablaQsp compflux.f90:107-157).
constexpr int kTraceCpb = 8;  // cells per CTA of adj_trace_kernel

// adjoint trace layout, [cell][local face][value][face point] like trace_at:
// the N points of a face, which consecutive lanes write and read, are
// adjacent (lf 1-based, nfp0 0-based, 12 values, the last one 0)
template <int N> __host__ __device__ __forceinline__ size_t adj_trace_at(size_t cell, int lf, int nfp0, int k)
{
    return ((cell * 4 + (size_t)(lf - 1)) * 12 + (size_t)k) * N + (size_t)nfp0;
}

template <int N>
__global__ void __launch_bounds__(128) adj_trace_kernel(int ncell, int vismode, const double *__restrict__ xbar,
                                                        double lam_scale, const double *__restrict__ q,
                                                        const double *__restrict__ met, const Ops ops,
                                                        double *__restrict__ at)
{
    using ML = MetLayout<N>;
    constexpr int NQ = 9 * N * N, NN = N * N, CPB = kTraceCpb;
    __shared__ __align__(16) double sMu[CPB * NQ];  // lambda source, then -lambda/J
    __shared__ __align__(16) double sQs[CPB * NQ];  // the state
    __shared__ double sB[CPB * NN];                 // Jac, 1/Jac, then the divB adjoint over Jac
    __shared__ __align__(8) unsigned long long sBar;
    __shared__ int sAbort;
    const int tid = threadIdx.x, c0 = blockIdx.x * CPB, ncl = min(CPB, ncell - c0);
    // the lambda source and state slices by TMA bulk copies when aligned
    const double *xsrc = xbar + (size_t)c0 * NQ, *qsrc = q + (size_t)c0 * NQ;
    const size_t bytes = (size_t)ncl * NQ * sizeof(double);
    const bool bulk = (((uintptr_t)xsrc | (uintptr_t)qsrc | bytes) & 15) == 0;
    if (tid == 0) {
        sAbort = 0;
        if (bulk) {
            mbar_init(&sBar, 1);
            mbar_expect_tx(&sBar, (unsigned)(2 * bytes));
            bulk_g2s(sMu, xsrc, (unsigned)bytes, &sBar);
            bulk_g2s(sQs, qsrc, (unsigned)bytes, &sBar);
        }
    }
    for (int k = tid; k < ncl * NN; k += 128) {
        const int c = k / NN;
        sB[k] = met[(size_t)(c0 + c) * ML::kSize + ML::kJac + (k - c * NN)];
    }
    if (!bulk)
        for (int k = tid; k < ncl * NQ; k += 128) {
            sMu[k] = xsrc[k];
            sQs[k] = qsrc[k];
        }
    if (bulk && tid == 0 && !mbar_wait_bounded(&sBar, 0)) {
        sAbort = 1;  // the copies did not complete; the caller sees stale traces
        mbar_wait_bounded(&sBar, 0);
    }
    __syncthreads();
    if (sAbort) return;
    // per solution point: the divB adjoint from the Powell source
    // (compresid.f90:60-76), over Jac
    double beta[(CPB * NN + 127) / 128];
    for (int k = tid, it = 0; k < ncl * NN; k += 128, it++) {
        const double *x = sMu + 9 * k;
        double db = 0.0;
        if (vismode == 1) {
            const double *qq = sQs + 9 * k;
            const double ri = 1.0 / qq[0], ux = qq[1] * ri, uy = qq[2] * ri, uz = qq[3] * ri;
            db = -lam_scale * (x[1] * qq[5] + x[2] * qq[6] + x[3] * qq[7] +
                               x[4] * ((ux * qq[5] + uy * qq[6]) + uz * qq[7]) + x[5] * ux + x[6] * uy + x[7] * uz);
        }
        const double rJ = 1.0 / sB[k];
        beta[it] = db * rJ;
        sB[k] = rJ;
    }
    __syncthreads();
    for (int k = tid; k < ncl * NQ; k += 128) sMu[k] = -(lam_scale * sMu[k]) * sB[k / 9];
    __syncthreads();
    for (int k = tid, it = 0; k < ncl * NN; k += 128, it++) sB[k] = beta[it];
    __syncthreads();
    // per face point: the transposed flux derivative and B gradient
    for (int t = tid; t < ncl * 4 * N; t += 128) {
        const int c = t / (4 * N), f = t - c * 4 * N;
        const int nfp = 1 + f % N, lf = 1 + f / N;
        int fam, line, r;
        face_point<N>(lf, nfp, fam, line, r);
        double fb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, bs = 0.0;
#pragma unroll
        for (int i = 0; i < N; i++) {
            const int sp = fam == 0 ? i + N * line : line + N * i;
            const double m = ops.M[r * N + i];
            const double *mu = sMu + c * NQ + 9 * sp;
#pragma unroll
            for (int k = 0; k < 9; k++) fb[k] += m * mu[k];
            bs += m * sB[c * NN + sp];
        }
        const double *nr = met + (size_t)(c0 + c) * ML::kSize + ML::normal(fam, line, r);
#pragma unroll
        for (int k = 0; k < 9; k++) at[adj_trace_at<N>(c0 + c, lf, nfp - 1, k)] = fb[k];
        at[adj_trace_at<N>(c0 + c, lf, nfp - 1, 9)] = bs * nr[0];
        at[adj_trace_at<N>(c0 + c, lf, nfp - 1, 10)] = bs * nr[1];
        at[adj_trace_at<N>(c0 + c, lf, nfp - 1, 11)] = 0.0;
    }
}

// The adjoint trace at face point f (0..4N-1) of one cell from global memory,
// in adj_trace_kernel's arithmetic: the reduction uses it to form again the
// next stage's traces of the cells that its records changed.
template <int N>
__device__ void adj_trace_point(size_t cell, int f, const double *xbar, const double *q, double scale,
                                const double *met, int vismode, const Ops &ops, double *at)
{
    using ML = MetLayout<N>;
    constexpr int NQ = 9 * N * N;
    const int nfp = 1 + f % N, lf = 1 + f / N;
    int fam, line, r;
    face_point<N>(lf, nfp, fam, line, r);
    const double *mc = met + cell * ML::kSize;
    double fb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, bs = 0.0;
    for (int i = 0; i < N; i++) {
        const int sp = fam == 0 ? i + N * line : line + N * i;
        const double *x = xbar + cell * NQ + 9 * sp;
        double db = 0.0;
        if (vismode == 1) {
            const double *qq = q + cell * NQ + 9 * sp;
            const double ri = 1.0 / qq[0], ux = qq[1] * ri, uy = qq[2] * ri, uz = qq[3] * ri;
            db = -scale * (x[1] * qq[5] + x[2] * qq[6] + x[3] * qq[7] + x[4] * ((ux * qq[5] + uy * qq[6]) + uz * qq[7]) +
                           x[5] * ux + x[6] * uy + x[7] * uz);
        }
        const double rJ = 1.0 / mc[ML::kJac + sp];
        const double m = ops.M[r * N + i];
        for (int k = 0; k < 9; k++) fb[k] += m * (-(scale * x[k]) * rJ);
        bs += m * (db * rJ);
    }
    const double *nr = mc + ML::normal(fam, line, r);
    for (int k = 0; k < 9; k++) at[adj_trace_at<N>(cell, lf, nfp - 1, k)] = fb[k];
    at[adj_trace_at<N>(cell, lf, nfp - 1, 9)] = bs * nr[0];
    at[adj_trace_at<N>(cell, lf, nfp - 1, 10)] = bs * nr[1];
    at[adj_trace_at<N>(cell, lf, nfp - 1, 11)] = 0.0;
}

// ---- running-max argmax records ----------------------------------------------------
// where the records go (passed by value: the out-of-line record path must
// not copy the kernel's argument block)
struct RecSink {
    AdjRec *recs;
    int cap;
    int *n;
    int *cnt;
    unsigned *err;
};

static __device__ __noinline__ void adj_record(RecSink rs, int cell, int slot, int kind, int counted, const double *d,
                                        const double *p)
{
    const int k = atomicAdd(rs.n, 1);
    if (k < rs.cap) {
        AdjRec &R = rs.recs[k];
        R.cell = cell;
        R.slot = slot;
        R.kind = kind;
        R.counted = counted;
        for (int m = 0; m < 9; m++) R.d[m] = d[m];
        for (int m = 0; m < 6; m++) R.p[m] = p ? p[m] : 0.0;
    } else {
        atomicOr(rs.err, kErrAdjointRecords);
    }
    if (counted) atomicAdd(rs.cnt + kind, 1);
}

// a face point whose wave speed (hit_eig) or velocity maximum (hit_um)
// equals the stage's new running max: the gradient of that value with
// respect to this cell's trace (and the free stream, through a ghost
// state); a shared face is counted by its left cell only
static __device__ __noinline__ void adj_record_face(RecSink rs, Freestream fs, int vismode, double c_h, bool hit_eig,
                                             bool hit_um, int cell, int slot, int kind, bool own_right,
                                             const double *own, const double *oth, double n0, double n1, int sign_l)
{
    const bool pair = kind == kFaceLeft || kind == kFaceRight;
    const double *ql = own_right ? oth : own, *qr = own_right ? own : oth;
    const double z[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int kk = 0; kk < 2; kk++) {
        if (!(kk == 0 ? hit_eig : hit_um)) continue;
        double d[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, dg[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, p[6] = {0, 0, 0, 0, 0, 0};
        double e2, u2;
        if (pair) {
            rusanov_vjp(ql, qr, n0, n1, sign_l, c_h, z, kk == 0 ? 1.0 : 0.0, kk == 1 ? 1.0 : 0.0,
                        own_right ? nullptr : d, own_right ? d : nullptr, e2, u2);
        } else {
            rusanov_vjp(own, oth, n0, n1, sign_l, c_h, z, kk == 0 ? 1.0 : 0.0, kk == 1 ? 1.0 : 0.0, d, dg, e2, u2);
            bc_ghost_vjp(kind, own, n0, n1, vismode, fs, dg, d, p);
        }
        adj_record(rs, cell, slot, kk, own_right ? 0 : 1, d, p);
    }
}

// ---- the stage VJP -------------------------------------------------------------
template <int N, int CPB>
__global__ void __launch_bounds__(adj_threads(N, CPB), 4) vjp_kernel(const VjpArgs a, const Ops ops)
{
    using ML = MetLayout<N>;
    constexpr int NT = adj_threads(N, CPB);
    constexpr int NQ = 9 * N * N, NP = N + 1, NN = N * N;
    constexpr int kF = 2 * N * NP * 9, kV = 2 * N * NP * 2, kO = 4 * N * 9, kP = 4 * N * 13, NM = 2 * ML::kFam;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sQ = reinterpret_cast<double *>(smem_raw);  // [CPB][NQ] q, then qbar of the sources, then qbar
    double *sA = sQ + CPB * NQ;                         // [CPB][NQ] lambda, then -lambda/J
    double *sQf = sA + CPB * NQ;                        // [CPB][2][N][NP][9] flux-point states
    double *sFb = sQf + CPB * kF;                       // [CPB][2][N][NP][9] flux adjoint, then state adjoint
    double *sVb = sFb + CPB * kF;                       // [CPB][2][N][NP][2] face-averaged Bx,By, then adjoint
    double *sQo = sVb + CPB * kV;                       // [CPB][4N][9] neighbour / ghost trace
    // [CPB][4N][13] per face point: the partner's signed flux adjoint (9) and
    // face-average adjoints (2), zero on boundary faces; the face's normal (2)
    double *sPa = sQo + CPB * kO;
    constexpr int NJ = ML::kJacPad;
    double *sJac = sPa + CPB * kP;                      // [CPB][NJ]
    double *sBeta = sJac + CPB * NJ;                    // [CPB][NN] adjoint of divB, over Jac
    double *sNrm = sBeta + CPB * NN;                    // [CPB][NM]
    double *sL = sNrm + CPB * NM;                       // [NP][N]
    double *sM = sL + NP * N;                           // [NP][N]
    double *sRed = sM + NP * N;                         // [8][32]

    const int tid = threadIdx.x;
    const int c0 = blockIdx.x * CPB;
    const int ncl = min(CPB, a.ncell - c0);

    // the tile's state, lambda source and metric slices by TMA bulk copies
    // when they are 16-byte aligned, else by loads: the split normals and Jac
    // straight into place, or the packed metric records into sQf (free until
    // the primal phase) for conversion
    __shared__ __align__(8) unsigned long long sBar;
    __shared__ int sAbort;
    const bool split = a.nrm != nullptr;  // uniform
    {
        const double *qsrc = a.q + (size_t)c0 * NQ, *msrc = a.met + (size_t)c0 * ML::kSize;
        const double *nsrc = split ? a.nrm + (size_t)c0 * NM : nullptr, *jsrc = split ? a.jac + (size_t)c0 * NJ : nullptr;
        const double *xsrc = a.xbar ? a.xbar + (size_t)c0 * NQ : nullptr;
        const size_t qbytes = (size_t)ncl * NQ * sizeof(double);
        const size_t mbytes = split ? 0 : (size_t)ncl * ML::kSize * sizeof(double);
        const size_t nbytes = split ? (size_t)ncl * NM * sizeof(double) : 0;
        const size_t jbytes = split ? (size_t)ncl * NJ * sizeof(double) : 0;
        const bool bulk = (((uintptr_t)qsrc | (uintptr_t)msrc | (uintptr_t)nsrc | (uintptr_t)jsrc | (uintptr_t)xsrc |
                            qbytes | mbytes | nbytes | jbytes) & 15) == 0;
        if (tid == 0) {
            sAbort = 0;
            if (bulk) {
                mbar_init(&sBar, 1);
                mbar_expect_tx(&sBar, (unsigned)(qbytes + mbytes + nbytes + jbytes + (xsrc ? qbytes : 0)));
                bulk_g2s(sQ, qsrc, (unsigned)qbytes, &sBar);
                if (split) {
                    bulk_g2s(sNrm, nsrc, (unsigned)nbytes, &sBar);
                    bulk_g2s(sJac, jsrc, (unsigned)jbytes, &sBar);
                } else {
                    bulk_g2s(sQf, msrc, (unsigned)mbytes, &sBar);
                }
                if (xsrc) bulk_g2s(sA, xsrc, (unsigned)qbytes, &sBar);
            }
        }
        // L2 prefetches of what later phases load from global memory: the RK
        // registers of the epilogue, and per shared face the partner's trace
        // and adjoint trace (each face's values are contiguous)
        if (tid == 0) {
            const size_t g0 = (size_t)c0 * NQ;
            const double *regs[3] = {a.ra, a.rb, a.out2 ? a.rc : nullptr};
            for (int m = 0; m < 3; m++)
                if (regs[m] && (((uintptr_t)(regs[m] + g0) | qbytes) & 15) == 0)
                    bulk_prefetch_l2(regs[m] + g0, (unsigned)qbytes);
        } else if (tid >= 32 && tid < 32 + ncl * 4) {
            const int c = (tid - 32) >> 2, lf = 1 + ((tid - 32) & 3);
            const int2 rec = a.faces[(size_t)(c0 + c) * 4 + (lf - 1)];
            const int kind = rec.y & 0xff;
            if (kind == kFaceLeft || kind == kFaceRight) {
                const int pc = rec.x, plf = (rec.y >> 8) & 0xff;
                // the face's 9N trace values, widened to 16-byte bounds (the
                // buffer, 288N bytes per cell, starts and ends on one)
                const uintptr_t t0 = (uintptr_t)(a.t_in + trace_at<N>(pc, plf, 0, 0)) & ~(uintptr_t)15;
                const uintptr_t t1 = ((uintptr_t)(a.t_in + trace_at<N>(pc, plf, 0, 9)) + 15) & ~(uintptr_t)15;
                if (((uintptr_t)a.t_in & 15) == 0) bulk_prefetch_l2((const void *)t0, (unsigned)(t1 - t0));
                if (a.xbar && ((uintptr_t)a.at & 15) == 0)
                    bulk_prefetch_l2(a.at + adj_trace_at<N>(pc, plf, 0, 0), 12 * N * sizeof(double));
            }
        }
        for (int k = tid; k < NP * N; k += NT) {
            sL[k] = ops.L[k];
            sM[k] = ops.M[k];
        }
        if (!bulk) {
            for (int k = tid; k < ncl * NQ; k += NT) {
                sQ[k] = __ldg(qsrc + k);
                if (xsrc) sA[k] = xsrc[k];
            }
            if (split) {
                for (int k = tid; k < ncl * NM; k += NT) sNrm[k] = __ldg(nsrc + k);
                for (int k = tid; k < ncl * NJ; k += NT) sJac[k] = __ldg(jsrc + k);
            } else {
                for (int k = tid; k < ncl * ML::kSize; k += NT) sQf[k] = __ldg(msrc + k);
            }
        }
        if (bulk && tid == 0 && !mbar_wait_bounded(&sBar, 0)) {
            atomicOr(a.err, kErrStagingTimeout);  // the copies did not complete
            sAbort = 1;
            mbar_wait_bounded(&sBar, 0);
        }
    }
    __syncthreads();
    if (sAbort) return;
    // lambda (first read two barriers on); the packed metric records, staged in
    // sQf, are converted before phase A overwrites sQf
    for (int k = tid; k < ncl * NQ; k += NT) sA[k] = a.xbar ? a.lam_scale * sA[k] : 0.0;
    if (!split) {
        for (int k = tid; k < ncl * ML::kSize; k += NT) {
            const int c = k / ML::kSize, o = k - c * ML::kSize;
            const double v = sQf[k];
            if (o < NM) sNrm[c * NM + o] = v;
            else if (o < NM + NN) sJac[c * NJ + (o - NM)] = v;
        }
        __syncthreads();
    }

    // ---- primal: flux-point states (phase A of the stage kernel) ----------------
    for (int t = tid; t < ncl * 2 * N * 9; t += NT) {
        const int v = t % 9, l = (t / 9) % N, f = (t / (9 * N)) % 2, c = t / (18 * N);
        const double *q = sQ + c * NQ;
        double qs[N];
#pragma unroll
        for (int s = 0; s < N; s++) qs[s] = f == 0 ? q[v + 9 * (s + N * l)] : q[v + 9 * (l + N * s)];
        double *o = sQf + c * kF + (f * N + l) * NP * 9 + v;
#pragma unroll
        for (int r = 0; r < NP; r++) {
            double acc = 0.0;
#pragma unroll
            for (int s = 0; s < N; s++) acc = acc + qs[s] * ops.L[r * N + s];
            o[r * 9] = acc;
        }
    }
    __syncthreads();

    // ---- primal: neighbour / ghost traces and face-averaged Bx, By; on the ---------
    // ---- other threads the partner's adjoint trace and the face normal -------------
    for (int t2 = tid; t2 < 2 * ncl * 4 * N; t2 += NT) {
        const bool part = t2 >= ncl * 4 * N;
        const int t = part ? t2 - ncl * 4 * N : t2;
        const int nfp = 1 + t % N, lf = 1 + (t / N) % 4, c = t / (4 * N);
        int fam, line, r;
        face_point<N>(lf, nfp, fam, line, r);
        const int2 rec = a.faces[(size_t)(c0 + c) * 4 + (lf - 1)];
        const int kind = rec.y & 0xff;
        const bool own_right = kind == kFaceRight;
        if (part) {
            const double *onrm = sNrm + c * NM + ML::normal(fam, line, r);
            double v[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, onrm[0], onrm[1]};
            if (kind == kFaceLeft || own_right) {
                const int pc = rec.x, plf = (rec.y >> 8) & 0xff;
                int pfam, pline, pr;
                face_point<N>(plf, N - nfp + 1, pfam, pline, pr);
                if (own_right) {  // the flux is formed with the left (partner) cell's normal
                    const double *pn = a.met + (size_t)pc * ML::kSize + ML::normal(pfam, pline, pr);
                    v[11] = __ldg(pn);
                    v[12] = __ldg(pn + 1);
                }
                // the partner's slot enters with sign_l * sign_r unless it is
                // the left cell's
                const int sign_l = own_right ? (pr == 0 ? -1 : 1) : (r == 0 ? -1 : 1);
                const int sign_r = own_right ? (r == N ? -1 : 1) : (pr == N ? -1 : 1);
                const double ps = own_right ? 1.0 : (double)(sign_l * sign_r);
                if (a.xbar) {
#pragma unroll
                    for (int k = 0; k < 9; k++) v[k] = ps * a.at[adj_trace_at<N>(pc, plf, N - nfp, k)];
                    if (a.vismode == 1) {
                        v[9] = a.at[adj_trace_at<N>(pc, plf, N - nfp, 9)];
                        v[10] = a.at[adj_trace_at<N>(pc, plf, N - nfp, 10)];
                    }
                }
            }
            double *pa = sPa + c * kP + (t % (4 * N)) * 13;
#pragma unroll
            for (int k = 0; k < 13; k++) pa[k] = v[k];
            continue;
        }
        const double *own = sQf + c * kF + ((fam * N + line) * NP + r) * 9;
        double oth[9];
        if (kind == kFaceLeft || own_right) {
            const int pc = rec.x, plf = (rec.y >> 8) & 0xff;
#pragma unroll
            for (int k = 0; k < 9; k++) oth[k] = a.t_in[trace_at<N>(pc, plf, N - nfp, k)];
        } else {
            const double *nrm = sNrm + c * NM + ML::normal(fam, line, r);
            bc_ghost<double, true>(kind, own, nrm[0], nrm[1], a.vismode, a.fs, oth);
        }
        double *so = sQo + c * kO + t % (4 * N) * 9;
#pragma unroll
        for (int k = 0; k < 9; k++) so[k] = oth[k];
        double *vs = sVb + c * kV + ((fam * N + line) * NP + r) * 2;
        const double *ql = own_right ? oth : own, *qr = own_right ? own : oth;
        vs[0] = 0.5 * ql[5] + 0.5 * qr[5];
        vs[1] = 0.5 * ql[6] + 0.5 * qr[6];
    }
    __syncthreads();

    // ---- per solution point: divB, the source adjoint, -lambda/J, divB adjoint ------
    for (int t = tid; t < ncl * NN; t += NT) {
        const int i = t % N, j = (t / N) % N, c = t / NN;
        const double rJ = 1.0 / sJac[c * NJ + i + N * j];
        const double *met = sNrm + c * NM;
        double divB = 0.0;
        if (a.vismode == 1) {
            // nablaQsp for Bx (x derivative) and By (y derivative)
            auto V = [&](int f, int l, int r, int g) -> double {
                return (r == 0 || r == N) ? sVb[c * kV + ((f * N + l) * NP + r) * 2 + g]
                                          : sQf[c * kF + ((f * N + l) * NP + r) * 9 + 5 + g];
            };
            double ax = 0.0, bx = 0.0, ay = 0.0, by = 0.0;
#pragma unroll
            for (int r = 0; r < NP; r++) {
                ax += V(0, j, r, 0) * sM[r * N + i] * met[ML::normal(0, j, r)];
                bx += V(1, i, r, 0) * sM[r * N + j] * met[ML::normal(1, i, r)];
                ay += V(0, j, r, 1) * sM[r * N + i] * met[ML::normal(0, j, r) + 1];
                by += V(1, i, r, 1) * sM[r * N + j] * met[ML::normal(1, i, r) + 1];
            }
            divB = ((ax + bx) + (ay + by)) * rJ;
        }
        double *qs = sQ + c * NQ + 9 * (i + N * j);
        double *lam = sA + c * NQ + 9 * (i + N * j);
        const double rho = qs[0], ri = 1.0 / rho, ux = qs[1] * ri, uy = qs[2] * ri, uz = qs[3] * ri;
        const double Bx = qs[5], By = qs[6], Bz = qs[7];
        double db = 0.0;
        if (a.vismode == 1)
            db = -(lam[1] * Bx + lam[2] * By + lam[3] * Bz + lam[4] * ((ux * Bx + uy * By) + uz * Bz) +
                   lam[5] * ux + lam[6] * uy + lam[7] * uz);
        // Powell and GLM sources (compresid.f90:60-78)
        const double ub = -divB * (lam[4] * Bx + lam[5]);
        const double vb = -divB * (lam[4] * By + lam[6]);
        const double wb = -divB * (lam[4] * Bz + lam[7]);
        double src[9];
        src[0] = -(ub * ux + vb * uy + wb * uz) * ri;
        src[1] = ub * ri;
        src[2] = vb * ri;
        src[3] = wb * ri;
        src[4] = 0.0;
        src[5] = -divB * (lam[1] + lam[4] * ux);
        src[6] = -divB * (lam[2] + lam[4] * uy);
        src[7] = -divB * (lam[3] + lam[4] * uz);
        src[8] = -a.alpha * lam[8];
#pragma unroll
        for (int k = 0; k < 9; k++) {
            qs[k] = src[k];
            lam[k] = -lam[k] * rJ;
        }
        sBeta[c * NN + i + N * j] = db * rJ;
    }
    __syncthreads();

    // ---- transposed flux derivative and B gradient: adjoints at the flux points ------
    for (int t = tid; t < ncl * 2 * N * 11; t += NT) {
        const int v = t % 11, l = (t / 11) % N, f = (t / (11 * N)) % 2, c = t / (22 * N);
        double x[N];
#pragma unroll
        for (int i = 0; i < N; i++) {
            const int sp = f == 0 ? i + N * l : l + N * i;
            x[i] = v < 9 ? sA[c * NQ + 9 * sp + v] : sBeta[c * NN + sp];
        }
#pragma unroll
        for (int r = 0; r < NP; r++) {
            double acc = 0.0;
#pragma unroll
            for (int i = 0; i < N; i++) acc += ops.M[r * N + i] * x[i];
            if (v < 9) {
                sFb[c * kF + ((f * N + l) * NP + r) * 9 + v] = acc;
            } else {
                const double n = sNrm[c * NM + ML::normal(f, l, r) + (v - 9)];
                sVb[c * kV + ((f * N + l) * NP + r) * 2 + (v - 9)] = acc * n;
            }
        }
    }
    __syncthreads();

    double cbar = 0.0, pb[6] = {0, 0, 0, 0, 0, 0};
    // The point adjoints: face points on the first kFaceWarps warps, interior
    // flux points on the others (adj_face_warps balances their rounds).  The
    // interior warps then add the interior flux points' share of the
    // transposed interpolation while the face warps finish.
    constexpr int kFaceWarps = adj_face_warps(N, CPB);
    const int wid = tid >> 5;
    if (wid >= kFaceWarps) {
        // ---- interior flux points ---------------------------------------------------
        const int nth = NT - 32 * kFaceWarps, me = tid - 32 * kFaceWarps;
        for (int t = me; t < ncl * 2 * N * (N - 1); t += nth) {
            const int r = 1 + t % (N - 1), l = (t / (N - 1)) % N, f = (t / ((N - 1) * N)) % 2,
                      c = t / (2 * N * (N - 1));
            const int slot = (f * N + l) * NP + r;
            const double *qf = sQf + c * kF + slot * 9;
            double *fb = sFb + c * kF + slot * 9;
            const double *nr = sNrm + c * NM + ML::normal(f, l, r);
            double qb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, um;
            cbar += iflux_vjp(qf, a.c_h, nr[0], nr[1], fb, qb, um, nullptr);
            if (a.vismode == 1) {
                qb[5] += sVb[c * kV + slot * 2];
                qb[6] += sVb[c * kV + slot * 2 + 1];
            }
#pragma unroll
            for (int k = 0; k < 9; k++) fb[k] = qb[k];
        }
        // the interior warps' own barrier: their flux-point adjoints are all in
        asm volatile("bar.sync 1, %0;" ::"r"(nth) : "memory");
        for (int t = me; t < ncl * NQ; t += nth) {
            const int v = t % 9, i = (t / 9) % N, j = (t / (9 * N)) % N, c = t / NQ;
            const double *gx = sFb + c * kF + (0 * N + j) * NP * 9 + v;  // xi-line j
            const double *gy = sFb + c * kF + (1 * N + i) * NP * 9 + v;  // eta-line i
            double acc = sQ[t];
#pragma unroll
            for (int r = 1; r < N; r++) acc += sL[r * N + i] * gx[r * 9] + sL[r * N + j] * gy[r * 9];
            sQ[t] = acc;
        }
    } else {
        // ---- face points ------------------------------------------------------------
        for (int t = tid; t < ncl * 4 * N; t += 32 * kFaceWarps) {
            const int nfp = 1 + t % N, lf = 1 + (t / N) % 4, c = t / (4 * N);
            int fam, line, r;
            face_point<N>(lf, nfp, fam, line, r);
            const int slot = (fam * N + line) * NP + r;
            const double *own = sQf + c * kF + slot * 9;
            const double *oth = sQo + c * kO + (t % (4 * N)) * 9;
            double *fown = sFb + c * kF + slot * 9;
            const int2 rec = a.faces[(size_t)(c0 + c) * 4 + (lf - 1)];
            const int kind = rec.y & 0xff;
            const bool pair = kind == kFaceLeft || kind == kFaceRight;
            const bool own_right = kind == kFaceRight;
            const double *pa = sPa + c * kP + (t % (4 * N)) * 13;
            const double n0 = pa[11], n1 = pa[12];
            int sign_l, sign_r;
            double fbar[9], vbx = 0.0, vby = 0.0;
            if (a.vismode == 1) {
                vbx = sVb[c * kV + slot * 2];
                vby = sVb[c * kV + slot * 2 + 1];
            }
            if (pair) {
                const int plf = (rec.y >> 8) & 0xff;
                int pfam, pline, pr;
                face_point<N>(plf, N - nfp + 1, pfam, pline, pr);
                sign_l = own_right ? (pr == 0 ? -1 : 1) : (r == 0 ? -1 : 1);
                sign_r = own_right ? (r == N ? -1 : 1) : (pr == N ? -1 : 1);
                const double ms = own_right ? (double)(sign_l * sign_r) : 1.0;
                // the partner's share (staged signed, zero without xbar)
#pragma unroll
                for (int k = 0; k < 9; k++) fbar[k] = ms * fown[k] + pa[k];
                if (a.vismode == 1) {
                    vbx += pa[9];
                    vby += pa[10];
                }
            } else {
                sign_l = r == 0 ? -1 : 1;
                sign_r = 1;
#pragma unroll
                for (int k = 0; k < 9; k++) fbar[k] = fown[k];
                if (kind == kFaceWall) {  // the objective: force on the wall faces
                    const double w = a.wq[line] * (double)sign_l;
                    fbar[1] += a.sx * w;
                    fbar[2] += a.sy * w;
                }
            }
            const double *ql = own_right ? oth : own, *qr = own_right ? own : oth;
            double qown[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, eig, um;
            // the face-averaged Bx, By feed the gradients of both cells
            qown[5] = 0.5 * vbx;
            qown[6] = 0.5 * vby;
            // this cell's share of the c_h adjoint comes from its own flux
            // slot (fown, weighted by the slot's sign)
            double wdc;
            if (pair) {
                wdc = rusanov_vjp(ql, qr, n0, n1, sign_l, a.c_h, fbar, 0.0, 0.0, own_right ? nullptr : qown,
                                  own_right ? qown : nullptr, eig, um, nullptr, fown);
            } else {
                double qgb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                qgb[5] = 0.5 * vbx;
                qgb[6] = 0.5 * vby;
                wdc = rusanov_vjp(own, oth, n0, n1, sign_l, a.c_h, fbar, 0.0, 0.0, qown, qgb, eig, um, nullptr, fown);
                bc_ghost_vjp(kind, own, n0, n1, a.vismode, a.fs, qgb, qown, pb);
            }
            cbar += (own_right ? (double)(sign_l * sign_r) : 1.0) * wdc;

#pragma unroll
            for (int k = 0; k < 9; k++) fown[k] = qown[k];
        }
    }
    __syncthreads();

    // the next stage's input state, for its adjoint traces, by a bulk copy into
    // sQf (no longer read) that lands during the steps below
    const bool fuse = a.at_next != nullptr;  // uniform
    const double *qn = fuse ? a.q_next + (size_t)c0 * NQ : nullptr;
    const bool qn_bulk = fuse && (((uintptr_t)qn | ((size_t)ncl * NQ * sizeof(double))) & 15) == 0;
    __shared__ __align__(8) unsigned long long sBarN;
    if (qn_bulk && tid == 0) {
        fence_proxy_async();
        mbar_init(&sBarN, 1);
        mbar_expect_tx(&sBarN, (unsigned)(ncl * NQ * sizeof(double)));
        bulk_g2s(sQf, qn, (unsigned)(ncl * NQ * sizeof(double)), &sBarN);
    }

    // ---- transposed interpolation, the face points' share (the interior flux ---------
    // ---- points' share is in): state adjoint at the solution points ------------------
    for (int t = tid; t < ncl * NQ; t += NT) {
        const int v = t % 9, i = (t / 9) % N, j = (t / (9 * N)) % N, c = t / NQ;
        const double *gx = sFb + c * kF + (0 * N + j) * NP * 9 + v;  // xi-line j
        const double *gy = sFb + c * kF + (1 * N + i) * NP * 9 + v;  // eta-line i
        sQ[t] += (sL[i] * gx[0] + sL[j] * gy[0]) + (sL[N * N + i] * gx[N * 9] + sL[N * N + j] * gy[N * 9]);
    }
    __syncthreads();

    // ---- RK reverse update, element-wise ----------------------------------------------
    // the register reads of kU elements are issued before their use, so that
    // each thread keeps several loads in flight
    {
        constexpr int kU = 4;
        const size_t g0 = (size_t)c0 * NQ;
        const int n = ncl * NQ;
        for (int e0 = tid; e0 < n; e0 += kU * NT) {
            double va[kU], vb[kU], vc[kU], vx[kU];
#pragma unroll
            for (int u = 0; u < kU; u++) {
                const int e = e0 + u * NT;
                const size_t g = g0 + (e < n ? e : 0);
                va[u] = a.ra ? a.ra[g] : 0.0;
                vb[u] = a.rb ? a.rb[g] : 0.0;
                vc[u] = a.out2 && a.rc ? a.rc[g] : 0.0;
                vx[u] = a.out2 ? a.xbar[g] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kU; u++) {
                const int e = e0 + u * NT;
                if (e >= n) break;
                const size_t g = g0 + e;
                double o = 0.0;
                if (a.ra) o = a.wa * va[u];
                if (a.rb) o = o + a.wb * vb[u];
                const double ov = o + sQ[e];
                a.out[g] = ov;
                if (fuse) sQ[e] = ov;
                if (a.out2) a.out2[g] = (a.rc ? a.wc * vc[u] : 0.0) + a.wd * vx[u];
            }
        }
    }

    // ---- the next reverse stage's adjoint traces from out (adj_trace_kernel's ----------
    // ---- arithmetic): -lambda/J and the divB adjoint per point, then per face point -----
    if (fuse) {
        if (!qn_bulk)
            for (int k = tid; k < ncl * NQ; k += NT) sQf[k] = qn[k];
        else if (tid == 0 && !mbar_wait_bounded(&sBarN, 0)) {
            atomicOr(a.err, kErrStagingTimeout);  // the copy did not complete
            sAbort = 1;
            mbar_wait_bounded(&sBarN, 0);
        }
        __syncthreads();
        if (sAbort) return;
        for (int k = tid; k < ncl * NN; k += NT) {
            double *x = sQ + 9 * k;
            double db = 0.0;
            if (a.vismode == 1) {
                const double *qq = sQf + 9 * k;
                const double ri = 1.0 / qq[0], ux = qq[1] * ri, uy = qq[2] * ri, uz = qq[3] * ri;
                db = -a.scale_next * (x[1] * qq[5] + x[2] * qq[6] + x[3] * qq[7] +
                                      x[4] * ((ux * qq[5] + uy * qq[6]) + uz * qq[7]) + x[5] * ux + x[6] * uy +
                                      x[7] * uz);
            }
            const int c = k / NN;
            const double rJ = 1.0 / sJac[c * NJ + (k - c * NN)];
            sBeta[k] = db * rJ;
#pragma unroll
            for (int m = 0; m < 9; m++) x[m] = -(a.scale_next * x[m]) * rJ;
        }
        __syncthreads();
        for (int t = tid; t < ncl * 4 * N; t += NT) {
            const int c = t / (4 * N), f = t - c * 4 * N;
            const int nfp = 1 + f % N, lf = 1 + f / N;
            int fam, line, r;
            face_point<N>(lf, nfp, fam, line, r);
            double fb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, bs = 0.0;
#pragma unroll
            for (int i = 0; i < N; i++) {
                const int sp = fam == 0 ? i + N * line : line + N * i;
                const double m = sM[r * N + i];
                const double *mu = sQ + c * NQ + 9 * sp;
#pragma unroll
                for (int k = 0; k < 9; k++) fb[k] += m * mu[k];
                bs += m * sBeta[c * NN + sp];
            }
            const double *nr = sNrm + c * NM + ML::normal(fam, line, r);
            double *o = a.at_next;
#pragma unroll
            for (int k = 0; k < 9; k++) o[adj_trace_at<N>(c0 + c, lf, nfp - 1, k)] = fb[k];
            o[adj_trace_at<N>(c0 + c, lf, nfp - 1, 9)] = bs * nr[0];
            o[adj_trace_at<N>(c0 + c, lf, nfp - 1, 10)] = bs * nr[1];
            o[adj_trace_at<N>(c0 + c, lf, nfp - 1, 11)] = 0.0;
        }
    }

    // ---- per-CTA sums of the c_h and free-stream adjoints ------------------------------
    {
        const int lane = tid & 31, wid = tid >> 5;
        constexpr int NW = NT / 32;
        double v[7] = {cbar, pb[0], pb[1], pb[2], pb[3], pb[4], pb[5]};
        // the free-stream adjoints are zero away from boundary faces: a warp
        // whose lanes all hold zero skips that sum
#pragma unroll
        for (int m = 0; m < 7; m++) {
            if (m == 0 || __any_sync(0xffffffffu, v[m] != 0.0)) v[m] = warp_sum(v[m]);
            if (lane == 0) sRed[m * 32 + wid] = v[m];
        }
        __syncthreads();
        if (tid < 7) {
            double s = 0.0;
            for (int w = 0; w < NW; w++) s += sRed[tid * 32 + w];
            a.part[(size_t)tid * gridDim.x + blockIdx.x] = s;
        }
    }
}

// ---- per-stage reduction and the running-max adjoint --------------------------------
// Sums the per-CTA partials in a fixed order; gives the adjoint accumulated
// for the running maxima to the points recorded for this stage (split
// equally among the points attaining the maximum, a shared face counted
// once); then restarts the accumulation at this stage's owner and adds this
// stage's c_h adjoint (dc/dL, dc/dU from the maxima it read).
// Where the VJP formed the next stage's adjoint traces from out, the cells
// that the records change get theirs formed again (next.at non-null).
constexpr int kRedThreads = 1024;
struct NextTraces {
    double *at;       // the next stage's adjoint traces (null: none formed yet)
    const double *q;  // its input state
    double scale;     // its lam_scale
    const double *met;
    int vismode;
};
template <int N>
static __global__ void __launch_bounds__(kRedThreads) adj_reduce_kernel(int nblk, const double *__restrict__ part,
                                                                 AdjScalars *acc, int owner_eig, int owner_um,
                                                                 double dc_dl, double dc_du,
                                                                 const AdjRec *__restrict__ recs, int *rec_n,
                                                                 int *rec_cnt, int rec_cap, double *out,
                                                                 const Ops ops, unsigned *err, NextTraces next)
{
    __shared__ double s[7][kRedThreads / 32];
    __shared__ double w[2];
    __shared__ double ps[6];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    // unrolled so that the loads of several partials are in flight at once
#pragma unroll 8
    for (int b = tid; b < nblk; b += kRedThreads)
#pragma unroll
        for (int m = 0; m < 7; m++) v[m] += part[(size_t)m * nblk + b];
#pragma unroll
    for (int m = 0; m < 7; m++) {
        v[m] = warp_sum(v[m]);
        if (lane == 0) s[m][wid] = v[m];
    }
    if (tid < 6) ps[tid] = 0.0;
    if (tid == 0) {
        const int ce = rec_cnt[0], cu = rec_cnt[1];
        w[0] = (owner_eig && ce > 0) ? acc->lam_eig / ce : 0.0;
        w[1] = (owner_um && cu > 0) ? acc->lam_um / cu : 0.0;
        if ((owner_eig && ce == 0) || (owner_um && cu == 0)) atomicOr(err, kErrAdjointMaxLost);
    }
    __syncthreads();
    const int nrec = min(*rec_n, rec_cap);
    const int NP = N + 1, NQ = 9 * N * N;
    for (int k = tid; k < nrec; k += kRedThreads) {
        const AdjRec &R = recs[k];
        const double wt = w[R.kind];
        if (wt == 0.0) continue;
        const int r = R.slot % NP, fl = R.slot / NP, line = fl % N, fam = fl / N;
        for (int sidx = 0; sidx < N; sidx++) {
            const int sp = fam == 0 ? sidx + N * line : line + N * sidx;
            const double l = wt * ops.L[r * N + sidx];
            double *o = out + (size_t)R.cell * NQ + 9 * sp;
            for (int m = 0; m < 9; m++) atomicAdd(o + m, l * R.d[m]);
        }
        for (int m = 0; m < 6; m++)
            if (R.p[m] != 0.0) atomicAdd(&ps[m], wt * R.p[m]);
    }
    __syncthreads();
    if (next.at)  // one warp per record, a lane per face point of its cell
        for (int k = wid; k < nrec; k += kRedThreads / 32) {
            const AdjRec &R = recs[k];
            if (w[R.kind] == 0.0) continue;
            for (int f = lane; f < 4 * N; f += 32)
                adj_trace_point<N>((size_t)R.cell, f, out, next.q, next.scale, next.met, next.vismode, ops, next.at);
        }
    if (tid == 0) {
        double t[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int x = 0; x < kRedThreads / 32; x++)
            for (int m = 0; m < 7; m++) t[m] += s[m][x];
        const double cb = t[0];
        for (int m = 0; m < 6; m++) acc->pbar[m] += t[1 + m] + ps[m];
        acc->cbar += cb;
        if ((owner_eig && rec_cnt[0] > 1) || (owner_um && rec_cnt[1] > 1)) acc->ties += 1.0;
        acc->lam_eig = (owner_eig ? 0.0 : acc->lam_eig) + cb * dc_dl;
        acc->lam_um = (owner_um ? 0.0 : acc->lam_um) + cb * dc_du;
        *rec_n = 0;
        rec_cnt[0] = 0;
        rec_cnt[1] = 0;
    }
}

// ---- where a running maximum was raised --------------------------------------------
// Each thread checks the recorded maxima of one CTA of the forward stage
// (cpb cells each; a block covers 128 of them).  For every CTA whose
// recorded maximum equals the stage's new running max, in ascending order,
// the block recomputes, in the exact form (its translation unit is compiled
// with -fmad=false, like the forward stage kernel), the wave speed and
// velocity maximum of its points and records the gradient of each one equal
// to the new maximum.
struct LocateArgs {
    int ncell, vismode, cpb;
    double c_h;
    Freestream fs;
    const double *q, *t_in, *met;
    const int2 *faces;
    const double *cta_max;  // per forward CTA (max eigv, max umax)
    int hit_eig, hit_um;    // which running maximum the stage raised
    double eig_max, um_max;
    RecSink rs;
};

constexpr int kLocateThreads = 128;

// the points of forward CTA `tile` (cpb cells) that attain the new maximum
template <int N>
__device__ void locate_tile(const LocateArgs &a, const Ops &ops, int tile, bool e, bool u)
{
    using ML = MetLayout<N>;
    constexpr int NQ = 9 * N * N, NP = N + 1;
    const int c0 = tile * a.cpb, ncl = min(a.cpb, a.ncell - c0);
    // flux-point state of line (fam, line) at point r, as phase A computes it
    auto interp = [&](int cell, int fam, int line, int r, double *qf) {
        const double *qc = a.q + (size_t)cell * NQ;
        for (int v = 0; v < 9; v++) {
            double acc = 0.0;
            for (int s = 0; s < N; s++) {
                const double x = fam == 0 ? qc[v + 9 * (s + N * line)] : qc[v + 9 * (line + N * s)];
                acc = acc + x * ops.L[r * N + s];
            }
            qf[v] = acc;
        }
    };
    const int nface = ncl * 4 * N, nint = ncl * 2 * N * (N - 1);
    for (int t = threadIdx.x; t < nface + nint; t += blockDim.x) {
        if (t < nface) {
            const int nfp = 1 + t % N, lf = 1 + (t / N) % 4, c = t / (4 * N);
            const int cell = c0 + c;
            int fam, line, r;
            face_point<N>(lf, nfp, fam, line, r);
            double own[9], oth[9];
            interp(cell, fam, line, r, own);
            const int2 rec = a.faces[(size_t)cell * 4 + (lf - 1)];
            const int kind = rec.y & 0xff;
            const bool pair = kind == kFaceLeft || kind == kFaceRight, own_right = kind == kFaceRight;
            const double *onrm = a.met + (size_t)cell * ML::kSize + ML::normal(fam, line, r);
            double n0 = onrm[0], n1 = onrm[1];
            int sign_l = r == 0 ? -1 : 1, sign_r = 1;
            if (pair) {
                const int pc = rec.x, plf = (rec.y >> 8) & 0xff;
                int pfam, pline, pr;
                face_point<N>(plf, N - nfp + 1, pfam, pline, pr);
                for (int k = 0; k < 9; k++) oth[k] = a.t_in[trace_at<N>(pc, plf, N - nfp, k)];
                if (!own_right) {
                    sign_r = pr == N ? -1 : 1;
                } else {
                    const double *pn = a.met + (size_t)pc * ML::kSize + ML::normal(pfam, pline, pr);
                    n0 = pn[0];
                    n1 = pn[1];
                    sign_l = pr == 0 ? -1 : 1;
                    sign_r = r == N ? -1 : 1;
                }
            } else {
                bc_ghost<double, true>(kind, own, n0, n1, a.vismode, a.fs, oth);
            }
            double Ql[9], Qr[9], Fl[9], Fr[9], eig, um = 0.0;
            for (int k = 0; k < 9; k++) {
                Ql[k] = own_right ? oth[k] : own[k];
                Qr[k] = own_right ? own[k] : oth[k];
            }
            rusanov<double, true>(Ql, Qr, Fl, Fr, n0, n1, sign_l, sign_r, a.c_h, eig, um);
            const bool he = e && eig == a.eig_max, hu = u && um == a.um_max;
            if (he || hu)
                adj_record_face(a.rs, a.fs, a.vismode, a.c_h, he, hu, cell, (fam * N + line) * NP + r, kind, own_right,
                                own, oth, n0, n1, sign_l);
        } else if (u) {
            const int k = t - nface;
            const int r = 1 + k % (N - 1), l = (k / (N - 1)) % N, f = (k / ((N - 1) * N)) % 2, c = k / (2 * N * (N - 1));
            double qf[9];
            interp(c0 + c, f, l, r, qf);
            // the velocity maximum as the forward's iflux forms it
            const double uu = qf[1] / qf[0], vv = qf[2] / qf[0], ww = qf[3] / qf[0];
            if (Max(Max(Abs(uu), Abs(vv)), Abs(ww)) == a.um_max) {
                double umd[9], qb[9], fz[9], um;
                for (int m = 0; m < 9; m++) fz[m] = qb[m] = 0.0;
                iflux_vjp(qf, a.c_h, 0.0, 0.0, fz, qb, um, umd);
                adj_record(a.rs, c0 + c, (f * N + l) * NP + r, 1, 1, umd, nullptr);
            }
        }
    }
}

template <int N>
__global__ void __launch_bounds__(kLocateThreads) adj_locate_kernel(const LocateArgs a, const Ops ops, int ntiles)
{
    __shared__ unsigned sE[kLocateThreads / 32], sU[kLocateThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    {
        const int bt = blockIdx.x * kLocateThreads + threadIdx.x;
        const bool e = bt < ntiles && a.hit_eig && a.cta_max[2 * bt] == a.eig_max;
        const bool u = bt < ntiles && a.hit_um && a.cta_max[2 * bt + 1] == a.um_max;
        const unsigned me = __ballot_sync(0xffffffffu, e), mu = __ballot_sync(0xffffffffu, u);
        if (lane == 0) {
            sE[wid] = me;
            sU[wid] = mu;
        }
    }
    __syncthreads();
    for (int w = 0; w < kLocateThreads / 32; w++)
        for (unsigned m = sE[w] | sU[w]; m; m &= m - 1) {
            const int bit = __ffs(m) - 1;
            const int tile = blockIdx.x * kLocateThreads + 32 * w + bit;
            const bool e = (sE[w] >> bit) & 1u, u = (sU[w] >> bit) & 1u;
            locate_tile<N>(a, ops, tile, e, u);
        }
}

// ---- the objective: force on the wall faces -------------------------------------------
// out[0..1] = sum over wall face points of w(line) * sign_l * f(1..2), f the
// wall face's Rusanov flux (BCFLUX wall state) at the state whose traces are
// t; one block, fixed summation order.
template <int N>
__global__ void __launch_bounds__(256) wall_force_kernel(int nw, const int2 *__restrict__ wall,
                                                         const double *__restrict__ t, const double *__restrict__ met,
                                                         int vismode, Freestream fs, const double *__restrict__ wq,
                                                         double *out)
{
    using ML = MetLayout<N>;
    __shared__ double s0[256], s1[256];
    const int tid = threadIdx.x;
    double fx = 0.0, fy = 0.0;
    for (int e = tid; e < nw * N; e += 256) {
        const int2 wf = wall[e / N];
        const int nfp = 1 + e % N, lf = wf.y;
        int fam, line, r;
        face_point<N>(lf, nfp, fam, line, r);
        const size_t own = trace_at<N>(wf.x, lf, nfp - 1, 0);  // variable k at own + k*N
        const double *nr = met + (size_t)wf.x * ML::kSize + ML::normal(fam, line, r);
        const int sign_l = r == 0 ? -1 : 1;
        double ql[9], gh[9], Fl[9], Fr[9], eig, um = 0.0;
        for (int k = 0; k < 9; k++) ql[k] = t[own + (size_t)k * N];
        bc_ghost<double, true>(kFaceWall, ql, nr[0], nr[1], vismode, fs, gh);
        rusanov<double, true>(ql, gh, Fl, Fr, nr[0], nr[1], sign_l, 1, 0.0, eig, um);
        const double w = wq[line] * (double)sign_l;
        fx += w * Fl[1];
        fy += w * Fl[2];
    }
    s0[tid] = fx;
    s1[tid] = fy;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (tid < h) {
            s0[tid] += s0[tid + h];
            s1[tid] += s1[tid + h];
        }
        __syncthreads();
    }
    if (tid == 0) {
        out[0] = s0[0];
        out[1] = s1[0];
    }
}

// launches compiled in the exact translation unit (adjoint_exact.cu)
cudaError_t launch_adj_locate(int N, int nblk, const LocateArgs &a, const Ops &ops, cudaStream_t st);
cudaError_t launch_wall_force(int N, int nw, const int2 *wall, const double *t, const double *met, int vismode,
                              const Freestream &fs, const double *wq, double *out, cudaStream_t st);

}  // namespace sddc
