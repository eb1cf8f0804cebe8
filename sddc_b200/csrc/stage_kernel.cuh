// The fused residual + RK stage kernel of the SDDC drop-in.
//
// One launch evaluates compresid (compresid.f90:1-80, compflux.f90:1-104,
// interfaceflux_all.f90:1-112, cyclocflux_all.f90:1-112, bcflux.f90:1-377,
// nablaQsp compflux.f90:107-157, the AV sensor AV.f90:1-142) for every cell
// and applies one RK stage update (iterations.f90:88-213) to it, so a stage
// reads the state once and writes it once.
//
// Work split: one CTA owns CPB consecutive cells and stages them in shared
// memory.  Phases, separated by __syncthreads:
//   A  Lagrange interpolation of every line of solution points to its N+1
//      flux points (one thread per cell x line index x variable: the xi-
//      and eta-line of one index share the operator row, so their sums go
//      through paired FMAs, FFMA2 in the mixed form);
//   B1 physical flux at the interior flux points (thread per point; the
//      FP64 and mixed forms form F n0 + G n1 directly along the normal);
//   B2 Rusanov flux at the 4N face points of each cell (thread per point).
//      The neighbour's trace at the face point comes from the trace buffer
//      (trace_at) that the stage producing the input published.  Each
//      shared face is evaluated by both of its cells, each with the
//      reference's left/right assignment, so both get the value the
//      reference scatters to them.  Its loads from global memory are issued
//      early in the FP64 and mixed forms: the face record before the
//      staging wait, the neighbour's trace and the normals before B1 (all
//      after B1 in the exact form);
//   C  divergence of the flux, gradient of (Bx, By) from the face-averaged
//      flux-point states, Powell and GLM sources (thread per solution point);
//   D  the AV smoothness sensor per cell (residual evaluations only);
//   E  in a time step, the RK stage update of each point by the thread of
//      phase C: the RK register slice was staged by TMA with the state, the
//      output is formed in shared memory and stored by one TMA bulk copy
//      while phase F runs; in a residual evaluation, the residual copy-out;
//   F  the face traces of the output state, published for the next stage.
// Running maxima of the wave speed and of the velocity (the c_h input of
// the next stage) go through atomicMax on five rotating slots, so that
// launches need no host synchronisation.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "physics.cuh"

namespace sddc {

constexpr int kMaxN = 6;

// threads per cell: one per face point (4N); the 6-cell tile gives each
// solution point its own thread where there are more of those (N*N > 4N, N
// >= 5), so that the residual phase takes one round (the fastest tile of all
// three forms at N = 5: 64 registers and 6 CTAs per SM in the mixed form)
__host__ __device__ constexpr int stage_tpc(int n, int cpb) { return cpb == 6 && n * n > 4 * n ? n * n : 4 * n; }
// threads of a CTA owning cpb cells, rounded up to whole warps
__host__ __device__ constexpr int stage_threads(int n, int cpb) { return (stage_tpc(n, cpb) * cpb + 31) / 32 * 32; }

// operators in kernel parameter space (row-major)
struct Ops {
    double L[(kMaxN + 1) * kMaxN];   // L[r*N + s]  = Lmat(r+1, s+1)
    double M[(kMaxN + 1) * kMaxN];   // M[r*N + s]  = Mmat(r+1, s+1)
    double H[(kMaxN - 1) * kMaxN];   // H[l*N + s]  = hhval(s+1, Xs_low(l+1))
    double HL[kMaxN * (kMaxN - 1)];  // HL[s*(N-1) + l] = hhval_low(l+1, Xs(s+1))
    float Lf[(kMaxN + 1) * kMaxN];
    float Mf[(kMaxN + 1) * kMaxN];
};

// how the stage output is formed from the residual r of the stage input q
enum RkKind : int {
    kRkNone = 0,     // residual evaluation only (compresid)
    kRkAxpy = 1,     // out = q + c0*r                                     RK_S5P3 stages 1-2, FiveStageRk stage 1
    kRkTwoReg = 2,   // out = (c1*a + c2*q) + c0*r                         RK_S5P3 stages 3-5, FiveStageRk stages 3-4
    kRkTwoRegT = 3,  // out = (c1*a + c2*q) + (c0*r)*c3                    FiveStageRk stage 2
    kRkFive = 4      // out = ((((c1*a + c2*b) + c3*c) + c4*q) + c5*d) + c0*r   FiveStageRk stage 5
};

// per-case data of a batch of independent cases sharing one launch
struct CaseParams {
    Freestream fs;
    double dt;
    double pad;
};

struct StageArgs {
    int ncell;
    int vismode;
    int artiv;
    int rk_kind;
    int slot_r, slot_w;
    double alpha;
    // RK coefficients of the stage: c[i] = cb[i] * dt when bit i of dt_mask
    // is set, else cb[i] (the products round as the host's would)
    double cb[8];
    unsigned dt_mask;
    double dt;                         // single case
    Freestream fs;                     // single case
    // batch: one tile per CTA (first cell, cells, case, 1 if the case's
    // first tile), per-case data and running maxima [case][5][2]; null for
    // a single case
    const int4 *tiles;
    int ntiles;
    // batch launched persistently: each CTA walks the tile table with a grid
    // stride (the table is ordered largest case first); 0: one CTA per tile
    int persistent;
    const CaseParams *cases;
    const double *__restrict__ q_in;   // (9,N,N,NCELL), never written during the stage
    double *q_out;                     // RK output (may be reg_a: FiveStageRk stage 5)
    const void *__restrict__ t_in;     // face traces of q_in, R[NCELL][4][9][N] (trace_at)
    void *t_out;                       // face traces of q_out (null: not produced)
    const double *reg_a;               // RK registers read by this stage
    const double *reg_b;
    const double *reg_c;
    const double *reg_d;
    double *resid_w;                   // residual copy (FiveStageRk stage 4 resid0)
    const double *__restrict__ met;    // packed metrics, per cell
    // the same metrics split for direct staging: normals in the arithmetic
    // type [NCELL][4N(N+1)] and Jac [NCELL][MetLayout::kJacPad]; null: the
    // kernel converts the packed record
    const void *__restrict__ nrm;
    const double *__restrict__ jac;
    int jac_inv;                       // jac holds 1/Jac (the forms other than the exact one)
    const int2 *__restrict__ faces;    // (cell, local face) records
    // remote traces of the processor faces of a decomposed run, [slot][nfp][9]
    // in the sending rank's point order (procintflux_all.f90:83-99)
    const void *__restrict__ proc_recv;
    double *maxima;                    // [5][2]: running max of eigv, umax
    double *__restrict__ sm_ind;       // (2,NCELL) AV sensor
    double *__restrict__ resid_out;    // (9,N,N,NCELL), residual evaluation only (null: not kept)
    double *__restrict__ grad_out;     // (9,2,N,N,NCELL), residual evaluation only (null: not kept)
    double *__restrict__ mon_part;     // per-CTA (sum resid^2, sum divB^2), or null
    double *__restrict__ cta_max;      // per-CTA (max eigv, max umax) of this stage, or null
    const double *__restrict__ visc;   // dFv + dGv (9,N,N,NCELL) of the viscous chain, or null (mu = eta0 = 0)
    unsigned *err_flags;
};

// packed per-cell metric record: normals of both flux-point families, then Jac
template <int N> struct MetLayout {
    static constexpr int kFam = 2 * N * (N + 1);       // doubles per family
    static constexpr int kJac = 2 * kFam;              // offset of Jac(i,j) at kJac + i + N*j
    static constexpr int kSize = (2 * kFam + N * N + 1) & ~1;
    static constexpr int kJacPad = (N * N + 1) & ~1;  // Jac per cell in the split layout (16-byte rows)
    // normal (S1(1,1:2) or S2(2,1:2)) of family f, line l, flux point r
    __host__ __device__ static constexpr int normal(int f, int l, int r) { return f * kFam + 2 * (l * (N + 1) + r); }
};

// error flag bits
enum : unsigned { kErrNonPositiveDensity = 1u, kErrNonFiniteWaveSpeed = 2u, kErrStagingTimeout = 16u };

// ---- one-dimensional TMA bulk copies into shared memory, completed on an
// mbarrier (PTX mbarrier.*, cp.async.bulk) -------------------------------------
__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_inval(unsigned long long *bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// dst and src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait (each try_wait may suspend the thread briefly); false if it
// gave up
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity)
{
    for (int it = 0; it < (1 << 22); it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// shared-memory writes of this thread made visible to the bulk-copy (async)
// proxy, before a barrier after which one thread issues a bulk store
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// shared -> global bulk store; src and dst 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_s2g(void *dst, const void *src, unsigned bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(src)),
                 "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// the issuing thread's bulk stores have read their shared-memory source
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// a hint that brings [src, src + bytes) into L2; src 16-byte aligned, bytes a
// multiple of 16, the range inside one allocation
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

template <int N, typename R, bool DIAG> struct Smem {
    static constexpr int NQ = 9 * N * N;
    static constexpr int NP = N + 1;
    static constexpr int NG = DIAG ? 9 : (sizeof(R) == 4 ? 1 : 2);  // variables of the face-averaged state kept
    // normals staged in shared memory (the mixed form's time step reads them
    // from global memory where used)
    static constexpr bool kStageNrm = DIAG || sizeof(R) == 8;
    // the mixed form's time step also keeps the block reductions at one slot
    // per warp and no AV operators (6 CTAs per SM at the 6-cell tile, N = 5)
    static constexpr bool kLean = !DIAG && sizeof(R) == 4;
    static constexpr int kF = 2 * N * NP * 9;   // R per cell: state then flux at every flux point
    static constexpr int kV = 2 * N * NP * NG;  // R per cell: face-averaged state at every flux point
    static constexpr int kLow = 2 * (N - 1) * (N - 1);
};

// Lagrange coefficient access in the arithmetic type
template <typename R> __device__ __forceinline__ R opL(const Ops &o, int i);
template <> __device__ __forceinline__ double opL<double>(const Ops &o, int i) { return o.L[i]; }
template <> __device__ __forceinline__ float opL<float>(const Ops &o, int i) { return o.Lf[i]; }
template <typename R> __device__ __forceinline__ R opM(const Ops &o, int i);
template <> __device__ __forceinline__ double opM<double>(const Ops &o, int i) { return o.M[i]; }
template <> __device__ __forceinline__ float opM<float>(const Ops &o, int i) { return o.Mf[i]; }


// two lanes of the arithmetic type through one paired FMA (FFMA2 for float,
// each component rounded as fmaf; for double two scalar multiply-adds, in
// the order a + x*y of the scalar code)
template <typename R> struct Pair2;
template <> struct Pair2<float> { using T = float2; };
template <> struct Pair2<double> { using T = double2; };
template <typename R> using P2 = typename Pair2<R>::T;
__device__ __forceinline__ float2 fma2(float2 x, float2 y, float2 z) { return __ffma2_rn(x, y, z); }
__device__ __forceinline__ double2 fma2(double2 x, double2 y, double2 z)
{
    return make_double2(z.x + x.x * y.x, z.y + x.y * y.y);
}
template <typename R> __device__ __forceinline__ P2<R> splat2(R v)
{
    P2<R> p;
    p.x = v;
    p.y = v;
    return p;
}

template <typename R> __device__ __forceinline__ P2<R> opL2(const Ops &o, int i) { return splat2<R>(opL<R>(o, i)); }
template <typename R> __device__ __forceinline__ P2<R> opM2(const Ops &o, int i) { return splat2<R>(opM<R>(o, i)); }

// local face lf (1..4), face point nfp (1..N) -> flux point (family, line, point)
// (face2fpconnec, initsetup.f90:347-383)
template <int N>
__device__ __forceinline__ void face_point(int lf, int nfp, int &fam, int &line, int &r)
{
    switch (lf) {
    case 1: fam = 1; line = nfp - 1; r = 0; break;       // (nfp, 1)
    case 2: fam = 0; line = nfp - 1; r = N; break;       // (N+1, nfp)
    case 3: fam = 1; line = N - nfp; r = N; break;       // (N-nfp+1, N+1)
    default: fam = 0; line = N - nfp; r = 0; break;      // (1, N-nfp+1)
    }
}

// face traces of a state, [cell][local face][variable][face point]: the N
// points of one face, which consecutive lanes read and write, are adjacent.
// lf is 1-based, nfp0 0-based.
template <int N> __host__ __device__ __forceinline__ size_t trace_at(size_t cell, int lf, int nfp0, int k)
{
    return ((cell * 4 + (size_t)(lf - 1)) * 9 + (size_t)k) * N + (size_t)nfp0;
}

template <typename T> __device__ __forceinline__ T warp_max(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int N, int CPB, typename R, bool DIAG> constexpr size_t stage_smem_bytes()
{
    using S = Smem<N, R, DIAG>;
    // sQ, sA, sJac; the sensor's sJz and sLow in residual evaluations only
    size_t d = (size_t)CPB * (2 * S::NQ + MetLayout<N>::kJacPad + (DIAG ? N * N + S::kLow : 0)) +
               4 * (S::kLean ? stage_threads(N, CPB) / 32 : 32) + (S::kLean ? 0 : 2 * (N - 1) * N);
    size_t r = (size_t)CPB * (S::kF + S::kV + (S::kStageNrm ? 2 * MetLayout<N>::kFam : 0)) + 2 * (N + 1) * N;
    return d * sizeof(double) + r * sizeof(R);
}

// CTAs per SM the kernel is compiled for: as many as the 228 KB of shared
// memory per SM hold (1 KB per CTA is the driver's), but no fewer than 96
// registers per thread (64 for the 6-cell tile: 6 CTAs of 160 threads at
// N = 5 in the mixed form, measured faster than 5 CTAs with 80 registers),
// and at most 8, except for the mixed form's 6-cell tile at N >= 4, which
// may take what shared memory allows up to the SM's 32 CTAs and 2048
// threads: 9 CTAs of 96 threads at N = 4 (70 registers; compiled for 8 it
// took 74, allocated as 80, and held 8; measured 5% faster)
template <int N, int CPB, typename R, bool DIAG> constexpr int stage_min_blocks()
{
    constexpr bool kWide = CPB == 6 && sizeof(R) == sizeof(float) && N >= 4;
    const int bmax = kWide ? (2048 / stage_threads(N, CPB) < 32 ? 2048 / stage_threads(N, CPB) : 32) : 8;
    int b = (int)((228 * 1024) / (stage_smem_bytes<N, CPB, R, DIAG>() + 1024));
    b = b < 1 ? 1 : (b > bmax ? bmax : b);
    while (b > 1 && 65536 / (stage_threads(N, CPB) * b) < (CPB == 6 ? 64 : 96)) b--;
    return b;
}

// One tile (CPB consecutive cells, or an entry of a batch's tile table) by
// the whole CTA; false if the staging copies timed out (the CTA stops).
// EXACT instantiations are compiled without FMA contraction (-fmad=false) in
// their own translation unit; they reproduce the reference's FP64 rounding.
template <int N, int CPB, typename R, bool DIAG, bool EXACT>
__device__ __forceinline__ bool stage_tile(const StageArgs &a, const Ops &ops, const int tile)
{
    constexpr bool EX = EXACT && (sizeof(R) == sizeof(double));
    // a time step of the forms other than the exact one needs only div B:
    // the face-averaged state is kept as its contravariant component
    // Bn = Bx n0 + By n1 at each flux point (this cell's normal), and div B
    // is the SD divergence of Bn (the same sum as the exact form's
    // d(Bx)/dx + d(By)/dy, associated differently)
    constexpr bool kBn = !DIAG && !EX;
    using S = Smem<N, R, DIAG>;
    using ML = MetLayout<N>;
    constexpr int NT = stage_threads(N, CPB);  // whole warps: the reductions use full-warp masks
    constexpr int NQ = S::NQ, NP = S::NP, NG = S::NG;
    constexpr int NN = N * N;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NM = 2 * ML::kFam;  // normals per cell
    constexpr int NJ = ML::kJacPad;
    double *sQ = reinterpret_cast<double *>(smem_raw);          // [CPB][NQ]
    double *sJac = sQ + CPB * NQ;                                // [CPB][NJ]
    double *sJz = sJac + CPB * NJ;                               // [CPB][NN]  Jz^2 for the sensor (DIAG)
    double *sLow = sJz + (DIAG ? CPB * NN : 0);                  // [CPB][kLow] (DIAG)
    constexpr int NWR = S::kLean ? NT / 32 : 32;
    double *sRed = sLow + (DIAG ? CPB * S::kLow : 0);            // [4][NWR] block reductions
    // residual (DIAG); in a time step the RK register, then the output
    double *sA = sRed + 4 * NWR;                                 // [CPB][NQ]
    double *sOpH = sA + CPB * NQ;                                // [N-1][N]  AV projection
    double *sOpHL = sOpH + (S::kLean ? 0 : (N - 1) * N);         // [N][N-1]  AV prolongation (DIAG)
    R *sNrm = reinterpret_cast<R *>(sOpHL + (S::kLean ? 0 : N * (N - 1)));  // [CPB][NM] flux-point normals
    R *sF = sNrm + (S::kStageNrm ? CPB * NM : 0);                // [CPB][2][N][NP][9]
    R *sV = sF + CPB * S::kF;                                    // [CPB][2][N][NP][NG]
    // operators read with lane-dependent indices live in shared memory
    // (divergent reads of kernel parameters serialise per address)
    R *sOpL = sV + CPB * S::kV;                                  // [NP][N]
    R *sOpM = sOpL + NP * N;                                     // [NP][N]

    const int tid = threadIdx.x;
    int c0, ncl, cs;
    bool first_tile;
    if (a.tiles) {
        const int4 tl = a.tiles[tile];
        c0 = tl.x;
        ncl = tl.y;
        cs = tl.z;
        first_tile = tl.w != 0;
    } else {
        c0 = tile * CPB;
        ncl = min(CPB, a.ncell - c0);  // cells of this CTA
        cs = 0;
        first_tile = tile == 0;
    }
    // per-case data is read where it is used (kept out of registers)
    double *maxima = a.maxima + 10 * cs;
    // the face record of this thread's face point (a cell has 4N face points
    // and at least 4N threads: one face point per thread at most), loaded
    // before the staging wait (in the exact form with the rest of the face
    // point's inputs, after B1: measured faster there)
    static_assert(stage_tpc(N, CPB) >= 4 * N, "one face point per thread at most");
    const bool has_fp = tid < ncl * 4 * N;
    int2 frec = make_int2(0, 0);
    if (!EX && has_fp) frec = __ldg(a.faces + (size_t)c0 * 4 + tid / N);

    // ---- stage the state, the metrics and the operators ------------------------
    // The tile's state slice goes to sQ, its normals to sNrm and Jac to sJac
    // (or, without the split metric arrays, its packed metric records to the
    // flux buffer, free until phase A, for conversion) and, in a stage that
    // reads one RK register, that register's slice to sA, by TMA bulk copies
    // that one thread issues when every slice is 16-byte aligned; otherwise
    // by batches of loads.
    __shared__ __align__(8) unsigned long long sBar;
    __shared__ int sAbort;
    double *sMetRaw = reinterpret_cast<double *>(sF);
    const bool split = a.nrm != nullptr;  // uniform
    const bool want_ra = !DIAG && (a.rk_kind == kRkTwoReg || a.rk_kind == kRkTwoRegT);
    const size_t qbytes = (size_t)ncl * NQ * sizeof(double);
    const size_t mbytes = split ? 0 : (size_t)ncl * ML::kSize * sizeof(double);
    const size_t nbytes = split ? (size_t)ncl * NM * sizeof(R) : 0;
    const size_t jbytes = split ? (size_t)ncl * NJ * sizeof(double) : 0;
    const double *qsrc = a.q_in + (size_t)c0 * NQ;
    const double *msrc0 = a.met + (size_t)c0 * ML::kSize;
    const R *nsrc = split ? reinterpret_cast<const R *>(a.nrm) + (size_t)c0 * NM : nullptr;
    const double *jsrc = split ? a.jac + (size_t)c0 * NJ : nullptr;
    const double *rsrc = want_ra ? a.reg_a + (size_t)c0 * NQ : nullptr;
    const bool bulk = ((uintptr_t)qsrc & 15) == 0 && (qbytes & 15) == 0 &&
                      (split ? (((uintptr_t)nsrc | (uintptr_t)jsrc | nbytes | jbytes) & 15) == 0
                             : (((uintptr_t)msrc0 | mbytes) & 15) == 0) &&
                      (!want_ra || ((uintptr_t)rsrc & 15) == 0);  // uniform in the CTA
    if (tid == 0) {
        sAbort = 0;
        if (bulk) {
            mbar_init(&sBar, 1);
            mbar_expect_tx(&sBar, (unsigned)(qbytes + mbytes + (S::kStageNrm ? nbytes : 0) + jbytes + (want_ra ? qbytes : 0)));
            bulk_g2s(sQ, qsrc, (unsigned)qbytes, &sBar);
            if (split) {
                if (S::kStageNrm) bulk_g2s(sNrm, nsrc, (unsigned)nbytes, &sBar);
                bulk_g2s(sJac, jsrc, (unsigned)jbytes, &sBar);
            } else {
                bulk_g2s(sMetRaw, msrc0, (unsigned)mbytes, &sBar);
            }
            if (want_ra) bulk_g2s(sA, rsrc, (unsigned)qbytes, &sBar);
        }
    }
    for (int k = tid; k < NP * N; k += NT) {
        sOpL[k] = opL<R>(ops, k);
        sOpM[k] = opM<R>(ops, k);
    }
    if constexpr (!S::kLean)
        for (int k = tid; k < (N - 1) * N; k += NT) {
            sOpH[k] = ops.H[k];
            sOpHL[k] = ops.HL[k];
        }
    if (!bulk) {
        // batches of kU independent loads per thread before their stores, so
        // that each thread keeps several loads in flight
        auto stage_copy = [&](auto *dst, const auto *src, int n) {
            constexpr int kU = 4;
            for (int k0 = tid; k0 < n; k0 += kU * NT) {
                decltype(+src[0]) v[kU];
#pragma unroll
                for (int u = 0; u < kU; u++) v[u] = k0 + u * NT < n ? __ldg(src + k0 + u * NT) : decltype(+src[0])(0);
#pragma unroll
                for (int u = 0; u < kU; u++)
                    if (k0 + u * NT < n) dst[k0 + u * NT] = v[u];
            }
        };
        stage_copy(sQ, qsrc, ncl * NQ);
        if (split) {
            if (S::kStageNrm) stage_copy(sNrm, nsrc, ncl * NM);
            stage_copy(sJac, jsrc, ncl * NJ);
        } else {
            stage_copy(sMetRaw, msrc0, ncl * ML::kSize);
        }
        if (want_ra) stage_copy(sA, rsrc, ncl * NQ);
    }
    const double eig_r = maxima[2 * a.slot_r], um_r = maxima[2 * a.slot_r + 1];
    // compflux.f90:6 -- running maxima of all previous stages
    const R c_h = (R)sqrt(eig_r * (eig_r - um_r));
    if (bulk && tid == 0 && !mbar_wait_bounded(&sBar, 0)) {
        // the copies did not complete: flag it, give them time to land in
        // this CTA's shared memory, and leave (every thread, below)
        atomicOr(a.err_flags, kErrStagingTimeout);
        sAbort = 1;
        mbar_wait_bounded(&sBar, 0);
    }
    __syncthreads();
    if (sAbort) return false;
    if (!split) {
        // the metric record: normals (rounded once to the arithmetic type) and Jac
        for (int k = tid; k < ncl * ML::kSize; k += NT) {
            const int c = k / ML::kSize, o = k - c * ML::kSize;
            const double v = sMetRaw[k];
            if (o < NM) { if (S::kStageNrm) sNrm[c * NM + o] = (R)v; }
            else if (o < NM + NN) sJac[c * NJ + (o - NM)] = v;
        }
        __syncthreads();
    }

    // ---- A: interpolate every line to its flux points ---------------------------
    // one thread per (cell, line index l, variable): xi-line l and eta-line l
    // together, their sums paired (both use the same operator row)
    for (int t = tid; t < ncl * N * 9; t += NT) {
        const int v = t % 9, l = (t / 9) % N, c = t / (9 * N);
        const double *q = sQ + c * NQ + v;
        P2<R> qs[N];
#pragma unroll
        for (int s = 0; s < N; s++) {
            qs[s].x = (R)q[9 * (s + N * l)];
            qs[s].y = (R)q[9 * (l + N * s)];
        }
        R *ox = sF + c * S::kF + l * NP * 9 + v;  // xi-line l (family 0)
        R *oy = ox + N * NP * 9;                   // eta-line l (family 1)
#pragma unroll
        for (int r = 0; r < NP; r++) {
            P2<R> acc = splat2<R>((R)0);
#pragma unroll
            for (int s = 0; s < N; s++) acc = fma2(qs[s], opL2<R>(ops, r * N + s), acc);
            ox[r * 9] = acc.x;
            oy[r * 9] = acc.y;
        }
    }
    __syncthreads();

    R eigmax = (R)0, umax = (R)0;
    unsigned err = 0;

    // ---- B2's inputs from global memory (the neighbour's trace or the
    // received remote trace, the normals).  The forms other than the exact
    // one gather them before B1, so that their latency overlaps the interior
    // fluxes (measured faster there; slower in the exact form, which gathers
    // them after B1)
    constexpr bool kGatherEarly = !EX;
    R other[9];
    R on0 = (R)0, on1 = (R)0, pn0 = (R)0, pn1 = (R)0;
    auto gather = [&]() {
        if (has_fp) {
            if constexpr (EX) frec = __ldg(a.faces + (size_t)c0 * 4 + tid / N);
            const int nfp = 1 + tid % N, lf = 1 + (tid / N) % 4, c = tid / (4 * N);
            int fam, line, r;
            face_point<N>(lf, nfp, fam, line, r);
            const int kind = frec.y & 0xff;
            if constexpr (S::kStageNrm) {
                const R *nrm = sNrm + c * NM + ML::normal(fam, line, r);
                on0 = nrm[0]; on1 = nrm[1];
            } else if (split) {
                const R *gn = reinterpret_cast<const R *>(a.nrm) + (size_t)(c0 + c) * NM + ML::normal(fam, line, r);
                on0 = __ldg(gn); on1 = __ldg(gn + 1);
            } else {
                const double *gn = a.met + (size_t)(c0 + c) * ML::kSize + ML::normal(fam, line, r);
                on0 = (R)__ldg(gn); on1 = (R)__ldg(gn + 1);
            }
            if (kind == kFaceProc) {
                // the received trace, remote point N+1-nfp (procintflux_all.f90:83-99)
                const R *rv = reinterpret_cast<const R *>(a.proc_recv) + ((size_t)frec.x * N + (N - nfp)) * 9;
#pragma unroll
                for (int k = 0; k < 9; k++) other[k] = rv[k];
            } else if (kind == kFaceLeft || kind == kFaceRight) {
                // partner point N-nfp+1 on the partner's local face; its trace was
                // published by the stage that produced q_in
                const int pc = frec.x, plf = (frec.y >> 8) & 0xff;
                const R *tp = reinterpret_cast<const R *>(a.t_in);
#pragma unroll
                for (int k = 0; k < 9; k++) other[k] = tp[trace_at<N>(pc, plf, N - nfp, k)];
                if (kind == kFaceRight) {
                    // the left (partner) cell's normal, from the split array or
                    // the packed record
                    int pfam, pline, pr;
                    face_point<N>(plf, N - nfp + 1, pfam, pline, pr);
                    if (split) {
                        const R *pn = reinterpret_cast<const R *>(a.nrm) + (size_t)pc * NM + ML::normal(pfam, pline, pr);
                        pn0 = __ldg(pn);
                        pn1 = __ldg(pn + 1);
                    } else {
                        const double *pn = a.met + (size_t)pc * ML::kSize + ML::normal(pfam, pline, pr);
                        pn0 = (R)__ldg(pn);
                        pn1 = (R)__ldg(pn + 1);
                    }
                }
            }
        }
    };
    if constexpr (kGatherEarly) gather();

    // ---- B1: interior flux points (inviscid_flux_interior) ---------------------
    // the normal of family f, line l, flux point r of cell c
    auto normal_at = [&](int c, int f, int l, int r, R &n0, R &n1) {
        if constexpr (S::kStageNrm) {
            const R *nrm = sNrm + c * NM + ML::normal(f, l, r);
            n0 = nrm[0]; n1 = nrm[1];
        } else if (split) {
            const R *gn = reinterpret_cast<const R *>(a.nrm) + (size_t)(c0 + c) * NM + ML::normal(f, l, r);
            n0 = __ldg(gn); n1 = __ldg(gn + 1);
        } else {
            const double *gn = a.met + (size_t)(c0 + c) * ML::kSize + ML::normal(f, l, r);
            n0 = (R)__ldg(gn); n1 = (R)__ldg(gn + 1);
        }
    };
    for (int t = tid; t < ncl * 2 * N * (N - 1); t += NT) {
        const int r = 1 + t % (N - 1), l = (t / (N - 1)) % N, f = (t / ((N - 1) * N)) % 2,
                  c = t / (2 * N * (N - 1));
        R *slot = sF + c * S::kF + ((f * N + l) * NP + r) * 9;
        R q[9];
#pragma unroll
        for (int k = 0; k < 9; k++) q[k] = slot[k];
        if (!(q[0] > (R)0)) err |= kErrNonPositiveDensity;
        R n0, n1;
        normal_at(c, f, l, r, n0, n1);
        if constexpr (EX) {
            // the reference's F and G, projected
            R F[9], G[9];
            iflux<R, EX>(q, c_h, umax, F, G);
#pragma unroll
            for (int k = 0; k < 9; k++) slot[k] = F[k] * n0 + G[k] * n1;
        } else {
            R Fn[9];
            iflux_n<R>(q, c_h, n0, n1, umax, Fn);
#pragma unroll
            for (int k = 0; k < 9; k++) slot[k] = Fn[k];
        }
        R *vs = sV + c * S::kV + ((f * N + l) * NP + r) * NG;
        if constexpr (DIAG) {
#pragma unroll
            for (int k = 0; k < 9; k++) vs[k] = q[k];
        } else {
            if constexpr (kBn) {
                vs[0] = q[5] * n0 + q[6] * n1;
            } else {
                vs[0] = q[5];
                vs[1] = q[6];
            }
        }
    }

    if constexpr (!kGatherEarly) gather();

    // ---- B2: face points (interfaceflux, CYCLOCFLUX, BCFLUX) -------------------
    if (has_fp) {
        const int nfp = 1 + tid % N, lf = 1 + (tid / N) % 4, c = tid / (4 * N);
        int fam, line, r;
        face_point<N>(lf, nfp, fam, line, r);
        R *slot = sF + c * S::kF + ((fam * N + line) * NP + r) * 9;
        R own[9], Fl[9], Fr[9];
#pragma unroll
        for (int k = 0; k < 9; k++) own[k] = slot[k];
        const int kind = frec.y & 0xff;
        R n0, n1;
        int sign_l, sign_r;
        const bool pair = kind == kFaceLeft || kind == kFaceRight;
        const bool own_right = kind == kFaceRight;
        if (kind == kFaceProc) {
            // PROCINTFLUX / CYCREMFLUX (procintflux_all.f90:104-151): this
            // cell is the left cell, with its own normal and sign_r = 1
            n0 = on0; n1 = on1;
            sign_l = r == 0 ? -1 : 1;
            sign_r = 1;
        } else if (pair) {
            int pfam, pline, pr;
            face_point<N>((frec.y >> 8) & 0xff, N - nfp + 1, pfam, pline, pr);
            if (!own_right) {
                n0 = on0; n1 = on1;
                sign_l = r == 0 ? -1 : 1;
                sign_r = pr == N ? -1 : 1;
            } else {
                n0 = pn0; n1 = pn1;
                sign_l = pr == 0 ? -1 : 1;
                sign_r = r == N ? -1 : 1;
            }
        } else {
            n0 = on0; n1 = on1;
            sign_l = r == 0 ? -1 : 1;
            sign_r = 1;
            bc_ghost<R, EX>(kind, own, n0, n1, a.vismode, a.cases ? a.cases[cs].fs : a.fs, other);
        }
        // left and right states by element-wise selects (arrays picked
        // through a pointer would live in local memory)
        R Ql[9], Qr[9];
#pragma unroll
        for (int k = 0; k < 9; k++) {
            Ql[k] = own_right ? other[k] : own[k];
            Qr[k] = own_right ? own[k] : other[k];
        }
        if (!(Ql[0] > (R)0) || !(Qr[0] > (R)0)) err |= kErrNonPositiveDensity;
        R eig_face;
        rusanov<R, EX>(Ql, Qr, Fl, Fr, n0, n1, sign_l, sign_r, c_h, eig_face, umax);
        if (!(Abs(eig_face) < (R)INFINITY)) err |= kErrNonFiniteWaveSpeed;
        if (eig_face > eigmax) eigmax = eig_face;
#pragma unroll
        for (int k = 0; k < 9; k++) slot[k] = own_right ? Fr[k] : Fl[k];
        R *vs = sV + c * S::kV + ((fam * N + line) * NP + r) * NG;
        if constexpr (DIAG) {
#pragma unroll
            for (int k = 0; k < 9; k++) vs[k] = (R)0.5 * Ql[k] + (R)0.5 * Qr[k];
        } else {
            const R bxa = (R)0.5 * Ql[5] + (R)0.5 * Qr[5], bya = (R)0.5 * Ql[6] + (R)0.5 * Qr[6];
            if constexpr (kBn) {
                vs[0] = bxa * on0 + bya * on1;  // this cell's normal
            } else {
                vs[0] = bxa;
                vs[1] = bya;
            }
        }
    }
    __syncthreads();

    // ---- C1: flux derivative along every line, in place ------------------------
    // one thread per (cell, line index, variable), the xi- and eta-line of
    // the index paired: the N+1 flux values of each line, d(i) = sum over r
    // of F(r) * M(r, i) in the reference's order (compresid.f90:14-32),
    // written over point slots 0..N-1 of the line
    for (int t = tid; t < ncl * N * 9; t += NT) {
        const int k = t % 9, l = (t / 9) % N, c = t / (9 * N);
        R *cx = sF + c * S::kF + l * NP * 9 + k;  // xi-line l
        R *cy = cx + N * NP * 9;                   // eta-line l
        P2<R> fv[NP];
#pragma unroll
        for (int r = 0; r < NP; r++) {
            fv[r].x = cx[r * 9];
            fv[r].y = cy[r * 9];
        }
#pragma unroll
        for (int i = 0; i < N; i++) {
            P2<R> d = splat2<R>((R)0);
#pragma unroll
            for (int r = 0; r < NP; r++) d = fma2(fv[r], opM2<R>(ops, r * N + i), d);
            cx[i * 9] = d.x;
            cy[i * 9] = d.y;
        }
    }
    __syncthreads();

    // ---- C: B gradient, sources and the residual per solution point ------------
    // in a time step the RK coefficients of the stage (phase E runs here)
    // formed where used, from the kernel parameters (not held in registers
    // through the phase)
    const double cdt = a.cases ? a.cases[cs].dt : a.dt;
    auto cf = [&](int i) -> double { return ((a.dt_mask >> i) & 1u) ? a.cb[i] * cdt : a.cb[i]; };
    double part_r = 0.0, part_d = 0.0;
    for (int t = tid; t < ncl * NN; t += NT) {
        const int i = t % N, j = (t / N) % N, c = t / NN;
        const int cell = c0 + c;
        const R *met = S::kStageNrm ? sNrm + c * NM : nullptr;  // used only where the normals are staged
        // Jac, or its reciprocal when the split array holds reciprocals (the
        // exact form divides by Jac, as the reference does; the others multiply
        // by 1/Jac, rounded once, on the host or here)
        const double Jv = sJac[c * NJ + i + N * j];
        double J = Jv, rJ = Jv;
        if constexpr (!EX) {
            if (!a.jac_inv) rJ = 1.0 / Jv;
        }
        const R *Fx = sF + c * S::kF + (0 * N + j) * NP * 9;  // xi-line j
        const R *Fy = sF + c * S::kF + (1 * N + i) * NP * 9;  // eta-line i
        const R *Vx = sV + c * S::kV + (0 * N + j) * NP * NG;
        const R *Vy = sV + c * S::kV + (1 * N + i) * NP * NG;
        // nablaQsp (compflux.f90:107-157) for the variables kept
        double gB[2][2] = {{0.0, 0.0}, {0.0, 0.0}};  // [Bx,By][x,y]
        // with vismode == 0 the reference never fills nablaQs; its divB
        // source then reads the zeros of the fresh allocation
        if constexpr (DIAG) {
            if (a.vismode != 1 && a.grad_out) {
                double *go = a.grad_out + (size_t)cell * (18 * NN) + 18 * (i + N * j);
                for (int k = 0; k < 18; k++) go[k] = 0.0;
            }
        }
        double divB = 0.0;
        if constexpr (kBn) {
            // div B from the contravariant component Bn at the flux points
            if (a.vismode == 1) {
                R sx = (R)0, sy = (R)0;
#pragma unroll
                for (int r = 0; r < NP; r++) sx = sx + Vx[r * NG] * sOpM[r * N + i];
#pragma unroll
                for (int r = 0; r < NP; r++) sy = sy + Vy[r * NG] * sOpM[r * N + j];
                divB = (double)(sx + sy) * rJ;
            }
        }
#pragma unroll
        for (int g = 0; g < NG; g++) {
            if (kBn || a.vismode != 1) break;
            R ax = (R)0, ay = (R)0, bx = (R)0, by = (R)0;
#pragma unroll
            for (int r = 0; r < NP; r++) {
                const R mx = Vx[r * NG + g] * sOpM[r * N + i];
                ax = ax + mx * met[ML::normal(0, j, r)];
                ay = ay + mx * met[ML::normal(0, j, r) + 1];
            }
#pragma unroll
            for (int r = 0; r < NP; r++) {
                const R my = Vy[r * NG + g] * sOpM[r * N + j];
                bx = bx + my * met[ML::normal(1, i, r)];
                by = by + my * met[ML::normal(1, i, r) + 1];
            }
            double gx, gy;
            if constexpr (EX) {
                gx = (double)(ax + bx) / J;
                gy = (double)(ay + by) / J;
            } else {
                gx = (double)(ax + bx) * rJ;
                gy = (double)(ay + by) * rJ;
            }
            const int var = DIAG ? g : g + 5;
            if (var == 5) { gB[0][0] = gx; gB[0][1] = gy; }
            if (var == 6) { gB[1][0] = gx; gB[1][1] = gy; }
            if constexpr (DIAG) {
                if (a.grad_out) {
                    double *go = a.grad_out + (size_t)cell * (18 * NN) + 18 * (i + N * j);
                    go[g] = gx;
                    go[9 + g] = gy;
                }
            }
        }
        if constexpr (!kBn) divB = gB[0][0] + gB[1][1];
        if constexpr (DIAG) {
            const double d = gB[1][0] - gB[0][1];
            sJz[c * NN + i + N * j] = d * d;
        }
        // compresid.f90:12-51 divergence of the inviscid flux: the line sums
        // of phase C1 sit in point slot i of xi-line j and slot j of eta-line i
        double res[9];
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const R dF = Fx[i * 9 + k], dG = Fy[j * 9 + k];
            res[k] = (double)(-(dF + dG));
            // the viscous chain (compresid.f90:34-49); it adds exactly +0.0
            // when mu == eta0 == 0, which only the exact form reproduces (it
            // turns a -0.0 residual into +0.0)
            if constexpr (EX) {
                if (a.vismode == 1) res[k] = res[k] + (a.visc ? a.visc[(size_t)cell * NQ + 9 * (i + N * j) + k] : 0.0);
            } else {
                if (a.vismode == 1 && a.visc) res[k] = res[k] + a.visc[(size_t)cell * NQ + 9 * (i + N * j) + k];
            }
        }
        // compresid.f90:53-78: 1/Jac, Powell 8-wave and GLM sources
        const double *q = sQ + c * NQ + 9 * (i + N * j);
        if constexpr (EX) {
#pragma unroll
            for (int k = 0; k < 9; k++) res[k] = res[k] / J;
        } else {
#pragma unroll
            for (int k = 0; k < 9; k++) res[k] = res[k] * rJ;
        }
        const double Bx = q[5], By = q[6], Bz = q[7], psi = q[8];
        double ux, uy, uz;
        if constexpr (EX) {
            ux = q[1] / q[0]; uy = q[2] / q[0]; uz = q[3] / q[0];
        } else {
            const double ri = 1.0 / q[0];
            ux = q[1] * ri; uy = q[2] * ri; uz = q[3] * ri;
        }
        res[1] = res[1] - divB * Bx;
        res[2] = res[2] - divB * By;
        res[3] = res[3] - divB * Bz;
        res[4] = res[4] - divB * ((ux * Bx + uy * By) + uz * Bz);
        res[5] = res[5] - divB * ux;
        res[6] = res[6] - divB * uy;
        res[7] = res[7] - divB * uz;
        res[8] = res[8] - a.alpha * psi;
        if (a.mon_part) {
#pragma unroll
            for (int k = 0; k < 9; k++) part_r += res[k] * res[k];
            part_d += divB * divB;
        }
        double *ap = sA + c * NQ + 9 * (i + N * j);
        if constexpr (DIAG) {
            // stage the residual for phase E's copy-out
#pragma unroll
            for (int k = 0; k < 9; k++) ap[k] = res[k];
        } else {
            // ---- E: the RK stage update of this point (iterations.f90:88-213);
            // the point's state and RK register slot are read by this thread
            // only, so the output goes to the register slot in place, and in
            // the float form a float copy over the state slot for phase F
            // element by element in order: float copy k overwrites bytes of
            // state element k/2 <= k, already read
            const size_t g = (size_t)cell * NQ + 9 * (i + N * j);
            const int kind = a.rk_kind;
            R *qf = reinterpret_cast<R *>(sQ + c * NQ + 9 * (i + N * j));
#pragma unroll
            for (int k = 0; k < 9; k++) {
                const double qk = q[k], r = res[k];
                double o;
                switch (kind) {
                case kRkAxpy: o = qk + cf(0) * r; break;
                case kRkTwoReg: o = (cf(1) * ap[k] + cf(2) * qk) + cf(0) * r; break;
                case kRkTwoRegT: o = (cf(1) * ap[k] + cf(2) * qk) + (cf(0) * r) * cf(3); break;
                default:
                    o = ((((cf(1) * a.reg_a[g + k] + cf(2) * a.reg_b[g + k]) + cf(3) * a.reg_c[g + k]) + cf(4) * qk) +
                         cf(5) * a.reg_d[g + k]) +
                        cf(0) * r;
                    break;
                }
                ap[k] = o;
                if (a.resid_w) a.resid_w[g + k] = r;
                if constexpr (sizeof(R) != sizeof(double)) qf[k] = (R)o;
            }
            fence_proxy_async();  // sA is the source of the bulk store below
        }
    }
    __syncthreads();

    // ---- D: AV smoothness sensor (comp_artificial_viscosity, AV.f90:14-83) ------
    const bool av = DIAG && a.artiv == 1 && a.vismode == 1;
    if constexpr (DIAG) if (av) {
        constexpr int NL = N - 1;
        // the sensed fields: density (v = 0) and Jz^2 (v = 1)
        auto field = [&](int c, int v, int is, int js) -> double {
            return v == 0 ? sQ[c * NQ + 9 * (is + N * js)] : sJz[c * NN + is + N * js];
        };
        // the flux buffer is free after phase C: it holds the separable
        // projection's intermediate products
        double *sTmp = reinterpret_cast<double *>(sF);  // [CPB][2][NL][N]
        if constexpr (EX) {
            // projection to the N-1 points with the reference's double sum
            for (int t = tid; t < ncl * 2 * NL * NL; t += NT) {
                const int isl = t % NL, jsl = (t / NL) % NL, v = (t / (NL * NL)) % 2, c = t / (2 * NL * NL);
                double acc = 0.0;
                for (int js = 0; js < N; js++)
#pragma unroll
                    for (int is = 0; is < N; is++)
                        acc = acc + field(c, v, is, js) * sOpH[isl * N + is] * sOpH[jsl * N + js];
                sLow[c * S::kLow + v * NL * NL + isl + NL * jsl] = acc;
            }
        } else {
            // the same projection as two one-dimensional passes
            for (int t = tid; t < ncl * 2 * NL * N; t += NT) {
                const int isl = t % NL, js = (t / NL) % N, v = (t / (NL * N)) % 2, c = t / (2 * NL * N);
                double acc = 0.0;
#pragma unroll
                for (int is = 0; is < N; is++) acc += field(c, v, is, js) * sOpH[isl * N + is];
                sTmp[((c * 2 + v) * N + js) * NL + isl] = acc;
            }
            __syncthreads();
            for (int t = tid; t < ncl * 2 * NL * NL; t += NT) {
                const int isl = t % NL, jsl = (t / NL) % NL, v = (t / (NL * NL)) % 2, c = t / (2 * NL * NL);
                double acc = 0.0;
#pragma unroll
                for (int js = 0; js < N; js++) acc += sTmp[((c * 2 + v) * N + js) * NL + isl] * sOpH[jsl * N + js];
                sLow[c * S::kLow + v * NL * NL + isl + NL * jsl] = acc;
            }
        }
        __syncthreads();
        // projection back to the solution points and the terms of the sensor
        // sum, one thread per (cell, variable, point); the face-state buffer
        // is free after phase C and holds the terms
        double *sTerm = reinterpret_cast<double *>(sV);  // [CPB][2][NN]
        if constexpr (!EX) {
            for (int t = tid; t < ncl * 2 * N * NL; t += NT) {
                const int is = t % N, jsl = (t / N) % NL, v = (t / (N * NL)) % 2, c = t / (2 * N * NL);
                const double *lo = sLow + c * S::kLow + v * NL * NL;
                double acc = 0.0;
#pragma unroll
                for (int isl = 0; isl < NL; isl++) acc += lo[isl + NL * jsl] * sOpHL[is * NL + isl];
                sTmp[((c * 2 + v) * NL + jsl) * N + is] = acc;
            }
            __syncthreads();
        }
        for (int t = tid; t < ncl * 2 * NN; t += NT) {
            const int is = t % N, js = (t / N) % N, v = (t / NN) % 2, c = t / (2 * NN);
            double hi = 0.0;
            if constexpr (EX) {
                const double *lo = sLow + c * S::kLow + v * NL * NL;
                for (int jsl = 0; jsl < NL; jsl++)
#pragma unroll
                    for (int isl = 0; isl < NL; isl++)
                        hi = hi + lo[isl + NL * jsl] * sOpHL[is * NL + isl] * sOpHL[js * NL + jsl];
            } else {
#pragma unroll
                for (int jsl = 0; jsl < NL; jsl++) hi += sTmp[((c * 2 + v) * NL + jsl) * N + is] * sOpHL[js * NL + jsl];
            }
            const double x = field(c, v, is, js);
            const double d = hi - x;
            sTerm[(c * 2 + v) * NN + is + N * js] = d * d / (x * x);
        }
        __syncthreads();
        // the sum in the reference's (js, is) order
        for (int t = tid; t < ncl * 2; t += NT) {
            const double *tm = sTerm + t * NN;
            double se = 0.0;
#pragma unroll
            for (int k = 0; k < NN; k++) se = se + tm[k];
            a.sm_ind[2 * (size_t)c0 + t] = log10(se);
        }
    }

    // ---- E: residual copy-out (residual evaluation) or the output store ---------
    const double *qout_src = nullptr;
    bool out_bulk = false;
    {
        const size_t g0 = (size_t)c0 * NQ;
        const int n = ncl * NQ;
        if constexpr (DIAG) {
            if (a.resid_out)
                for (int e = tid; e < n; e += NT) a.resid_out[g0 + e] = sA[e];
        } else {
            // the output slice (formed in sA by phase C) to q_out: one bulk
            // store issued by one thread, read from shared memory while phase
            // F runs, or coalesced stores when the slice is not 16-byte aligned
            double *dst = a.q_out + g0;
            out_bulk = (((uintptr_t)dst | (size_t)n * sizeof(double)) & 15) == 0;
            if (out_bulk) {
                if (tid == 0) bulk_s2g(dst, sA, (unsigned)(n * sizeof(double)));
            } else {
                for (int e = tid; e < n; e += NT) dst[e] = sA[e];
            }
            qout_src = sA;
        }
    }

    // ---- F: face traces of the output state for the next stage's neighbours ---
    // (the barrier after phase C orders its output before these reads: in a
    // time step nothing between them writes shared memory)
    if (!DIAG && a.t_out) {
        R *to = reinterpret_cast<R *>(a.t_out);
        // the output state: sA (double), or its float copy over the state
        // slots (9 floats at the start of each point's 9 doubles)
        constexpr int PS = sizeof(R) == sizeof(double) ? 9 : 18;  // R per point
        const R *qo = sizeof(R) == sizeof(double) ? reinterpret_cast<const R *>(qout_src)
                                                  : reinterpret_cast<const R *>(sQ);
        if constexpr (sizeof(R) == sizeof(double)) {
            // one thread per (cell, family, variable, line): the line's N
            // values give the traces at both of its ends (r = 0 and r = N),
            // each summed in order as phase A sums them (measured faster than
            // one thread per face point in the FP64 forms, slower in the mixed)
            for (int t = tid; t < ncl * 2 * 9 * N; t += NT) {
                const int line = t % N, k = (t / N) % 9, fam = (t / (9 * N)) % 2, c = t / (18 * N);
                const R *q = qo + c * (PS * NN) + (fam == 0 ? PS * N * line : PS * line) + k;
                const int stride = fam == 0 ? PS : PS * N;
                R qs[N];
#pragma unroll
                for (int s = 0; s < N; s++) qs[s] = q[stride * s];
                R a0 = (R)0, aN = (R)0;
#pragma unroll
                for (int s = 0; s < N; s++) {
                    a0 = a0 + qs[s] * sOpL[s];
                    aN = aN + qs[s] * sOpL[N * N + s];
                }
                // the faces at the line's ends (face_point inverted): xi line j
                // ends on local faces 4 (point N-j) and 2 (point j+1), eta
                // line i on local faces 1 (point i+1) and 3 (point N-i)
                const int lf0 = fam == 0 ? 4 : 1, nfp0 = fam == 0 ? N - line : line + 1;
                const int lfN = fam == 0 ? 2 : 3, nfpN = fam == 0 ? line + 1 : N - line;
                to[trace_at<N>(c0 + c, lf0, nfp0 - 1, k)] = a0;
                to[trace_at<N>(c0 + c, lfN, nfpN - 1, k)] = aN;
            }
        } else {
            for (int t = tid; t < ncl * 4 * N; t += NT) {  // one thread per face point
                const int nfp = 1 + t % N, lf = 1 + (t / N) % 4, c = t / (4 * N);
                int fam, line, r;
                face_point<N>(lf, nfp, fam, line, r);
                const R *q = qo + c * (PS * NN) + (fam == 0 ? PS * N * line : PS * line);
                const int stride = fam == 0 ? PS : PS * N;
                // variables in pairs (8-byte loads of the float copy, paired FMAs)
                P2<R> Ls[N];
#pragma unroll
                for (int s = 0; s < N; s++) Ls[s] = splat2<R>(sOpL[r * N + s]);
#pragma unroll
                for (int k = 0; k < 8; k += 2) {
                    P2<R> acc = splat2<R>((R)0);
#pragma unroll
                    for (int s = 0; s < N; s++)
                        acc = fma2(*reinterpret_cast<const P2<R> *>(q + k + stride * s), Ls[s], acc);
                    to[trace_at<N>(c0 + c, lf, nfp - 1, k)] = acc.x;
                    to[trace_at<N>(c0 + c, lf, nfp - 1, k + 1)] = acc.y;
                }
                {
                    R acc = (R)0;
#pragma unroll
                    for (int s = 0; s < N; s++) acc = acc + q[8 + stride * s] * Ls[s].x;
                    to[trace_at<N>(c0 + c, lf, nfp - 1, 8)] = acc;
                }
            }
        }
    }

    // ---- reductions ------------------------------------------------------------
    {
        const int lane = tid & 31, wid = tid >> 5;
        constexpr int NW = (NT + 31) / 32;
        double em, um;
        if constexpr (sizeof(R) == sizeof(float)) {
            // the maxima are non-negative (never raised by NaN), and
            // non-negative floats order as their bit patterns
            em = (double)__uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(eigmax)));
            um = (double)__uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(umax)));
        } else {
            em = warp_max((double)eigmax);
            um = warp_max((double)umax);
        }
        unsigned e = __reduce_or_sync(0xffffffffu, err);
        double pr = 0.0, pd = 0.0;
        if (a.mon_part) {
            pr = warp_sum(part_r);
            pd = warp_sum(part_d);
        }
        if (lane == 0) {
            sRed[wid] = em;
            sRed[NWR + wid] = um;
            sRed[2 * NWR + wid] = pr;
            sRed[3 * NWR + wid] = pd;
            if (e) atomicOr(a.err_flags, e);
        }
        __syncthreads();
        if (tid == 0) {
            double m0 = 0.0, m1 = 0.0, s0 = 0.0, s1 = 0.0;
            for (int w = 0; w < NW; w++) {
                m0 = sRed[w] > m0 ? sRed[w] : m0;
                m1 = sRed[NWR + w] > m1 ? sRed[NWR + w] : m1;
                s0 += sRed[2 * NWR + w];
                s1 += sRed[3 * NWR + w];
            }
            atomic_max_nonneg(&maxima[2 * a.slot_w], m0);
            atomic_max_nonneg(&maxima[2 * a.slot_w + 1], m1);
            if (first_tile) {  // carry the previous stages' maxima forward
                // (re-read: slot_r is not written during the stage)
                atomic_max_nonneg(&maxima[2 * a.slot_w], maxima[2 * a.slot_r]);
                atomic_max_nonneg(&maxima[2 * a.slot_w + 1], maxima[2 * a.slot_r + 1]);
            }
            if (a.mon_part) {
                a.mon_part[2 * tile] = s0;
                a.mon_part[2 * tile + 1] = s1;
            }
            if (a.cta_max) {  // where the running maxima were raised (the adjoint's argmax)
                a.cta_max[2 * tile] = m0;
                a.cta_max[2 * tile + 1] = m1;
            }
            // the bulk store must have read sA before the CTA's shared memory
            // goes or the next tile reuses it; the staging barrier is free
            if (out_bulk) bulk_wait_read();
            if (bulk) mbar_inval(&sBar);
        }
    }
    return true;
}

// a batch's stage as a persistent launch: each CTA walks the tile table with
// a grid stride
template <int N, int CPB, typename R, bool DIAG, bool EXACT>
__device__ __forceinline__ void stage_tiles_persistent(const StageArgs &a, const Ops &ops)
{
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        if (!stage_tile<N, CPB, R, DIAG, EXACT>(a, ops, t)) return;
        __syncthreads();  // tile t's last shared-memory reads before tile t+grid stages
    }
}

// One CTA per tile.  The persistent walk is a kernel of its own, so that the
// one-tile kernel carries no loop state.
template <int N, int CPB, typename R, bool DIAG, bool EXACT>
__global__ void __launch_bounds__(stage_threads(N, CPB), (stage_min_blocks<N, CPB, R, DIAG>()))
    stage_kernel(const StageArgs a, const Ops ops)
{
    stage_tile<N, CPB, R, DIAG, EXACT>(a, ops, blockIdx.x);
}

template <int N, int CPB, typename R, bool DIAG, bool EXACT>
__global__ void __launch_bounds__(stage_threads(N, CPB), (stage_min_blocks<N, CPB, R, DIAG>()))
    stage_kernel_persistent(const StageArgs a, const Ops ops)
{
    stage_tiles_persistent<N, CPB, R, DIAG, EXACT>(a, ops);
}

// Face traces of a state: T[trace_at(cell, lf, nfp, k)] = sum_s Q(k, line
// points) * L(r, s) at the flux point of local face lf, face point nfp -- the
// same interpolation, in the same order and type, as phase A and phase F.
template <int N, typename R, bool EXACT>  // EXACT: compiled with -fmad=false, like phase A
__global__ void trace_kernel(int ncell, const double *__restrict__ q, R *__restrict__ t, const Ops ops)
{
    const size_t n = (size_t)ncell * 4 * N * 9;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        // e = trace_at(c, lf, nfp - 1, k)
        const int nfp = 1 + (int)(e % N), k = (int)((e / N) % 9), lf = 1 + (int)((e / (9 * N)) % 4);
        const size_t c = e / (36 * N);
        int fam, line, r;
        face_point<N>(lf, nfp, fam, line, r);
        const double *qc = q + c * (9 * N * N);
        R acc = (R)0;
#pragma unroll
        for (int s = 0; s < N; s++) {
            const double x = fam == 0 ? qc[k + 9 * (s + N * line)] : qc[k + 9 * (line + N * s)];
            acc = acc + (R)x * opL<R>(ops, r * N + s);
        }
        t[e] = acc;
    }
}

}  // namespace sddc
