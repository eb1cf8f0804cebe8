// Host runtime of the discrete adjoint: sddc_vjp_resid and sddc_adjoint_run
// (include/sddc.h).
//
// The forward run of sddc_adjoint_run uses the exact FP64 stage kernel with
// a per-stage history of the running maxima (stage g reads slot g and writes
// slot g+1), stores the state every checkpoint_every steps, and evaluates
// the wall force after each step of the objective window.  The reverse sweep
// walks the segments backwards: it recomputes a segment's stage states from
// its checkpoint (all five stage inputs of every step, with their face
// traces), then runs the reverse stages of each step:
//   Qb4 = a54 Qb5 + c5 R'(Q4)^T Qb5      Qb2  = a52 Qb5
//   Qb3 = a43 Qb4 + c4 R'(Q3)^T Qb4      Qb0  = a40 Qb4
//   Qb2 += a32 Qb3 + c3 R'(Q2)^T Qb3     Qb0 += a30 Qb3
//   Qb1 = Qb2 + c2 R'(Q1)^T Qb2
//   Qb0 += Qb1 + c1 R'(Q0)^T Qb1 (+ dJ/dQ0 when Q0 is in the window)
// (RK_S5P3, iterations.f90:158-213, with c_k = b_k dt), each as an
// adjoint-trace launch, a VJP launch with the update as its epilogue, and a
// one-block reduction carrying the c_h adjoint.  Where a stage raised a
// running maximum, the forward stage kernel's per-CTA maxima point to the
// CTAs that hold it, and the exact-form locate kernel (adjoint_exact.cu)
// records the gradient at the points attaining it, found by equality.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "adjoint_kernel.cuh"
#include "context_impl.h"

using namespace sddc;

namespace sddc {

struct AdjWs {
    int grid = 0;            // VJP CTAs
    double *at = nullptr;    // adjoint traces, ncell * 4N * 12 (adj_trace_at)
    double *at2 = nullptr;   // the next stage's, formed by the VJP epilogue
    bool at_ready = false;   // at holds the current stage's traces already
    double *part = nullptr;  // [grid][8]
    AdjScalars *acc = nullptr;
    AdjRec *recs = nullptr;
    int rec_cap = 0;
    int *rec_n = nullptr;  // [0]: records, [1..2]: counted points per kind
    double *lam = nullptr, *qbar = nullptr, *tq = nullptr;  // sddc_vjp_resid scratch
    int2 *wall = nullptr;  // (cell, local face) of the wall faces
    int nwall = 0;
    double wq[kMaxN] = {};   // quadrature weights of the solution points
    double *host = nullptr;  // pinned read-back
    size_t bytes = 0;
};

void adjoint_free(sddc_ctx *ctx)
{
    AdjWs *w = ctx->adj;
    if (!w) return;
    void *b[] = {w->at, w->at2, w->part, w->acc, w->recs, w->rec_n, w->lam, w->qbar, w->tq, w->wall};
    for (void *p : b) cudaFree(p);
    if (w->host) cudaFreeHost(w->host);
    delete w;
    ctx->adj = nullptr;
}

}  // namespace sddc

namespace {

#define CKA(call)                                                             \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return cuda_err(ctx, e_, #call);               \
    } while (0)

template <int N>
cudaError_t launch_adj_trace_n(sddc_ctx *ctx, const double *xbar, double scale, const double *q, double *at)
{
    adj_trace_kernel<N><<<(ctx->ncell + kTraceCpb - 1) / kTraceCpb, 128, 0, ctx->stream>>>(
        ctx->ncell, ctx->p.vismode, xbar, scale, q, ctx->met, ctx->ops, at);
    return cudaGetLastError();
}

cudaError_t launch_adj_trace(sddc_ctx *ctx, const double *xbar, double scale, const double *q, double *at)
{
    switch (ctx->N) {
    case 2: return launch_adj_trace_n<2>(ctx, xbar, scale, q, at);
    case 3: return launch_adj_trace_n<3>(ctx, xbar, scale, q, at);
    case 4: return launch_adj_trace_n<4>(ctx, xbar, scale, q, at);
    case 5: return launch_adj_trace_n<5>(ctx, xbar, scale, q, at);
    default: return launch_adj_trace_n<6>(ctx, xbar, scale, q, at);
    }
}

template <int N> cudaError_t launch_vjp_n(sddc_ctx *ctx, const VjpArgs &a)
{
    constexpr int CPB = kAdjCpb;
    const size_t smem = vjp_smem_doubles<N, CPB>() * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(vjp_kernel<N, CPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    vjp_kernel<N, CPB><<<(ctx->ncell + CPB - 1) / CPB, adj_threads(N, CPB), smem, ctx->stream>>>(a, ctx->ops);
    return cudaGetLastError();
}

cudaError_t launch_vjp(sddc_ctx *ctx, const VjpArgs &a)
{
    switch (ctx->N) {
    case 2: return launch_vjp_n<2>(ctx, a);
    case 3: return launch_vjp_n<3>(ctx, a);
    case 4: return launch_vjp_n<4>(ctx, a);
    case 5: return launch_vjp_n<5>(ctx, a);
    default: return launch_vjp_n<6>(ctx, a);
    }
}

template <int N>
cudaError_t launch_adj_reduce_n(sddc_ctx *ctx, int own_eig, int own_um, double dl, double du, double *out,
                                const NextTraces &nt)
{
    AdjWs *w = ctx->adj;
    adj_reduce_kernel<N><<<1, kRedThreads, 0, ctx->stream>>>(w->grid, w->part, w->acc, own_eig, own_um, dl, du, w->recs,
                                                             w->rec_n, w->rec_n + 1, w->rec_cap, out, ctx->ops,
                                                             ctx->err_flags, nt);
    return cudaGetLastError();
}

cudaError_t launch_adj_reduce(sddc_ctx *ctx, int own_eig, int own_um, double dl, double du, double *out,
                              const NextTraces &nt)
{
    switch (ctx->N) {
    case 2: return launch_adj_reduce_n<2>(ctx, own_eig, own_um, dl, du, out, nt);
    case 3: return launch_adj_reduce_n<3>(ctx, own_eig, own_um, dl, du, out, nt);
    case 4: return launch_adj_reduce_n<4>(ctx, own_eig, own_um, dl, du, out, nt);
    case 5: return launch_adj_reduce_n<5>(ctx, own_eig, own_um, dl, du, out, nt);
    default: return launch_adj_reduce_n<6>(ctx, own_eig, own_um, dl, du, out, nt);
    }
}

Freestream ctx_fs(const sddc_ctx *ctx)
{
    return Freestream{ctx->p.rinf, ctx->p.pinf, ctx->p.uinf, ctx->p.vinf, ctx->p.bxinf, ctx->p.byinf};
}

cudaError_t wall_force(sddc_ctx *ctx, const double *t, double *out)
{
    const AdjWs *w = ctx->adj;
    return launch_wall_force(ctx->N, w->nwall, w->wall, t, ctx->met, ctx->p.vismode, ctx_fs(ctx), ctx->wq, out,
                             ctx->stream);
}

int ensure_ws(sddc_ctx *ctx)
{
    if (ctx->adj) return SDDC_OK;
    auto *w = new AdjWs();
    ctx->adj = w;
    const size_t nc = ctx->ncell, N = ctx->N;
    w->grid = (ctx->ncell + kAdjCpb - 1) / kAdjCpb;
    w->rec_cap = (int)std::min<size_t>(nc * 4 * N, (size_t)1 << 24);
    const size_t tr = nc * 4 * N * 9;
    int rc;
    if ((rc = alloc(ctx, (void **)&w->at, nc * 4 * N * 12 * sizeof(double), "adjoint traces")) ||
        (rc = alloc(ctx, (void **)&w->at2, nc * 4 * N * 12 * sizeof(double), "adjoint traces")) ||
        (rc = alloc(ctx, (void **)&w->part, (size_t)w->grid * 8 * sizeof(double), "adjoint partials")) ||
        (rc = alloc(ctx, (void **)&w->acc, sizeof(AdjScalars), "adjoint scalars")) ||
        (rc = alloc(ctx, (void **)&w->recs, (size_t)w->rec_cap * sizeof(AdjRec), "argmax records")) ||
        (rc = alloc(ctx, (void **)&w->rec_n, 4 * sizeof(int), "record counters")) ||
        (rc = alloc(ctx, (void **)&w->lam, ctx->nq * sizeof(double), "adjoint input")) ||
        (rc = alloc(ctx, (void **)&w->qbar, ctx->nq * sizeof(double), "adjoint output")) ||
        (rc = alloc(ctx, (void **)&w->tq, tr * sizeof(double), "traces")))
        return rc;
    w->bytes = nc * 4 * N * 12 * 8 + (size_t)w->grid * 64 + sizeof(AdjScalars) + (size_t)w->rec_cap * sizeof(AdjRec) +
               16 + 2 * ctx->nq * 8 + tr * 8;
    CKA(cudaMallocHost((void **)&w->host, 64 * sizeof(double)));
    CKA(cudaMemsetAsync(w->rec_n, 0, 4 * sizeof(int), ctx->stream));
    CKA(cudaMemcpyAsync(w->host, ctx->wq, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    // the wall faces from the connectivity records
    std::vector<int2> fr(nc * 4), wl;
    CKA(cudaMemcpyAsync(fr.data(), ctx->faces, fr.size() * sizeof(int2), cudaMemcpyDeviceToHost, ctx->stream));
    CKA(cudaStreamSynchronize(ctx->stream));
    for (size_t k = 0; k < N; k++) w->wq[k] = w->host[k];
    for (size_t k = 0; k < fr.size(); k++)
        if ((fr[k].y & 0xff) == kFaceWall) wl.push_back(make_int2((int)(k / 4), (int)(k % 4) + 1));
    w->nwall = (int)wl.size();
    if ((rc = alloc(ctx, (void **)&w->wall, std::max<size_t>(wl.size(), 1) * sizeof(int2), "wall faces"))) return rc;
    w->bytes += std::max<size_t>(wl.size(), 1) * sizeof(int2);
    if (!wl.empty())
        CKA(cudaMemcpyAsync(w->wall, wl.data(), wl.size() * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
    CKA(cudaStreamSynchronize(ctx->stream));
    return SDDC_OK;
}

int check_adjoint_ctx(sddc_ctx *ctx)
{
    int rc = ready(ctx);
    if (rc) return rc;
    if (ctx->ncase) return set_err(ctx, SDDC_ESTATE, "the adjoint runs one case (no batch)");
    if (ctx->p.k_stage != 3) return set_err(ctx, SDDC_EINVAL, "the adjoint differentiates RK_S5P3 (k_stage = 3)");
    if (ctx->visc) return set_err(ctx, SDDC_EINVAL, "the adjoint differentiates the ideal chain (mu = eta0 = 0)");
    if (!ctx->ibfproc.empty() || ctx->exch)
        return set_err(ctx, SDDC_ESTATE, "the adjoint runs a whole case on one GPU (no processor faces)");
    return ensure_ws(ctx);
}

// one reverse stage: the adjoint traces, the VJP with its RK epilogue, and
// the reduction (record weights, c_h adjoint carried to the owner stage)
struct RevStage {
    const double *q, *t;  // stage input state and its face traces
    const double *xbar;   // adjoint of the stage output (null: objective seeds only)
    double scale;         // c_k of the stage
    const double *ra = nullptr, *rb = nullptr;
    double wa = 0.0, wb = 0.0;
    double *out = nullptr;
    const double *rc = nullptr;
    double wc = 0.0, wd = 0.0;
    double *out2 = nullptr;
    double sx = 0.0, sy = 0.0;
    double L = 0.0, U = 0.0, Lnext = 0.0, Unext = 0.0;  // maxima read by the stage and after it
    const double *cta_max = nullptr;  // the forward stage's per-CTA maxima
    bool reduce = true;
    // the next reverse stage (whose output adjoint is out): its input state and
    // c_k, for its adjoint traces in this stage's epilogue (null: not known yet)
    const double *q_next = nullptr;
    double scale_next = 0.0;
};

int reverse_stage(sddc_ctx *ctx, const RevStage &s)
{
    AdjWs *w = ctx->adj;
    if (s.xbar && !w->at_ready) CKA(launch_adj_trace(ctx, s.xbar, s.scale, s.q, w->at));
    double *at_next = s.q_next ? w->at2 : nullptr;
    const double c_h = std::sqrt(s.L * (s.L - s.U));
    VjpArgs a{};
    a.ncell = ctx->ncell;
    a.vismode = ctx->p.vismode;
    a.alpha = 2.0;  // initsetup.f90:165
    a.c_h = c_h;
    a.fs = ctx_fs(ctx);
    a.q = s.q;
    a.t_in = s.t;
    a.xbar = s.xbar;
    a.lam_scale = s.scale;
    a.at = w->at;
    a.met = ctx->met;
    if (ctx->nrm_double && !ctx->jac_inv) {  // an exact context holds double normals and Jac
        a.nrm = static_cast<const double *>(ctx->nrm);
        a.jac = ctx->jac;
    }
    a.faces = ctx->faces;
    a.ra = s.ra;
    a.rb = s.rb;
    a.wa = s.wa;
    a.wb = s.wb;
    a.out = s.out;
    a.rc = s.rc;
    a.wc = s.wc;
    a.wd = s.wd;
    a.out2 = s.out2;
    a.sx = s.sx;
    a.sy = s.sy;
    for (int i = 0; i < kMaxN; i++) a.wq[i] = w->wq[i];
    a.part = w->part;
    a.err = ctx->err_flags;
    a.q_next = s.q_next;
    a.scale_next = s.scale_next;
    a.at_next = at_next;
    CKA(launch_vjp(ctx, a));
    // the traces formed for the next stage become the current ones (the
    // reduction below corrects the cells its records change)
    if (at_next) std::swap(w->at, w->at2);
    w->at_ready = at_next != nullptr;
    const bool own_eig = s.reduce && s.Lnext > s.L, own_um = s.reduce && s.Unext > s.U;
    if (own_eig || own_um) {  // record where the stage raised a running maximum
        LocateArgs l{};
        l.ncell = ctx->ncell;
        l.vismode = ctx->p.vismode;
        l.cpb = ctx->cpb;
        l.c_h = c_h;
        l.fs = a.fs;
        l.q = s.q;
        l.t_in = s.t;
        l.met = ctx->met;
        l.faces = ctx->faces;
        l.cta_max = s.cta_max;
        l.hit_eig = own_eig;
        l.hit_um = own_um;
        l.eig_max = s.Lnext;
        l.um_max = s.Unext;
        l.rs = RecSink{w->recs, w->rec_cap, w->rec_n, w->rec_n + 1, ctx->err_flags};
        CKA(launch_adj_locate(ctx->N, (ctx->ncell + ctx->cpb - 1) / ctx->cpb, l, ctx->ops, ctx->stream));
    }
    if (!s.reduce) return SDDC_OK;
    double dl = 0.0, du = 0.0;
    if (c_h > 0.0) {  // c = sqrt(L (L - U))
        dl = (2.0 * s.L - s.U) / (2.0 * c_h);
        du = -s.L / (2.0 * c_h);
    }
    const NextTraces nt{at_next, s.q_next, s.scale_next, ctx->met, ctx->p.vismode};
    CKA(launch_adj_reduce(ctx, own_eig, own_um, dl, du, s.out, nt));
    return SDDC_OK;
}

int adjoint_flags(sddc_ctx *ctx)
{
    CKA(cudaMemcpyAsync(ctx->adj->host, ctx->err_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CKA(cudaStreamSynchronize(ctx->stream));
    unsigned f;
    std::memcpy(&f, ctx->adj->host, sizeof(unsigned));
    if (f & (kErrAdjointMaxLost | kErrAdjointRecords)) {
        CKA(cudaMemsetAsync(ctx->err_flags, 0, sizeof(unsigned), ctx->stream));
        CKA(cudaStreamSynchronize(ctx->stream));
        if (f & kErrAdjointRecords) return set_err(ctx, SDDC_ENUMERIC, "adjoint: more points attain a running maximum than the record buffer holds");
        return set_err(ctx, SDDC_ENUMERIC, "adjoint: no point reproduces a recorded running maximum");
    }
    return check_flags(ctx);
}

// the RK_S5P3 stage table (iterations.f90:179-210): output = (c1*ra + c2*q) + c0*dt*R(q)
struct FwdStage {
    int kind, in, out, ra;
    double c[3];
};
const FwdStage kS5P3[5] = {{kRkAxpy, 0, 1, -1, {B10, 0, 0}},
                           {kRkAxpy, 1, 2, -1, {B21, 0, 0}},
                           {kRkTwoReg, 2, 3, 0, {B32, A30, A32}},
                           {kRkTwoReg, 3, 4, 0, {B43, A40, A43}},
                           {kRkTwoReg, 4, 5, 2, {B54, A52, A54}}};

// forward steps through the stage store: S[5m + k] is the input of stage k
// of local step m (S[5m] its start state), T the matching face traces;
// stage g = 5*step + k reads running-max slot g of hist and writes slot g+1
// (a rerun writes the values already there); launched on st
int forward_steps(sddc_ctx *ctx, double dt, int step0, int nsteps, double *const *S, double *const *T, double *hist,
                  int n1, int n2, double *force, double *cmax, cudaStream_t st)
{
    const size_t fgrid = (ctx->ncell + ctx->cpb - 1) / ctx->cpb;
    for (int m = 0; m < nsteps; m++) {
        for (int k = 0; k < 5; k++) {
            const FwdStage &f = kS5P3[k];
            StageArgs a = base_args(ctx);
            a.maxima = hist;
            a.dt = dt;
            a.rk_kind = f.kind;
            a.q_in = S[5 * m + f.in];
            a.t_in = T[5 * m + f.in];
            a.q_out = S[5 * m + f.out];
            a.t_out = T[5 * m + f.out];
            a.reg_a = f.ra >= 0 ? S[5 * m + f.ra] : nullptr;
            a.cb[0] = f.c[0];
            a.cb[1] = f.c[1];
            a.cb[2] = f.c[2];
            a.dt_mask = 1u;
            const int g = 5 * (step0 + m) + k;
            a.slot_r = g;
            a.slot_w = g + 1;
            a.cta_max = cmax + (size_t)(5 * m + k) * 2 * fgrid;
            if (!ctx->nrm_double || ctx->jac_inv) {
                // the exact kernel reads double normals and Jac itself: convert
                // the packed record
                a.nrm = nullptr;
                a.jac = nullptr;
                a.jac_inv = 0;
            }
            CKA(launch_stage_exact(ctx->N, ctx->cpb, false, a, ctx->ops, st));
        }
        const int n = step0 + m + 1;
        if (force && n >= n1 && n <= n2) CKA(wall_force(ctx, T[5 * (m + 1)], force + 2 * n));
    }
    return SDDC_OK;
}

// device buffers of one run, released on every exit path
struct RunBufs {
    std::vector<void *> p;
    size_t bytes = 0;
    ~RunBufs()
    {
        for (void *x : p) cudaFree(x);
    }
    int get(sddc_ctx *ctx, double **out, size_t n, const char *what)
    {
        int rc = alloc(ctx, (void **)out, n * sizeof(double), what);
        if (rc == SDDC_OK) {
            p.push_back(*out);
            bytes += n * sizeof(double);
        }
        return rc;
    }
};

}  // namespace

extern "C" int sddc_vjp_resid(sddc_ctx *ctx, const double *Rbar, double *Qbar, double *parbar)
{
    if (!ctx || !Rbar || !Qbar) return set_err(ctx, SDDC_EINVAL, "sddc_vjp_resid: NULL argument");
    int rc = check_adjoint_ctx(ctx);
    if (rc) return rc;
    AdjWs *w = ctx->adj;
    CKA(cudaMemcpyAsync(w->lam, Rbar, ctx->nq * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CKA(launch_trace_exact(ctx->N, ctx->ncell, ctx->reg[0], w->tq, ctx->ops, ctx->stream));
    CKA(cudaMemcpyAsync(w->host, ctx->maxima + 2 * ctx->slot, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CKA(cudaMemsetAsync(w->acc, 0, sizeof(AdjScalars), ctx->stream));
    CKA(cudaStreamSynchronize(ctx->stream));
    w->at_ready = false;
    RevStage s;
    s.q = ctx->reg[0];
    s.t = w->tq;
    s.xbar = w->lam;
    s.scale = 1.0;
    s.out = w->qbar;
    s.L = s.Lnext = w->host[0];
    s.U = s.Unext = w->host[1];
    if ((rc = reverse_stage(ctx, s))) return rc;
    CKA(cudaMemcpyAsync(Qbar, w->qbar, ctx->nq * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    AdjScalars acc;
    CKA(cudaMemcpyAsync(w->host, w->acc, sizeof(AdjScalars), cudaMemcpyDeviceToHost, ctx->stream));
    CKA(cudaStreamSynchronize(ctx->stream));
    std::memcpy(&acc, w->host, sizeof(AdjScalars));
    if (parbar) {
        parbar[0] = acc.cbar;
        for (int m = 0; m < 6; m++) parbar[1 + m] = acc.pbar[m];
    }
    return adjoint_flags(ctx);
}

extern "C" int sddc_adjoint_run(sddc_ctx *ctx, const sddc_adjoint_opts *o, double *obj, double *Qbar0,
                                double *parbar, sddc_adjoint_stats *stats)
{
    if (!ctx || !o) return set_err(ctx, SDDC_EINVAL, "sddc_adjoint_run: NULL argument");
    if (!(o->dt > 0.0)) return set_err(ctx, SDDC_EINVAL, "dt must be positive");
    if (o->nsteps < 1) return set_err(ctx, SDDC_EINVAL, "nsteps must be positive");
    if (o->n1 < 0 || o->n1 > o->n2 || o->n2 > o->nsteps)
        return set_err(ctx, SDDC_EINVAL, "the window must satisfy 0 <= n1 <= n2 <= nsteps");
    if (o->checkpoint_every < 0) return set_err(ctx, SDDC_EINVAL, "checkpoint_every must be >= 0");
    const double U2 = ctx->p.uinf * ctx->p.uinf + ctx->p.vinf * ctx->p.vinf;
    if (!(ctx->p.rinf > 0.0) || !(U2 > 0.0))
        return set_err(ctx, SDDC_EINVAL, "C_D and C_L need rinf > 0 and a nonzero free-stream velocity");
    int rc = check_adjoint_ctx(ctx);
    if (rc) return rc;
    AdjWs *w = ctx->adj;
    if (w->nwall == 0 && (o->w_drag != 0.0 || o->w_lift != 0.0))
        return set_err(ctx, SDDC_EINVAL, "the objective needs wall faces (IBFWAL)");
    const bool grad = Qbar0 || parbar;
    const int ns = o->nsteps, K = o->checkpoint_every ? o->checkpoint_every : 20;
    const int nseg = (ns + K - 1) / K;
    const int segmax = std::min(K, ns);
    const size_t nq = ctx->nq, tr = (size_t)ctx->ncell * 4 * ctx->N * 9;
    const double D = o->diameter > 0.0 ? o->diameter : 1.0;

    RunBufs rb;
    std::vector<double *> ckpt(nseg), S(5 * segmax + 1), T(5 * segmax + 1);
    double *hist = nullptr, *force = nullptr, *cmax = nullptr, *A[6] = {};
    for (int s = 0; s < nseg; s++)
        if ((rc = rb.get(ctx, &ckpt[s], nq, "checkpoint"))) return rc;
    for (int i = 0; i <= 5 * segmax; i++)
        if ((rc = rb.get(ctx, &S[i], nq, "stage state")) || (rc = rb.get(ctx, &T[i], tr, "stage traces"))) return rc;
    if ((rc = rb.get(ctx, &hist, 2 * ((size_t)5 * ns + 1), "running maxima")) ||
        (rc = rb.get(ctx, &force, 2 * ((size_t)ns + 1), "wall force")) ||
        (rc = rb.get(ctx, &cmax, (size_t)5 * segmax * 2 * ((ctx->ncell + ctx->cpb - 1) / ctx->cpb), "CTA maxima")))
        return rc;
    if (grad)
        for (auto &a : A)
            if ((rc = rb.get(ctx, &a, nq, "adjoint register"))) return rc;
    // the reverse sweep recomputes segment s - 1 into a second stage store
    // (with its own per-CTA maxima) on a second stream while it reverses
    // segment s from the first
    const bool overlap = grad && nseg > 1;
    std::vector<double *> S2(overlap ? 5 * segmax + 1 : 0), T2(overlap ? 5 * segmax + 1 : 0);
    double *cmax2 = nullptr;
    if (overlap) {
        for (int i = 0; i <= 5 * segmax; i++)
            if ((rc = rb.get(ctx, &S2[i], nq, "stage state")) || (rc = rb.get(ctx, &T2[i], tr, "stage traces"))) return rc;
        if ((rc = rb.get(ctx, &cmax2, (size_t)5 * segmax * 2 * ((ctx->ncell + ctx->cpb - 1) / ctx->cpb), "CTA maxima")))
            return rc;
    }

    // streams and events of the overlapped reverse sweep; on every exit the
    // streams are drained (before the run buffers go) and the context's
    // stream is restored
    struct Overlap {
        sddc_ctx *ctx = nullptr;
        cudaStream_t saved = nullptr, rs = nullptr, hs = nullptr;  // recompute stream, reverse stream
        cudaEvent_t ready[2] = {}, freed[2] = {}, join = nullptr;
        ~Overlap()
        {
            if (rs) cudaStreamSynchronize(rs);
            if (hs) cudaStreamSynchronize(hs);
            if (saved) ctx->stream = saved;
            for (cudaEvent_t e : {ready[0], ready[1], freed[0], freed[1], join})
                if (e) cudaEventDestroy(e);
            if (rs) cudaStreamDestroy(rs);
            if (hs) cudaStreamDestroy(hs);
        }
    } ov;
    ov.ctx = ctx;

    cudaEvent_t ev[3];
    for (auto &e : ev) CKA(cudaEventCreate(&e));
    struct EvGuard {
        cudaEvent_t *e;
        ~EvGuard()
        {
            for (int i = 0; i < 3; i++) cudaEventDestroy(e[i]);
        }
    } evg{ev};

    // ---- forward run -------------------------------------------------------------
    CKA(cudaMemsetAsync(hist, 0, 2 * ((size_t)5 * ns + 1) * sizeof(double), ctx->stream));
    CKA(cudaMemcpyAsync(hist, ctx->maxima + 2 * ctx->slot, 2 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CKA(cudaMemsetAsync(force, 0, 2 * ((size_t)ns + 1) * sizeof(double), ctx->stream));
    CKA(cudaMemcpyAsync(ckpt[0], ctx->reg[0], nq * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CKA(cudaEventRecord(ev[0], ctx->stream));
    for (int s = 0; s < nseg; s++) {
        const int step0 = s * K, nst = std::min(K, ns - step0);
        CKA(cudaMemcpyAsync(S[0], ckpt[s], nq * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        CKA(launch_trace_exact(ctx->N, ctx->ncell, S[0], T[0], ctx->ops, ctx->stream));
        if (s == 0 && o->n1 == 0) CKA(wall_force(ctx, T[0], force));
        if ((rc = forward_steps(ctx, o->dt, step0, nst, S.data(), T.data(), hist, o->n1, o->n2, force, cmax,
                                ctx->stream)))
            return rc;
        if (s + 1 < nseg)
            CKA(cudaMemcpyAsync(ckpt[s + 1], S[5 * nst], nq * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    }
    CKA(cudaEventRecord(ev[1], ctx->stream));
    std::vector<double> H(2 * ((size_t)5 * ns + 1)), Fh(2 * ((size_t)ns + 1));
    CKA(cudaMemcpyAsync(H.data(), hist, H.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CKA(cudaMemcpyAsync(Fh.data(), force, Fh.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CKA(cudaStreamSynchronize(ctx->stream));
    if ((rc = check_flags(ctx))) return rc;

    // objective: C = 2 F . e / (rho |U|^2 D), e the free-stream direction (drag)
    // or its left normal (lift)
    const double Um = std::sqrt(U2), dx = ctx->p.uinf / Um, dy = ctx->p.vinf / Um;
    const double norm = 2.0 / (ctx->p.rinf * U2 * D);
    const int M = o->n2 - o->n1 + 1;
    double cd = 0.0, cl = 0.0;
    for (int n = o->n1; n <= o->n2; n++) {
        cd += norm * (Fh[2 * n] * dx + Fh[2 * n + 1] * dy);
        cl += norm * (-Fh[2 * n] * dy + Fh[2 * n + 1] * dx);
    }
    cd /= M;
    cl /= M;
    if (obj) {
        obj[0] = o->w_drag * cd + o->w_lift * cl;
        obj[1] = cd;
        obj[2] = cl;
    }
    // dJ/dF at a state of the window
    const double sx = norm / M * (o->w_drag * dx - o->w_lift * dy);
    const double sy = norm / M * (o->w_drag * dy + o->w_lift * dx);

    int owners = 0, ties = 0;
    float rev_ms = 0.0f;
    if (grad) {
        // ---- reverse sweep ---------------------------------------------------------
        if (overlap) {
            int lo = 0, hi = 0;
            CKA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            CKA(cudaStreamCreateWithPriority(&ov.rs, cudaStreamNonBlocking, lo));
            CKA(cudaStreamCreateWithPriority(&ov.hs, cudaStreamNonBlocking, hi));
            for (cudaEvent_t *e : {&ov.ready[0], &ov.ready[1], &ov.freed[0], &ov.freed[1], &ov.join})
                CKA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
            // the reverse sweep on the high-priority stream (the forward run
            // is complete: the stream was synchronised above)
            ov.saved = ctx->stream;
            ctx->stream = ov.hs;
        }
        CKA(cudaMemsetAsync(w->acc, 0, sizeof(AdjScalars), ctx->stream));
        CKA(cudaMemsetAsync(w->rec_n, 0, 4 * sizeof(int), ctx->stream));
        w->at_ready = false;
        double *Ab[6] = {A[0], A[1], A[2], A[3], A[4], A[5]};
        // the final state: dJ/dQ(n = nsteps)
        {
            const int last = ns - (nseg - 1) * K;
            RevStage r;
            r.q = S[5 * last];
            r.t = T[5 * last];
            r.xbar = nullptr;
            r.scale = 0.0;
            r.out = Ab[5];
            const bool in = ns >= o->n1 && ns <= o->n2;
            r.sx = in ? sx : 0.0;
            r.sy = in ? sy : 0.0;
            r.reduce = false;
            r.q_next = S[5 * last - 1];  // stage 5 of the last step: input Q4
            r.scale_next = B54 * o->dt;
            if ((rc = reverse_stage(ctx, r))) return rc;
        }
        // the two stage stores: store cur holds the segment being reversed,
        // the other one receives the next (earlier) segment on the recompute
        // stream.  The reverse sweep runs on a stream of the highest priority,
        // so that the recompute takes only the SMs it leaves idle (the
        // one-block reductions, the tails of its launches).
        std::vector<double *> *SS[2] = {&S, &S2}, *TT[2] = {&T, &T2};
        double *CM[2] = {cmax, cmax2};
        int cur = 0;
        auto recompute = [&](int seg, int buf, cudaStream_t st) -> int {
            const int s0 = seg * K, n = std::min(K, ns - s0);
            CKA(cudaMemcpyAsync((*SS[buf])[0], ckpt[seg], nq * sizeof(double), cudaMemcpyDeviceToDevice, st));
            CKA(launch_trace_exact(ctx->N, ctx->ncell, (*SS[buf])[0], (*TT[buf])[0], ctx->ops, st));
            return forward_steps(ctx, o->dt, s0, n, SS[buf]->data(), TT[buf]->data(), hist, 0, -1, nullptr, CM[buf], st);
        };
        for (int s = nseg - 1; s >= 0; s--) {
            const int step0 = s * K, nst = std::min(K, ns - step0);
            if (overlap && s > 0) {  // segment s - 1 into the other store, once segment s + 1 has left it
                if (s < nseg - 1) CKA(cudaStreamWaitEvent(ov.rs, ov.freed[1 - cur], 0));
                if ((rc = recompute(s - 1, 1 - cur, ov.rs))) return rc;
                CKA(cudaEventRecord(ov.ready[1 - cur], ov.rs));
            }
            if (s < nseg - 1) CKA(cudaStreamWaitEvent(ctx->stream, ov.ready[cur], 0));
            double *const *S_ = SS[cur]->data(), *const *T_ = TT[cur]->data();
            double *cmax_ = CM[cur];
            for (int m = nst - 1; m >= 0; m--) {
                const int n = step0 + m, i = 5 * m;
                const size_t fgrid = (ctx->ncell + ctx->cpb - 1) / ctx->cpb;
                auto maxima = [&](RevStage &r, int k) {
                    const size_t g = (size_t)5 * n + k;
                    r.cta_max = cmax_ + (size_t)(5 * m + k) * 2 * fgrid;
                    r.L = H[2 * g];
                    r.U = H[2 * g + 1];
                    r.Lnext = H[2 * g + 2];
                    r.Unext = H[2 * g + 3];
                    if (r.Lnext > r.L || r.Unext > r.U) owners++;
                };
                RevStage r5;  // stage 5: input Q4 = S_[i+4]
                r5.q = S_[i + 4]; r5.t = T_[i + 4]; r5.xbar = Ab[5]; r5.scale = B54 * o->dt;
                r5.ra = Ab[5]; r5.wa = A54; r5.out = Ab[4]; r5.wd = A52; r5.out2 = Ab[2];
                r5.q_next = S_[i + 3]; r5.scale_next = B43 * o->dt;
                maxima(r5, 4);
                if ((rc = reverse_stage(ctx, r5))) return rc;
                RevStage r4;  // stage 4: input Q3 = S_[i+3]
                r4.q = S_[i + 3]; r4.t = T_[i + 3]; r4.xbar = Ab[4]; r4.scale = B43 * o->dt;
                r4.ra = Ab[4]; r4.wa = A43; r4.out = Ab[3]; r4.wd = A40; r4.out2 = Ab[0];
                r4.q_next = S_[i + 2]; r4.scale_next = B32 * o->dt;
                maxima(r4, 3);
                if ((rc = reverse_stage(ctx, r4))) return rc;
                RevStage r3;  // stage 3: input Q2 = S_[i+2]
                r3.q = S_[i + 2]; r3.t = T_[i + 2]; r3.xbar = Ab[3]; r3.scale = B32 * o->dt;
                r3.ra = Ab[2]; r3.wa = 1.0; r3.rb = Ab[3]; r3.wb = A32; r3.out = Ab[2];
                r3.rc = Ab[0]; r3.wc = 1.0; r3.wd = A30; r3.out2 = Ab[0];
                r3.q_next = S_[i + 1]; r3.scale_next = B21 * o->dt;
                maxima(r3, 2);
                if ((rc = reverse_stage(ctx, r3))) return rc;
                RevStage r2;  // stage 2: input Q1 = S_[i+1]
                r2.q = S_[i + 1]; r2.t = T_[i + 1]; r2.xbar = Ab[2]; r2.scale = B21 * o->dt;
                r2.ra = Ab[2]; r2.wa = 1.0; r2.out = Ab[1];
                r2.q_next = S_[i]; r2.scale_next = B10 * o->dt;
                maxima(r2, 1);
                if ((rc = reverse_stage(ctx, r2))) return rc;
                RevStage r1;  // stage 1: input Q0 = S_[i], the state after n steps
                r1.q = S_[i]; r1.t = T_[i]; r1.xbar = Ab[1]; r1.scale = B10 * o->dt;
                r1.ra = Ab[0]; r1.wa = 1.0; r1.rb = Ab[1]; r1.wb = 1.0; r1.out = Ab[0];
                const bool in = n >= o->n1 && n <= o->n2;
                r1.sx = in ? sx : 0.0;
                r1.sy = in ? sy : 0.0;
                if (m > 0) {  // stage 5 of step n - 1 (its input is recomputed with the segment)
                    r1.q_next = S_[i - 1];
                    r1.scale_next = B54 * o->dt;
                }
                maxima(r1, 0);
                if ((rc = reverse_stage(ctx, r1))) return rc;
                std::swap(Ab[0], Ab[5]);  // the adjoint of the state after n steps
            }
            if (overlap) CKA(cudaEventRecord(ov.freed[cur], ctx->stream));
            cur = 1 - cur;
        }
        CKA(cudaEventRecord(ev[2], ctx->stream));
        if (overlap) {  // back to the context's stream, after the sweep
            CKA(cudaEventRecord(ov.join, ov.hs));
            CKA(cudaStreamWaitEvent(ov.saved, ov.join, 0));
            ctx->stream = ov.saved;
            ov.saved = nullptr;
        }
        if (Qbar0) CKA(cudaMemcpyAsync(Qbar0, Ab[5], nq * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CKA(cudaMemcpyAsync(w->host, w->acc, sizeof(AdjScalars), cudaMemcpyDeviceToHost, ctx->stream));
        CKA(cudaStreamSynchronize(ctx->stream));
        AdjScalars acc;
        std::memcpy(&acc, w->host, sizeof(AdjScalars));
        if (parbar)
            for (int m = 0; m < 6; m++) parbar[m] = acc.pbar[m];
        ties = (int)acc.ties;
        CKA(cudaEventElapsedTime(&rev_ms, ev[1], ev[2]));
        if ((rc = adjoint_flags(ctx))) return rc;
    }
    float fwd_ms = 0.0f;
    CKA(cudaEventElapsedTime(&fwd_ms, ev[0], ev[1]));
    if (stats) {
        stats->forward_ms = fwd_ms;
        stats->reverse_ms = rev_ms;
        stats->device_bytes = (double)(rb.bytes + w->bytes);
        stats->owner_stages = owners;
        stats->tie_stages = ties;
    }

    // ---- the context continues from the final state -------------------------------
    {
        const int last = ns - (nseg - 1) * K;
        double *fin = S[5 * last];
        if (grad && nseg > 1) {  // the stage store now holds the first segment: rerun the last one
            const int step0 = (nseg - 1) * K;
            CKA(cudaMemcpyAsync(S[0], ckpt[nseg - 1], nq * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
            CKA(launch_trace_exact(ctx->N, ctx->ncell, S[0], T[0], ctx->ops, ctx->stream));
            if ((rc = forward_steps(ctx, o->dt, step0, last, S.data(), T.data(), hist, 0, -1, nullptr, cmax,
                                    ctx->stream)))
                return rc;
        }
        CKA(cudaMemcpyAsync(ctx->reg[0], fin, nq * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        const double *hl = &H[2 * (size_t)5 * ns];
        std::vector<double> mx(2 * kSlots);
        for (int k = 0; k < kSlots; k++) {
            mx[2 * k] = hl[0];
            mx[2 * k + 1] = hl[1];
        }
        CKA(cudaMemcpyAsync(ctx->maxima, mx.data(), mx.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        CKA(cudaStreamSynchronize(ctx->stream));
        ctx->slot = 0;
        ctx->ctime += ns * o->dt;
        ctx->traces_stale = true;
    }
    return SDDC_OK;
}
