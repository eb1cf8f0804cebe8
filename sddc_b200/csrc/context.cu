// Host runtime of the SDDC drop-in: the C ABI of include/sddc.h.
//
// A context owns every device buffer of one case: the RK registers, the
// packed metrics, the per-(cell, local face) connectivity records, the
// running maxima and the diagnostics.  Table conversion (Fortran layout ->
// device layout) happens once in sddc_set_tables; afterwards a time step is
// five launches of the fused stage kernel on the context's stream, captured
// in a CUDA graph.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "context_impl.h"
#include "sd_basis.h"
#include "tables_pack.h"
#include "visc_kernel.cuh"

using namespace sddc;

namespace {

// muAV from the sensor and epsilon0 (AV.f90:106-140); epsilon0 uses the
// running max of the wave speed after the evaluation.
__global__ void muav_kernel(int ncell, int N, double h_msh, const double *sm_ind, const double *maxima, int slot,
                            double *muav)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const double eps0 = maxima[2 * slot] * h_msh / (double)(N - 1) * 0.05;
    const double lo[2] = {-5.0, -3.0}, hi[2] = {0.0, 1.0};
    for (int v = 0; v < 2; v++) {
        const double s = sm_ind[2 * (size_t)c + v];
        const double k = (hi[v] - lo[v]) * 0.5, s0 = (hi[v] + lo[v]) * 0.5;
        double m;
        if (s < lo[v]) m = 0.0;
        else if (s > hi[v]) m = eps0;
        else m = eps0 / 2.0 * (1.0 + sin(kPi * (s - s0) / 2.0 / k));
        muav[2 * (size_t)c + v] = m;
    }
}

// fixed-order sum of per-CTA partials (deterministic)
__global__ void sum_pairs_kernel(int n, const double *part, double *out)
{
    __shared__ double s0[kMonThreads], s1[kMonThreads];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < n; i += kMonThreads) {
        a += part[2 * i];
        b += part[2 * i + 1];
    }
    s0[threadIdx.x] = a;
    s1[threadIdx.x] = b;
    __syncthreads();
    for (int w = kMonThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            s0[threadIdx.x] += s0[threadIdx.x + w];
            s1[threadIdx.x] += s1[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = s0[0];
        out[1] = s1[0];
    }
}

// per-cell integrals of density and energy: sum_ij Jac * w_i * w_j * Q
__global__ void integrals_kernel(int ncell, int N, const double *q, const double *met, int met_size, int jac_off,
                                 const double *w, double *part)
{
    __shared__ double s0[kMonThreads], s1[kMonThreads];
    double a = 0.0, b = 0.0;
    const int NN = N * N;
    for (size_t t = blockIdx.x * (size_t)kMonThreads + threadIdx.x; t < (size_t)ncell * NN;
         t += (size_t)gridDim.x * kMonThreads) {
        const size_t c = t / NN;
        const int k = (int)(t % NN), i = k % N, j = k / N;
        const double wt = met[c * met_size + jac_off + k] * w[i] * w[j];
        a += wt * q[9 * t];
        b += wt * q[9 * t + 4];
    }
    s0[threadIdx.x] = a;
    s1[threadIdx.x] = b;
    __syncthreads();
    for (int s = kMonThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            s0[threadIdx.x] += s0[threadIdx.x + s];
            s1[threadIdx.x] += s1[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = s0[0];
        part[2 * blockIdx.x + 1] = s1[0];
    }
}

// quadrature weights of the solution points: w_i = integral over [0,1] of
// the Lagrange basis i (moment equations sum_i w_i x_i^k = 1/(k+1))
std::vector<double> sp_weights(const double *Xs, int N)
{
    std::vector<double> A(N * N), b(N);
    for (int k = 0; k < N; k++) {
        for (int i = 0; i < N; i++) A[k * N + i] = std::pow(Xs[i], k);
        b[k] = 1.0 / (k + 1);
    }
    for (int col = 0; col < N; col++) {  // Gaussian elimination, partial pivoting
        int piv = col;
        for (int r = col + 1; r < N; r++)
            if (std::fabs(A[r * N + col]) > std::fabs(A[piv * N + col])) piv = r;
        for (int c = 0; c < N; c++) std::swap(A[col * N + c], A[piv * N + c]);
        std::swap(b[col], b[piv]);
        for (int r = col + 1; r < N; r++) {
            const double f = A[r * N + col] / A[col * N + col];
            for (int c = col; c < N; c++) A[r * N + c] -= f * A[col * N + c];
            b[r] -= f * b[col];
        }
    }
    std::vector<double> w(N);
    for (int r = N - 1; r >= 0; r--) {
        double s = b[r];
        for (int c = r + 1; c < N; c++) s -= A[r * N + c] * w[c];
        w[r] = s / A[r * N + r];
    }
    return w;
}

}  // namespace

int sddc::met_size(int N) { return met_record_doubles(N); }

int sddc::set_err(sddc_ctx *c, int code, const std::string &m)
{
    if (c) c->err = m;
    return code;
}

int sddc::cuda_err(sddc_ctx *c, cudaError_t e, const char *what)
{
    return set_err(c, SDDC_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

extern "C" const char *sddc_last_error(const sddc_ctx *ctx) { return ctx ? ctx->err.c_str() : "NULL context"; }

static void free_all(sddc_ctx *ctx)
{
    output_free(ctx);
    for (auto &g : ctx->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    for (auto &r : ctx->reg) cudaFree(r), r = nullptr;
    for (auto &t : ctx->trace) cudaFree(t), t = nullptr;
    void *bufs[] = {ctx->met, ctx->nrm, ctx->jac, ctx->faces, ctx->maxima, ctx->sm_ind, ctx->muav, ctx->resid, ctx->grad,
                    ctx->mon_part, ctx->mon_out, ctx->int_part, ctx->wq, ctx->err_flags,
                    ctx->case_dev, ctx->tiles_rk, ctx->tiles_diag, ctx->visc_grad, ctx->visc_gt,
                    ctx->visc_rv, ctx->met2, ctx->max_scratch, ctx->proc_cells};
    for (void *b : bufs) cudaFree(b);
    if (ctx->host_small) cudaFreeHost(ctx->host_small);
    adjoint_free(ctx);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
}

extern "C" void sddc_destroy(sddc_ctx *ctx)
{
    if (!ctx) return;
    cudaStreamSynchronize(ctx->stream);
    free_all(ctx);
    delete ctx;
}

int sddc::alloc(sddc_ctx *ctx, void **p, size_t bytes, const char *what)
{
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_err(ctx, SDDC_ENOMEM, std::string("cudaMalloc ") + what + ": " + cudaGetErrorString(e));
    }
    return SDDC_OK;
}

extern "C" int sddc_create(sddc_ctx **out, const sddc_params *p)
{
    if (!out || !p) return SDDC_EINVAL;
    *out = nullptr;
    auto *ctx = new sddc_ctx();
    ctx->p = *p;
    auto bad = [&](const std::string &m) {
        int r = set_err(ctx, SDDC_EINVAL, m);
        *out = ctx;  // hand the context back so the caller can read the message
        return r;
    };
    if (p->N < 2 || p->N > kMaxN) return bad("N must be in [2, 6]");
    if (p->ncell < 1) return bad("ncell must be positive");
    if (p->vismode != 0 && p->vismode != 1) return bad("vismode must be 0 or 1");
    if (p->k_stage != 3 && p->k_stage != 5) return bad("k_stage can be only 3 or 5 (iterations.f90:22-31)");
    if (p->precision < SDDC_FP64_EXACT || p->precision > SDDC_MIXED) return bad("unknown precision");
    if (!(p->mu >= 0.0) || !(p->eta0 >= 0.0)) return bad("mu and eta0 must be non-negative");
    if (p->cells_per_cta != 0 && p->cells_per_cta != 4 && p->cells_per_cta != 6 && p->cells_per_cta != 8 &&
        p->cells_per_cta != 16)
        return bad("cells_per_cta must be 0, 4, 6, 8 or 16");
    ctx->N = p->N;
    ctx->ncell = p->ncell;
    ctx->cpb = p->cells_per_cta ? p->cells_per_cta : 8;
    if (!ctx->p.ncellglob) ctx->p.ncellglob = p->ncell;
    ctx->msize = met_size(p->N);
    ctx->nq = (size_t)9 * p->N * p->N * p->ncell;
    ctx->grid = (p->ncell + ctx->cpb - 1) / ctx->cpb;
    *out = ctx;
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    const int nreg = p->k_stage == 5 ? 6 : 4;
    int rc;
    ctx->trace_bytes = (size_t)p->ncell * 4 * p->N * 9 * (p->precision == SDDC_MIXED ? sizeof(float) : sizeof(double));
    for (int r = 0; r < nreg; r++) {
        if ((rc = alloc(ctx, (void **)&ctx->reg[r], ctx->nq * sizeof(double), "state register"))) return rc;
        if ((rc = alloc(ctx, &ctx->trace[r], ctx->trace_bytes, "face traces"))) return rc;
    }
    const size_t nc = p->ncell;
    const int diag_grid = (p->ncell + 7) / 8;
    const int mon_blocks = std::max(ctx->grid, diag_grid);
    ctx->nrm_double = p->precision != SDDC_MIXED;
    ctx->jac_inv = p->precision != SDDC_FP64_EXACT;
    const size_t n_nrm = nc * 4 * p->N * (p->N + 1), n_jac = nc * ((p->N * p->N + 1) & ~1);
    if ((rc = alloc(ctx, (void **)&ctx->met, nc * ctx->msize * sizeof(double), "metrics")) ||
        (rc = alloc(ctx, &ctx->nrm, n_nrm * (ctx->nrm_double ? sizeof(double) : sizeof(float)), "normals")) ||
        (rc = alloc(ctx, (void **)&ctx->jac, n_jac * sizeof(double), "Jacobians")) ||
        (rc = alloc(ctx, (void **)&ctx->faces, nc * 4 * sizeof(int2), "faces")) ||
        (rc = alloc(ctx, (void **)&ctx->maxima, kSlots * 2 * sizeof(double), "maxima")) ||
        (rc = alloc(ctx, (void **)&ctx->sm_ind, nc * 2 * sizeof(double), "sensor")) ||
        (rc = alloc(ctx, (void **)&ctx->muav, nc * 2 * sizeof(double), "muAV")) ||
        (rc = alloc(ctx, (void **)&ctx->mon_part, (size_t)mon_blocks * 2 * sizeof(double), "monitor")) ||
        (rc = alloc(ctx, (void **)&ctx->mon_out, 4 * sizeof(double), "monitor")) ||
        (rc = alloc(ctx, (void **)&ctx->int_part, 1024 * 2 * sizeof(double), "integrals")) ||
        (rc = alloc(ctx, (void **)&ctx->wq, kMaxN * sizeof(double), "weights")) ||
        (rc = alloc(ctx, (void **)&ctx->err_flags, sizeof(unsigned), "flags")))
        return rc;
    // the viscous chain runs only with vismode = 1 (compflux.f90:36)
    ctx->visc = p->vismode == 1 && (p->mu != 0.0 || p->eta0 != 0.0);
    if (ctx->visc) {
        if ((rc = alloc(ctx, (void **)&ctx->visc_grad, 2 * ctx->nq * sizeof(double), "viscous gradients")) ||
            (rc = alloc(ctx, (void **)&ctx->visc_gt, nc * 4 * p->N * 18 * sizeof(double), "gradient traces")) ||
            (rc = alloc(ctx, (void **)&ctx->visc_rv, ctx->nq * sizeof(double), "viscous residual")) ||
            (rc = alloc(ctx, (void **)&ctx->met2, nc * 4 * p->N * 2 * sizeof(double), "face metrics")))
            return rc;
    }
    CK(cudaMallocHost((void **)&ctx->host_small, 64 * sizeof(double)));
    CK(cudaMemsetAsync(ctx->maxima, 0, kSlots * 2 * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(ctx->err_flags, 0, sizeof(unsigned), ctx->stream));
    CK(cudaMemsetAsync(ctx->sm_ind, 0, nc * 2 * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(ctx->mon_part, 0, (size_t)mon_blocks * 2 * sizeof(double), ctx->stream));

    // operators from the SD points; Lmat/Mmat are replaced by the caller's
    // tables in sddc_set_tables
    const int N = p->N, NL = N - 1;
    double Xs[kMaxN], Xf[kMaxN + 1], Xl[kMaxN], Xlf[kMaxN + 1];
    sd_points(N, Xs, Xf);
    sd_points(NL, Xl, Xlf);
    for (int l = 0; l < NL; l++)
        for (int s = 0; s < N; s++) ctx->ops.H[l * N + s] = lagrange(Xs, N, s + 1, Xl[l]);
    for (int s = 0; s < N; s++)
        for (int l = 0; l < NL; l++) ctx->ops.HL[s * NL + l] = lagrange(Xl, NL, l + 1, Xs[s]);
    std::vector<double> w = sp_weights(Xs, N);
    CK(cudaMemcpyAsync(ctx->wq, w.data(), N * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SDDC_OK;
}

extern "C" int sddc_set_tables(sddc_ctx *ctx, const double *Lmat, const double *Mmat, const double *S1,
                               const double *S2, const double *Jac, const int *IF2C, int nface,
                               const int *ibfinter, int ninter, const int *ibfinl, int ninlet, const int *ibfout,
                               int noutlet, const int *ibfwal, int nwall, const int *ibfsymp, int nsymp,
                               const int *ibfree, int nfree, const int *cyc2fpair, int npair)
{
    if (!ctx) return SDDC_EINVAL;
    if (!Lmat || !Mmat || !S1 || !S2 || !Jac || !IF2C || nface < 1)
        return set_err(ctx, SDDC_EINVAL, "sddc_set_tables: NULL table or nface < 1");
    const int N = ctx->N, N1 = N + 1, NC = ctx->ncell;
    for (int r = 0; r < N1; r++)
        for (int s = 0; s < N; s++) {
            ctx->ops.L[r * N + s] = Lmat[r + N1 * s];
            ctx->ops.M[r * N + s] = Mmat[r + N1 * s];
            ctx->ops.Lf[r * N + s] = (float)Lmat[r + N1 * s];
            ctx->ops.Mf[r * N + s] = (float)Mmat[r + N1 * s];
        }
    // packed metrics: S1(1,1:2,r,j), S2(2,1:2,i,r), Jac(i,j)
    std::vector<double> met((size_t)NC * ctx->msize, 0.0);
    pack_metric_records(N, NC, S1, S2, Jac, met.data());
    const int kFam = 2 * N * N1, kJac = 2 * kFam;
    // the same, split: normals (rounded once to the form's type) and Jac
    // (its IEEE reciprocal for the forms that multiply by 1/Jac) padded to
    // an even count, so that a tile's slices are 16-byte aligned
    const int NJ = (N * N + 1) & ~1;
    std::vector<double> nrm_d, jac((size_t)NC * NJ, 0.0);
    std::vector<float> nrm_f;
    if (ctx->nrm_double) nrm_d.resize((size_t)NC * kJac);
    else nrm_f.resize((size_t)NC * kJac);
    for (size_t c = 0; c < (size_t)NC; c++) {
        const double *m = &met[c * ctx->msize];
        for (int o = 0; o < kJac; o++) {
            if (ctx->nrm_double) nrm_d[c * kJac + o] = m[o];
            else nrm_f[c * kJac + o] = (float)m[o];
        }
        for (int k = 0; k < N * N; k++) jac[c * NJ + k] = ctx->jac_inv ? 1.0 / m[kJac + k] : m[kJac + k];
    }
    // per-(cell, local face) records from the reference's face lists
    std::vector<int2> fr((size_t)NC * 4);
    FaceLists fl{IF2C, nface, ibfinter, ninter, ibfinl, ninlet, ibfout, noutlet, ibfwal, nwall,
                 ibfsymp, nsymp, ibfree, nfree, cyc2fpair, npair};
    fl.ibfproc = ctx->ibfproc.data();
    fl.nproc = (int)ctx->ibfproc.size();
    static_assert(sizeof(int2) == 2 * sizeof(int), "face records are int pairs");
    const std::string msg = build_face_records(NC, fl, reinterpret_cast<int *>(fr.data()));
    if (!msg.empty()) return set_err(ctx, SDDC_EINVAL, "sddc_set_tables: " + msg);
    if (!ctx->ibfproc.empty()) {
        // each exchange slot's own (cell, local face), IF2C(K,1) and IF2C(K,3)
        std::vector<int2> pc(ctx->ibfproc.size());
        for (size_t b = 0; b < pc.size(); b++) {
            const int K = ctx->ibfproc[b];
            pc[b] = make_int2(IF2C[K - 1] - 1, IF2C[(K - 1) + (size_t)nface * 2]);
        }
        cudaFree(ctx->proc_cells);
        ctx->proc_cells = nullptr;
        int rc = alloc(ctx, (void **)&ctx->proc_cells, pc.size() * sizeof(int2), "processor faces");
        if (rc) return rc;
        CK(cudaMemcpyAsync(ctx->proc_cells, pc.data(), pc.size() * sizeof(int2), cudaMemcpyHostToDevice,
                           ctx->stream));
    }
    std::vector<double> met2;
    if (ctx->visc) {
        // the normal row the adiabatic-wall gradient state reads
        // (bcflux.f90:527-583): S1(2,1:2) at xi face points (local faces 2,
        // 4), S2(1,1:2) at eta face points (1, 3)
        met2.assign((size_t)NC * 4 * N * 2, 0.0);
        for (size_t c = 0; c < (size_t)NC; c++)
            for (int lf = 1; lf <= 4; lf++)
                for (int nfp = 1; nfp <= N; nfp++) {
                    int ifp, jfp;  // face2fpconnec, initsetup.f90:347-383
                    switch (lf) {
                    case 1: ifp = nfp; jfp = 1; break;
                    case 2: ifp = N1; jfp = nfp; break;
                    case 3: ifp = N - nfp + 1; jfp = N1; break;
                    default: ifp = 1; jfp = N - nfp + 1; break;
                    }
                    double *o = &met2[((c * 4 + (lf - 1)) * N + (nfp - 1)) * 2];
                    if (lf % 2 == 0) {
                        const size_t b = 4 * ((ifp - 1) + (size_t)N1 * ((jfp - 1) + (size_t)N * c));
                        o[0] = S1[b + 1];
                        o[1] = S1[b + 3];
                    } else {
                        const size_t b = 4 * ((ifp - 1) + (size_t)N * ((jfp - 1) + (size_t)N1 * c));
                        o[0] = S2[b + 0];
                        o[1] = S2[b + 2];
                    }
                }
        CK(cudaMemcpyAsync(ctx->met2, met2.data(), met2.size() * sizeof(double), cudaMemcpyHostToDevice,
                           ctx->stream));
    }
    CK(cudaMemcpyAsync(ctx->met, met.data(), met.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if (ctx->nrm_double)
        CK(cudaMemcpyAsync(ctx->nrm, nrm_d.data(), nrm_d.size() * sizeof(double), cudaMemcpyHostToDevice,
                           ctx->stream));
    else
        CK(cudaMemcpyAsync(ctx->nrm, nrm_f.data(), nrm_f.size() * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
    CK(cudaMemcpyAsync(ctx->jac, jac.data(), jac.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->faces, fr.data(), fr.size() * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->tables = true;
    ctx->traces_stale = true;
    ctx->proc_stale = true;
    return SDDC_OK;
}

// ---------------------------------------------------------- decomposed runs

extern "C" int sddc_set_proc_faces(sddc_ctx *ctx, int nproc, const int *ibfproc)
{
    if (!ctx) return SDDC_EINVAL;
    if (ctx->tables) return set_err(ctx, SDDC_ESTATE, "sddc_set_proc_faces comes before sddc_set_tables");
    if (nproc < 0 || (nproc > 0 && !ibfproc)) return set_err(ctx, SDDC_EINVAL, "sddc_set_proc_faces: bad list");
    if (ctx->visc) return set_err(ctx, SDDC_EINVAL, "decomposed runs need the ideal chain (mu = eta0 = 0)");
    ctx->ibfproc.assign(ibfproc, ibfproc + nproc);
    return SDDC_OK;
}

extern "C" int sddc_set_exchange(sddc_ctx *ctx, sddc_exchange_fn fn, void *user, void *send_dev, void *recv_dev,
                                 double *maxima_dev)
{
    if (!ctx) return SDDC_EINVAL;
    if (!ctx->tables) return set_err(ctx, SDDC_ESTATE, "sddc_set_exchange comes after sddc_set_tables");
    if (ctx->ncase) return set_err(ctx, SDDC_ESTATE, "a batch is not decomposed");
    if (!fn || !maxima_dev || (!ctx->ibfproc.empty() && (!send_dev || !recv_dev)))
        return set_err(ctx, SDDC_EINVAL, "sddc_set_exchange: NULL function or buffer");
    ctx->exch = fn;
    ctx->exch_user = user;
    ctx->proc_send = send_dev;
    ctx->proc_recv = recv_dev;
    ctx->proc_max = maxima_dev;
    ctx->proc_stale = true;
    return SDDC_OK;
}

namespace {
// send[slot][nfp][k] = trace of the slot's own (cell, local face), the
// reference's SBUFC order (procintflux_all.f90:49-70)
template <typename T>
__global__ void proc_pack_kernel(int nproc, int N, const int2 *__restrict__ pc, const T *__restrict__ tr,
                                 T *__restrict__ send)
{
    const int n = nproc * N * 9;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int k = e % 9, nfp0 = (e / 9) % N, b = e / (9 * N);
        const int2 c = pc[b];
        send[e] = tr[((size_t)c.x * 4 + (c.y - 1)) * 9 * N + (size_t)k * N + nfp0];  // trace_at
    }
}
}  // namespace

// The exchange of a decomposed run after the traces of register `reg`
// exist and the running maxima of `slot` are this rank's: pack, hand the
// maxima to the host buffer, call the host, take the reduced maxima back.
static int exchange(sddc_ctx *ctx, int reg, int slot)
{
    const int nproc = (int)ctx->ibfproc.size();
    if (!ctx->exch) {
        if (nproc) return set_err(ctx, SDDC_ESTATE, "processor faces need sddc_set_exchange");
        return SDDC_OK;
    }
    if (nproc) {
        const int n = nproc * ctx->N * 9, nb = std::min((n + 255) / 256, 4096);
        if (ctx->p.precision == SDDC_MIXED)
            proc_pack_kernel<float><<<nb, 256, 0, ctx->stream>>>(
                nproc, ctx->N, ctx->proc_cells, reinterpret_cast<const float *>(ctx->trace[reg]),
                reinterpret_cast<float *>(ctx->proc_send));
        else
            proc_pack_kernel<double><<<nb, 256, 0, ctx->stream>>>(
                nproc, ctx->N, ctx->proc_cells, reinterpret_cast<const double *>(ctx->trace[reg]),
                reinterpret_cast<double *>(ctx->proc_send));
        CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(ctx->proc_max, ctx->maxima + 2 * slot, 2 * sizeof(double), cudaMemcpyDeviceToDevice,
                       ctx->stream));
    if (ctx->exch(ctx->exch_user) != 0) return set_err(ctx, SDDC_ECUDA, "the host's exchange failed");
    CK(cudaMemcpyAsync(ctx->maxima + 2 * slot, ctx->proc_max, 2 * sizeof(double), cudaMemcpyDeviceToDevice,
                       ctx->stream));
    return SDDC_OK;
}

// face traces of the current state (register 0), computed by the form's own
// translation unit so they round exactly as its stage kernel's
static int refresh_traces(sddc_ctx *ctx)
{
    cudaError_t e;
    switch (ctx->p.precision) {
    case SDDC_FP64_EXACT: e = launch_trace_exact(ctx->N, ctx->ncell, ctx->reg[0], ctx->trace[0], ctx->ops, ctx->stream); break;
    case SDDC_FP64: e = launch_trace_fp64(ctx->N, ctx->ncell, ctx->reg[0], ctx->trace[0], ctx->ops, ctx->stream); break;
    default: e = launch_trace_mixed(ctx->N, ctx->ncell, ctx->reg[0], ctx->trace[0], ctx->ops, ctx->stream); break;
    }
    if (e != cudaSuccess) return cuda_err(ctx, e, "trace kernel");
    ctx->traces_stale = false;
    return SDDC_OK;
}

extern "C" int sddc_set_state(sddc_ctx *ctx, const double *Q, double ctime, double eigvmax, double umax)
{
    if (!ctx || !Q) return set_err(ctx, SDDC_EINVAL, "sddc_set_state: NULL argument");
    CK(cudaMemcpyAsync(ctx->reg[0], Q, ctx->nq * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    // every running-max slot of every case starts from the given maxima
    std::vector<double> mx(2 * kSlots * std::max(ctx->ncase, 1));
    for (size_t s = 0; s < mx.size() / 2; s++) {
        mx[2 * s] = eigvmax;
        mx[2 * s + 1] = umax;
    }
    CK(cudaMemcpyAsync(ctx->maxima, mx.data(), mx.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if (ctx->tables) {
        int rc = refresh_traces(ctx);
        if (rc) return rc;
    } else {
        ctx->traces_stale = true;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->ctime = ctime;
    ctx->slot = 0;
    ctx->state = true;
    ctx->proc_stale = true;
    return SDDC_OK;
}

StageArgs sddc::base_args(sddc_ctx *ctx)
{
    StageArgs a{};
    a.ncell = ctx->ncell;
    a.vismode = ctx->p.vismode;
    a.artiv = ctx->p.artiv;
    a.alpha = 2.0;  // initsetup.f90:165
    a.fs = Freestream{ctx->p.rinf, ctx->p.pinf, ctx->p.uinf, ctx->p.vinf, ctx->p.bxinf, ctx->p.byinf};
    a.met = ctx->met;
    a.nrm = ctx->nrm;
    a.jac = ctx->jac;
    a.jac_inv = ctx->jac_inv ? 1 : 0;
    a.faces = ctx->faces;
    a.proc_recv = ctx->proc_recv;
    a.maxima = ctx->maxima;
    a.sm_ind = ctx->sm_ind;
    a.err_flags = ctx->err_flags;
    return a;
}

// the viscous chain of the stage input (two launches); the stage kernel then
// adds its dFv + dGv
static cudaError_t launch_visc(sddc_ctx *ctx, const double *q_in, const void *t_in)
{
    ViscArgs v{};
    v.ncell = ctx->ncell;
    v.vismode = ctx->p.vismode;
    v.mu = ctx->p.mu;
    v.eta0 = ctx->p.eta0;
    v.fs = Freestream{ctx->p.rinf, ctx->p.pinf, ctx->p.uinf, ctx->p.vinf, ctx->p.bxinf, ctx->p.byinf};
    v.q = q_in;
    v.t_in = t_in;
    v.met = ctx->met;
    v.met2 = ctx->met2;
    v.faces = ctx->faces;
    v.grad = ctx->visc_grad;
    v.gt = ctx->visc_gt;
    v.rv = ctx->visc_rv;
    switch (ctx->p.precision) {
    case SDDC_FP64_EXACT: return launch_visc_exact(ctx->N, v, ctx->ops, ctx->stream);
    case SDDC_FP64: return launch_visc_fp64(ctx->N, v, ctx->ops, ctx->stream);
    default: return launch_visc_mixed(ctx->N, v, ctx->ops, ctx->stream);
    }
}

static cudaError_t launch(sddc_ctx *ctx, bool diag, const StageArgs &a_in)
{
    StageArgs a = a_in;
    if (ctx->visc) {
        cudaError_t e = launch_visc(ctx, a.q_in, a.t_in);
        if (e != cudaSuccess) return e;
        a.visc = ctx->visc_rv;
    }
    if (ctx->ncase) {  // a batch: one CTA per tile of the case-aligned tile table
        a.tiles = diag ? ctx->tiles_diag : ctx->tiles_rk;
        a.ntiles = diag ? ctx->ntiles_diag : ctx->ntiles_rk;
        a.cases = ctx->case_dev;
        a.persistent = ctx->persistent ? 1 : 0;
    }
    switch (ctx->p.precision) {
    case SDDC_FP64_EXACT: return launch_stage_exact(ctx->N, ctx->cpb, diag, a, ctx->ops, ctx->stream);
    case SDDC_FP64: return launch_stage_fp64(ctx->N, ctx->cpb, diag, a, ctx->ops, ctx->stream);
    default: return launch_stage_mixed(ctx->N, ctx->cpb, diag, a, ctx->ops, ctx->stream);
    }
}

int sddc::ready(sddc_ctx *ctx)
{
    if (!ctx) return SDDC_EINVAL;
    if (!ctx->tables) return set_err(ctx, SDDC_ESTATE, "tables not set (call sddc_set_tables)");
    if (!ctx->state) return set_err(ctx, SDDC_ESTATE, "state not set (call sddc_set_state)");
    if (ctx->traces_stale) return refresh_traces(ctx);
    return SDDC_OK;
}

// before a residual evaluation of a decomposed run: the exchange of the
// current state's traces, once after set_state or set_tables
static int proc_ready(sddc_ctx *ctx)
{
    if (!ctx->proc_stale) return SDDC_OK;
    int rc = exchange(ctx, 0, ctx->slot);
    if (rc) return rc;
    ctx->proc_stale = false;
    return SDDC_OK;
}

int sddc::check_flags(sddc_ctx *ctx)
{
    CK(cudaMemcpyAsync(ctx->host_small, ctx->err_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned f;
    std::memcpy(&f, ctx->host_small, sizeof(unsigned));
    if (f) {
        CK(cudaMemsetAsync(ctx->err_flags, 0, sizeof(unsigned), ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        std::string m = "device numerics:";
        if (f & kErrNonPositiveDensity) m += " non-positive density";
        if (f & kErrNonFiniteWaveSpeed) m += " non-finite wave speed";
        if (f & kErrStagingTimeout) m += " staging copy timed out";
        return set_err(ctx, SDDC_ENUMERIC, m);
    }
    return SDDC_OK;
}

extern "C" int sddc_compresid(sddc_ctx *ctx)
{
    int rc = ready(ctx);
    if (!rc) rc = proc_ready(ctx);
    if (rc) return rc;
    const size_t nc = ctx->ncell;
    if (!ctx->resid) {
        if ((rc = alloc(ctx, (void **)&ctx->resid, ctx->nq * sizeof(double), "resid")) ||
            (rc = alloc(ctx, (void **)&ctx->grad, 2 * ctx->nq * sizeof(double), "nablaQs")))
            return rc;
    }
    (void)nc;
    StageArgs a = base_args(ctx);
    a.rk_kind = kRkNone;
    a.q_in = ctx->reg[0];
    a.t_in = ctx->trace[0];
    a.slot_r = ctx->slot;
    a.slot_w = (ctx->slot + 1) % kSlots;
    a.resid_out = ctx->resid;
    a.grad_out = ctx->grad;
    a.mon_part = ctx->mon_part;
    CK(launch(ctx, true, a));
    // a decomposed run reduces the maxima over the ranks (compflux.f90:10-11)
    if ((rc = exchange(ctx, 0, a.slot_w))) return rc;
    ctx->slot = a.slot_w;
    ctx->sensor_stale = false;
    ctx->mon_nblk = ctx->ncase ? ctx->ntiles_diag : (ctx->ncell + 7) / 8;
    CK(cudaStreamSynchronize(ctx->stream));
    return check_flags(ctx);
}

// the launches of one time step, starting from running-max slot s0; in a
// decomposed run (xrc not null) each stage is followed by the exchange of its
// output's traces and maxima, whose status goes to *xrc
static cudaError_t enqueue_step(sddc_ctx *ctx, double dt, int s0, int *xrc = nullptr)
{
    double **P = ctx->reg;
    StageArgs a = base_args(ctx);
    a.dt = dt;
    // stage table: kind, registers, base coefficients and which of them are
    // multiplied by the case's dt (in the kernel, as the host would)
    struct St {
        int kind;
        int in, out, ra, rb, rc, rd, rw;
        double c[6];
        unsigned mask;
    };
    St st[5];
    if (ctx->p.k_stage == 3) {  // RK_S5P3, iterations.f90:179-210
        st[0] = {kRkAxpy, 0, 1, -1, -1, -1, -1, -1, {B10}, 1u};
        st[1] = {kRkAxpy, 1, 2, -1, -1, -1, -1, -1, {B21}, 1u};
        st[2] = {kRkTwoReg, 2, 1, 0, -1, -1, -1, -1, {B32, A30, A32}, 1u};
        st[3] = {kRkTwoReg, 1, 3, 0, -1, -1, -1, -1, {B43, A40, A43}, 1u};
        st[4] = {kRkTwoReg, 3, 0, 2, -1, -1, -1, -1, {B54, A52, A54}, 1u};
    } else {  // FiveStageRk, iterations.f90:103-152
        st[0] = {kRkAxpy, 0, 1, -1, -1, -1, -1, -1, {F11}, 1u};
        st[1] = {kRkTwoRegT, 1, 2, 0, -1, -1, -1, -1, {F23, F21, F22, 1.0}, 8u};
        st[2] = {kRkTwoReg, 2, 3, 0, -1, -1, -1, -1, {F33, F31, F32}, 1u};
        st[3] = {kRkTwoReg, 3, 4, 0, -1, -1, -1, 5, {F43, F41, F42}, 1u};
        st[4] = {kRkFive, 4, 0, 0, 2, 3, 5, -1, {F56, F51, F52, F53, F54, F55}, 1u | 32u};
    }
    a.artiv = 0;  // the sensor is evaluated on request (sensor_stale)
    ctx->last_in = st[4].in;
    for (int k = 0; k < 5; k++) {
        a.rk_kind = st[k].kind;
        a.q_in = P[st[k].in];
        a.q_out = P[st[k].out];
        a.t_in = ctx->trace[st[k].in];
        a.t_out = ctx->trace[st[k].out];
        a.reg_a = st[k].ra >= 0 ? P[st[k].ra] : nullptr;
        a.reg_b = st[k].rb >= 0 ? P[st[k].rb] : nullptr;
        a.reg_c = st[k].rc >= 0 ? P[st[k].rc] : nullptr;
        a.reg_d = st[k].rd >= 0 ? P[st[k].rd] : nullptr;
        a.resid_w = st[k].rw >= 0 ? P[st[k].rw] : nullptr;
        for (int i = 0; i < 6; i++) a.cb[i] = st[k].c[i];
        a.dt_mask = st[k].mask;
        a.slot_r = (s0 + k) % kSlots;
        a.slot_w = (s0 + k + 1) % kSlots;
        a.mon_part = k == 4 ? ctx->mon_part : nullptr;
        cudaError_t e = launch(ctx, false, a);
        if (e != cudaSuccess) return e;
        if (xrc && (*xrc = exchange(ctx, st[k].out, a.slot_w))) return cudaSuccess;
    }
    return cudaSuccess;
}

static int run_steps(sddc_ctx *ctx, double dt, int nsteps);

extern "C" int sddc_rk_step(sddc_ctx *ctx, double dt, int nsteps)
{
    int rc = ready(ctx);
    if (rc) return rc;
    if (ctx->ncase) return set_err(ctx, SDDC_ESTATE, "a batch steps with sddc_rk_step_cases");
    if (nsteps < 0) return set_err(ctx, SDDC_EINVAL, "nsteps < 0");
    if (!(dt > 0.0)) return set_err(ctx, SDDC_EINVAL, "dt must be positive");
    return run_steps(ctx, dt, nsteps);
}

extern "C" int sddc_rk_step_cases(sddc_ctx *ctx, int nsteps)
{
    int rc = ready(ctx);
    if (rc) return rc;
    if (!ctx->ncase) return set_err(ctx, SDDC_ESTATE, "no batch: call sddc_set_cases first");
    if (nsteps < 0) return set_err(ctx, SDDC_EINVAL, "nsteps < 0");
    return run_steps(ctx, 0.0, nsteps);  // each case's dt lives on the device
}

static int run_steps(sddc_ctx *ctx, double dt, int nsteps)
{
    if (ctx->exch || !ctx->ibfproc.empty()) {
        // a decomposed run: stage by stage, the host's exchange between them
        int rc = proc_ready(ctx);
        if (rc) return rc;
        for (int s = 0; s < nsteps; s++) {
            int xrc = 0;
            cudaError_t e = enqueue_step(ctx, dt, ctx->slot, &xrc);
            if (e != cudaSuccess) return cuda_err(ctx, e, "stage launch");
            if (xrc) return xrc;
            ctx->ctime += dt;
            ctx->sensor_stale = true;
            ctx->mon_nblk = ctx->grid;
        }
        CK(cudaStreamSynchronize(ctx->stream));
        return check_flags(ctx);
    }
    for (int s = 0; s < nsteps; s++) {
        const int s0 = ctx->slot;
        cudaGraphExec_t &g = ctx->graph[s0];
        if (g && ctx->graph_dt[s0] != dt) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
        if (!g && s > 0) {  // first step of a call runs eagerly (kernel attributes, warm-up)
            cudaGraph_t graph;
            CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = enqueue_step(ctx, dt, s0);
            cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &graph);
            if (e != cudaSuccess) return cuda_err(ctx, e, "stage launch (capture)");
            if (e2 != cudaSuccess) return cuda_err(ctx, e2, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&g, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return cuda_err(ctx, e, "cudaGraphInstantiate");
            ctx->graph_dt[s0] = dt;
        }
        if (g) {
            CK(cudaGraphLaunch(g, ctx->stream));
        } else {
            cudaError_t e = enqueue_step(ctx, dt, s0);
            if (e != cudaSuccess) return cuda_err(ctx, e, "stage launch");
        }
        ctx->ctime += dt;  // ctime = ctime0 + dt after the last stage (iterations.f90:211)
        ctx->sensor_stale = true;
        ctx->mon_nblk = ctx->ncase ? ctx->ntiles_rk : ctx->grid;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return check_flags(ctx);
}

// the AV sensor of the last stage's input (see sensor_stale): a residual
// evaluation of that register that keeps only the sensor, with the maxima
// the stage read, on a copy of the running maxima
static int refresh_sensor(sddc_ctx *ctx)
{
    const size_t nmax = (size_t)kSlots * 2 * std::max(ctx->ncase, 1);
    if (!ctx->max_scratch) {
        int rc = alloc(ctx, (void **)&ctx->max_scratch, nmax * sizeof(double), "maxima copy");
        if (rc) return rc;
    }
    CK(cudaMemcpyAsync(ctx->max_scratch, ctx->maxima, nmax * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    StageArgs a = base_args(ctx);
    a.rk_kind = kRkNone;
    a.maxima = ctx->max_scratch;
    a.q_in = ctx->reg[ctx->last_in];
    a.t_in = ctx->trace[ctx->last_in];
    a.slot_r = (ctx->slot + kSlots - 1) % kSlots;  // the slot the last stage read
    a.slot_w = ctx->slot;
    CK(launch(ctx, true, a));
    ctx->sensor_stale = false;
    return SDDC_OK;
}

// muAV (2,NCELL) of the current state into ctx->muav, on the stream
int sddc::device_muav(sddc_ctx *ctx)
{
    if (ctx->sensor_stale && ctx->exch && ctx->p.artiv == 1 && ctx->p.vismode == 1)
        return set_err(ctx, SDDC_ESTATE,
                       "the AV sensor after steps of a decomposed run is not formed; call sddc_compresid first");
    if (ctx->sensor_stale && ctx->p.artiv == 1 && ctx->p.vismode == 1) {
        int rc = refresh_sensor(ctx);
        if (rc) return rc;
    }
    const double h = std::sqrt(ctx->p.dxcycl * ctx->p.dycycl / (double)ctx->p.ncellglob);
    muav_kernel<<<(ctx->ncell + 255) / 256, 256, 0, ctx->stream>>>(ctx->ncell, ctx->N, h, ctx->sm_ind, ctx->maxima,
                                                                   ctx->slot, ctx->muav);
    CK(cudaGetLastError());
    return SDDC_OK;
}

extern "C" int sddc_get_state(sddc_ctx *ctx, double *Q, double *resid, double *nablaQs, double *muAV,
                              double *sm_ind)
{
    if (!ctx) return SDDC_EINVAL;
    if ((sm_ind || muAV) && ctx->sensor_stale && ctx->exch && ctx->p.artiv == 1 && ctx->p.vismode == 1)
        return set_err(ctx, SDDC_ESTATE,
                       "the AV sensor after steps of a decomposed run is not formed; call sddc_compresid first");
    if (sm_ind && ctx->sensor_stale && ctx->p.artiv == 1 && ctx->p.vismode == 1) {
        int rc = refresh_sensor(ctx);
        if (rc) return rc;
    }
    if (Q) CK(cudaMemcpyAsync(Q, ctx->reg[0], ctx->nq * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if ((resid || nablaQs) && !ctx->resid)
        return set_err(ctx, SDDC_ESTATE, "no residual kept: call sddc_compresid first");
    if (resid) CK(cudaMemcpyAsync(resid, ctx->resid, ctx->nq * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (nablaQs)
        CK(cudaMemcpyAsync(nablaQs, ctx->grad, 2 * ctx->nq * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (muAV && ctx->ncase) return set_err(ctx, SDDC_ESTATE, "muAV is per case; read sm_ind for a batch");
    if (muAV) {
        int rc = device_muav(ctx);
        if (rc) return rc;
        CK(cudaMemcpyAsync(muAV, ctx->muav, 2 * (size_t)ctx->ncell * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream));
    }
    if (sm_ind)
        CK(cudaMemcpyAsync(sm_ind, ctx->sm_ind, 2 * (size_t)ctx->ncell * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SDDC_OK;
}

extern "C" int sddc_monitor(sddc_ctx *ctx, double *residsum, double *divbsum, double *mass, double *energy)
{
    int rc = ready(ctx);
    if (rc) return rc;
    sum_pairs_kernel<<<1, kMonThreads, 0, ctx->stream>>>(ctx->mon_nblk, ctx->mon_part, ctx->mon_out);
    CK(cudaGetLastError());
    const int ib = 1024;
    integrals_kernel<<<ib, kMonThreads, 0, ctx->stream>>>(ctx->ncell, ctx->N, ctx->reg[0], ctx->met, ctx->msize,
                                                          2 * (2 * ctx->N * (ctx->N + 1)), ctx->wq, ctx->int_part);
    CK(cudaGetLastError());
    sum_pairs_kernel<<<1, kMonThreads, 0, ctx->stream>>>(ib, ctx->int_part, ctx->mon_out + 2);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->host_small, ctx->mon_out, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (residsum) *residsum = ctx->host_small[0];
    if (divbsum) *divbsum = ctx->host_small[1];
    if (mass) *mass = ctx->host_small[2];
    if (energy) *energy = ctx->host_small[3];
    return SDDC_OK;
}

extern "C" int sddc_get_maxima(sddc_ctx *ctx, double *eigvmax, double *umax, double *c_h, double *ctime)
{
    if (!ctx) return SDDC_EINVAL;
    CK(cudaMemcpyAsync(ctx->host_small, ctx->maxima + 2 * ctx->slot, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const double e = ctx->host_small[0], u = ctx->host_small[1];
    if (eigvmax) *eigvmax = e;
    if (umax) *umax = u;
    if (c_h) *c_h = std::sqrt(e * (e - u));
    if (ctime) *ctime = ctx->ctime;
    return SDDC_OK;
}

extern "C" int sddc_state_device_ptr(sddc_ctx *ctx, double **q_dev)
{
    if (!ctx || !q_dev) return SDDC_EINVAL;
    *q_dev = ctx->reg[0];
    return SDDC_OK;
}

extern "C" int sddc_get_stream(sddc_ctx *ctx, void **stream)
{
    if (!ctx || !stream) return SDDC_EINVAL;
    *stream = (void *)ctx->stream;
    return SDDC_OK;
}

// ---------------------------------------------------------------- batches

static int build_tiles(sddc_ctx *ctx, int cpb, int4 **dev, int *count)
{
    // persistent launches walk the table with a grid stride, largest case
    // first; otherwise the cases in their order
    std::vector<int> order(ctx->ncase);
    for (int c = 0; c < ctx->ncase; c++) order[c] = c;
    if (ctx->persistent)
        std::stable_sort(order.begin(), order.end(),
                         [&](int x, int y) { return ctx->cases[x].ncell > ctx->cases[y].ncell; });
    std::vector<int4> tiles;
    for (int c : order) {
        const sddc_case &k = ctx->cases[c];
        for (int first = 0; first < k.ncell; first += cpb)
            tiles.push_back(make_int4(k.first_cell + first, std::min(cpb, k.ncell - first), c, first == 0 ? 1 : 0));
    }
    cudaFree(*dev);
    *dev = nullptr;
    int rc = alloc(ctx, (void **)dev, tiles.size() * sizeof(int4), "tile table");
    if (rc) return rc;
    CK(cudaMemcpyAsync(*dev, tiles.data(), tiles.size() * sizeof(int4), cudaMemcpyHostToDevice, ctx->stream));
    *count = (int)tiles.size();
    return SDDC_OK;
}

extern "C" int sddc_set_cases(sddc_ctx *ctx, int ncase, const sddc_case *cases)
{
    if (ctx && ctx->visc) return set_err(ctx, SDDC_EINVAL, "batches run the ideal chain only (mu = eta0 = 0)");
    if (ctx && (ctx->exch || !ctx->ibfproc.empty())) return set_err(ctx, SDDC_ESTATE, "a batch is not decomposed");
    if (!ctx || ncase < 1 || !cases) return set_err(ctx, SDDC_EINVAL, "sddc_set_cases: bad arguments");
    // the cases must tile the cell range in order
    int next = 0;
    for (int c = 0; c < ncase; c++) {
        if (cases[c].first_cell != next || cases[c].ncell < 1)
            return set_err(ctx, SDDC_EINVAL, "case " + std::to_string(c) + " does not start where the previous ends");
        if (!(cases[c].dt > 0.0)) return set_err(ctx, SDDC_EINVAL, "case " + std::to_string(c) + ": dt must be positive");
        next += cases[c].ncell;
    }
    if (next != ctx->ncell) return set_err(ctx, SDDC_EINVAL, "the cases do not cover the context's cells");
    ctx->ncase = ncase;
    ctx->cases.assign(cases, cases + ncase);
    std::vector<CaseParams> cp(ncase);
    for (int c = 0; c < ncase; c++) {
        const sddc_case &k = cases[c];
        cp[c].fs = Freestream{k.rinf, k.pinf, k.uinf, k.vinf, k.bxinf, k.byinf};
        cp[c].dt = k.dt;
        cp[c].pad = 0.0;
    }
    int rc;
    cudaFree(ctx->case_dev);
    ctx->case_dev = nullptr;
    if ((rc = alloc(ctx, (void **)&ctx->case_dev, ncase * sizeof(CaseParams), "case table"))) return rc;
    CK(cudaMemcpyAsync(ctx->case_dev, cp.data(), ncase * sizeof(CaseParams), cudaMemcpyHostToDevice, ctx->stream));
    if ((rc = build_tiles(ctx, ctx->cpb, &ctx->tiles_rk, &ctx->ntiles_rk))) return rc;
    if ((rc = build_tiles(ctx, 8, &ctx->tiles_diag, &ctx->ntiles_diag))) return rc;
    // per-case running maxima and per-tile monitor partials
    cudaFree(ctx->maxima);
    cudaFree(ctx->mon_part);
    ctx->maxima = nullptr;
    ctx->mon_part = nullptr;
    const int nmon = std::max(ctx->ntiles_rk, ctx->ntiles_diag);
    if ((rc = alloc(ctx, (void **)&ctx->maxima, (size_t)ncase * kSlots * 2 * sizeof(double), "maxima")) ||
        (rc = alloc(ctx, (void **)&ctx->mon_part, (size_t)nmon * 2 * sizeof(double), "monitor")))
        return rc;
    CK(cudaMemsetAsync(ctx->maxima, 0, (size_t)ncase * kSlots * 2 * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(ctx->mon_part, 0, (size_t)nmon * 2 * sizeof(double), ctx->stream));
    for (auto &g : ctx->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->state = false;  // the maxima were reset: set the state again
    ctx->mon_nblk = 0;
    return SDDC_OK;
}

extern "C" int sddc_set_persistent(sddc_ctx *ctx, int on)
{
    if (!ctx) return SDDC_EINVAL;
    ctx->persistent = on != 0;
    if (ctx->ncase) {  // the tile tables in the launch's order
        int rc;
        if ((rc = build_tiles(ctx, ctx->cpb, &ctx->tiles_rk, &ctx->ntiles_rk)) ||
            (rc = build_tiles(ctx, 8, &ctx->tiles_diag, &ctx->ntiles_diag)))
            return rc;
    }
    for (auto &g : ctx->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    CK(cudaStreamSynchronize(ctx->stream));
    return SDDC_OK;
}

extern "C" int sddc_get_case_maxima(sddc_ctx *ctx, int icase, double *eigvmax, double *umax)
{
    if (!ctx) return SDDC_EINVAL;
    if (icase < 0 || icase >= std::max(ctx->ncase, 1)) return set_err(ctx, SDDC_EINVAL, "case index out of range");
    CK(cudaMemcpyAsync(ctx->host_small, ctx->maxima + (size_t)icase * kSlots * 2 + 2 * ctx->slot,
                       2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (eigvmax) *eigvmax = ctx->host_small[0];
    if (umax) *umax = ctx->host_small[1];
    return SDDC_OK;
}
