// Output from the device state: the reference's restart file
// (WRITE_ALL_DATA_PARALLEL, write_data.f90:1-83) and Tecplot file
// (tecplotter2d + tecpost_parallel, tecplotter.f90:1-415), both written every
// nwrite iterations at iterations.f90:77-80.
//
// The file write is taken off the stepping path.  On the context's stream a
// write call only snapshots what it needs (a device-to-device copy of the
// state, or the plot-node kernel into a plot buffer) and records an event; a
// side stream copies the snapshot to pinned host memory after that event, and
// a host thread waits for the copy and writes the file while the next steps
// run.  Each kind of output has one snapshot, one pinned buffer and one writer
// thread, so a restart and a Tecplot file are written side by side; a second
// write of the same kind waits (on the host) until the first file is written.
//
// This unit is compiled without multiply-add contraction: the plot-node
// values are the reference's FP64 operations in the reference's order, so
// they match the CPU restatement bit for bit before the conversion to float.
#include <condition_variable>
#include <mutex>
#include <thread>

#include "context_impl.h"
#include "output_format.h"
#include "sd_basis.h"

using namespace sddc;

namespace sddc {

constexpr int kPlotOut = 11;  // rho u v w p Bx By Bz psi muAV etaAV
enum { kJobRestart = 0, kJobTecplot = 1 };

// One thread per plot node: tecplotter2d (tecplotter.f90:16-54) for that
// node.  The cells that touch the node are visited in ascending order, as the
// reference's cell loop adds them; each adds its interpolant at the node,
// sum over js (outer) and is (inner) of Q * h_is(xsi) * h_js(eta), and its
// muAV.  Then the division by gnode_factor and the conversion to rho, u, v,
// w, p (the gas pressure without the psi term, as tecplotter2d has it),
// Bx, By, Bz, psi.  out is [kPlotOut][plotnodes].
__global__ void plot_nodes_kernel(int plotnodes, int N, int nre, const double *__restrict__ q,
                                  const double *__restrict__ muav, const int *__restrict__ node_ptr,
                                  const int *__restrict__ node_pts, const int *__restrict__ gfac,
                                  const double *__restrict__ hv, double *__restrict__ out)
{
    const int nd = blockIdx.x * blockDim.x + threadIdx.x;
    if (nd >= plotnodes) return;
    const int np1 = nre + 1, npt = np1 * np1, nn = N * N;
    double acc[9], av0 = 0.0, av1 = 0.0;
#pragma unroll
    for (int v = 0; v < 9; v++) acc[v] = 0.0;
    for (int k = node_ptr[nd]; k < node_ptr[nd + 1]; k++) {
        const int code = node_pts[k];
        const int c = code / npt, r = code - c * npt, jj = r / np1, ii = r - jj * np1;
        const double *qc = q + (size_t)c * 9 * nn;
        const double *hx = hv + ii * N, *hy = hv + jj * N;
        double s[9];
#pragma unroll
        for (int v = 0; v < 9; v++) s[v] = 0.0;
        for (int js = 0; js < N; js++) {
            const double hj = hy[js];
            for (int is = 0; is < N; is++) {
                const double hi = hx[is];
                const double *qp = qc + 9 * (is + N * js);
#pragma unroll
                for (int v = 0; v < 9; v++) s[v] = s[v] + qp[v] * hi * hj;
            }
        }
#pragma unroll
        for (int v = 0; v < 9; v++) acc[v] = acc[v] + s[v];
        if (muav) {
            av0 = av0 + muav[2 * (size_t)c];
            av1 = av1 + muav[2 * (size_t)c + 1];
        }
    }
    const double g = (double)gfac[nd];
    double Qs[9];
#pragma unroll
    for (int v = 0; v < 9; v++) Qs[v] = acc[v] / g;
    const double u = Qs[1] / Qs[0], vv = Qs[2] / Qs[0], w = Qs[3] / Qs[0];
    const double norm_u = u * u + vv * vv + w * w;
    const double norm_b = Qs[5] * Qs[5] + Qs[6] * Qs[6] + Qs[7] * Qs[7];
    const double p = (Qs[4] - 0.5 * Qs[0] * norm_u - 0.5 * norm_b) * (kGam - 1.0);
    const size_t P = (size_t)plotnodes;
    out[0 * P + nd] = Qs[0];
    out[1 * P + nd] = u;
    out[2 * P + nd] = vv;
    out[3 * P + nd] = w;
    out[4 * P + nd] = p;
    out[5 * P + nd] = Qs[5];
    out[6 * P + nd] = Qs[6];
    out[7 * P + nd] = Qs[7];
    out[8 * P + nd] = Qs[8];
    out[9 * P + nd] = av0 / g;
    out[10 * P + nd] = av1 / g;
}

struct Output {
    struct Job {
        int kind;
        std::string path;
        int iter;
        double ctime;
        std::vector<int> icg;
    };
    int device = 0, N = 0, ncell = 0;
    cudaStream_t copy = nullptr;
    cudaEvent_t ev_in[2] = {}, ev_out[2] = {};
    // plot mesh (sddc_set_plot)
    int nre = 0, plotnodes = 0, plotcells = 0;
    std::vector<double> plotx;
    std::vector<int> connec;
    int *node_ptr = nullptr, *node_pts = nullptr, *gfac = nullptr;
    double *hv = nullptr;
    // snapshots (device) and their pinned host copies
    double *d_buf[2] = {}, *h_buf[2] = {};
    size_t buf_doubles[2] = {};
    // background writers, one per kind; a kind holds at most one job
    std::thread worker[2];
    std::mutex mu;
    std::condition_variable cv;
    Job job[2];
    bool queued[2] = {false, false};
    bool busy[2] = {false, false};  // the kind's buffers are held by a queued or running job
    bool stop = false;
    int err = 0;
    std::string msg;

    void run(int kind);
    void wait_kind(int kind)
    {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return !busy[kind]; });
    }
    void wait_all()
    {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return !busy[0] && !busy[1]; });
    }
    void free_plot()
    {
        cudaFree(node_ptr);
        cudaFree(node_pts);
        cudaFree(gfac);
        cudaFree(hv);
        node_ptr = node_pts = gfac = nullptr;
        hv = nullptr;
        plotnodes = plotcells = nre = 0;
    }
};

void Output::run(int kind)
{
    cudaSetDevice(device);
    for (;;) {
        Job j;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return stop || queued[kind]; });
            if (!queued[kind]) return;
            j = std::move(job[kind]);
            queued[kind] = false;
        }
        int rc = SDDC_OK;
        std::string em;
        const cudaError_t e = cudaEventSynchronize(ev_out[j.kind]);
        if (e != cudaSuccess) {
            rc = SDDC_ECUDA;
            em = std::string("output copy: ") + cudaGetErrorString(e);
        } else if (j.kind == kJobRestart) {
            if (fmt::write_restart(j.path.c_str(), j.iter, j.ctime, N, ncell, j.icg.empty() ? nullptr : j.icg.data(),
                                   h_buf[kJobRestart], em))
                rc = SDDC_EIO;
        } else {
            const double *h = h_buf[kJobTecplot];
            const size_t P = (size_t)plotnodes;
            fmt::PlotVar vars[fmt::kPlotVars] = {{plotx.data(), 2}, {plotx.data() + 1, 2}};
            for (int v = 0; v < kPlotOut; v++) vars[2 + v] = {h + v * P, 1};
            if (fmt::write_tecplot(j.path.c_str(), j.ctime, plotnodes, plotcells, vars, connec.data(), em))
                rc = SDDC_EIO;
        }
        std::lock_guard<std::mutex> lk(mu);
        busy[j.kind] = false;
        if (rc && !err) {
            err = rc;
            msg = em;
        }
        cv.notify_all();
    }
}

}  // namespace sddc

void sddc::output_free(sddc_ctx *ctx)
{
    Output *o = ctx->out;
    if (!o) return;
    {
        std::lock_guard<std::mutex> lk(o->mu);
        o->stop = true;
    }
    o->cv.notify_all();
    for (auto &w : o->worker)
        if (w.joinable()) w.join();  // each writes what is queued first
    o->free_plot();
    for (int k = 0; k < 2; k++) {
        cudaFree(o->d_buf[k]);
        if (o->h_buf[k]) cudaFreeHost(o->h_buf[k]);
        if (o->ev_in[k]) cudaEventDestroy(o->ev_in[k]);
        if (o->ev_out[k]) cudaEventDestroy(o->ev_out[k]);
    }
    if (o->copy) cudaStreamDestroy(o->copy);
    delete o;
    ctx->out = nullptr;
}

static int output_init(sddc_ctx *ctx)
{
    if (ctx->out) return SDDC_OK;
    auto *o = new Output();
    ctx->out = o;
    o->N = ctx->N;
    o->ncell = ctx->ncell;
    CK(cudaGetDevice(&o->device));
    CK(cudaStreamCreateWithFlags(&o->copy, cudaStreamNonBlocking));
    for (int k = 0; k < 2; k++) {
        CK(cudaEventCreateWithFlags(&o->ev_in[k], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&o->ev_out[k], cudaEventDisableTiming));
    }
    for (int k = 0; k < 2; k++) o->worker[k] = std::thread([o, k] { o->run(k); });
    return SDDC_OK;
}

// device snapshot and pinned host buffer of one kind, at least n doubles
static int output_buffers(sddc_ctx *ctx, int kind, size_t n)
{
    Output *o = ctx->out;
    if (o->buf_doubles[kind] >= n) return SDDC_OK;
    cudaFree(o->d_buf[kind]);
    if (o->h_buf[kind]) cudaFreeHost(o->h_buf[kind]);
    o->d_buf[kind] = o->h_buf[kind] = nullptr;
    o->buf_doubles[kind] = 0;
    int rc = alloc(ctx, (void **)&o->d_buf[kind], n * sizeof(double), "output snapshot");
    if (rc) return rc;
    cudaError_t e = cudaMallocHost((void **)&o->h_buf[kind], n * sizeof(double));
    if (e != cudaSuccess) {
        cudaGetLastError();
        o->h_buf[kind] = nullptr;
        return set_err(ctx, SDDC_ENOMEM, std::string("cudaMallocHost output buffer: ") + cudaGetErrorString(e));
    }
    o->buf_doubles[kind] = n;
    return SDDC_OK;
}

// snapshot on the context's stream is done: copy it to the pinned buffer on
// the side stream and hand the job to the writer
static int output_submit(sddc_ctx *ctx, Output::Job &&job, size_t n)
{
    Output *o = ctx->out;
    const int k = job.kind;
    CK(cudaEventRecord(o->ev_in[k], ctx->stream));
    CK(cudaStreamWaitEvent(o->copy, o->ev_in[k], 0));
    CK(cudaMemcpyAsync(o->h_buf[k], o->d_buf[k], n * sizeof(double), cudaMemcpyDeviceToHost, o->copy));
    CK(cudaEventRecord(o->ev_out[k], o->copy));
    {
        std::lock_guard<std::mutex> lk(o->mu);
        o->busy[k] = true;
        o->queued[k] = true;
        o->job[k] = std::move(job);
    }
    o->cv.notify_all();
    return SDDC_OK;
}

// the plot-node kernel into the Tecplot snapshot buffer, on the stream
static int launch_plot(sddc_ctx *ctx)
{
    Output *o = ctx->out;
    if (!o || !o->plotnodes) return set_err(ctx, SDDC_ESTATE, "no plot mesh: call sddc_set_plot first");
    if (ctx->ncase) return set_err(ctx, SDDC_ESTATE, "Tecplot output is per case: write each case from its own context");
    int rc = output_buffers(ctx, kJobTecplot, (size_t)kPlotOut * o->plotnodes);
    if (rc) return rc;
    // muAV exists in the reference only with vismode = 1 and ARTIV = 1
    // (initsetup.f90:36-41); otherwise the plot's muAV and etaAV are 0
    const double *mu = nullptr;
    if (ctx->p.vismode == 1 && ctx->p.artiv == 1) {
        if ((rc = device_muav(ctx))) return rc;
        mu = ctx->muav;
    }
    plot_nodes_kernel<<<(o->plotnodes + 255) / 256, 256, 0, ctx->stream>>>(
        o->plotnodes, ctx->N, o->nre, ctx->reg[0], mu, o->node_ptr, o->node_pts, o->gfac, o->hv,
        o->d_buf[kJobTecplot]);
    CK(cudaGetLastError());
    return SDDC_OK;
}

extern "C" int sddc_set_plot(sddc_ctx *ctx, int nre, int plotnodes, int plotcells, const double *plotx,
                             const int *gnumnode, const int *gnode_factor, const int *connec)
{
    if (!ctx) return SDDC_EINVAL;
    if (!ctx->tables) return set_err(ctx, SDDC_ESTATE, "tables not set (call sddc_set_tables)");
    int rc = SDDC_OK;
    if (nre < 1 || nre > 64 || plotnodes < 1 || !plotx || !gnumnode || !gnode_factor || !connec)
        return set_err(ctx, SDDC_EINVAL, "sddc_set_plot: bad arguments");
    const int np1 = nre + 1;
    const size_t npt = (size_t)np1 * np1, npts = npt * ctx->ncell;
    if (npts >= ((size_t)1 << 31)) return set_err(ctx, SDDC_EINVAL, "sddc_set_plot: plot mesh too large");
    if ((size_t)plotcells != (size_t)nre * nre * ctx->ncell)
        return set_err(ctx, SDDC_EINVAL, "sddc_set_plot: plotcells must be nre^2 * NCELL");
    // node -> its (cell, ii, jj) points, cells ascending
    std::vector<int> cnt(plotnodes + 1, 0);
    for (size_t i = 0; i < npts; i++) {
        const int g = gnumnode[i];
        if (g < 1 || g > plotnodes) return set_err(ctx, SDDC_EINVAL, "sddc_set_plot: gnumnode out of range");
        cnt[g]++;
    }
    for (int g = 0; g < plotnodes; g++)
        if (gnode_factor[g] < 1) return set_err(ctx, SDDC_EINVAL, "sddc_set_plot: gnode_factor must be >= 1");
    for (size_t i = 0; i < 4 * (size_t)plotcells; i++)
        if (connec[i] < 1 || connec[i] > plotnodes) return set_err(ctx, SDDC_EINVAL, "sddc_set_plot: connec out of range");
    std::vector<int> ptr(plotnodes + 1, 0), pts(npts);
    for (int g = 1; g <= plotnodes; g++) ptr[g] = ptr[g - 1] + cnt[g];
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    for (int c = 0; c < ctx->ncell; c++)
        for (int jj = 0; jj < np1; jj++)
            for (int ii = 0; ii < np1; ii++) {
                const int g = gnumnode[ii + np1 * (jj + (size_t)np1 * c)] - 1;
                pts[fill[g]++] = (int)(c * npt) + jj * np1 + ii;
            }
    // Lagrange basis of the solution points at the plot points (i / nre)
    double Xs[kMaxN], Xf[kMaxN + 1];
    sd_points(ctx->N, Xs, Xf);
    std::vector<double> hv((size_t)np1 * ctx->N);
    for (int i = 0; i < np1; i++)
        for (int s = 0; s < ctx->N; s++) hv[i * ctx->N + s] = lagrange(Xs, ctx->N, s + 1, (double)i / (double)nre);
    if ((rc = output_init(ctx))) return rc;
    Output *o = ctx->out;
    o->wait_kind(kJobTecplot);  // a queued Tecplot file still reads the old mesh
    o->free_plot();
    if ((rc = alloc(ctx, (void **)&o->node_ptr, ptr.size() * sizeof(int), "plot nodes")) ||
        (rc = alloc(ctx, (void **)&o->node_pts, pts.size() * sizeof(int), "plot points")) ||
        (rc = alloc(ctx, (void **)&o->gfac, (size_t)plotnodes * sizeof(int), "gnode_factor")) ||
        (rc = alloc(ctx, (void **)&o->hv, hv.size() * sizeof(double), "plot basis")))
        return rc;
    CK(cudaMemcpyAsync(o->node_ptr, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(o->node_pts, pts.data(), pts.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(o->gfac, gnode_factor, (size_t)plotnodes * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(o->hv, hv.data(), hv.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    // the snapshot and pinned buffers now, not in the first write call
    if ((rc = output_buffers(ctx, kJobTecplot, (size_t)kPlotOut * plotnodes))) return rc;
    o->plotx.assign(plotx, plotx + 2 * (size_t)plotnodes);
    o->connec.assign(connec, connec + 4 * (size_t)plotcells);
    o->nre = nre;
    o->plotnodes = plotnodes;
    o->plotcells = plotcells;
    return SDDC_OK;
}

extern "C" int sddc_plot_nodes(sddc_ctx *ctx, double *plotq, double *plotav)
{
    int rc = ready(ctx);
    if (rc) return rc;
    Output *o = ctx->out;
    if (!o || !o->plotnodes) return set_err(ctx, SDDC_ESTATE, "no plot mesh: call sddc_set_plot first");
    o->wait_kind(kJobTecplot);
    if ((rc = launch_plot(ctx))) return rc;
    const size_t P = (size_t)o->plotnodes;
    std::vector<double> h(kPlotOut * P);
    CK(cudaMemcpyAsync(h.data(), o->d_buf[kJobTecplot], h.size() * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (size_t i = 0; i < P; i++) {
        if (plotq)
            for (int v = 0; v < 9; v++) plotq[9 * i + v] = h[v * P + i];
        if (plotav) {
            plotav[2 * i] = h[9 * P + i];
            plotav[2 * i + 1] = h[10 * P + i];
        }
    }
    return check_flags(ctx);
}

extern "C" int sddc_write_tecplot(sddc_ctx *ctx, const char *path)
{
    int rc = ready(ctx);
    if (rc) return rc;
    Output *o = ctx->out;
    if (!o || !o->plotnodes) return set_err(ctx, SDDC_ESTATE, "no plot mesh: call sddc_set_plot first");
    o->wait_kind(kJobTecplot);
    if ((rc = launch_plot(ctx))) return rc;
    Output::Job j{kJobTecplot, path ? std::string(path) : "./TEC/" + fmt::tecplot_name(ctx->ctime), 0, ctx->ctime,
                  {}};
    return output_submit(ctx, std::move(j), (size_t)kPlotOut * o->plotnodes);
}

extern "C" int sddc_write_restart(sddc_ctx *ctx, const char *path, int iter, const int *icg)
{
    int rc = ready(ctx);
    if (rc) return rc;
    if ((rc = output_init(ctx))) return rc;
    Output *o = ctx->out;
    o->wait_kind(kJobRestart);
    if ((rc = output_buffers(ctx, kJobRestart, ctx->nq))) return rc;
    CK(cudaMemcpyAsync(o->d_buf[kJobRestart], ctx->reg[0], ctx->nq * sizeof(double), cudaMemcpyDeviceToDevice,
                       ctx->stream));
    Output::Job j{kJobRestart, path ? std::string(path) : fmt::restart_name(iter), iter, ctx->ctime, {}};
    if (icg) j.icg.assign(icg, icg + ctx->ncell);
    return output_submit(ctx, std::move(j), ctx->nq);
}

extern "C" int sddc_output_wait(sddc_ctx *ctx)
{
    if (!ctx) return SDDC_EINVAL;
    Output *o = ctx->out;
    if (!o) return SDDC_OK;
    o->wait_all();
    std::lock_guard<std::mutex> lk(o->mu);
    const int e = o->err;
    const std::string m = o->msg;
    o->err = 0;
    o->msg.clear();
    return e ? set_err(ctx, e, m) : SDDC_OK;
}
