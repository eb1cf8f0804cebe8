// Residual evaluation that allocates no device memory (sddc_compresid_noalloc).
//
// For callers that cannot call cudaMalloc: a host whose device memory is all
// handed out by its own pool or budget (a Fortran or C++ solver that
// pre-allocates the GPU at start-up), or a plugin inside another framework
// that owns the allocator.  The call synchronises the caller's stream before
// it returns.  The caller
// passes every input and output as device memory it already holds; the
// working memory the residual needs beyond those (the face traces of the
// state, the running-maxima slots, the AV sensor and the fault flags) lives
// in one file-scope __device__ array of fixed size, which every GPU that
// loads the library keeps until the process exits.

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/sddc.h"
#include "sd_basis.h"
#include "stage_kernel.cuh"
#include "tables_pack.h"

namespace sddc {
cudaError_t launch_stage_exact(int N, int cpb, bool diag, const StageArgs &a, const Ops &ops, cudaStream_t st);
cudaError_t launch_stage_fp64(int N, int cpb, bool diag, const StageArgs &a, const Ops &ops, cudaStream_t st);
cudaError_t launch_stage_mixed(int N, int cpb, bool diag, const StageArgs &a, const Ops &ops, cudaStream_t st);
cudaError_t launch_trace_exact(int N, int ncell, const double *q, void *t, const Ops &ops, cudaStream_t st);
cudaError_t launch_trace_fp64(int N, int ncell, const double *q, void *t, const Ops &ops, cudaStream_t st);
cudaError_t launch_trace_mixed(int N, int ncell, const double *q, void *t, const Ops &ops, cudaStream_t st);
}  // namespace sddc

using namespace sddc;

namespace {

// The shared working memory.  In host code this name is only a stand-in
// for the symbol: its device address comes from cudaGetSymbolAddress.
constexpr size_t kScratchBytes = SDDC_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void *g_scratch_ptr[kMaxDevices] = {};  // device address of g_scratch, per device

// layout inside the scratch array (each part 256-byte aligned)
struct ScratchLayout {
    size_t maxima, flags, sm_ind, trace, total;
};

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

ScratchLayout layout(const sddc_params &p)
{
    ScratchLayout s;
    const size_t elem = p.precision == SDDC_MIXED ? sizeof(float) : sizeof(double);
    s.maxima = 0;                                               // [5][2] doubles
    s.flags = up256(s.maxima + 10 * sizeof(double));            // unsigned
    s.sm_ind = up256(s.flags + sizeof(unsigned));               // (2, NCELL) doubles
    s.trace = up256(s.sm_ind + 2 * (size_t)p.ncell * sizeof(double));
    s.total = s.trace + (size_t)p.ncell * 4 * p.N * 9 * elem;   // face traces
    return s;
}

thread_local std::string g_noalloc_err;

int fail(int code, const std::string &m)
{
    g_noalloc_err = m;
    return code;
}

// device address of the scratch array on the current device, looked up once
// per device by the first call on it (that first call should come before any
// stream capture on the device)
int scratch_on_current_device(unsigned char **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(SDDC_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(SDDC_EINVAL, "device index beyond the supported range");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(SDDC_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = ptr;
    }
    *out = static_cast<unsigned char *>(g_scratch_ptr[dev]);
    return SDDC_OK;
}

}  // namespace

extern "C" const char *sddc_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

extern "C" size_t sddc_noalloc_scratch_bytes(void) { return kScratchBytes; }

extern "C" int sddc_noalloc_packed_sizes(int N, int ncell, size_t *met_doubles, size_t *face_ints)
{
    if (N < 2 || N > kMaxN || ncell < 1) return fail(SDDC_EINVAL, "N must be in [2, 6] and ncell positive");
    if (met_doubles) *met_doubles = (size_t)ncell * met_record_doubles(N);
    if (face_ints) *face_ints = (size_t)ncell * 4 * 2;
    return SDDC_OK;
}

extern "C" int sddc_noalloc_pack_tables(int N, int ncell, const double *S1, const double *S2, const double *Jac,
                                        const int *IF2C, int nface, const int *ibfinter, int ninter,
                                        const int *ibfinl, int ninlet, const int *ibfout, int noutlet,
                                        const int *ibfwal, int nwall, const int *ibfsymp, int nsymp,
                                        const int *ibfree, int nfree, const int *cyc2fpair, int npair,
                                        double *met_out, int *faces_out)
{
    size_t nmet = 0, nfi = 0;
    int rc = sddc_noalloc_packed_sizes(N, ncell, &nmet, &nfi);
    if (rc) return rc;
    if (!S1 || !S2 || !Jac || !IF2C || nface < 1 || !met_out || !faces_out)
        return fail(SDDC_EINVAL, "sddc_noalloc_pack_tables: NULL table or nface < 1");
    pack_metric_records(N, ncell, S1, S2, Jac, met_out);
    const FaceLists fl{IF2C, nface, ibfinter, ninter, ibfinl, ninlet, ibfout, noutlet, ibfwal, nwall,
                       ibfsymp, nsymp, ibfree, nfree, cyc2fpair, npair};
    const std::string msg = build_face_records(ncell, fl, faces_out);
    if (!msg.empty()) return fail(SDDC_EINVAL, "face lists: " + msg);
    return SDDC_OK;
}

extern "C" int sddc_compresid_noalloc(const sddc_params *p, const double *Lmat, const double *Mmat,
                                      const double *q_dev, const double *met_dev, const int *faces_dev,
                                      double eigvmax, double umax, double *resid_dev, double *nablaqs_dev,
                                      double *maxima_out, void *stream)
{
    if (!p || !Lmat || !Mmat || !q_dev || !met_dev || !faces_dev || !resid_dev || !nablaqs_dev)
        return fail(SDDC_EINVAL, "sddc_compresid_noalloc: NULL argument");
    if (p->N < 2 || p->N > kMaxN || p->ncell < 1) return fail(SDDC_EINVAL, "N must be in [2, 6] and ncell positive");
    if (p->precision < SDDC_FP64_EXACT || p->precision > SDDC_MIXED) return fail(SDDC_EINVAL, "unknown precision");
    if (p->vismode != 0 && p->vismode != 1) return fail(SDDC_EINVAL, "vismode must be 0 or 1");
    if (p->mu != 0.0 || p->eta0 != 0.0) return fail(SDDC_EINVAL, "mu and eta0 must be 0");
    const ScratchLayout L = layout(*p);
    if (L.total > kScratchBytes)
        return fail(SDDC_EINVAL, "case too large for the fixed scratch array: needs " + std::to_string(L.total) +
                                     " bytes, the array holds " + std::to_string(kScratchBytes));
    unsigned char *scratch = nullptr;
    int rc = scratch_on_current_device(&scratch);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int N = p->N, N1 = N + 1, NL = N - 1;

    // operators (kernel parameters, no device memory)
    Ops ops{};
    for (int r = 0; r < N1; r++)
        for (int s = 0; s < N; s++) {
            ops.L[r * N + s] = Lmat[r + N1 * s];
            ops.M[r * N + s] = Mmat[r + N1 * s];
            ops.Lf[r * N + s] = (float)Lmat[r + N1 * s];
            ops.Mf[r * N + s] = (float)Mmat[r + N1 * s];
        }
    double Xs[kMaxN], Xf[kMaxN + 1], Xl[kMaxN], Xlf[kMaxN + 1];
    sd_points(N, Xs, Xf);
    sd_points(NL, Xl, Xlf);
    for (int l = 0; l < NL; l++)
        for (int s = 0; s < N; s++) ops.H[l * N + s] = lagrange(Xs, N, s + 1, Xl[l]);
    for (int s = 0; s < N; s++)
        for (int l = 0; l < NL; l++) ops.HL[s * NL + l] = lagrange(Xl, NL, l + 1, Xs[s]);

    // clear what must start from zero; seed every running-max slot
    double *maxima = reinterpret_cast<double *>(scratch + L.maxima);
    unsigned *flags = reinterpret_cast<unsigned *>(scratch + L.flags);
    double seed[10];
    for (int s = 0; s < 5; s++) {
        seed[2 * s] = eigvmax;
        seed[2 * s + 1] = umax;
    }
    cudaError_t e = cudaMemcpyAsync(maxima, seed, sizeof(seed), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(flags, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return fail(SDDC_ECUDA, std::string("scratch set-up: ") + cudaGetErrorString(e));

    void *trace = scratch + L.trace;
    switch (p->precision) {
    case SDDC_FP64_EXACT: e = launch_trace_exact(N, p->ncell, q_dev, trace, ops, st); break;
    case SDDC_FP64: e = launch_trace_fp64(N, p->ncell, q_dev, trace, ops, st); break;
    default: e = launch_trace_mixed(N, p->ncell, q_dev, trace, ops, st); break;
    }
    if (e != cudaSuccess) return fail(SDDC_ECUDA, std::string("trace kernel: ") + cudaGetErrorString(e));

    StageArgs a{};
    a.ncell = p->ncell;
    a.vismode = p->vismode;
    a.artiv = p->artiv;
    a.alpha = 2.0;  // initsetup.f90:165
    a.fs = Freestream{p->rinf, p->pinf, p->uinf, p->vinf, p->bxinf, p->byinf};
    a.rk_kind = kRkNone;
    a.q_in = q_dev;
    a.t_in = trace;
    a.met = met_dev;
    a.faces = reinterpret_cast<const int2 *>(faces_dev);
    a.maxima = maxima;
    a.slot_r = 0;
    a.slot_w = 1;
    a.sm_ind = reinterpret_cast<double *>(scratch + L.sm_ind);
    a.resid_out = resid_dev;
    a.grad_out = nablaqs_dev;
    a.mon_part = nullptr;
    a.err_flags = flags;
    switch (p->precision) {
    case SDDC_FP64_EXACT: e = launch_stage_exact(N, 8, true, a, ops, st); break;
    case SDDC_FP64: e = launch_stage_fp64(N, 8, true, a, ops, st); break;
    default: e = launch_stage_mixed(N, 8, true, a, ops, st); break;
    }
    if (e != cudaSuccess) return fail(SDDC_ECUDA, std::string("stage kernel: ") + cudaGetErrorString(e));

    // running maxima after the evaluation and the fault flags
    double out[2];
    unsigned f = 0;
    e = cudaMemcpyAsync(out, maxima + 2, sizeof(out), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&f, flags, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(SDDC_ECUDA, std::string("read-back: ") + cudaGetErrorString(e));
    if (maxima_out) {
        maxima_out[0] = out[0];
        maxima_out[1] = out[1];
    }
    if (f) return fail(SDDC_ENUMERIC, "device numerics: non-positive density or non-finite wave speed");
    return SDDC_OK;
}
