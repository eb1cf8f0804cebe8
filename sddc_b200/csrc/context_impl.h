// Internal declarations shared by the host runtime's translation units
// (context.cu: the forward drop-in; adjoint.cu: the discrete adjoint).
// Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/sddc.h"
#include "stage_kernel.cuh"

#define SDDC_INTERNAL __attribute__((visibility("hidden")))

namespace sddc {
struct AdjWs;
struct Output;
cudaError_t launch_stage_exact(int N, int cpb, bool diag, const StageArgs &a, const Ops &ops, cudaStream_t st);
cudaError_t launch_stage_fp64(int N, int cpb, bool diag, const StageArgs &a, const Ops &ops, cudaStream_t st);
cudaError_t launch_stage_mixed(int N, int cpb, bool diag, const StageArgs &a, const Ops &ops, cudaStream_t st);
cudaError_t launch_trace_exact(int N, int ncell, const double *q, void *t, const Ops &ops, cudaStream_t st);
cudaError_t launch_trace_fp64(int N, int ncell, const double *q, void *t, const Ops &ops, cudaStream_t st);
cudaError_t launch_trace_mixed(int N, int ncell, const double *q, void *t, const Ops &ops, cudaStream_t st);
struct ViscArgs;
cudaError_t launch_visc_exact(int N, const ViscArgs &a, const Ops &ops, cudaStream_t st);
cudaError_t launch_visc_fp64(int N, const ViscArgs &a, const Ops &ops, cudaStream_t st);
cudaError_t launch_visc_mixed(int N, const ViscArgs &a, const Ops &ops, cudaStream_t st);
}  // namespace sddc


namespace sddc {

constexpr int kSlots = 5;     // rotating running-max slots
constexpr int kRegs = 6;      // RK registers (FiveStageRk needs six)
constexpr int kMonThreads = 256;

// RK_S5P3 coefficients, iterations.f90:164-174
constexpr double A30 = 0.355909775063327, A32 = 0.644090224936674, A40 = 0.367933791638137,
                 A43 = 0.632066208361863, A52 = 0.237593836598569, A54 = 0.762406163401431,
                 B10 = 0.377268915331368, B21 = 0.377268915331368, B32 = 0.242995220537396,
                 B43 = 0.238458932846290, B54 = 0.287632146308408;
// FiveStageRk coefficients, iterations.f90:108-150
constexpr double F11 = 0.39175222700392, F21 = 0.44437049406734, F22 = 0.55562950593266,
                 F23 = 0.36841059262959, F31 = 0.6201018513854, F32 = 0.3798981486146,
                 F33 = 0.25189177424738, F41 = 0.17807995410773, F42 = 0.82192004589227,
                 F43 = 0.54497475021237, F51 = 0.00683325884039, F52 = 0.51723167208978,
                 F53 = 0.12759831133288, F54 = 0.34833675773694, F55 = 0.08460416338212,
                 F56 = 0.22600748319395;

}  // namespace sddc

struct sddc_ctx {
    using Ops = sddc::Ops;
    using CaseParams = sddc::CaseParams;
    sddc_params p{};
    int N = 0, ncell = 0, cpb = 8, msize = 0, grid = 0;
    size_t nq = 0;  // doubles per state
    cudaStream_t stream = nullptr;
    std::string err;
    double *reg[sddc::kRegs] = {};
    void *trace[sddc::kRegs] = {};  // face traces of each register (float in the mixed form)
    size_t trace_bytes = 0;
    double *met = nullptr;
    // the metrics split for the stage kernel's staging copies: normals in the
    // form's arithmetic type [NCELL][4N(N+1)] and Jac [NCELL][kJacPad]
    void *nrm = nullptr;
    double *jac = nullptr;
    bool nrm_double = true;  // normals stored as double (FP64 forms)
    bool jac_inv = false;    // jac holds 1/Jac (the forms other than the exact one)
    int2 *faces = nullptr;
    double *maxima = nullptr;  // [sddc::kSlots][2]
    double *sm_ind = nullptr, *muav = nullptr, *resid = nullptr, *grad = nullptr;
    double *mon_part = nullptr, *mon_out = nullptr, *int_part = nullptr, *wq = nullptr;
    unsigned *err_flags = nullptr;
    double *host_small = nullptr;  // pinned scratch for small read-backs
    Ops ops{};
    int slot = 0;  // slot holding the running maxima after the last evaluation
    // The AV sensor enters no residual (its coefficients are zero,
    // getrusanov.f90:326,328), so the RK stages skip it; when muAV or SM_IND
    // is read after steps, it is evaluated from the last stage's input
    // register with the maxima that stage read, which is what the reference
    // holds after RK_S5P3 / FiveStageRk.
    bool sensor_stale = false;
    int last_in = 0;            // register that was the last stage's input
    double *max_scratch = nullptr;  // copy of the maxima for that evaluation
    int mon_nblk = 0;  // CTAs of the last launch that wrote monitor partials
    bool tables = false, state = false;
    bool traces_stale = true;  // trace[0] does not match reg[0] yet
    double ctime = 0.0;
    cudaGraphExec_t graph[sddc::kSlots] = {};
    double graph_dt[sddc::kSlots] = {};
    // batch of independent cases (sddc_set_cases); ncase == 0 for one case
    int ncase = 0;
    std::vector<sddc_case> cases;
    CaseParams *case_dev = nullptr;
    int4 *tiles_rk = nullptr, *tiles_diag = nullptr;
    int ntiles_rk = 0, ntiles_diag = 0;
    bool persistent = false;  // batch stages as grid-stride persistent launches
    // discrete adjoint work space (adjoint.cu), created on first use
    sddc::AdjWs *adj = nullptr;
    // viscous / resistive chain (vismode = 1 with mu or eta0 nonzero)
    bool visc = false;
    double *visc_grad = nullptr;  // nablaQs (9,2,N,N,NCELL)
    double *visc_gt = nullptr;    // gradient traces [cell][lf][nfp][18]
    double *visc_rv = nullptr;    // dFv + dGv (9,N,N,NCELL)
    double *met2 = nullptr;       // [cell][lf][nfp][2]: the other normal row at each face point
    // restart / Tecplot output (output.cu), created on first use
    sddc::Output *out = nullptr;
    // decomposed run: processor faces (slot order) and the host's exchange
    std::vector<int> ibfproc;
    int2 *proc_cells = nullptr;  // [slot]: own cell (0-based), own local face
    sddc_exchange_fn exch = nullptr;
    void *exch_user = nullptr;
    void *proc_send = nullptr, *proc_recv = nullptr;
    double *proc_max = nullptr;
    bool proc_stale = false;  // the exchange of the current state's traces is due
};


namespace sddc {
SDDC_INTERNAL int set_err(sddc_ctx *c, int code, const std::string &m);
SDDC_INTERNAL int cuda_err(sddc_ctx *c, cudaError_t e, const char *what);
SDDC_INTERNAL int alloc(sddc_ctx *ctx, void **p, size_t bytes, const char *what);
SDDC_INTERNAL int ready(sddc_ctx *ctx);
SDDC_INTERNAL int check_flags(sddc_ctx *ctx);
SDDC_INTERNAL int met_size(int N);
SDDC_INTERNAL StageArgs base_args(sddc_ctx *ctx);
SDDC_INTERNAL void adjoint_free(sddc_ctx *ctx);
SDDC_INTERNAL void output_free(sddc_ctx *ctx);
SDDC_INTERNAL int device_muav(sddc_ctx *ctx);
}  // namespace sddc

#define CK(call)                                                              \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return cuda_err(ctx, e_, #call);               \
    } while (0)

