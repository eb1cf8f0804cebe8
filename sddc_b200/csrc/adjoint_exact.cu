// The adjoint's kernels that must round as the exact forward stage kernel
// does (compiled with -fmad=false, like stage_exact.cu): locating the points
// that raised a running maximum (found by equality with the recorded
// maximum) and the wall force of the objective.

#include "adjoint_kernel.cuh"

namespace sddc {

template <int N> static void locate_n(int nblk, const LocateArgs &a, const Ops &ops, cudaStream_t st)
{
    // one thread per forward CTA checks its recorded maxima
    adj_locate_kernel<N><<<(nblk + kLocateThreads - 1) / kLocateThreads, kLocateThreads, 0, st>>>(a, ops, nblk);
}

cudaError_t launch_adj_locate(int N, int nblk, const LocateArgs &a, const Ops &ops, cudaStream_t st)
{
    switch (N) {
    case 2: locate_n<2>(nblk, a, ops, st); break;
    case 3: locate_n<3>(nblk, a, ops, st); break;
    case 4: locate_n<4>(nblk, a, ops, st); break;
    case 5: locate_n<5>(nblk, a, ops, st); break;
    default: locate_n<6>(nblk, a, ops, st); break;
    }
    return cudaGetLastError();
}

template <int N>
static void wall_n(int nw, const int2 *wall, const double *t, const double *met, int vismode, const Freestream &fs,
                   const double *wq, double *out, cudaStream_t st)
{
    wall_force_kernel<N><<<1, 256, 0, st>>>(nw, wall, t, met, vismode, fs, wq, out);
}

cudaError_t launch_wall_force(int N, int nw, const int2 *wall, const double *t, const double *met, int vismode,
                              const Freestream &fs, const double *wq, double *out, cudaStream_t st)
{
    switch (N) {
    case 2: wall_n<2>(nw, wall, t, met, vismode, fs, wq, out, st); break;
    case 3: wall_n<3>(nw, wall, t, met, vismode, fs, wq, out, st); break;
    case 4: wall_n<4>(nw, wall, t, met, vismode, fs, wq, out, st); break;
    case 5: wall_n<5>(nw, wall, t, met, vismode, fs, wq, out, st); break;
    default: wall_n<6>(nw, wall, t, met, vismode, fs, wq, out, st); break;
    }
    return cudaGetLastError();
}

}  // namespace sddc
