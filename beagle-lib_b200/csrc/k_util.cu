// Small device utilities used by the host instance: filling pre-order root
// partials with the state frequencies.
#include "b200_kernels.h"
#include "b200_vec.cuh"

namespace b200 {

namespace {

// dest[p][c][i] = freqs[i] for i < S, 0 for the padded states
// (CPU/BeagleCPUImpl.hpp:621-676, beagleSetRootPrePartials).  One thread per
// four-state group (Sg is a multiple of 4): one vector store each.
template <typename Real>
__global__ void k_fill_root(Real* dest, const double* __restrict__ freqs, int S, int Sg,
                            size_t ngroups) {
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroups) return;
    const int i0 = 4 * (int)(g % (size_t)(Sg / 4));
    Real v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = (i0 + q < S) ? (Real)freqs[i0 + q] : Real(0);
    st4(dest + 4 * g, v);
}

// The same for several instances (b200_batch.cpp): 256 values per CTA.
template <typename Real>
__global__ void k_fill_batch(const FillSeg* __restrict__ segs, int nseg) {
    __shared__ int s_seg;
    if (threadIdx.x == 0) {
        int lo = 0, hi = nseg - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (segs[mid].first_cta <= (int)blockIdx.x) lo = mid;
            else hi = mid - 1;
        }
        s_seg = lo;
    }
    __syncthreads();
    const FillSeg sg = segs[s_seg];
    const long long idx = (long long)(blockIdx.x - sg.first_cta) * blockDim.x + threadIdx.x;
    if (idx >= sg.n) return;
    const int i = (int)(idx % sg.Sg);
    static_cast<Real*>(sg.dest)[idx] = (i < sg.S) ? (Real)sg.freqs[i] : Real(0);
}

}  // namespace

template <typename Real>
cudaError_t launch_fill_batch(const FillSeg* d_segs, int nseg, int ncta, cudaStream_t s) {
    if (nseg == 0 || ncta == 0) return cudaSuccess;
    k_fill_batch<Real><<<ncta, 256, 0, s>>>(d_segs, nseg);
    return cudaGetLastError();
}

template cudaError_t launch_fill_batch<float>(const FillSeg*, int, int, cudaStream_t);
template cudaError_t launch_fill_batch<double>(const FillSeg*, int, int, cudaStream_t);

template <typename Real>
cudaError_t launch_fill_root(void* dest, const double* freqs, const Dims& d, cudaStream_t s) {
    const size_t ng = (size_t)d.Pp * d.C * d.Sg / 4;
    k_fill_root<Real><<<(unsigned)((ng + 255) / 256), 256, 0, s>>>(static_cast<Real*>(dest), freqs,
                                                                    d.S, d.Sg, ng);
    return cudaGetLastError();
}

template cudaError_t launch_fill_root<float>(void*, const double*, const Dims&, cudaStream_t);
template cudaError_t launch_fill_root<double>(void*, const double*, const Dims&, cudaStream_t);

}  // namespace b200
