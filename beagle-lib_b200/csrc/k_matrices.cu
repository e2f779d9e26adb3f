// Transition matrices on the device: P(t) from the eigen cube in FP64, and
// the matrix-pair operations (convolution, transpose).
//
// P[c][i][j] = max(0, sum_k cube[i][j][k] * exp(lambda_k * (t * r_c))),
// dP = sum_k cube[i][j][k] * (lambda_k r_c) e^(..), d2P with (lambda_k r_c)^2,
// following CPU/EigenDecompositionCube.hpp:105-322 (cube from :69-100); with
// model categories, category c takes its own eigen system and r_c = 1
// (:326-470).  The
// missing-state column of the reference's padded layout is not stored here:
// its value travels with each matrix (1 for P, 0 for derivatives).
#include "b200_kernels.h"

namespace b200 {

namespace {

// One block per (job, category, slice of the entries).  exp(.) is evaluated
// once per eigenvalue in shared memory; each thread then forms entries (i, j)
// with a sequential FP64 sum over k (the reference's order), clamps P at 0
// and rounds to Real.  The cube is stored [i][k][j], so for each k a warp's
// consecutive entries of a row read consecutive words.
template <typename Real>
__global__ void __launch_bounds__(256)
k_update_matrices(const MatJob* __restrict__ jobs, int S, int Sg) {
    extern __shared__ double sh[];
    double* ex = sh;
    double* e1 = sh + S;
    double* e2 = sh + 2 * S;
    const MatJob jb = jobs[blockIdx.x];
    const int c = blockIdx.y;
    const int C = gridDim.y;
    const double* cube = jb.cube;
    const double* evals = jb.evals;
    double r;
    if (jb.cat_eig) {           // CPU/EigenDecompositionCube.hpp:326-470: no category rate
        const int e = jb.cat_eig[c];
        cube += (size_t)e * S * S * S;
        evals += (size_t)e * S;
        r = 1.0;
    } else {
        r = jb.rates[c];
    }
    const double t = jb.tlen ? *jb.tlen : jb.t;
    for (int k = threadIdx.x; k < S; k += blockDim.x) {
        const double lam = evals[k];
        const double v = exp(lam * (t * r));
        const double sl = lam * r;
        ex[k] = v;
        e1[k] = sl * v;
        e2[k] = sl * sl * v;
    }
    __syncthreads();
    Real* P = static_cast<Real*>(jb.p) + (size_t)c * Sg * Sg;
    Real* D1 = jb.d1 ? static_cast<Real*>(jb.d1) + (size_t)c * Sg * Sg : nullptr;
    Real* D2 = jb.d2 ? static_cast<Real*>(jb.d2) + (size_t)c * Sg * Sg : nullptr;
    (void)C;
    for (int idx = blockIdx.z * blockDim.x + threadIdx.x; idx < Sg * Sg;
         idx += gridDim.z * blockDim.x) {
        const int i = idx / Sg, j = idx - (idx / Sg) * Sg;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        if (i < S && j < S) {
            const double* cu = cube + (size_t)i * S * S + j;
            if (D1) {
                for (int k = 0; k < S; ++k) {
                    const double cv = cu[(size_t)k * S];
                    s0 += cv * ex[k];
                    s1 += cv * e1[k];
                    s2 += cv * e2[k];
                }
            } else {
                for (int k = 0; k < S; ++k) s0 += cu[(size_t)k * S] * ex[k];
            }
            if (!(s0 > 0.0)) s0 = 0.0;
        }
        P[idx] = (Real)s0;
        if (D1) D1[idx] = (Real)s1;
        if (D2) D2[idx] = (Real)s2;
        const size_t tix = (size_t)c * Sg * Sg + j * Sg + i;   // transposed image
        static_cast<Real*>(jb.pt)[tix] = (Real)s0;
        if (D1) static_cast<Real*>(jb.d1t)[tix] = (Real)s1;
        if (D2) static_cast<Real*>(jb.d2t)[tix] = (Real)s2;
    }
}

// The same for small state counts (Sg <= 8, at most 64 entries a matrix):
// a 256-thread block takes 256 / Sg^2 (job, category) items, one group of
// Sg^2 threads each, instead of one item with most threads idle.  Each
// group's exponentials go to its own slice of shared memory.
template <typename Real, int SG>
__global__ void __launch_bounds__(256)
k_update_matrices_small(const MatJob* __restrict__ jobs, int nitems, int C, int S) {
    constexpr int E = SG * SG, G = 256 / E;
    __shared__ double ex[G][SG], e1[G][SG], e2[G][SG];
    const int g = threadIdx.x / E, e = threadIdx.x - (threadIdx.x / E) * E;
    const int item = blockIdx.x * G + g;
    const bool active = g < G && item < nitems;
    const int c = active ? item % C : 0;
    const MatJob& jb = jobs[active ? item / C : 0];
    const double* cube = jb.cube;
    const double* evals = jb.evals;
    double r;
    if (jb.cat_eig) {           // CPU/EigenDecompositionCube.hpp:326-470: no category rate
        const int ce = jb.cat_eig[c];
        cube += (size_t)ce * S * S * S;
        evals += (size_t)ce * S;
        r = 1.0;
    } else {
        r = jb.rates[c];
    }
    if (active && e < S) {
        const double t = jb.tlen ? *jb.tlen : jb.t;
        const double lam = evals[e];
        const double v = exp(lam * (t * r));
        const double sl = lam * r;
        ex[g][e] = v;
        e1[g][e] = sl * v;
        e2[g][e] = sl * sl * v;
    }
    __syncthreads();
    if (!active) return;
    const size_t off = (size_t)c * SG * SG;
    Real* P = static_cast<Real*>(jb.p) + off;
    Real* D1 = jb.d1 ? static_cast<Real*>(jb.d1) + off : nullptr;
    Real* D2 = jb.d2 ? static_cast<Real*>(jb.d2) + off : nullptr;
    const int i = e / SG, j = e - (e / SG) * SG;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    if (i < S && j < S) {
        const double* cu = cube + (size_t)i * S * S + j;
        if (D1) {
            for (int k = 0; k < S; ++k) {
                const double cv = cu[(size_t)k * S];
                s0 += cv * ex[g][k];
                s1 += cv * e1[g][k];
                s2 += cv * e2[g][k];
            }
        } else {
            for (int k = 0; k < S; ++k) s0 += cu[(size_t)k * S] * ex[g][k];
        }
        if (!(s0 > 0.0)) s0 = 0.0;
    }
    P[e] = (Real)s0;
    if (D1) D1[e] = (Real)s1;
    if (D2) D2[e] = (Real)s2;
    const size_t tix = off + j * SG + i;   // transposed image
    static_cast<Real*>(jb.pt)[tix] = (Real)s0;
    if (D1) static_cast<Real*>(jb.d1t)[tix] = (Real)s1;
    if (D2) static_cast<Real*>(jb.d2t)[tix] = (Real)s2;
}

// op 0: out = a . b (convolution, CPU/BeagleCPUImpl.hpp:1096-1160);
// op 1: out = transpose(a) (CPU/BeagleCPUImpl.hpp:1175-1222).
// `out` holds 2n pointers: the n results, then their transposed images.
template <typename Real>
__global__ void k_matrix_pairs(const void* const* a, const void* const* b, void* const* out,
                               int op, int S, int Sg) {
    const int m = blockIdx.x, c = blockIdx.y;
    const size_t off = (size_t)c * Sg * Sg;
    const Real* A = static_cast<const Real*>(a[m]) + off;
    Real* O = static_cast<Real*>(out[m]) + off;
    Real* OT = static_cast<Real*>(out[gridDim.x + m]) + off;
    for (int idx = threadIdx.x; idx < Sg * Sg; idx += blockDim.x) {
        const int i = idx / Sg, j = idx - (idx / Sg) * Sg;
        Real v = 0;
        if (i < S && j < S) {
            if (op == 0) {
                const Real* B = static_cast<const Real*>(b[m]) + off;
                Real acc = 0;
                for (int k = 0; k < S; ++k) acc += A[i * Sg + k] * B[k * Sg + j];
                v = acc;
            } else {
                v = A[j * Sg + i];
            }
        }
        O[idx] = v;
        OT[j * Sg + i] = v;
    }
}

}  // namespace

template <typename Real>
cudaError_t launch_update_matrices(const MatJob* d_jobs, int njobs, const Dims& d,
                                   cudaStream_t s) {
    if (njobs == 0) return cudaSuccess;
    const int nitems = njobs * d.C;
    if (d.Sg == 4) {
        k_update_matrices_small<Real, 4><<<(nitems + 15) / 16, 256, 0, s>>>(d_jobs, nitems, d.C,
                                                                            d.S);
        return cudaGetLastError();
    }
    if (d.Sg == 8) {
        k_update_matrices_small<Real, 8><<<(nitems + 3) / 4, 256, 0, s>>>(d_jobs, nitems, d.C,
                                                                          d.S);
        return cudaGetLastError();
    }
    // Entries split over blocks in slices of 1024 (4 a thread): 4 slices for
    // 61 states, one for 20 or fewer.
    dim3 grid(njobs, d.C, (d.Sg * d.Sg + 1023) / 1024);
    k_update_matrices<Real><<<grid, 256, 3 * d.S * sizeof(double), s>>>(d_jobs, d.S, d.Sg);
    return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_matrix_pairs(const void* const* d_a, const void* const* d_b,
                                void* const* d_out, int n, int op, const Dims& d,
                                cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    dim3 grid(n, d.C);
    k_matrix_pairs<Real><<<grid, 256, 0, s>>>(d_a, d_b, d_out, op, d.S, d.Sg);
    return cudaGetLastError();
}

template cudaError_t launch_update_matrices<float>(const MatJob*, int, const Dims&, cudaStream_t);
template cudaError_t launch_update_matrices<double>(const MatJob*, int, const Dims&, cudaStream_t);
template cudaError_t launch_matrix_pairs<float>(const void* const*, const void* const*,
                                                void* const*, int, int, const Dims&, cudaStream_t);
template cudaError_t launch_matrix_pairs<double>(const void* const*, const void* const*,
                                                 void* const*, int, int, const Dims&, cudaStream_t);

}  // namespace b200
