// Per-turn bunch diagnostics on the device: Diagnostics_full2::do_update
// (bunch/diagnostics_full2.cc:16-37) -- number and real number of
// particles, mean, standard deviation, min/max of x, y, cdt, second
// moments, correlations and the emittances of calculate_emittances
// (diagnostics_full2_host.cc) -- computed and appended to a device record
// array without a host round trip, so a propagate call with diagnostics
// still runs (and replays as a CUDA graph) without synchronising.
//
// Record layout (kDiagRecord doubles): num_particles, real_num, mean[6],
// std[6], min[3], max[3], mom2[36] (row major), corr[36], emitx, emity,
// emitz, emitxy, emitxyz.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "sb2_kernels.h"

namespace sb2 {

// sums of the six coordinates and min/max of x, y, cdt over live particles
// (core_diagnostics.cc:105-111 calculate_mean, :364-419 calculate_min/max)
__global__ void __launch_bounds__(256) diag_sums_kernel(const double* __restrict__ parts, int64_t stride,
                                                        const uint8_t* __restrict__ masks, int64_t n,
                                                        double* partials)
{
    __shared__ double s_red[8][12];
    double acc[12] = {0, 0, 0, 0, 0, 0, 1e100, 1e100, 1e100, -1e100, -1e100, -1e100};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (!masks[i]) continue;
        double v[6];
        for (int j = 0; j < 6; ++j) v[j] = parts[i + j * stride];
        for (int j = 0; j < 6; ++j) acc[j] += v[j];
        for (int j = 0; j < 3; ++j) {
            acc[6 + j] = fmin(acc[6 + j], v[2 * j]);
            acc[9 + j] = fmax(acc[9 + j], v[2 * j]);
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int j = 0; j < 12; ++j) {
        double v = acc[j];
        for (int off = 16; off > 0; off >>= 1) {
            const double u = __shfl_down_sync(0xffffffffu, v, off);
            v = j < 6 ? v + u : (j < 9 ? fmin(v, u) : fmax(v, u));
        }
        if (lane == 0) s_red[w][j] = v;
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        const int j = threadIdx.x;
        double v = s_red[0][j];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k)
            v = j < 6 ? v + s_red[k][j] : (j < 9 ? fmin(v, s_red[k][j]) : fmax(v, s_red[k][j]));
        partials[blockIdx.x * 12 + j] = v;
    }
}

// mean = sums / n_total (the reference divides by the bunch's total
// number), min, max: fixed-order reduction of the block partials
__global__ void diag_mean_kernel(const double* __restrict__ partials, int nb, const BunchCounters* __restrict__ c,
                                 double* tmp)
{
    if (threadIdx.x >= 12) return;
    const int j = threadIdx.x;
    double v = partials[j];
    for (int k = 1; k < nb; ++k) {
        const double u = partials[k * 12 + j];
        v = j < 6 ? v + u : (j < 9 ? fmin(v, u) : fmax(v, u));
    }
    tmp[j] = j < 6 ? v / c->n_total : v;
}

// determinant of the leading k x k block of a 6 x 6 matrix (Gaussian
// elimination with partial pivoting)
__device__ double det_lead(const double m[6][6], int k)
{
    double a[6][6];
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) a[i][j] = m[i][j];
    double det = 1.0;
    for (int col = 0; col < k; ++col) {
        int piv = col;
        for (int r = col + 1; r < k; ++r)
            if (fabs(a[r][col]) > fabs(a[piv][col])) piv = r;
        if (a[piv][col] == 0.0) return 0.0;
        if (piv != col) {
            for (int j = 0; j < k; ++j) {
                const double t = a[col][j];
                a[col][j] = a[piv][j];
                a[piv][j] = t;
            }
            det = -det;
        }
        det *= a[col][col];
        for (int r = col + 1; r < k; ++r) {
            const double f = a[r][col] / a[col][col];
            for (int j = col; j < k; ++j) a[r][j] -= f * a[col][j];
        }
    }
    return det;
}

__device__ double eliminate_small_negative(double x)
{ // diagnostics_full2_host.cc:8-17
    return (x < 0 && x > -1.0e-15) ? 0.0 : x;
}

// second moments from the central partials (moments_kernel with the mean),
// the derived quantities, one record appended at *count (if it fits)
__global__ void diag_final_kernel(const double* __restrict__ partials, int nb, const BunchCounters* __restrict__ c,
                                  const double* __restrict__ tmp, double* records, int32_t* count, int capacity)
{
    __shared__ double s_acc[21];
    if (threadIdx.x < 21) {
        double v = 0.0;
        for (int k = 0; k < nb; ++k) v += partials[k * 27 + 6 + threadIdx.x];
        s_acc[threadIdx.x] = v;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const int idx = *count;
    *count = idx + 1;
    if (idx >= capacity) return;
    double* r = records + (int64_t)idx * kDiagRecord;
    const double nt = c->n_total;
    double m2[6][6];
    int t = 0;
    for (int j = 0; j < 6; ++j)
        for (int k = 0; k <= j; ++k) {
            m2[j][k] = m2[k][j] = s_acc[t] / nt;
            ++t;
        }
    r[0] = c->n_total;
    r[1] = c->real_num;
    for (int j = 0; j < 6; ++j) r[2 + j] = tmp[j];
    for (int j = 0; j < 6; ++j) r[8 + j] = sqrt(m2[j][j]);
    for (int j = 0; j < 6; ++j) r[14 + j] = tmp[6 + j]; // min[3], max[3]
    for (int j = 0; j < 6; ++j)
        for (int k = 0; k < 6; ++k) {
            r[20 + j * 6 + k] = m2[j][k];
            r[56 + j * 6 + k] = m2[j][k] / sqrt(m2[j][j] * m2[k][k]);
        }
    for (int pl = 0; pl < 3; ++pl) {
        const double d = m2[2 * pl][2 * pl] * m2[2 * pl + 1][2 * pl + 1] - m2[2 * pl + 1][2 * pl] * m2[2 * pl][2 * pl + 1];
        r[92 + pl] = sqrt(eliminate_small_negative(d));
    }
    r[95] = sqrt(eliminate_small_negative(det_lead(m2, 4)));
    r[96] = sqrt(eliminate_small_negative(det_lead(m2, 6)));
}

// update_total_num (bunch_particles.cc:388) after a checkin: n_valid =
// n_total = number of set masks, counted on the device (16 bytes per thread
// per load, one atomic per block)
__global__ void __launch_bounds__(256) count_valid_kernel(const uint8_t* __restrict__ masks, int64_t n,
                                                          bool aligned16, BunchCounters* c)
{
    __shared__ int s_part[8];
    int cnt = 0;
    const int64_t nv = aligned16 ? n / 16 : 0; // caller-owned masks may start anywhere
    const uint4* m16 = reinterpret_cast<const uint4*>(masks);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv; i += (int64_t)gridDim.x * blockDim.x) {
        const uint4 v = m16[i];
        const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; ++k)
            for (int b = 0; b < 4; ++b) cnt += ((w[k] >> (8 * b)) & 0xffu) != 0;
    }
    for (int64_t i = nv * 16 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        cnt += masks[i] != 0;
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += s_part[k];
        if (t) atomicAdd(&c->n_valid, t);
    }
}

__global__ void count_valid_finish_kernel(BunchCounters* c) { c->n_total = c->n_valid; }

cudaError_t launch_count_valid(const uint8_t* masks, int64_t n, BunchCounters* c, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(&c->n_valid, 0, sizeof(int32_t), s);
    if (e) return e;
    if (n > 0) {
        const int64_t blocks = std::min<int64_t>((n / 16 + 255) / 256 + 1, 148 * 8);
        count_valid_kernel<<<(int)blocks, 256, 0, s>>>(masks, n, ((uintptr_t)masks & 15) == 0, c);
    }
    count_valid_finish_kernel<<<1, 1, 0, s>>>(c);
    return cudaGetLastError();
}

// FP64 issue-rate probe: eight independent fused multiply-add chains per
// thread, so the FP64 pipe, not latency, bounds the kernel.  The values
// stay finite (|a| < 1) and the sums are stored so no chain is dropped.
__global__ void __launch_bounds__(256) fp64_fma_probe_kernel(double* out, int iters, double a, double b)
{
    double r0 = threadIdx.x * 1e-6, r1 = r0 + 0.125, r2 = r0 + 0.25, r3 = r0 + 0.375;
    double r4 = r0 + 0.5, r5 = r0 + 0.625, r6 = r0 + 0.75, r7 = r0 + 0.875;
    for (int i = 0; i < iters; ++i) {
        r0 = __fma_rn(r0, a, b);
        r1 = __fma_rn(r1, a, b);
        r2 = __fma_rn(r2, a, b);
        r3 = __fma_rn(r3, a, b);
        r4 = __fma_rn(r4, a, b);
        r5 = __fma_rn(r5, a, b);
        r6 = __fma_rn(r6, a, b);
        r7 = __fma_rn(r7, a, b);
    }
    out[blockIdx.x * (int64_t)blockDim.x + threadIdx.x] = ((r0 + r1) + (r2 + r3)) + ((r4 + r5) + (r6 + r7));
}

cudaError_t launch_fp64_probe(double* out, int blocks, int iters, cudaStream_t s)
{
    fp64_fma_probe_kernel<<<blocks, 256, 0, s>>>(out, iters, 0.9999999, 1e-7);
    return cudaGetLastError();
}

cudaError_t launch_diagnostics(const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                               const BunchCounters* counters, double* partials, int nb, double* tmp, double* records,
                               int32_t* count, int capacity, cudaStream_t s)
{
    diag_sums_kernel<<<nb, 256, 0, s>>>(parts, stride, masks, n, partials);
    diag_mean_kernel<<<1, 32, 0, s>>>(partials, nb, counters, tmp);
    cudaError_t e = launch_moments(parts, stride, masks, n, tmp, partials, nb, s);
    if (e) return e;
    diag_final_kernel<<<1, 32, 0, s>>>(partials, nb, counters, tmp, records, count, capacity);
    return cudaGetLastError();
}

} // namespace sb2
