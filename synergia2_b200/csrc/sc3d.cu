// 3D open-boundary Hockney solver kernels for sm_100a (FP64 path).
//
// Layouts in HBM (x fastest everywhere):
//   rho, phi   dense real (gz, gy, gx) on the original grid
//   S          complex spectrum [nz][ny][nkxp], nkx = nx/2+1 (padded even)
//   Ghat       real octant [nz/2+1][ny/2+1][nx/2+1]: the transform of the
//              mirrored Green function is real and even in every axis, so
//              only this octant is built and read
//   E          (gz, gy, gx) cells x {ex, ey, ez, 0} FP64 (32 B per cell)
//
// The convolution phi = IFFT(FFT(rho_padded) * FFT(G2)) of
// space_charge_3d_open_hockney.cc:642-676 is computed in five line passes
// that skip the zero padding: x (pairs of real rows packed as one complex
// FFT), y (first gy inputs), z forward + Ghat multiply + z inverse in one
// kernel (first gz inputs, first gz outputs), y inverse (first gy outputs),
// x inverse (Hermitian pairs, first gx outputs).  Each pass stages a tile of
// lines in shared memory and runs a Stockham transform there with radix-8/4/2
// butterflies in registers.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>

#include "sb2_kernels.h"

namespace sb2 {

constexpr double kPi = 3.14159265358979323846;
constexpr double kE = 1.602176565e-19;
constexpr double kCl = 299792458.0;
constexpr double kMu0 = 4 * kPi * 1.0e-7;
constexpr double kEps0 = 1.0 / (kCl * kCl * kMu0);

// ---------------------------------------------------------------------------
// bookkeeping + domain (one block)
// ---------------------------------------------------------------------------

__device__ double smallest_non_tiny(double val, double o1, double o2, double tiny)
{ // space_charge_3d_open_hockney.cc:94-109
    if (val > tiny) return val;
    if ((o1 > tiny) && (o2 > tiny)) return fmin(o1, o2);
    return fmax(o1, o2);
}

__global__ void __launch_bounds__(256) book_domain_kernel(const __grid_constant__ DomainParams p)
{
    __shared__ double s_sum[256][6];
    // fixed-order reduction of the per-block moment partials
    if (p.compute_domain && !p.domain_fixed) {
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int b = threadIdx.x; b < p.n_partials; b += blockDim.x)
            for (int j = 0; j < 6; ++j) acc[j] += p.moment_partials[b * 6 + j];
        for (int j = 0; j < 6; ++j) s_sum[threadIdx.x][j] = acc[j];
        __syncthreads();
        for (int w = 128; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w)
                for (int j = 0; j < 6; ++j) s_sum[threadIdx.x][j] += s_sum[threadIdx.x + w][j];
            __syncthreads();
        }
    }
    if (threadIdx.x != 0) return;

    // bookkeeping: aperture operations then update_total_num per operator
    // (independent_operator.cc:94-133, aperture_operation.h:14-24,
    // bunch.h:363-370)
    BunchCounters c = *p.counters;
    for (int o = 0; o < p.book.n_operators; ++o) {
        int nd_op = 0;
        for (int s = p.book.slot_begin[o]; s < p.book.slot_end[o]; ++s) {
            int nd = p.ap_counts[s];
            p.ap_counts[s] = 0;
            int el = p.book.slot_elem[s];
            if (p.elem_charge && el >= 0 && nd) p.elem_charge[el] += nd * c.real_num / c.n_total;
            nd_op += nd;
            c.n_valid -= nd;
        }
        int old_total = c.n_total;
        c.n_total = c.n_valid;
        c.real_num = old_total ? c.n_total * c.real_num / old_total : 0.0;
    }
    *p.counters = c;
    if (!p.compute_domain) return;

    ScState st = *p.sc;
    st.error = 0;
    double size[3], offset[3];
    if (p.domain_fixed) {
        for (int i = 0; i < 3; ++i) {
            size[i] = p.fixed_size[i];
            offset[i] = p.fixed_offset[i];
        }
    } else {
        // update_domain :494-540; calculate_spatial_mean_stddev
        // core_diagnostics.cc:422-460 (divides by n_total)
        double ms[6];
        for (int j = 0; j < 3; ++j) {
            ms[j] = s_sum[0][j] / c.n_total;
            ms[j + 3] = sqrt((s_sum[0][j + 3]) / c.n_total - ms[j] * ms[j]);
        }
        for (int j = 0; j < 6; ++j) st.mean_std[j] = ms[j];
        const double tiny = 1.0e-10;
        if ((ms[3] < tiny) && (ms[4] < tiny) && (ms[5] < tiny)) {
            st.error = 1;
            st.valid = 0;
            *p.sc = st;
            return;
        }
        offset[0] = ms[0];
        offset[1] = ms[1];
        offset[2] = ms[2];
        size[0] = p.n_sigma * smallest_non_tiny(ms[3], ms[4], ms[5], tiny);
        size[1] = p.n_sigma * smallest_non_tiny(ms[4], ms[3], ms[5], tiny);
        size[2] = p.n_sigma * smallest_non_tiny(ms[5], ms[3], ms[4], tiny);
        if (p.grid_entire_period) {
            offset[2] = 0.0;
            size[2] = p.z_period;
        }
    }
    // Rectangular_grid_domain rectangular_grid_domain.h:20-36 (original and
    // doubled domains)
    for (int i = 0; i < 3; ++i) {
        st.left[i] = offset[i] - size[i] / 2.0;
        st.h[i] = size[i] / (1.0 * p.g[i]);
        st.ih[i] = 1.0 / st.h[i];
        st.dh[i] = (size[i] * 2.0) / (1.0 * p.dg[i]);
    }
    // deposit weight deposit.cc:608-610
    st.w0 = (c.real_num / c.n_total) * p.charge * kE / (st.h[0] * st.h[1] * st.h[2]);
    // get_normalization_force :708-735
    double norm = st.h[0] * st.h[1] * st.h[2];
    norm *= 1.0 / (4.0 * kPi * kEps0);
    norm *= 1.0;
    if (p.green_linear) norm *= 1.0 / (st.h[2] * st.h[2]);
    norm *= 1.0 / (p.dg[0] * p.dg[1] * p.dg[2]);
    st.fn_norm = norm;
    // apply_kick :753-770
    double q = p.charge * kE;
    double unit_conversion = kCl / (1e9 * kE);
    st.factor = p.kick_scale * unit_conversion * q * p.time_step * st.fn_norm /
                (p.pref * p.gamma * p.gamma * p.beta);
    st.valid = 1;
    *p.sc = st;
}

// ---------------------------------------------------------------------------
// deposit (FP64, global atomics): sv_zyx_rho_reducer_non_periodic
// deposit.cc:309-394; edges excluded deposit.cc:23-30
// ---------------------------------------------------------------------------
__device__ __forceinline__ void leftmost_d(double pos, double left, double inv, int& idx, double& off)
{
    double s = (pos - left) * inv - 0.5;
    idx = (int)floor(s);
    off = s - idx;
}

// Particles whose stencils start in the same cell are summed inside the
// warp first (a segmented shuffle scan over runs of equal cell keys), so a
// cell-ordered bunch issues one set of 8 atomics per run instead of per
// particle; with no equal neighbours the scan is skipped.
__global__ void __launch_bounds__(256) deposit_kernel(const double* __restrict__ parts, int64_t stride,
                                                      const uint8_t* __restrict__ masks, int64_t n,
                                                      const ScState* __restrict__ scp, double* rho,
                                                      int gx, int gy, int gz)
{
    const ScState& sc = *scp;
    if (!sc.valid) return;
    const double lx = sc.left[0], ly = sc.left[1], lz = sc.left[2];
    const double ihx = sc.ih[0], ihy = sc.ih[1], ihz = sc.ih[2];
    const double w0 = sc.w0;
    const int lane = threadIdx.x & 31;
    const int64_t wstride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t wb = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) - lane; wb < n; wb += wstride) {
        const int64_t i = wb + lane;
        int ix = 0, iy = 0, iz = 0;
        int64_t key = -1;
        double w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (i < n && masks[i]) {
            double ox, oy, oz;
            leftmost_d(parts[i], lx, ihx, ix, ox);
            leftmost_d(parts[i + 2 * stride], ly, ihy, iy, oy);
            leftmost_d(parts[i + 4 * stride], lz, ihz, iz, oz);
            if (ix >= -1 && ix < gx && iy >= -1 && iy < gy && iz >= -1 && iz < gz) {
                key = ((int64_t)(iz + 1) * (gy + 1) + (iy + 1)) * (gx + 1) + (ix + 1);
                double aox = 1.0 - ox, aoy = 1.0 - oy, aoz = 1.0 - oz;
                w[0] = w0 * aox * aoy * aoz;
                w[1] = w0 * ox * aoy * aoz;
                w[2] = w0 * aox * oy * aoz;
                w[3] = w0 * ox * oy * aoz;
                w[4] = w0 * aox * aoy * oz;
                w[5] = w0 * ox * aoy * oz;
                w[6] = w0 * aox * oy * oz;
                w[7] = w0 * ox * oy * oz;
            }
        }
        const int64_t prev = __shfl_up_sync(0xffffffffu, key, 1);
        const int64_t next = __shfl_down_sync(0xffffffffu, key, 1);
        const bool head = lane == 0 || prev != key;
        const bool tail = lane == 31 || next != key;
        const unsigned heads = __ballot_sync(0xffffffffu, head);
        if (heads != 0xffffffffu) { // some run longer than one particle
            unsigned le;
            asm("mov.u32 %0, %%lanemask_le;" : "=r"(le));
            const int seg = 31 - __clz(heads & le);
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                double v = w[c];
                for (int o = 1; o < 32; o <<= 1) {
                    double u = __shfl_up_sync(0xffffffffu, v, o);
                    if (lane - o >= seg) v += u;
                }
                w[c] = v;
            }
        }
        if (!tail || key < 0) continue;
        bool x0 = ix > 0 && ix < gx - 1, x1 = ix + 1 > 0 && ix + 1 < gx - 1;
        bool y0 = iy > 0 && iy < gy - 1, y1 = iy + 1 > 0 && iy + 1 < gy - 1;
        bool z0 = iz > 0 && iz < gz - 1, z1 = iz + 1 > 0 && iz + 1 < gz - 1;
        int64_t base = (int64_t)iz * gx * gy;
        if (z0) {
            if (y0 && x0) atomicAdd(&rho[base + iy * gx + ix], w[0]);
            if (y0 && x1) atomicAdd(&rho[base + iy * gx + ix + 1], w[1]);
            if (y1 && x0) atomicAdd(&rho[base + (iy + 1) * gx + ix], w[2]);
            if (y1 && x1) atomicAdd(&rho[base + (iy + 1) * gx + ix + 1], w[3]);
        }
        base = (int64_t)(iz + 1) * gx * gy;
        if (z1) {
            if (y0 && x0) atomicAdd(&rho[base + iy * gx + ix], w[4]);
            if (y0 && x1) atomicAdd(&rho[base + iy * gx + ix + 1], w[5]);
            if (y1 && x0) atomicAdd(&rho[base + (iy + 1) * gx + ix], w[6]);
            if (y1 && x1) atomicAdd(&rho[base + (iy + 1) * gx + ix + 1], w[7]);
        }
    }
}

// ---------------------------------------------------------------------------
// Green function octant: alg_g2_linear :230-348 / alg_g2_pointlike :136-228
// evaluated for ix <= gx, iy <= gy, iz <= gz (doubled shape = 2 * shape,
// so this octant plus mirroring is the whole doubled-grid G2)
// ---------------------------------------------------------------------------
__global__ void green_octant_kernel(const ScState* __restrict__ scp, double* G, int gx0, int gy0, int gz0,
                                    int linear)
{
    const ScState& sc = *scp;
    if (!sc.valid) return;
    const int ox = gx0 + 1, oy = gy0 + 1, oz = gz0 + 1;
    const int64_t total = (int64_t)ox * oy * oz;
    const double hx = sc.dh[0], hy = sc.dh[1], hz = sc.dh[2];
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        int ix = (int)(t % ox);
        int iy = (int)((t / ox) % oy);
        int iz = (int)(t / ((int64_t)ox * oy));
        double Gv;
        if (!linear) {
            double G000 = 2.8 / fmin(hx, fmin(hy, hz));
            double dx = ix * hx, dy = iy * hy, dz = iz * hz;
            Gv = (ix == 0 && iy == 0 && iz == 0) ? G000 : 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
        } else {
            double rr0 = hx * hx + hy * hy;
            double r10 = sqrt(hx * hx + hy * hy + hz * hz);
            double G000 = (2.0 / rr0) * (hz * r10 + rr0 * log((hz + r10) / sqrt(rr0)) - hz * hz);
            double z = iz * hz; // iz <= gz0
            double y = iy * hy, x = ix * hx;
            double rr = x * x + y * y;
            double s0 = sqrt(rr + z * z);
            double sn = sqrt(rr + (z - hz) * (z - hz));
            double sp = sqrt(rr + (z + hz) * (z + hz));
            Gv = 2.0 * s0 - sn - sp;
            const double epsz = 1e-12 * hz;
            double T1, T2, r1, r2;
            if (z < -hz) {
                r1 = (sn - z + hz) / (s0 - z);
                T1 = (hz - z) * log(r1);
                r2 = (s0 - z) / (sp - z - hz);
                T2 = (hz + z) * log(r2);
                Gv += T1 + T2;
            } else if (fabs(z + hz) < epsz) {
                r1 = (sn - z + hz) / (s0 - z);
                T1 = (hz - z) * log(r1);
                Gv += T1;
            } else if (fabs(z) < epsz) {
                if (fabs(x) + fabs(y) < 2. * epsz) {
                    Gv += hz * G000;
                } else {
                    r1 = (sqrt(hz * hz + rr) + hz) / sqrt(rr);
                    Gv += 2.0 * hz * log(r1);
                }
            } else if (fabs(z - hz) < epsz) {
                r1 = (sp + z + hz) / (s0 + z);
                T1 = (hz + z) * log(r1);
                Gv += T1;
            } else if (z > hz) {
                r1 = (s0 + z) / (sn + z - hz);
                T1 = (hz - z) * log(r1);
                r2 = (sp + z + hz) / (s0 + z);
                T2 = (hz + z) * log(r2);
                Gv += T1 + T2;
            }
        }
        G[t] = Gv;
    }
}

// ---------------------------------------------------------------------------
// Shared-memory Stockham FFT with radix-8/4/2 butterflies in registers.
// A tile holds `nl` lines of length L (power of two, 8..4096) at pitch L in
// shared memory; each pass reads every element once, does one radix-R
// butterfly per (line, j) in registers and writes the Stockham-ordered
// result to the other buffer.  Input and output are in natural order.
// tw[k] = exp(-2 pi i k / L) for k < L; `sign` > 0 selects the inverse.
// ---------------------------------------------------------------------------
// Complex helpers for double2 (FP64 path) and float2 (mixed path).
template <typename C> struct CxT;
template <> struct CxT<double2> { typedef double R; };
template <> struct CxT<float2> { typedef float R; };
__device__ __forceinline__ double2 mkc(double x, double y, double2*) { return make_double2(x, y); }
__device__ __forceinline__ float2 mkc(float x, float y, float2*) { return make_float2(x, y); }
template <typename C>
__device__ __forceinline__ C cplx(typename CxT<C>::R x, typename CxT<C>::R y) { return mkc(x, y, (C*)nullptr); }
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) { return cplx<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return cplx<C>(a.x + b.x, a.y + b.y); }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { return cplx<C>(a.x - b.x, a.y - b.y); }
// multiply by -i (forward) or +i (inverse)
template <typename C>
__device__ __forceinline__ C rot90(C a, bool inv) { return inv ? cplx<C>(-a.y, a.x) : cplx<C>(a.y, -a.x); }

// In-register DFT of size R (2, 4, 8) in natural order: X[k] = sum_r v[r] w^(rk),
// w = exp(-/+ 2 pi i / R).
template <int RAD, typename C>
struct DftReg;

template <typename C>
struct DftReg<2, C> {
    static __device__ __forceinline__ void run(C* v, bool)
    {
        C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <typename C>
struct DftReg<4, C> {
    static __device__ __forceinline__ void run(C* v, bool inv)
    {
        C s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        C s13 = cadd(v[1], v[3]), d13 = rot90(csub(v[1], v[3]), inv);
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        v[1] = cadd(d02, d13);
        v[3] = csub(d02, d13);
    }
};

template <typename C>
struct DftReg<8, C> {
    static __device__ __forceinline__ void run(C* v, bool inv)
    {
        typedef typename CxT<C>::R R;
        const R h = (R)0.70710678118654752440;
        // radix-2 first stage (decimation in frequency)
        C a[4], b[4];
        for (int r = 0; r < 4; ++r) {
            a[r] = cadd(v[r], v[r + 4]);
            b[r] = csub(v[r], v[r + 4]);
        }
        // twiddles w8^r on the difference branch
        b[1] = inv ? cplx<C>(h * (b[1].x - b[1].y), h * (b[1].x + b[1].y))
                   : cplx<C>(h * (b[1].x + b[1].y), h * (b[1].y - b[1].x));
        b[2] = rot90(b[2], inv);
        b[3] = inv ? cplx<C>(-h * (b[3].x + b[3].y), h * (b[3].x - b[3].y))
                   : cplx<C>(h * (b[3].y - b[3].x), -h * (b[3].x + b[3].y));
        DftReg<4, C>::run(a, inv); // even outputs
        DftReg<4, C>::run(b, inv); // odd outputs
        for (int k = 0; k < 4; ++k) {
            v[2 * k] = a[k];
            v[2 * k + 1] = b[k];
        }
    }
};

template <int RAD, typename C>
__device__ __forceinline__ void stockham_pass(const C* __restrict__ src, C* __restrict__ dst, int nl, int L, int Ns,
                                              const C* __restrict__ tw, bool inv)
{
    // element j of line li sits at j * nl + li: consecutive threads take
    // consecutive lines, so every read and write below is contiguous
    const int T = L / RAD;
    const int total = nl * T;
    const int tstep = L / (Ns * RAD);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int j = t / nl, li = t - j * nl;
        const int k = j & (Ns - 1);
        C v[RAD];
#pragma unroll
        for (int r = 0; r < RAD; ++r) v[r] = src[(j + r * T) * nl + li];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < RAD; ++r) {
                C w = tw[(k * r * tstep) & (L - 1)];
                if (inv) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        DftReg<RAD, C>::run(v, inv);
        const int idxD = (j / Ns) * Ns * RAD + k;
#pragma unroll
        for (int r = 0; r < RAD; ++r) dst[(idxD + r * Ns) * nl + li] = v[r];
    }
}

// FFT of the nl lines in b0 (layout j * nl + li); returns the buffer
// holding the result.
template <typename C>
__device__ C* smem_fft(C* b0, C* b1, int nl, int L, const C* __restrict__ tw, bool inv)
{
    C* src = b0;
    C* dst = b1;
    int Ns = 1;
    while (Ns < L) {
        const int rem = L / Ns;
        if (rem >= 8 && rem != 16) {
            stockham_pass<8>(src, dst, nl, L, Ns, tw, inv);
            Ns *= 8;
        } else if (rem >= 4) {
            stockham_pass<4>(src, dst, nl, L, Ns, tw, inv);
            Ns *= 4;
        } else {
            stockham_pass<2>(src, dst, nl, L, Ns, tw, inv);
            Ns *= 2;
        }
        __syncthreads();
        C* t = src;
        src = dst;
        dst = t;
    }
    return src;
}

constexpr int kFftTile = 2048; // complex elements per line tile (32 KB; two tiles per CTA)
constexpr int kFftSmemBytes = 2 * kFftTile * 16;
constexpr int kFftThreads = 256;

// XF: pairs of real rows (y, y+1) of rho -> S rows (r2c, first gx inputs)
// Global storage of the spectrum is C (double2, or float2 for the mixed
// path); every pass converts to double2 on load and computes in FP64 in
// shared memory and registers, so the mixed path only rounds at the five
// pass boundaries.
__device__ __forceinline__ double2 to_d(double2 v) { return v; }
__device__ __forceinline__ double2 to_d(float2 v) { return make_double2(v.x, v.y); }
template <typename C> __device__ __forceinline__ C from_d(double2 v);
template <> __device__ __forceinline__ double2 from_d<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 from_d<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }

// XF: pairs of real rows (y, y+1) of rho -> S rows (r2c, first gx inputs)
template <typename C>
__global__ void __launch_bounds__(kFftThreads) fft_xf_kernel(const double* __restrict__ rho, C* S,
                                                             const double2* __restrict__ tw, Dims d,
                                                             const ScState* __restrict__ scp)
{
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* sm = (double2*)sm_raw;
    if (!scp->valid) return;
    const int L = d.nx, nl = kFftTile / L;
    const int npy = (d.gy + 1) / 2;
    const int64_t nlines = (int64_t)npy * d.gz;
    const int64_t l0 = (int64_t)blockIdx.x * nl;
    const int nlt = (int)min((int64_t)nl, nlines - l0);
    if (nlt <= 0) return;
    double2* b0 = sm;
    double2* b1 = sm + kFftTile;
    for (int idx = threadIdx.x; idx < nlt * L; idx += blockDim.x) {
        int li = idx / L, j = idx - li * L;
        int64_t l = l0 + li;
        int pr = (int)(l % npy), z = (int)(l / npy);
        int ya = 2 * pr, yb = ya + 1;
        double2 v = make_double2(0.0, 0.0);
        if (j < d.gx) {
            v.x = rho[((int64_t)z * d.gy + ya) * d.gx + j];
            if (yb < d.gy) v.y = rho[((int64_t)z * d.gy + yb) * d.gx + j];
        }
        b0[j * nlt + li] = v;
    }
    __syncthreads();
    double2* r = smem_fft(b0, b1, nlt, L, tw, false);
    const int nk = d.nkx;
    for (int idx = threadIdx.x; idx < nlt * nk; idx += blockDim.x) {
        int li = idx / nk, k = idx - li * nk;
        int64_t l = l0 + li;
        int pr = (int)(l % npy), z = (int)(l / npy);
        int ya = 2 * pr, yb = ya + 1;
        double2 Z = r[k * nlt + li], Zn = r[((L - k) & (L - 1)) * nlt + li];
        double2 A = make_double2((Z.x + Zn.x) * 0.5, (Z.y - Zn.y) * 0.5);
        double2 B = make_double2((Z.y + Zn.y) * 0.5, -(Z.x - Zn.x) * 0.5);
        S[((int64_t)z * d.ny + ya) * d.nkxp + k] = from_d<C>(A);
        if (yb < d.gy) S[((int64_t)z * d.ny + yb) * d.nkxp + k] = from_d<C>(B);
    }
}

// Y passes: lines (kx, z<gz) along y.  forward: first gy inputs, all ny
// outputs; inverse: all inputs, first gy outputs.
template <typename C>
__global__ void __launch_bounds__(kFftThreads) fft_y_kernel(C* S, const double2* __restrict__ tw, Dims d,
                                                            int inverse, const ScState* __restrict__ scp)
{
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* sm = (double2*)sm_raw;
    if (!scp->valid) return;
    const int L = d.ny, nl = kFftTile / L;
    const int64_t nlines = (int64_t)d.nkx * d.gz;
    const int64_t l0 = (int64_t)blockIdx.x * nl;
    const int nlt = (int)min((int64_t)nl, nlines - l0);
    if (nlt <= 0) return;
    double2* b0 = sm;
    double2* b1 = sm + kFftTile;
    const int nin = inverse ? L : d.gy;
    for (int idx = threadIdx.x; idx < nlt * L; idx += blockDim.x) {
        int j = idx / nlt, li = idx - j * nlt; // consecutive threads: consecutive kx
        int64_t l = l0 + li;
        int kx = (int)(l % d.nkx), z = (int)(l / d.nkx);
        double2 v = make_double2(0.0, 0.0);
        if (j < nin) v = to_d(S[((int64_t)z * d.ny + j) * d.nkxp + kx]);
        b0[j * nlt + li] = v;
    }
    __syncthreads();
    double2* r = smem_fft(b0, b1, nlt, L, tw, inverse != 0);
    const int nout = inverse ? d.gy : L;
    for (int idx = threadIdx.x; idx < nlt * nout; idx += blockDim.x) {
        int j = idx / nlt, li = idx - j * nlt;
        int64_t l = l0 + li;
        int kx = (int)(l % d.nkx), z = (int)(l / d.nkx);
        S[((int64_t)z * d.ny + j) * d.nkxp + kx] = from_d<C>(r[j * nlt + li]);
    }
}

// Z pass: lines (kx, ky) along z: forward (first gz inputs), multiply by
// the real octant Ghat(kx, min(ky, ny-ky), min(kz, nz-kz)), inverse, first gz
// outputs.  (alg_cplx_multiplier :350-372 fused between the transforms.)
template <typename C>
__global__ void __launch_bounds__(kFftThreads) fft_z_conv_kernel(C* S, const double* __restrict__ Ghat,
                                                                 const double2* __restrict__ tw, Dims d,
                                                                 const ScState* __restrict__ scp)
{
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* sm = (double2*)sm_raw;
    if (!scp->valid) return;
    const int L = d.nz, nl = kFftTile / L;
    const int64_t nlines = (int64_t)d.nkx * d.ny;
    const int64_t l0 = (int64_t)blockIdx.x * nl;
    const int nlt = (int)min((int64_t)nl, nlines - l0);
    if (nlt <= 0) return;
    double2* b0 = sm;
    double2* b1 = sm + kFftTile;
    for (int idx = threadIdx.x; idx < nlt * L; idx += blockDim.x) {
        int j = idx / nlt, li = idx - j * nlt;
        int64_t l = l0 + li;
        int kx = (int)(l % d.nkx), ky = (int)(l / d.nkx);
        double2 v = make_double2(0.0, 0.0);
        if (j < d.gz) v = to_d(S[((int64_t)j * d.ny + ky) * d.nkxp + kx]);
        b0[j * nlt + li] = v;
    }
    __syncthreads();
    double2* r = smem_fft(b0, b1, nlt, L, tw, false);
    double2* o = (r == b0) ? b1 : b0;
    const int ogx = d.nx / 2 + 1, ogy = d.ny / 2 + 1;
    for (int idx = threadIdx.x; idx < nlt * L; idx += blockDim.x) {
        int kz = idx / nlt, li = idx - kz * nlt;
        int64_t l = l0 + li;
        int kx = (int)(l % d.nkx), ky = (int)(l / d.nkx);
        int my = ky <= d.ny / 2 ? ky : d.ny - ky;
        int mz = kz <= d.nz / 2 ? kz : d.nz - kz;
        const double g = Ghat[((int64_t)mz * ogy + my) * ogx + kx];
        double2 v = r[kz * nlt + li];
        r[kz * nlt + li] = make_double2(v.x * g, v.y * g);
    }
    __syncthreads();
    double2* q = smem_fft(r, o, nlt, L, tw, true);
    for (int idx = threadIdx.x; idx < nlt * d.gz; idx += blockDim.x) {
        int j = idx / nlt, li = idx - j * nlt;
        int64_t l = l0 + li;
        int kx = (int)(l % d.nkx), ky = (int)(l / d.nkx);
        S[((int64_t)j * d.ny + ky) * d.nkxp + kx] = from_d<C>(q[j * nlt + li]);
    }
}

// XI: Hermitian pairs of spectrum rows -> real rows (y, y+1) of phi (c2r,
// first gx outputs); imaginary parts of the k = 0 and k = nx/2 terms are
// ignored as a c2r transform does.
template <typename C, typename RO>
__global__ void __launch_bounds__(kFftThreads) fft_xi_kernel(const C* __restrict__ S, RO* phi,
                                                             const double2* __restrict__ tw, Dims d,
                                                             const ScState* __restrict__ scp)
{
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* sm = (double2*)sm_raw;
    if (!scp->valid) return;
    const int L = d.nx, nl = kFftTile / L;
    const int npy = (d.gy + 1) / 2;
    const int64_t nlines = (int64_t)npy * d.gz;
    const int64_t l0 = (int64_t)blockIdx.x * nl;
    const int nlt = (int)min((int64_t)nl, nlines - l0);
    if (nlt <= 0) return;
    double2* b0 = sm;
    double2* b1 = sm + kFftTile;
    const int half = L / 2;
    for (int idx = threadIdx.x; idx < nlt * L; idx += blockDim.x) {
        int li = idx / L, j = idx - li * L;
        int64_t l = l0 + li;
        int pr = (int)(l % npy), z = (int)(l / npy);
        int ya = 2 * pr, yb = ya + 1;
        int k = j <= half ? j : L - j;
        double2 A = to_d(S[((int64_t)z * d.ny + ya) * d.nkxp + k]);
        double2 B = (yb < d.gy) ? to_d(S[((int64_t)z * d.ny + yb) * d.nkxp + k]) : make_double2(0.0, 0.0);
        if (k == 0 || k == half) {
            A.y = 0.0;
            B.y = 0.0;
        }
        if (j > half) {
            A.y = -A.y;
            B.y = -B.y;
        }
        b0[j * nlt + li] = make_double2(A.x - B.y, A.y + B.x);
    }
    __syncthreads();
    double2* r = smem_fft(b0, b1, nlt, L, tw, true);
    for (int idx = threadIdx.x; idx < nlt * d.gx; idx += blockDim.x) {
        int li = idx / d.gx, j = idx - li * d.gx;
        int64_t l = l0 + li;
        int pr = (int)(l % npy), z = (int)(l / npy);
        int ya = 2 * pr, yb = ya + 1;
        double2 v = r[j * nlt + li];
        phi[((int64_t)z * d.gy + ya) * d.gx + j] = (RO)v.x;
        if (yb < d.gy) phi[((int64_t)z * d.gy + yb) * d.gx + j] = (RO)v.y;
    }
}

// Ghat passes on the real octant (ox, oy, oz) = (nx/2+1, ny/2+1, nz/2+1):
// axis 0/1/2 transforms even real lines rebuilt by mirroring; real part of
// the first L/2+1 outputs stored back in place.  The transform of a real
// even line is real, so two lines ride in one complex FFT (line 2q as the
// real part, line 2q+1 as the imaginary part) and come out as its real and
// imaginary parts.
__global__ void __launch_bounds__(kFftThreads) fft_green_kernel(double* G, const double2* __restrict__ tw,
                                                                int axis, int L, int ox, int oy, int oz,
                                                                const ScState* __restrict__ scp)
{
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* sm = (double2*)sm_raw;
    if (!scp->valid) return;
    const int nl = kFftTile / L; // complex lines (line pairs) per CTA
    const int half = L / 2;
    int64_t nlines, sj;
    if (axis == 0) { nlines = (int64_t)oy * oz; sj = 1; }
    else if (axis == 1) { nlines = (int64_t)ox * oz; sj = ox; }
    else { nlines = (int64_t)ox * oy; sj = (int64_t)ox * oy; }
    const int64_t npairs = (nlines + 1) / 2;
    const int64_t l0 = (int64_t)blockIdx.x * nl;
    const int nlt = (int)min((int64_t)nl, npairs - l0);
    if (nlt <= 0) return;
    double2* b0 = sm;
    double2* b1 = sm + kFftTile;
    auto line_base = [&](int64_t l) -> int64_t {
        if (axis == 0) return l * ox;                                  // (y, z) rows
        if (axis == 1) return (l % ox) + (l / ox) * (int64_t)ox * oy;  // (kx, z)
        return l;                                                      // (kx, ky)
    };
    for (int idx = threadIdx.x; idx < nlt * L; idx += blockDim.x) {
        int li, j;
        if (axis == 0) { li = idx / L; j = idx - li * L; }
        else { j = idx / nlt; li = idx - j * nlt; }
        const int m = j <= half ? j : L - j;
        const int64_t la = 2 * (l0 + li), lb = la + 1;
        const double va = G[line_base(la) + m * sj];
        const double vb = lb < nlines ? G[line_base(lb) + m * sj] : 0.0;
        b0[j * nlt + li] = make_double2(va, vb);
    }
    __syncthreads();
    double2* r = smem_fft(b0, b1, nlt, L, tw, false);
    for (int idx = threadIdx.x; idx < nlt * (half + 1); idx += blockDim.x) {
        int li, k;
        if (axis == 0) { li = idx / (half + 1); k = idx - li * (half + 1); }
        else { k = idx / nlt; li = idx - k * nlt; }
        const int64_t la = 2 * (l0 + li), lb = la + 1;
        const double2 v = r[k * nlt + li];
        G[line_base(la) + k * sj] = v.x;
        if (lb < nlines) G[line_base(lb) + k * sj] = v.y;
    }
}

// E = -grad phi by central differences on interior cells of the original
// grid, zero on the boundary: alg_force_extractor_doubled_domain
// space_charge_3d_kernels.h:217-307 (h of the doubled domain).
__device__ __forceinline__ void store_e(double2* E, int64_t i, double ex, double ey, double ez)
{
    E[2 * i] = make_double2(ex, ey);
    E[2 * i + 1] = make_double2(ez, 0.0);
}
__device__ __forceinline__ void store_e(float4* E, int64_t i, float ex, float ey, float ez)
{
    E[i] = make_float4(ex, ey, ez, 0.0f);
}

template <typename R, typename EV>
__global__ void efield_kernel(const R* __restrict__ phi, EV* E, int gx, int gy, int gz,
                              const ScState* __restrict__ scp)
{
    const ScState& sc = *scp;
    if (!sc.valid) return;
    const R ihx = (R)(0.5 / sc.dh[0]), ihy = (R)(0.5 / sc.dh[1]), ihz = (R)(0.5 / sc.dh[2]);
    const int64_t total = (int64_t)gx * gy * gz;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        int ix = (int)(i % gx);
        int iy = (int)((i / gx) % gy);
        int iz = (int)(i / ((int64_t)gx * gy));
        R ex = 0, ey = 0, ez = 0;
        if (!(ix == 0 || ix == gx - 1 || iy == 0 || iy == gy - 1 || iz == 0 || iz == gz - 1)) {
            ex = -(phi[i + 1] - phi[i - 1]) * ihx;
            ey = -(phi[i + gx] - phi[i - gx]) * ihy;
            ez = -(phi[i + (int64_t)gx * gy] - phi[i - (int64_t)gx * gy]) * ihz;
        }
        store_e(E, i, ex, ey, ez);
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int sm_count()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

cudaError_t launch_book_domain(const DomainParams& p, cudaStream_t s)
{
    book_domain_kernel<<<1, 256, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_deposit(const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                           const ScState* sc, double* rho, int gx, int gy, int gz, cudaStream_t s)
{
    deposit_kernel<<<sm_count() * 8, 256, 0, s>>>(parts, stride, masks, n, sc, rho, gx, gy, gz);
    return cudaGetLastError();
}

template <typename C>
static cudaError_t set_fft_smem_t()
{
    const int bytes = kFftSmemBytes;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(fft_xf_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
    if ((e = cudaFuncSetAttribute(fft_y_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
    if ((e = cudaFuncSetAttribute(fft_z_conv_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
    if ((e = cudaFuncSetAttribute(fft_xi_kernel<C, typename CxT<C>::R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  bytes)))
        return e;
    return cudaSuccess;
}

static cudaError_t set_fft_smem()
{
    static bool done = false;
    if (done) return cudaSuccess;
    cudaError_t e;
    if ((e = set_fft_smem_t<double2>())) return e;
    if ((e = set_fft_smem_t<float2>())) return e;
    if ((e = cudaFuncSetAttribute(fft_green_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kFftSmemBytes)))
        return e;
    done = true;
    return cudaSuccess;
}

static inline int ceil_div64(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Ghat from the current domain: octant G, then the three even-line passes.
cudaError_t launch_green(const ScState* sc, double* G, const Dims& d, int linear, const double2* tw_x,
                         const double2* tw_y, const double2* tw_z, cudaStream_t s)
{
    cudaError_t e = set_fft_smem();
    if (e) return e;
    const int ox = d.nx / 2 + 1, oy = d.ny / 2 + 1, oz = d.nz / 2 + 1;
    green_octant_kernel<<<sm_count() * 4, 256, 0, s>>>(sc, G, d.gx, d.gy, d.gz, linear);
    const size_t sh = kFftSmemBytes;
    // one CTA per kFftTile / L line pairs
    fft_green_kernel<<<ceil_div64(((int64_t)oy * oz + 1) / 2, kFftTile / d.nx), kFftThreads, sh, s>>>(
        G, tw_x, 0, d.nx, ox, oy, oz, sc);
    fft_green_kernel<<<ceil_div64(((int64_t)ox * oz + 1) / 2, kFftTile / d.ny), kFftThreads, sh, s>>>(
        G, tw_y, 1, d.ny, ox, oy, oz, sc);
    fft_green_kernel<<<ceil_div64(((int64_t)ox * oy + 1) / 2, kFftTile / d.nz), kFftThreads, sh, s>>>(
        G, tw_z, 2, d.nz, ox, oy, oz, sc);
    return cudaGetLastError();
}

template <typename C>
static cudaError_t convolve_t(const double* rho, C* S, const double* Ghat, typename CxT<C>::R* phi, const Dims& d,
                              const double2* tw_x, const double2* tw_y, const double2* tw_z, const ScState* sc,
                              cudaStream_t s)
{
    cudaError_t e = set_fft_smem();
    if (e) return e;
    const size_t sh = kFftSmemBytes;
    const int npy = (d.gy + 1) / 2;
    fft_xf_kernel<C><<<ceil_div64((int64_t)npy * d.gz, kFftTile / d.nx), kFftThreads, sh, s>>>(rho, S, tw_x, d, sc);
    fft_y_kernel<C><<<ceil_div64((int64_t)d.nkx * d.gz, kFftTile / d.ny), kFftThreads, sh, s>>>(S, tw_y, d, 0, sc);
    fft_z_conv_kernel<C><<<ceil_div64((int64_t)d.nkx * d.ny, kFftTile / d.nz), kFftThreads, sh, s>>>(S, Ghat, tw_z, d, sc);
    fft_y_kernel<C><<<ceil_div64((int64_t)d.nkx * d.gz, kFftTile / d.ny), kFftThreads, sh, s>>>(S, tw_y, d, 1, sc);
    fft_xi_kernel<C, typename CxT<C>::R>
        <<<ceil_div64((int64_t)npy * d.gz, kFftTile / d.nx), kFftThreads, sh, s>>>(S, phi, tw_x, d, sc);
    return cudaGetLastError();
}

// rho -> phi through the five line passes (FP64).
cudaError_t launch_convolve(const double* rho, double2* S, const double* Ghat, double* phi, const Dims& d,
                            const double2* tw_x, const double2* tw_y, const double2* tw_z, const ScState* sc,
                            cudaStream_t s)
{
    return convolve_t<double2>(rho, S, Ghat, phi, d, tw_x, tw_y, tw_z, sc, s);
}

// rho (FP64 accumulation) -> phi in FP32 (mixed precision: FP32 spectrum
// and potential storage, FP64 butterflies).
cudaError_t launch_convolve_f32(const double* rho, float2* S, const double* Ghat, float* phi, const Dims& d,
                                const double2* tw_x, const double2* tw_y, const double2* tw_z, const ScState* sc,
                                cudaStream_t s)
{
    return convolve_t<float2>(rho, S, Ghat, phi, d, tw_x, tw_y, tw_z, sc, s);
}

cudaError_t launch_efield(const double* phi, double2* E, int gx, int gy, int gz, const ScState* sc, cudaStream_t s)
{
    int64_t total = (int64_t)gx * gy * gz;
    int nb = (int)std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 16);
    efield_kernel<double, double2><<<nb, 256, 0, s>>>(phi, E, gx, gy, gz, sc);
    return cudaGetLastError();
}

cudaError_t launch_efield_f32(const float* phi, float4* E, int gx, int gy, int gz, const ScState* sc, cudaStream_t s)
{
    int64_t total = (int64_t)gx * gy * gz;
    int nb = (int)std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 16);
    efield_kernel<float, float4><<<nb, 256, 0, s>>>(phi, E, gx, gy, gz, sc);
    return cudaGetLastError();
}

} // namespace sb2
