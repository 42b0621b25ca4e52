// Register-resident Stockham FFT for the line passes of the Hockney solver.
//
// A CTA transforms W lines of length L (a power of two, 8..2048).  Each line
// is handled by L/8 threads holding 8 complex values in registers; a pass of
// radix R (8, 4 or 2) is 8/R butterflies per thread, done in registers, and
// consecutive passes exchange their values through one shared-memory tile
// (W x L complex values).  The first pass reads its inputs straight from global
// memory and the last pass writes its outputs straight back, so a length-L
// transform costs (passes - 1) shared-memory round trips and no extra global
// traffic; a forward transform, a pointwise product and an inverse transform
// chain in registers (the inverse runs its radices in reverse order, so its
// first pass consumes exactly the values the forward's last pass produced).
//
// Index conventions (Stockham, natural order in and out):
//   pass p has radix R and span Ns (product of the earlier radices);
//   butterfly b (0 <= b < L/R) of thread t is b = t * (8/R) + q;
//   its inputs are positions b + r L/R (r < R), scaled by w^(k r L/(Ns R))
//   with k = b mod Ns, w = exp(-2 pi i / L) (conjugated for the inverse);
//   its outputs are positions (b - k) R + k + r Ns.
// The first pass (Ns = 1) therefore reads positions b + r L/R and the last
// pass (Ns R = L) writes positions b + r L/R_last.
#pragma once
#include <cuda_runtime.h>

namespace sb2 {
namespace fft {

constexpr int kE = 8; // complex values per thread

// Complex arithmetic in the transform's compute type: double2 (FP64 path) or
// float2 (FP32 butterflies of the mixed-precision path).
template <typename C> struct CxR;
template <> struct CxR<double2> { typedef double R; };
template <> struct CxR<float2> { typedef float R; };
__device__ __forceinline__ double2 mk(double2, double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 mk(float2, float a, float b) { return make_float2(a, b); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk(a, a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk(a, a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b)
{
    return mk(a, a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by -i (forward) or +i (inverse)
template <typename C> __device__ __forceinline__ C rot90(C a, bool inv) { return inv ? mk(a, -a.y, a.x) : mk(a, a.y, -a.x); }

// In-register DFT of size R in natural order: X[k] = sum_r v[r] w^(rk).
template <int R>
struct Dft;
template <>
struct Dft<2> {
    template <typename C>
    static __device__ __forceinline__ void run(C* v, bool)
    {
        C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};
template <>
struct Dft<4> {
    template <typename C>
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
template <>
struct Dft<8> {
    template <typename C>
    static __device__ __forceinline__ void run(C* v, bool inv)
    {
        typedef typename CxR<C>::R R;
        const R h = (R)0.70710678118654752440; // cos(pi/4)
        C a[4], b[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            a[r] = cadd(v[r], v[r + 4]);
            b[r] = csub(v[r], v[r + 4]);
        }
        // w8^r on the difference branch (decimation in frequency)
        b[1] = inv ? mk(b[1], h * (b[1].x - b[1].y), h * (b[1].x + b[1].y))
                   : mk(b[1], h * (b[1].x + b[1].y), h * (b[1].y - b[1].x));
        b[2] = rot90(b[2], inv);
        b[3] = inv ? mk(b[3], -h * (b[3].x + b[3].y), h * (b[3].x - b[3].y))
                   : mk(b[3], h * (b[3].y - b[3].x), -h * (b[3].x + b[3].y));
        Dft<4>::run(a, inv);
        Dft<4>::run(b, inv);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[2 * k] = a[k];
            v[2 * k + 1] = b[k];
        }
    }
};

// Radix plans.  A length L = 8^k * rem (rem 1, 2 or 4) takes k radix-8
// passes and, if rem > 1, one pass of radix rem: plan 0 runs the 8s first,
// plan 1 the radix-rem pass first (the autotuner picks one per propagator);
// REV runs a plan backwards.  Lengths that are powers of 8 have one plan.
__host__ __device__ constexpr int npasses(int L)
{
    int n = 0;
    while (L > 1) {
        L /= (L >= 8 ? 8 : L);
        ++n;
    }
    return n;
}
__host__ __device__ constexpr int rem_radix(int L)
{
    while (L >= 8) L /= 8;
    return L;
}
__host__ __device__ constexpr int radix_fwd(int L, int p, int plan)
{
    const int rem = rem_radix(L), n = npasses(L);
    if (rem == 1) return 8;
    return plan == 0 ? (p < n - 1 ? 8 : rem) : (p == 0 ? rem : 8);
}
// the plan a length actually has (1 only where the two plans differ)
template <int L>
__host__ __device__ constexpr int plan_of(int plan)
{
    return rem_radix(L) > 1 ? plan : 0;
}
template <int L, bool REV, int PLAN = 0>
__host__ __device__ constexpr int radix_at(int p)
{
    return REV ? radix_fwd(L, npasses(L) - 1 - p, PLAN) : radix_fwd(L, p, PLAN);
}
template <int L, bool REV, int PLAN = 0>
__host__ __device__ constexpr int span_at(int p)
{
    int ns = 1;
    for (int i = 0; i < p; ++i) ns *= radix_at<L, REV, PLAN>(i);
    return ns;
}
template <int L, bool REV, int PLAN = 0>
__host__ __device__ constexpr int first_radix() { return radix_at<L, REV, PLAN>(0); }
template <int L, bool REV, int PLAN = 0>
__host__ __device__ constexpr int last_radix() { return radix_at<L, REV, PLAN>(npasses(L) - 1); }

// CTA shape for length L: 256 threads up to L = 512 (two CTAs per SM at the
// pass kernels' ~110 registers, so one CTA's loads overlap another's
// arithmetic), 512 beyond; W lines.
template <int L>
struct Shape {
    static_assert(L >= 8 && L <= 2048 && (L & (L - 1)) == 0, "FFT length");
    static constexpr int TPL = L / kE;                                   // threads per line
    static constexpr int THREADS = L <= 512 ? 256 : 512;
    static constexpr int W = THREADS / TPL;                              // lines per CTA
    static constexpr int PITCH = L + L / 8;                              // x-major line pitch (skewed)
};

// Shared-memory tile layouts.  LMajor: line index fastest (passes along y and
// z: the W lines of a CTA are W consecutive x positions, so global rows are
// contiguous); XMajor: position fastest with one pad slot per 8 (passes along
// x, where a line is contiguous in global memory).
template <int L>
struct LMajor {
    static __device__ __forceinline__ int at(int li, int pos) { return pos * Shape<L>::W + li; }
    static __device__ __forceinline__ int line() { return (int)threadIdx.x % Shape<L>::W; }
    static __device__ __forceinline__ int thr() { return (int)threadIdx.x / Shape<L>::W; }
    static constexpr int kSmemElems = Shape<L>::W * L;
};
template <int L>
struct XMajor {
    static __device__ __forceinline__ int at(int li, int pos) { return li * Shape<L>::PITCH + pos + (pos >> 3); }
    static __device__ __forceinline__ int line() { return (int)threadIdx.x / Shape<L>::TPL; }
    static __device__ __forceinline__ int thr() { return (int)threadIdx.x % Shape<L>::TPL; }
    static constexpr int kSmemElems = Shape<L>::W * Shape<L>::PITCH;
};

// One pass's arithmetic on the registers: twiddles, then the butterflies.
template <int L, int R, typename C>
__device__ __forceinline__ void pass_math(C* v, int t, int Ns, const C* __restrict__ tw, bool inv)
{
    constexpr int NB = kE / R;
    const int tstep = L / (Ns * R);
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int b = t * NB + q;
        const int k = b & (Ns - 1);
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                C w = __ldg(&tw[(k * r * tstep) & (L - 1)]);
                if (inv) w.y = -w.y;
                v[q * R + r] = cmul(v[q * R + r], w);
            }
        }
        Dft<R>::run(v + q * R, inv);
    }
}

// Stores the registers of pass p (radix R, span Ns) at their output positions.
template <int L, int R, class LAY, typename C>
__device__ __forceinline__ void pass_store(const C* v, int li, int t, int Ns, C* sm)
{
    constexpr int NB = kE / R;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int b = t * NB + q;
        const int k = b & (Ns - 1);
        const int base = (b - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) sm[LAY::at(li, base + r * Ns)] = v[q * R + r];
    }
}

// Loads the inputs of a pass of radix R (positions b + r L/R).
template <int L, int R, class LAY, typename C>
__device__ __forceinline__ void pass_load(C* v, int li, int t, const C* sm)
{
    constexpr int NB = kE / R;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int b = t * NB + q;
#pragma unroll
        for (int r = 0; r < R; ++r) v[q * R + r] = sm[LAY::at(li, b + r * (L / R))];
    }
}

// Position held by register e of thread t in the first pass (inputs) or the
// last pass (outputs) of a plan whose first/last radix is R: b + r L/R.
template <int L, int R>
__device__ __forceinline__ int io_pos(int t, int e)
{
    constexpr int NB = kE / R;
    return (t * NB + e / R) + (e % R) * (L / R);
}

// The passes of one transform.  On entry v holds the first pass's inputs,
// on return the last pass's outputs.  Every thread of the CTA calls it (it
// synchronises the CTA).
template <int L, bool REV, class LAY, int PLAN = 0, int P = 0, typename C>
__device__ __forceinline__ void run_passes(C* v, int li, int t, C* sm, const C* __restrict__ tw, bool inv)
{
    if constexpr (P < npasses(L)) {
        constexpr int R = radix_at<L, REV, PLAN>(P);
        constexpr int Ns = span_at<L, REV, PLAN>(P);
        pass_math<L, R, C>(v, t, Ns, tw, inv);
        if constexpr (P + 1 < npasses(L)) {
            constexpr int R2 = radix_at<L, REV, PLAN>(P + 1);
            pass_store<L, R, LAY, C>(v, li, t, Ns, sm);
            __syncthreads();
            pass_load<L, R2, LAY, C>(v, li, t, sm);
            __syncthreads();
            run_passes<L, REV, LAY, PLAN, P + 1, C>(v, li, t, sm, tw, inv);
        }
    }
}

} // namespace fft
} // namespace sb2
