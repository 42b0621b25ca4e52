// 3D open-boundary Hockney solver kernels for sm_100a.
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
// x inverse (Hermitian pairs, first gx outputs).  Each pass holds its lines
// in registers and runs a Stockham transform with radix-8/4/2 butterflies,
// exchanging values between radix passes through shared memory (fft.cuh).
#include <cuda_runtime.h>
#include <algorithm>
#include <type_traits>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "fft.cuh"
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

__device__ __forceinline__ void book_domain_body(const DomainParams& p)
{
    __shared__ double s_sum[256][6];
    // fixed-order reduction of the per-block moment partials (a bunch split
    // over ranks takes the sums of all ranks from xchg instead)
    if (p.compute_domain && !p.domain_fixed && p.xchg) {
        if (threadIdx.x == 0)
            for (int j = 0; j < 6; ++j) s_sum[0][j] = p.xchg[j];
    } else if (p.compute_domain && !p.domain_fixed) {
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
        int nd_op = 0, nd_all = 0;
        for (int s = p.book.slot_begin[o]; s < p.book.slot_end[o]; ++s) {
            int nd = p.ap_counts[s];
            p.ap_counts[s] = 0;
            int el = p.book.slot_elem[s];
            if (p.elem_charge && el >= 0 && nd) p.elem_charge[el] += nd * c.real_num / c.n_total;
            nd_op += nd;
            if (p.xchg) nd_all += (int)llrint(p.xchg[6 + s]);
            c.n_valid -= nd;
        }
        int old_total = c.n_total;
        // update_total_num: total = sum over ranks of the valid counts
        c.n_total = p.xchg ? old_total - nd_all : c.n_valid;
        c.real_num = old_total ? c.n_total * c.real_num / old_total : 0.0;
        if (p.step_records && p.book.op_record[o] >= 0) {
            if (p.rec_cursor) {
                const int r = *p.rec_cursor;
                if (r < p.rec_cap) p.step_records[r] = c;
                *p.rec_cursor = r + 1;
            } else {
                p.step_records[p.book.op_record[o]] = c;
            }
        }
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

__global__ void __launch_bounds__(256) book_domain_kernel(const __grid_constant__ DomainParams p) { book_domain_body(p); }

// one block per bunch of a batch in lockstep
__global__ void __launch_bounds__(256) book_domain_list_kernel(const DomainParams* __restrict__ items)
{
    book_domain_body(items[blockIdx.x]);
}

// grid (x, nitems): item blockIdx.y zeroes its range
__global__ void zero_list_kernel(const ZeroItem* __restrict__ items)
{
    const ZeroItem it = items[blockIdx.y];
    double* d = (double*)it.ptr;
    const int64_t n = it.bytes / 8;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = 0.0;
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
// warp first (lanes grouped by cell key, in any order), so every distinct
// cell of the warp costs one set of 8 atomics -- also when the cell-ordered
// working copy has aged and equal keys are no longer adjacent.
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
    const unsigned full = 0xffffffffu;
    const int64_t wstride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t wb = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) - lane; wb < n; wb += wstride) {
        const int64_t i = wb + lane;
        int ix = 0, iy = 0, iz = 0;
        double ox = 0.0, oy = 0.0, oz = 0.0;
        int key = -1;
        if (i < n && masks[i]) {
            leftmost_d(parts[i], lx, ihx, ix, ox);
            leftmost_d(parts[i + 2 * stride], ly, ihy, iy, oy);
            leftmost_d(parts[i + 4 * stride], lz, ihz, iz, oz);
            if (ix >= -1 && ix < gx && iy >= -1 && iy < gy && iz >= -1 && iz < gz)
                key = ((iz + 1) * (gy + 1) + (iy + 1)) * (gx + 1) + (ix + 1);
        }
        double w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (key >= 0) {
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
        // Lanes whose stencils start in the same cell (__match_any_sync,
        // in any lane order) sum their 8 weights by a tree over their ranks
        // among those peers: in each round a lane adds the partial sum of the
        // next peer above it that is still live, and the peers whose rank
        // has the round's bit set drop out.  The lowest peer ends up with the
        // group's sums and issues its 8 atomics.
        const unsigned peers = __match_any_sync(full, key);
        unsigned below;
        asm("mov.u32 %0, %%lanemask_lt;" : "=r"(below));
        const bool leader = (peers & below) == 0;
        unsigned rest = peers & ~below & ~(1u << lane); // peers above this lane
        int rank = __popc(peers & below);
        while (__any_sync(full, rest != 0)) {
            const int nxt = __ffs(rest) - 1;
            const int from = nxt < 0 ? lane : nxt;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const double t = __shfl_sync(full, w[c], from);
                if (nxt >= 0) w[c] += t;
            }
            rest &= ~__ballot_sync(full, rank & 1);
            rank >>= 1;
        }
        const bool tail = leader;
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
// Deposit by shared-memory tiles (same weights as deposit_kernel; only the
// summation differs).
//
// A CTA takes kDepT * K consecutive particles of the (cell-ordered) bunch.
//   1. coalesced: each thread loads K particles (stride kDepT), computes the
//      stencil cell and the CIC offsets, and stores them in shared memory at
//      the particle's slot of a per-thread-consecutive layout (slot(i) =
//      i + i / K: thread t later reads particles t*K .. t*K+K-1, conflict
//      free); the CTA reduces the bounding box of the stencil cells.
//   2. if the box's grid points fit the tile (kDepTile points), each thread
//      walks its K consecutive particles summing the 8 corner weights of a
//      run of equal cells in FP64 registers (the bunch is ordered by cell, so
//      runs are long) and adds each finished run to the tile; the last run of
//      every thread is first summed over the warp's lanes with the same cell
//      (a transpose reduction when the whole warp shares one cell, the dense
//      core of a freshly ordered bunch; peer groups otherwise).  The tile
//      holds fixed-point sums in 32-bit words, because 32-bit integer
//      atomics are native in shared memory while FP64 (and 64-bit integer)
//      shared atomics are compare-and-swap loops: a run's corner weight is
//      w0 * u with u in [0, 32 K], u * 2^kFrac (< 2^63) is rounded to an
//      integer and split into three 21-bit digits, each added to its own word
//      (every addition carries at least one particle, so a word takes at most
//      kDepT * K <= 2^11 additions of < 2^21 and does not overflow).
//      Resolution 2^-kFrac w0 per addition, far below FP64 summation noise;
//      integer sums do not depend on the order of the additions.
//   3. the tile's non-zero interior points go to rho, the three digits
//      recombined in FP64 and scaled by w0 2^-kFrac, with one global FP64
//      atomic each -- the only global atomics, on the points the CTA's box
//      shares with its neighbours' boxes.
// A chunk whose box does not fit (tails of the bunch, or a bunch that is not
// cell ordered) deposits straight to rho with per-warp peer groups, as
// deposit_kernel does.  Only stencil cells with 0 <= i <= g-2 in every axis
// can reach an interior grid point (0 < i < g-1, deposit.cc:23-30); others
// are skipped.
// ---------------------------------------------------------------------------
constexpr int kDepT = 256;
constexpr int kDepTile = 1536;

template <int K>
struct DepositSmem {
    static constexpr int kSlots = kDepT * (K + 1);
    // fixed-point scale: one addition carries the sum u <= 32 K of a warp's
    // peer group, so u * 2^kFrac <= 2^63 (three 21-bit digits)
    static constexpr int kFrac = K <= 4 ? 56 : 55;
    // the chunk's particles in cell order, slot(i) = i + i / K
    double ox[kSlots], oy[kSlots], oz[kSlots];
    int16_t lk[kSlots];                             // tile cell of the stencil's lower corner
    uint32_t d0[kDepTile], d1[kDepTile], d2[kDepTile]; // d0: cell counts, then offsets, then digit 0
    int32_t box[kDepT / 32][6];
    int32_t wsum[kDepT / 32];
    int32_t nvalid;
};
static_assert(kDepTile < 32768, "tile cells are stored as int16");

// The 8 CIC weights of one particle divided by w0: products of the offsets
// (deposit.cc:309-394 multiplies w0 in front; factored out here and applied
// when the tile is flushed, the same product to rounding).
__device__ __forceinline__ void cic_unit_weights(double ox, double oy, double oz, double* u)
{
    const double aox = 1.0 - ox, aoy = 1.0 - oy, aoz = 1.0 - oz;
    u[0] = aox * aoy * aoz;
    u[1] = ox * aoy * aoz;
    u[2] = aox * oy * aoz;
    u[3] = ox * oy * aoz;
    u[4] = aox * aoy * oz;
    u[5] = ox * aoy * oz;
    u[6] = aox * oy * oz;
    u[7] = ox * oy * oz;
}

__device__ __forceinline__ void cic_weights(double w0, double ox, double oy, double oz, double* w)
{
    const double aox = 1.0 - ox, aoy = 1.0 - oy, aoz = 1.0 - oz;
    w[0] = w0 * aox * aoy * aoz;
    w[1] = w0 * ox * aoy * aoz;
    w[2] = w0 * aox * oy * aoz;
    w[3] = w0 * ox * oy * aoz;
    w[4] = w0 * aox * aoy * oz;
    w[5] = w0 * ox * aoy * oz;
    w[6] = w0 * aox * oy * oz;
    w[7] = w0 * ox * oy * oz;
}

// Sums w over the lanes of the warp whose `key` is equal (peer groups, in any
// lane order, by a tree over the lanes' ranks among their peers); returns
// true on the lowest lane of each group, which then holds the group's sums.
// Every lane of the warp calls it.
__device__ __forceinline__ bool peer_sum8(int key, double* w)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned peers = __match_any_sync(full, key);
    unsigned below;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(below));
    unsigned rest = peers & ~below & ~(1u << lane);
    int rank = __popc(peers & below);
    while (__any_sync(full, rest != 0)) {
        const int nxt = __ffs(rest) - 1;
        const int from = nxt < 0 ? lane : nxt;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const double t = __shfl_sync(full, w[c], from);
            if (nxt >= 0) w[c] += t;
        }
        rest &= ~__ballot_sync(full, rank & 1);
        rank >>= 1;
    }
    return (peers & below) == 0;
}

// Sum of a[0..7] over the warp's 32 lanes, corner c ending on lanes 4c..4c+3:
// each halving exchange keeps half of the values (9 FP64 shuffles in all).
__device__ __forceinline__ double transpose_sum8(const double* a)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    double h4[4], h2[2];
    const bool b16 = lane & 16, b8 = lane & 8, b4 = lane & 4;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double keep = b16 ? a[k + 4] : a[k], send = b16 ? a[k] : a[k + 4];
        h4[k] = keep + __shfl_xor_sync(full, send, 16);
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const double keep = b8 ? h4[k + 2] : h4[k], send = b8 ? h4[k] : h4[k + 2];
        h2[k] = keep + __shfl_xor_sync(full, send, 8);
    }
    double h = (b4 ? h2[1] : h2[0]) + __shfl_xor_sync(full, b4 ? h2[0] : h2[1], 4);
    h += __shfl_xor_sync(full, h, 2);
    h += __shfl_xor_sync(full, h, 1);
    return h; // corner (b16 ? 4 : 0) + (b8 ? 2 : 0) + (b4 ? 1 : 0) = lane >> 2
}

template <int K>
__device__ __forceinline__ void tile_add(DepositSmem<K>& sm, int at, double u, double scale)
{
    const unsigned long long q = __double2ull_rn(u * scale);
    atomicAdd(&sm.d0[at], (uint32_t)(q & 0x1fffffu));
    atomicAdd(&sm.d1[at], (uint32_t)((q >> 21) & 0x1fffffu));
    atomicAdd(&sm.d2[at], (uint32_t)(q >> 42));
}

template <int K, typename RT>
__device__ __forceinline__ void deposit_tile_body(const double* __restrict__ parts, int64_t stride,
                                                  const uint8_t* __restrict__ masks, int64_t n,
                                                  const ScState* __restrict__ scp, RT* rho, int gx, int gy, int gz,
                                                  int vb)
{
    extern __shared__ __align__(16) unsigned char dep_raw[];
    DepositSmem<K>& sm = *reinterpret_cast<DepositSmem<K>*>(dep_raw);
    const ScState& sc = *scp;
    if (!sc.valid) return;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int64_t base = (int64_t)vb * (kDepT * K);
    const unsigned full = 0xffffffffu;

    // 1. cells and offsets of this thread's K particles (stride kDepT), kept
    //    in registers; the CTA's bounding box of stencil cells
    int cell[K];
    double ox[K], oy[K], oz[K];
    {
        double px[K], py[K], pz[K];
        uint8_t pm[K];
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const int64_t i = base + j * kDepT + t;
            pm[j] = 0;
            if (i < n) {
                pm[j] = masks[i];
                px[j] = parts[i];
                py[j] = parts[i + 2 * stride];
                pz[j] = parts[i + 4 * stride];
            }
        }
        const double lx = sc.left[0], ly = sc.left[1], lz = sc.left[2];
        const double ihx = sc.ih[0], ihy = sc.ih[1], ihz = sc.ih[2];
#pragma unroll
        for (int j = 0; j < K; ++j) {
            cell[j] = -1;
            ox[j] = oy[j] = oz[j] = 0.0;
            if (pm[j]) {
                int ix, iy, iz;
                leftmost_d(px[j], lx, ihx, ix, ox[j]);
                leftmost_d(py[j], ly, ihy, iy, oy[j]);
                leftmost_d(pz[j], lz, ihz, iz, oz[j]);
                if (ix >= 0 && ix <= gx - 2 && iy >= 0 && iy <= gy - 2 && iz >= 0 && iz <= gz - 2)
                    cell[j] = ix | (iy << 10) | (iz << 20);
            }
        }
    }
    int bmin[3] = {1 << 30, 1 << 30, 1 << 30}, bmax[3] = {-1, -1, -1};
#pragma unroll
    for (int j = 0; j < K; ++j)
        if (cell[j] >= 0) {
            const int c[3] = {cell[j] & 1023, (cell[j] >> 10) & 1023, cell[j] >> 20};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                bmin[a] = min(bmin[a], c[a]);
                bmax[a] = max(bmax[a], c[a]);
            }
        }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        bmin[a] = __reduce_min_sync(full, bmin[a]);
        bmax[a] = __reduce_max_sync(full, bmax[a]);
    }
    if (lane == 0) {
        sm.box[warp][0] = bmin[0]; sm.box[warp][1] = bmin[1]; sm.box[warp][2] = bmin[2];
        sm.box[warp][3] = bmax[0]; sm.box[warp][4] = bmax[1]; sm.box[warp][5] = bmax[2];
    }
    __syncthreads();
    {
        const int w = lane & (kDepT / 32 - 1);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            bmin[a] = __reduce_min_sync(full, sm.box[w][a]);
            bmax[a] = __reduce_max_sync(full, sm.box[w][3 + a]);
        }
    }
    if (bmax[0] < 0) return; // no particle of the chunk reaches an interior point
    const int BX = bmax[0] - bmin[0] + 2, BY = bmax[1] - bmin[1] + 2, BZ = bmax[2] - bmin[2] + 2;
    const int BXY = BX * BY, V = BXY * BZ;
    const double w0 = sc.w0;

    if (V <= kDepTile) {
        // 2. counting sort of the chunk by tile cell: counts (warp-aggregated
        //    32-bit shared atomics, which also give each particle its rank in
        //    its cell), exclusive scan, particles written to their cell-ordered
        //    slots.  Runs of equal cells are then as long as the chunk allows,
        //    however far the particles have drifted since the bunch's last
        //    re-sort.
        int lk[K], rk[K];
#pragma unroll
        for (int j = 0; j < K; ++j)
            lk[j] = cell[j] < 0 ? -1
                                : (((cell[j] >> 20) - bmin[2]) * BY + (((cell[j] >> 10) & 1023) - bmin[1])) * BX +
                                      ((cell[j] & 1023) - bmin[0]);
        for (int v = t; v < V; v += kDepT) sm.d0[v] = 0u;
        __syncthreads();
        unsigned below;
        asm("mov.u32 %0, %%lanemask_lt;" : "=r"(below));
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const unsigned peers = __match_any_sync(full, lk[j]);
            const int lead = __ffs(peers) - 1;
            int r0 = 0;
            if (lane == lead && lk[j] >= 0) r0 = (int)atomicAdd(&sm.d0[lk[j]], (uint32_t)__popc(peers));
            rk[j] = __shfl_sync(full, r0, lead) + __popc(peers & below);
        }
        __syncthreads();
        {   // exclusive scan of the counts, E consecutive cells per thread
            const int E = (V + kDepT - 1) / kDepT;
            const int v0 = t * E;
            int tot = 0;
            for (int e = 0; e < E; ++e)
                if (v0 + e < V) tot += (int)sm.d0[v0 + e];
            int inc = tot;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(full, inc, o);
                if (lane >= o) inc += u;
            }
            if (lane == 31) sm.wsum[warp] = inc;
            __syncthreads();
            int run = inc - tot;
            for (int w = 0; w < warp; ++w) run += sm.wsum[w];
            if (t == kDepT - 1) sm.nvalid = run + tot;
            for (int e = 0; e < E; ++e)
                if (v0 + e < V) {
                    const int c = (int)sm.d0[v0 + e];
                    sm.d0[v0 + e] = (uint32_t)run;
                    run += c;
                }
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < K; ++j)
            if (lk[j] >= 0) {
                const int dest = (int)sm.d0[lk[j]] + rk[j];
                const int sl = dest + dest / K;
                sm.lk[sl] = (int16_t)lk[j];
                sm.ox[sl] = ox[j];
                sm.oy[sl] = oy[j];
                sm.oz[sl] = oz[j];
            }
        __syncthreads();
        const int nvalid = sm.nvalid;
        for (int v = t; v < V; v += kDepT) {
            sm.d0[v] = 0u;
            sm.d1[v] = 0u;
            sm.d2[v] = 0u;
        }
        __syncthreads();
        // 3. each thread's K consecutive cell-ordered particles: runs of equal
        //    cells summed in FP64 registers, finished runs into the tile
        const double scale = (double)(1ull << DepositSmem<K>::kFrac);
        const int off[8] = {0, 1, BX, BX + 1, BXY, BXY + 1, BXY + BX, BXY + BX + 1};
        int cur = -1;
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const int pos = t * K + j;
            if (pos >= nvalid) continue;
            const int sj = pos + pos / K;
            const int c = sm.lk[sj];
            double u[8];
            cic_unit_weights(sm.ox[sj], sm.oy[sj], sm.oz[sj], u);
            if (c != cur) {
                if (cur >= 0)
#pragma unroll
                    for (int q = 0; q < 8; ++q) tile_add(sm, cur + off[q], acc[q], scale);
                cur = c;
#pragma unroll
                for (int q = 0; q < 8; ++q) acc[q] = u[q];
            } else {
#pragma unroll
                for (int q = 0; q < 8; ++q) acc[q] += u[q];
            }
        }
        if (__all_sync(full, cur == __shfl_sync(full, cur, 0))) {
            // one cell for the whole warp: lane l ends with corner (l >> 2) of
            // the warp's sum
            const double v = transpose_sum8(acc);
            const int c = lane >> 2;
            if (cur >= 0 && (lane & 3) == 0) tile_add(sm, cur + (c & 1) + ((c >> 1) & 1) * BX + (c >> 2) * BXY, v, scale);
        } else if (peer_sum8(cur, acc) && cur >= 0) {
#pragma unroll
            for (int q = 0; q < 8; ++q) tile_add(sm, cur + off[q], acc[q], scale);
        }
        __syncthreads();
        // 4. the tile's interior points to rho
        const double back = w0 / scale;
        // v / BX and r / BY through float reciprocals: (v + 0.5) / BX lies at
        // least 0.5 / BX from an integer, and with v < 2^22 / BX the float
        // rounding stays below that, so the truncation is the integer quotient
        const float ibx = 1.0f / (float)BX, iby = 1.0f / (float)BY;
        for (int v = t; v < V; v += kDepT) {
            const uint32_t a0 = sm.d0[v], a1 = sm.d1[v], a2 = sm.d2[v];
            if ((a0 | a1 | a2) == 0u) continue;
            const int r = (int)(((float)v + 0.5f) * ibx);
            const int rz = (int)(((float)r + 0.5f) * iby);
            const int X = bmin[0] + (v - r * BX), Y = bmin[1] + (r - rz * BY), Z = bmin[2] + rz;
            if (X > 0 && X < gx - 1 && Y > 0 && Y < gy - 1 && Z > 0 && Z < gz - 1) {
                const double sum = ((double)a2 * 4398046511104.0 + (double)a1 * 2097152.0) + (double)a0;
                atomicAdd(&rho[((int64_t)Z * gy + Y) * gx + X], (RT)(sum * back));
            }
        }
        return;
    }

    // box too large for the tile: per-warp peer groups straight to rho
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const int c = cell[j];
        double w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (c >= 0) cic_weights(w0, ox[j], oy[j], oz[j], w);
        if (!peer_sum8(c, w) || c < 0) continue;
        const int ix = c & 1023, iy = (c >> 10) & 1023, iz = c >> 20;
        const bool x0 = ix > 0, x1 = ix + 1 < gx - 1;
        const bool y0 = iy > 0, y1 = iy + 1 < gy - 1;
        const bool z0 = iz > 0, z1 = iz + 1 < gz - 1;
        const int64_t b0 = (int64_t)iz * gx * gy + (int64_t)iy * gx + ix;
        const int64_t P = (int64_t)gx * gy;
        if (z0) {
            if (y0 && x0) atomicAdd(&rho[b0], (RT)w[0]);
            if (y0 && x1) atomicAdd(&rho[b0 + 1], (RT)w[1]);
            if (y1 && x0) atomicAdd(&rho[b0 + gx], (RT)w[2]);
            if (y1 && x1) atomicAdd(&rho[b0 + gx + 1], (RT)w[3]);
        }
        if (z1) {
            if (y0 && x0) atomicAdd(&rho[b0 + P], (RT)w[4]);
            if (y0 && x1) atomicAdd(&rho[b0 + P + 1], (RT)w[5]);
            if (y1 && x0) atomicAdd(&rho[b0 + P + gx], (RT)w[6]);
            if (y1 && x1) atomicAdd(&rho[b0 + P + gx + 1], (RT)w[7]);
        }
    }
}

template <int K, typename RT>
__global__ void __launch_bounds__(kDepT) deposit_tile_kernel(const double* __restrict__ parts, int64_t stride,
                                                             const uint8_t* __restrict__ masks, int64_t n,
                                                             const ScState* __restrict__ scp, RT* rho, int gx,
                                                             int gy, int gz)
{
    deposit_tile_body<K, RT>(parts, stride, masks, n, scp, rho, gx, gy, gz, blockIdx.x);
}

// The deposits of many bunches with one grid shape: item i on blocks
// [first[i], first[i+1]).
template <int K, typename RT>
__global__ void __launch_bounds__(kDepT) deposit_list_kernel(const DepositItem* __restrict__ items,
                                                             const int* __restrict__ first, int nitems, int gx,
                                                             int gy, int gz)
{
    int lo = 0, hi = nitems;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (first[mid] <= (int)blockIdx.x)
            lo = mid;
        else
            hi = mid;
    }
    const DepositItem it = items[lo];
    deposit_tile_body<K, RT>(it.parts, it.stride, it.masks, it.n, it.sc, (RT*)it.rho, gx, gy, gz,
                             (int)blockIdx.x - first[lo]);
}

// ---------------------------------------------------------------------------
// Green function octant: alg_g2_linear :230-348 / alg_g2_pointlike :136-228
// evaluated for ix <= gx, iy <= gy, iz <= gz (doubled shape = 2 * shape,
// so this octant plus mirroring is the whole doubled-grid G2)
// ---------------------------------------------------------------------------
// Linear (z-integrated) Green function on the octant, one chunk of a z
// column per thread.  With s(k) = sqrt(x^2 + y^2 + (k hz)^2) and P(k) =
// s(k) + k hz, the reference's per-point terms are
//   2 s(k) - s(k-1) - s(k+1) + (hz - z) log(P(k)/P(k-1)) + (hz + z) log(P(k+1)/P(k))
// (alg_g2_linear, space_charge_3d_open_hockney.cc:237-348, z = k hz >= 0 on
// the octant; k = 0 and k = 1 take the reference's special cases), so along
// a column every square root and every logarithm is shared by neighbouring
// points: one sqrt and one log per point instead of three and two.
// 4 points per thread: 139K threads on the 64^2 x 128 octant (0.035 ms per
// step at C1 against 0.040 with 16, 0.038 with 8 or 2)
constexpr int kGreenChunk = 4;

__global__ void green_octant_kernel(const ScState* __restrict__ scp, double* G, int gx0, int gy0, int gz0,
                                    int linear, const ConvItem* __restrict__ list)
{
    if (list) { // item blockIdx.y of a batch in lockstep
        scp = list[blockIdx.y].sc;
        G = list[blockIdx.y].ghat;
    }
    const ScState& sc = *scp;
    if (!sc.valid) return;
    const int ox = gx0 + 1, oy = gy0 + 1, oz = gz0 + 1;
    const double hx = sc.dh[0], hy = sc.dh[1], hz = sc.dh[2];
    if (!linear) { // alg_g2_pointlike :136-180
        const int64_t total = (int64_t)ox * oy * oz;
        const double G000 = 2.8 / fmin(hx, fmin(hy, hz));
        for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
             t += (int64_t)gridDim.x * blockDim.x) {
            const unsigned tt = (unsigned)t, r = tt / (unsigned)ox; // total < 2^31
            const int ix = (int)(tt - r * (unsigned)ox);
            const int iy = (int)(r % (unsigned)oy);
            const int iz = (int)(r / (unsigned)oy);
            const double dx = ix * hx, dy = iy * hy, dz = iz * hz;
            G[t] = (ix == 0 && iy == 0 && iz == 0) ? G000 : 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
        }
        return;
    }
    const double rr0 = hx * hx + hy * hy;
    const double r10 = sqrt(hx * hx + hy * hy + hz * hz);
    const double G000 = (2.0 / rr0) * (hz * r10 + rr0 * log((hz + r10) / sqrt(rr0)) - hz * hz);
    const double epsz = 1e-12 * hz;
    const int nchunks = (oz + kGreenChunk - 1) / kGreenChunk;
    const int64_t total = (int64_t)ox * oy * nchunks;
    const int64_t plane = (int64_t)ox * oy;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const unsigned tt = (unsigned)t, r = tt / (unsigned)ox; // total < 2^31
        const int ix = (int)(tt - r * (unsigned)ox);
        const int iy = (int)(r % (unsigned)oy);
        const int c = (int)(r / (unsigned)oy);
        const int k0 = c * kGreenChunk, k1 = min(oz, k0 + kGreenChunk);
        const double x = ix * hx, y = iy * hy;
        const double rr = x * x + y * y;
        auto sk = [&](int k) { const double z = k * hz; return sqrt(rr + z * z); };
        double s_m = sk(k0 - 1), s_0 = sk(k0), s_p = sk(k0 + 1);
        // log(P(k0)/P(k0-1)), needed from k0 >= 2 on
        double lr_m = k0 >= 2 ? log((s_0 + k0 * hz) / (s_m + (k0 - 1) * hz)) : 0.0;
        double* out = G + (int64_t)iy * ox + ix;
        for (int k = k0; k < k1; ++k) {
            const double z = k * hz;
            const double lr_p = log((s_p + (k + 1) * hz) / (s_0 + z)); // log(P(k+1)/P(k))
            double Gv = 2.0 * s_0 - s_m - s_p;
            if (k == 0) {
                if (fabs(x) + fabs(y) < 2. * epsz)
                    Gv += hz * G000;
                else
                    Gv += 2.0 * hz * log((sqrt(hz * hz + rr) + hz) / sqrt(rr));
            } else if (k == 1) {
                Gv += (hz + z) * lr_p;
            } else {
                Gv += (hz - z) * lr_m + (hz + z) * lr_p;
            }
            out[(int64_t)k * plane] = Gv;
            s_m = s_0;
            s_0 = s_p;
            s_p = sk(k + 2);
            lr_m = lr_p;
        }
    }
}

// ---------------------------------------------------------------------------
// Line passes of the convolution (register-resident FFT, fft.cuh).  Global
// storage of the spectrum is C (double2, or float2 for the mixed path); the
// butterflies, the twiddles and the shared-memory exchanges are in W
// (double2, or float2 for FP32 butterflies).  FP64 storage with FP64
// butterflies is the drop-in; float2 storage rounds only at the five pass
// boundaries when W is double2.
// ---------------------------------------------------------------------------
template <typename C> struct CxT;
template <> struct CxT<double2> { typedef double R; };
template <> struct CxT<float2> { typedef float R; };
template <typename W> __device__ __forceinline__ W cvt_c(double2 v);
template <typename W> __device__ __forceinline__ W cvt_c(float2 v);
template <> __device__ __forceinline__ double2 cvt_c<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ double2 cvt_c<double2>(float2 v) { return make_double2(v.x, v.y); }
template <> __device__ __forceinline__ float2 cvt_c<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <> __device__ __forceinline__ float2 cvt_c<float2>(float2 v) { return v; }
template <typename W> __device__ __forceinline__ W czero() { return cvt_c<W>(make_double2(0.0, 0.0)); }

// XF: pairs of real rows (y, y+1) of rho -> S rows (r2c, first gx inputs).
// Lines l = (pair, z); the last pass goes through shared memory so that
// each output k can combine Z[k] and Z[L-k].
template <int L, int PLAN, typename RI, typename C, typename W>
__global__ void __launch_bounds__(fft::Shape<L>::THREADS) fft_xf_kernel(const RI* __restrict__ rho, C* S,
                                                                        const W* __restrict__ tw, Dims d,
                                                                        const ScState* __restrict__ scp,
                                                                        const ConvItem* __restrict__ list)
{
    if (list) { // item blockIdx.z of a batch in lockstep
        rho = (const RI*)list[blockIdx.z].rho;
        S = (C*)list[blockIdx.z].S;
        scp = list[blockIdx.z].sc;
    }
    typedef fft::XMajor<L> LAY;
    typedef typename CxT<W>::R R;
    constexpr int NW = fft::Shape<L>::W, TPL = fft::Shape<L>::TPL;
    constexpr int R0 = fft::first_radix<L, false, PLAN>(), RL = fft::last_radix<L, false, PLAN>();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    W* sm = (W*)sm_raw;
    if (!scp->valid) return;
    const int li = LAY::line(), t = LAY::thr();
    const int npy = (d.gy + 1) / 2;
    const int64_t nlines = (int64_t)npy * d.gz;
    const int64_t l = (int64_t)blockIdx.x * NW + li;
    const bool ok = l < nlines;
    const int z = ok ? (int)((unsigned)l / (unsigned)npy) : 0, pr = ok ? (int)l - z * npy : 0; // nlines < 2^31
    const int ya = 2 * pr, yb = ya + 1;
    const RI* ra = rho + ((int64_t)z * d.gy + ya) * d.gx;
    const RI* rb = rho + ((int64_t)z * d.gy + yb) * d.gx;
    W v[fft::kE];
#pragma unroll
    for (int e = 0; e < fft::kE; ++e) {
        const int pos = fft::io_pos<L, R0>(t, e);
        v[e] = czero<W>();
        if (ok && pos < d.gx) {
            v[e].x = (R)ra[pos];
            if (yb < d.gy) v[e].y = (R)rb[pos];
        }
    }
    fft::run_passes<L, false, LAY, PLAN>(v, li, t, sm, tw, false);
#pragma unroll
    for (int e = 0; e < fft::kE; ++e) sm[LAY::at(li, fft::io_pos<L, RL>(t, e))] = v[e];
    __syncthreads();
    if (!ok) return;
    C* sa = S + ((int64_t)z * d.ny + ya) * d.nkxp;
    C* sb = S + ((int64_t)z * d.ny + yb) * d.nkxp;
    const R half = (R)0.5;
    for (int k = t; k < d.nkx; k += TPL) {
        const W Z = sm[LAY::at(li, k)], Zn = sm[LAY::at(li, (L - k) & (L - 1))];
        sa[k] = cvt_c<C>(fft::mk(Z, (Z.x + Zn.x) * half, (Z.y - Zn.y) * half));
        if (yb < d.gy) sb[k] = cvt_c<C>(fft::mk(Z, (Z.y + Zn.y) * half, -(Z.x - Zn.x) * half));
    }
}

// Y passes: lines (kx, z < gz) along y, NW consecutive kx per CTA.  forward:
// first gy inputs, all ny outputs; inverse: all inputs, first gy outputs.
template <int L, int PLAN, typename C, typename W, bool INV>
__global__ void __launch_bounds__(fft::Shape<L>::THREADS) fft_y_kernel(C* S, const W* __restrict__ tw, Dims d,
                                                                       const ScState* __restrict__ scp,
                                                                       const ConvItem* __restrict__ list)
{
    if (list) {
        S = (C*)list[blockIdx.z].S;
        scp = list[blockIdx.z].sc;
    }
    typedef fft::LMajor<L> LAY;
    constexpr int NW = fft::Shape<L>::W;
    constexpr int R0 = fft::first_radix<L, false, PLAN>(), RL = fft::last_radix<L, false, PLAN>();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    W* sm = (W*)sm_raw;
    if (!scp->valid) return;
    const int li = LAY::line(), t = LAY::thr();
    // lines (kx, z) numbered z * nkxp + kx over the padded row pitch, so no
    // CTA idles on a row's last column (nkx = nx / 2 + 1 is odd)
    const int l = blockIdx.x * NW + li;
    const int z = (int)((unsigned)l / (unsigned)d.nkxp), kx = l - z * d.nkxp;
    const bool ok = kx < d.nkx && z < d.gz;
    C* col = S + (int64_t)(ok ? z : 0) * d.ny * d.nkxp + (ok ? kx : 0);
    const int nin = INV ? L : d.gy;
    W v[fft::kE];
#pragma unroll
    for (int e = 0; e < fft::kE; ++e) {
        const int pos = fft::io_pos<L, R0>(t, e);
        v[e] = (ok && pos < nin) ? cvt_c<W>(col[(int64_t)pos * d.nkxp]) : czero<W>();
    }
    fft::run_passes<L, false, LAY, PLAN>(v, li, t, sm, tw, INV);
    if (!ok) return;
    const int nout = INV ? d.gy : L;
#pragma unroll
    for (int e = 0; e < fft::kE; ++e) {
        const int pos = fft::io_pos<L, RL>(t, e);
        if (pos < nout) col[(int64_t)pos * d.nkxp] = cvt_c<C>(v[e]);
    }
}

// Z pass: lines (kx, ky) along z: forward (first gz inputs), multiply by the
// real octant Ghat(kx, min(ky, ny-ky), min(kz, nz-kz)) in registers, inverse
// (radices reversed, so it starts from the registers), first gz outputs.
// (alg_cplx_multiplier space_charge_3d_open_hockney.cc:350-372 fused between
// the transforms.)
template <int L, int PLAN, typename C, typename W>
__global__ void __launch_bounds__(fft::Shape<L>::THREADS) fft_z_conv_kernel(C* S, const double* __restrict__ Ghat,
                                                                            const W* __restrict__ tw, Dims d,
                                                                            const ScState* __restrict__ scp,
                                                                            const ConvItem* __restrict__ list)
{
    if (list) {
        S = (C*)list[blockIdx.z].S;
        Ghat = list[blockIdx.z].ghat;
        scp = list[blockIdx.z].sc;
    }
    typedef fft::LMajor<L> LAY;
    typedef typename CxT<W>::R R;
    constexpr int NW = fft::Shape<L>::W;
    constexpr int R0 = fft::first_radix<L, false, PLAN>(), RL = fft::last_radix<L, false, PLAN>();
    constexpr int RI = fft::last_radix<L, true, PLAN>();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    W* sm = (W*)sm_raw;
    if (!scp->valid) return;
    const int li = LAY::line(), t = LAY::thr();
    // lines (kx, ky) numbered ky * nkxp + kx (see the y pass)
    const int l = blockIdx.x * NW + li;
    const int ky0 = (int)((unsigned)l / (unsigned)d.nkxp), kx0 = l - ky0 * d.nkxp;
    const bool ok = kx0 < d.nkx && ky0 < d.ny;
    const int kx = ok ? kx0 : 0, ky = ok ? ky0 : 0;
    C* col = S + (int64_t)ky * d.nkxp + kx;
    const int64_t zs = (int64_t)d.ny * d.nkxp;
    W v[fft::kE];
#pragma unroll
    for (int e = 0; e < fft::kE; ++e) {
        const int pos = fft::io_pos<L, R0>(t, e);
        v[e] = (ok && pos < d.gz) ? cvt_c<W>(col[pos * zs]) : czero<W>();
    }
    fft::run_passes<L, false, LAY, PLAN>(v, li, t, sm, tw, false);
    const int ogx = d.nx / 2 + 1, ogy = d.ny / 2 + 1;
    const int my = ky <= d.ny / 2 ? ky : d.ny - ky;
    const double* gcol = Ghat + (int64_t)my * ogx + (ok ? kx : 0);
#pragma unroll
    for (int e = 0; e < fft::kE; ++e) {
        const int kz = fft::io_pos<L, RL>(t, e);
        const int mz = kz <= L / 2 ? kz : L - kz;
        const R g = ok ? (R)__ldg(&gcol[(int64_t)mz * ogy * ogx]) : (R)0;
        v[e] = fft::mk(v[e], v[e].x * g, v[e].y * g);
    }
    fft::run_passes<L, true, LAY, PLAN>(v, li, t, sm, tw, true);
    if (!ok) return;
#pragma unroll
    for (int e = 0; e < fft::kE; ++e) {
        const int pos = fft::io_pos<L, RI>(t, e);
        if (pos < d.gz) col[pos * zs] = cvt_c<C>(v[e]);
    }
}

// XI: Hermitian pairs of spectrum rows -> real rows (y, y+1) of phi (c2r,
// first gx outputs); imaginary parts of the k = 0 and k = nx/2 terms are
// ignored as a c2r transform does.
template <int L, int PLAN, typename C, typename W, typename RO>
__global__ void __launch_bounds__(fft::Shape<L>::THREADS) fft_xi_kernel(const C* __restrict__ S, RO* phi,
                                                                        const W* __restrict__ tw, Dims d,
                                                                        const ScState* __restrict__ scp,
                                                                        const ConvItem* __restrict__ list)
{
    if (list) {
        S = (const C*)list[blockIdx.z].S;
        phi = (RO*)list[blockIdx.z].phi;
        scp = list[blockIdx.z].sc;
    }
    typedef fft::XMajor<L> LAY;
    constexpr int NW = fft::Shape<L>::W;
    constexpr int R0 = fft::first_radix<L, false, PLAN>(), RL = fft::last_radix<L, false, PLAN>();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    W* sm = (W*)sm_raw;
    if (!scp->valid) return;
    const int li = LAY::line(), t = LAY::thr();
    const int npy = (d.gy + 1) / 2;
    const int64_t nlines = (int64_t)npy * d.gz;
    const int64_t l = (int64_t)blockIdx.x * NW + li;
    const bool ok = l < nlines;
    const int z = ok ? (int)((unsigned)l / (unsigned)npy) : 0, pr = ok ? (int)l - z * npy : 0; // nlines < 2^31
    const int ya = 2 * pr, yb = ya + 1;
    const C* sa = S + ((int64_t)z * d.ny + ya) * d.nkxp;
    const C* sb = S + ((int64_t)z * d.ny + yb) * d.nkxp;
    constexpr int half = L / 2;
    W v[fft::kE];
#pragma unroll
    for (int e = 0; e < fft::kE; ++e) {
        const int j = fft::io_pos<L, R0>(t, e);
        const int k = j <= half ? j : L - j;
        W A = czero<W>(), B = czero<W>();
        if (ok) {
            A = cvt_c<W>(sa[k]);
            if (yb < d.gy) B = cvt_c<W>(sb[k]);
        }
        if (k == 0 || k == half) {
            A.y = 0;
            B.y = 0;
        }
        if (j > half) {
            A.y = -A.y;
            B.y = -B.y;
        }
        v[e] = fft::mk(A, A.x - B.y, A.y + B.x);
    }
    fft::run_passes<L, false, LAY, PLAN>(v, li, t, sm, tw, true);
    if (!ok) return;
    RO* pa = phi + ((int64_t)z * d.gy + ya) * d.gx;
    RO* pb = phi + ((int64_t)z * d.gy + yb) * d.gx;
#pragma unroll
    for (int e = 0; e < fft::kE; ++e) {
        const int j = fft::io_pos<L, RL>(t, e);
        if (j < d.gx) {
            pa[j] = (RO)v[e].x;
            if (yb < d.gy) pb[j] = (RO)v[e].y;
        }
    }
}

// Ghat passes on the real octant (ox, oy, oz) = (nx/2+1, ny/2+1, nz/2+1):
// along axis 0/1/2, each line is mirrored to the even real line of length L
// and transformed; the real parts of the first L/2+1 outputs are stored back
// in place.  The transform of a real even line is real, so two lines ride in
// one complex transform (lines 2c and 2c+1 as its real and imaginary parts)
// and come out as its real and imaginary parts.  Axis 0 (x rows, contiguous)
// uses the x-major tile; axes 1 and 2 take W consecutive line pairs.
template <int L, int AXIS, int PLAN>
__global__ void __launch_bounds__(fft::Shape<L>::THREADS) fft_green_kernel(double* G,
                                                                           const double2* __restrict__ tw, int ox,
                                                                           int oy, int oz,
                                                                           const ScState* __restrict__ scp,
                                                                           const ConvItem* __restrict__ list)
{
    if (list) {
        G = list[blockIdx.z].ghat;
        scp = list[blockIdx.z].sc;
    }
    typedef typename std::conditional<AXIS == 0, fft::XMajor<L>, fft::LMajor<L>>::type LAY;
    constexpr int W = fft::Shape<L>::W;
    constexpr int R0 = fft::first_radix<L, false, PLAN>(), RL = fft::last_radix<L, false, PLAN>();
    constexpr int half = L / 2;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* sm = (double2*)sm_raw;
    if (!scp->valid) return;
    const int li = LAY::line(), t = LAY::thr();
    int64_t nlines, sj;
    if (AXIS == 0) { nlines = (int64_t)oy * oz; sj = 1; }
    else if (AXIS == 1) { nlines = (int64_t)ox * oz; sj = ox; }
    else { nlines = (int64_t)ox * oy; sj = (int64_t)ox * oy; }
    auto line_base = [&](int64_t l) -> int64_t {
        if (AXIS == 0) return l * ox;                                  // (y, z) rows
        if (AXIS == 1) { // (kx, z); nlines < 2^31
            const int zz = (int)((unsigned)l / (unsigned)ox);
            return (l - (int64_t)zz * ox) + zz * (int64_t)ox * oy;
        }
        return l;                                                      // (kx, ky)
    };
    const int64_t c = (int64_t)blockIdx.x * W + li;
    const int64_t la = 2 * c, lb = la + 1;
    const bool oka = la < nlines, okb = lb < nlines;
    const double* ga = G + (oka ? line_base(la) : 0);
    const double* gb = G + (okb ? line_base(lb) : 0);
    double2 v[fft::kE];
#pragma unroll
    for (int e = 0; e < fft::kE; ++e) {
        const int j = fft::io_pos<L, R0>(t, e);
        const int m = j <= half ? j : L - j;
        v[e] = make_double2(oka ? ga[m * sj] : 0.0, okb ? gb[m * sj] : 0.0);
    }
    fft::run_passes<L, false, LAY, PLAN>(v, li, t, sm, tw, false);
    double* wa = G + (oka ? line_base(la) : 0);
    double* wb = G + (okb ? line_base(lb) : 0);
#pragma unroll
    for (int e = 0; e < fft::kE; ++e) {
        const int k = fft::io_pos<L, RL>(t, e);
        if (k <= half) {
            if (oka) wa[k * sj] = v[e].x;
            if (okb) wb[k * sj] = v[e].y;
        }
    }
}

// E = -grad phi by central differences on interior cells of the original
// grid, zero on the boundary: alg_force_extractor_doubled_domain
// space_charge_3d_kernels.h:217-307 (h of the doubled domain).
// one 32-byte store per FP64 cell {ex, ey, ez, 0} (the field is 32-byte
// aligned: the kick reads each cell with one 32-byte load)
__device__ __forceinline__ void store_e(double2* E, int64_t i, double ex, double ey, double ez)
{
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(E + 2 * i), "d"(ex), "d"(ey), "d"(ez), "d"(0.0)
                 : "memory");
}
__device__ __forceinline__ void store_e(float4* E, int64_t i, float ex, float ey, float ez)
{
    E[i] = make_float4(ex, ey, ez, 0.0f);
}

// One warp per x row (iy, iz): the row's indices come from one 32-bit
// division instead of three 64-bit ones per point.
template <typename R, typename EV>
__global__ void efield_kernel(const R* __restrict__ phi, EV* E, int gx, int gy, int gz,
                              const ScState* __restrict__ scp, const ConvItem* __restrict__ list)
{
    if (list) { // item blockIdx.y of a batch in lockstep
        phi = (const R*)list[blockIdx.y].phi;
        E = (EV*)list[blockIdx.y].E;
        scp = list[blockIdx.y].sc;
    }
    const ScState& sc = *scp;
    if (!sc.valid) return;
    const R ihx = (R)(0.5 / sc.dh[0]), ihy = (R)(0.5 / sc.dh[1]), ihz = (R)(0.5 / sc.dh[2]);
    const int rows = gy * gz, lane = threadIdx.x & 31;
    const int nw = (int)((gridDim.x * blockDim.x) >> 5);
    const int64_t plane = (int64_t)gx * gy;
    for (int r = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); r < rows; r += nw) {
        const int iz = r / gy, iy = r - iz * gy;
        const bool yz_in = iy > 0 && iy < gy - 1 && iz > 0 && iz < gz - 1;
        const int64_t row = (int64_t)r * gx;
        for (int ix = lane; ix < gx; ix += 32) {
            const int64_t i = row + ix;
            R ex = 0, ey = 0, ez = 0;
            if (yz_in && ix > 0 && ix < gx - 1) {
                ex = -(phi[i + 1] - phi[i - 1]) * ihx;
                ey = -(phi[i + gx] - phi[i - gx]) * ihy;
                ez = -(phi[i + plane] - phi[i - plane]) * ihz;
            }
            store_e(E, i, ex, ey, ez);
        }
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

// Sharded bunch: this rank's moment sums (fixed-order reduction of the block
// partials) and discard counts per aperture slot, to be summed over ranks.
__global__ void __launch_bounds__(256) shard_pack_kernel(const __grid_constant__ DomainParams p, int nslots,
                                                         double* xchg)
{
    __shared__ double s_sum[256][6];
    const bool sums = p.compute_domain && !p.domain_fixed;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (sums)
        for (int b = threadIdx.x; b < p.n_partials; b += blockDim.x)
            for (int j = 0; j < 6; ++j) acc[j] += p.moment_partials[b * 6 + j];
    for (int j = 0; j < 6; ++j) s_sum[threadIdx.x][j] = acc[j];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int j = 0; j < 6; ++j) s_sum[threadIdx.x][j] += s_sum[threadIdx.x + w][j];
        __syncthreads();
    }
    if (threadIdx.x < 6) xchg[threadIdx.x] = s_sum[0][threadIdx.x];
    for (int k = threadIdx.x; k < nslots; k += blockDim.x) xchg[6 + k] = (double)p.ap_counts[k];
}

__global__ void shard_count_kernel(const BunchCounters* c, double* xchg) { xchg[0] = (double)c->n_valid; }
__global__ void shard_total_kernel(BunchCounters* c, const double* xchg) { c->n_total = (int)llrint(xchg[0]); }

cudaError_t launch_shard_pack(const DomainParams& p, int nslots, double* xchg, cudaStream_t s)
{
    shard_pack_kernel<<<1, 256, 0, s>>>(p, nslots, xchg);
    return cudaGetLastError();
}
cudaError_t launch_shard_count(const BunchCounters* c, double* xchg, cudaStream_t s)
{
    shard_count_kernel<<<1, 1, 0, s>>>(c, xchg);
    return cudaGetLastError();
}
cudaError_t launch_shard_total(BunchCounters* c, const double* xchg, cudaStream_t s)
{
    shard_total_kernel<<<1, 1, 0, s>>>(c, xchg);
    return cudaGetLastError();
}

cudaError_t launch_book_domain(const DomainParams& p, cudaStream_t s)
{
    book_domain_kernel<<<1, 256, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_book_domain_list(const DomainParams* items, int nitems, cudaStream_t s)
{
    book_domain_list_kernel<<<nitems, 256, 0, s>>>(items);
    return cudaGetLastError();
}

cudaError_t launch_zero_list(const ZeroItem* items, int nitems, cudaStream_t s)
{
    zero_list_kernel<<<dim3(std::max(1, sm_count() * 8 / nitems), nitems), 256, 0, s>>>(items);
    return cudaGetLastError();
}

#ifndef SB2_DEPOSIT_CTAS
#define SB2_DEPOSIT_CTAS 8 // CTAs per SM of the grid-stride deposit (5 / 8 / 16: 0.163 / 0.142 / 0.146 ms per C1 step)
#endif
template <int K, typename RT>
static cudaError_t deposit_tile(const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                                const ScState* sc, RT* rho, int gx, int gy, int gz, cudaStream_t s)
{
    const int bytes = (int)sizeof(DepositSmem<K>);
    static cudaError_t once =
        cudaFuncSetAttribute(deposit_tile_kernel<K, RT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (once) return once;
    const int64_t chunk = (int64_t)kDepT * K;
    const int64_t nb = (n + chunk - 1) / chunk;
    if (nb > 0)
        deposit_tile_kernel<K, RT><<<(unsigned)nb, kDepT, bytes, s>>>(parts, stride, masks, n, sc, rho, gx, gy, gz);
    return cudaGetLastError();
}

// Deposit variant: SB2_DEPOSIT=tile (default: shared-memory tiles of 256 x K
// particles, K from SB2_DEPOSIT_K, 4 or 8) or warp (per-warp peer groups and
// global atomics only).
static int deposit_variant()
{
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("SB2_DEPOSIT");
        const char* k = getenv("SB2_DEPOSIT_K");
        v = (e && !strcmp(e, "warp")) ? 0 : ((k && atoi(k) == 8) ? 8 : 4);
    }
    return v;
}

int deposit_default_chunk() { return deposit_variant(); }

cudaError_t launch_deposit_k(int chunk, const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                             const ScState* sc, double* rho, int gx, int gy, int gz, cudaStream_t s)
{
    switch (chunk) {
    case 4: return deposit_tile<4, double>(parts, stride, masks, n, sc, rho, gx, gy, gz, s);
    case 8: return deposit_tile<8, double>(parts, stride, masks, n, sc, rho, gx, gy, gz, s);
    default:
        deposit_kernel<<<sm_count() * SB2_DEPOSIT_CTAS, 256, 0, s>>>(parts, stride, masks, n, sc, rho, gx, gy, gz);
        return cudaGetLastError();
    }
}

cudaError_t launch_deposit_f32_k(int chunk, const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                                 const ScState* sc, float* rho, int gx, int gy, int gz, cudaStream_t s)
{
    return chunk == 8 ? deposit_tile<8, float>(parts, stride, masks, n, sc, rho, gx, gy, gz, s)
                      : deposit_tile<4, float>(parts, stride, masks, n, sc, rho, gx, gy, gz, s);
}

cudaError_t launch_deposit(const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                           const ScState* sc, double* rho, int gx, int gy, int gz, cudaStream_t s)
{
    switch (deposit_variant()) {
    case 4: return deposit_tile<4, double>(parts, stride, masks, n, sc, rho, gx, gy, gz, s);
    case 8: return deposit_tile<8, double>(parts, stride, masks, n, sc, rho, gx, gy, gz, s);
    default:
        deposit_kernel<<<sm_count() * SB2_DEPOSIT_CTAS, 256, 0, s>>>(parts, stride, masks, n, sc, rho, gx, gy, gz);
        return cudaGetLastError();
    }
}

int deposit_list_blocks(int64_t n) { return (int)((n + kDepT * 4 - 1) / (kDepT * 4)); }

template <typename RT>
static cudaError_t deposit_list(const DepositItem* items, const int* first, int nitems, int nblocks, int gx, int gy,
                                int gz, cudaStream_t s)
{
    const int bytes = (int)sizeof(DepositSmem<4>);
    static cudaError_t once =
        cudaFuncSetAttribute(deposit_list_kernel<4, RT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (once) return once;
    if (nblocks > 0) deposit_list_kernel<4, RT><<<nblocks, kDepT, bytes, s>>>(items, first, nitems, gx, gy, gz);
    return cudaGetLastError();
}

cudaError_t launch_deposit_list(bool f32, const DepositItem* items, const int* first, int nitems, int nblocks, int gx,
                                int gy, int gz, cudaStream_t s)
{
    return f32 ? deposit_list<float>(items, first, nitems, nblocks, gx, gy, gz, s)
               : deposit_list<double>(items, first, nitems, nblocks, gx, gy, gz, s);
}

cudaError_t launch_deposit_f32(const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                               const ScState* sc, float* rho, int gx, int gy, int gz, cudaStream_t s)
{
    return deposit_tile<4, float>(parts, stride, masks, n, sc, rho, gx, gy, gz, s);
}

static inline int ceil_div64(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Dynamic shared memory of an FFT pass kernel (above 48 KB for L >= 512):
// raised once per kernel instantiation.
template <typename KERN>
static cudaError_t fft_smem(KERN* k, int bytes)
{
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

#define SB2_FFT_LENGTHS(X) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048)

// Every launcher below runs one bunch (list null, nitems 1) or, for a batch
// in lockstep, nitems bunches of the same grid shape whose pointers are in
// the device array `list` (the kernels take item blockIdx.z, or blockIdx.y
// for the field and the octant).
template <int L, int PLAN>
static cudaError_t green_passes_axis0(double* G, const double2* tw, int ox, int oy, int oz, const ScState* sc,
                                      const ConvItem* list, int nitems, cudaStream_t s)
{
    typedef fft::XMajor<L> LAY;
    const int bytes = LAY::kSmemElems * 16;
    static cudaError_t once = fft_smem(fft_green_kernel<L, 0, PLAN>, bytes);
    if (once) return once;
    const int64_t pairs = ((int64_t)oy * oz + 1) / 2;
    dim3 grid(ceil_div64(pairs, fft::Shape<L>::W), 1, nitems);
    fft_green_kernel<L, 0, PLAN><<<grid, fft::Shape<L>::THREADS, bytes, s>>>(G, tw, ox, oy, oz, sc, list);
    return cudaSuccess;
}
template <int L, int AXIS, int PLAN>
static cudaError_t green_passes_lmajor(double* G, const double2* tw, int ox, int oy, int oz, const ScState* sc,
                                       const ConvItem* list, int nitems, cudaStream_t s)
{
    typedef fft::LMajor<L> LAY;
    const int bytes = LAY::kSmemElems * 16;
    static cudaError_t once = fft_smem(fft_green_kernel<L, AXIS, PLAN>, bytes);
    if (once) return once;
    const int64_t nlines = AXIS == 1 ? (int64_t)ox * oz : (int64_t)ox * oy;
    dim3 grid(ceil_div64((nlines + 1) / 2, fft::Shape<L>::W), 1, nitems);
    fft_green_kernel<L, AXIS, PLAN><<<grid, fft::Shape<L>::THREADS, bytes, s>>>(G, tw, ox, oy, oz, sc, list);
    return cudaSuccess;
}

static cudaError_t green_t(const ScState* sc, double* G, const Dims& d, int linear, const double2* tw_x,
                           const double2* tw_y, const double2* tw_z, const ConvItem* list, int nitems, cudaStream_t s)
{
    const int ox = d.nx / 2 + 1, oy = d.ny / 2 + 1, oz = d.nz / 2 + 1;
    const int nb = list ? std::max(1, sm_count() * 4 / nitems) : sm_count() * 4;
    green_octant_kernel<<<dim3(nb, nitems), 256, 0, s>>>(sc, G, d.gx, d.gy, d.gz, linear, list);
    cudaError_t e = cudaSuccess;
#define SB2_G0(LL) case LL: e = d.plan ? green_passes_axis0<LL, fft::plan_of<LL>(1)>(G, tw_x, ox, oy, oz, sc, list, nitems, s) \
                                   : green_passes_axis0<LL, 0>(G, tw_x, ox, oy, oz, sc, list, nitems, s); break;
#define SB2_G1(LL) case LL: e = d.plan ? green_passes_lmajor<LL, 1, fft::plan_of<LL>(1)>(G, tw_y, ox, oy, oz, sc, list, nitems, s) \
                                   : green_passes_lmajor<LL, 1, 0>(G, tw_y, ox, oy, oz, sc, list, nitems, s); break;
#define SB2_G2(LL) case LL: e = d.plan ? green_passes_lmajor<LL, 2, fft::plan_of<LL>(1)>(G, tw_z, ox, oy, oz, sc, list, nitems, s) \
                                   : green_passes_lmajor<LL, 2, 0>(G, tw_z, ox, oy, oz, sc, list, nitems, s); break;
    switch (d.nx) { SB2_FFT_LENGTHS(SB2_G0) default: return cudaErrorInvalidValue; }
    if (e) return e;
    switch (d.ny) { SB2_FFT_LENGTHS(SB2_G1) default: return cudaErrorInvalidValue; }
    if (e) return e;
    switch (d.nz) { SB2_FFT_LENGTHS(SB2_G2) default: return cudaErrorInvalidValue; }
    if (e) return e;
#undef SB2_G0
#undef SB2_G1
#undef SB2_G2
    return cudaGetLastError();
}

// Ghat from the current domain: octant G, then the three even-line passes.
cudaError_t launch_green(const ScState* sc, double* G, const Dims& d, int linear, const double2* tw_x,
                         const double2* tw_y, const double2* tw_z, cudaStream_t s)
{
    return green_t(sc, G, d, linear, tw_x, tw_y, tw_z, nullptr, 1, s);
}

cudaError_t launch_green_list(const ConvItem* items, int nitems, const Dims& d, int linear, const double2* tw_x,
                              const double2* tw_y, const double2* tw_z, cudaStream_t s)
{
    return green_t(nullptr, nullptr, d, linear, tw_x, tw_y, tw_z, items, nitems, s);
}

template <int L, int PLAN, typename RI, typename C, typename W>
static cudaError_t pass_xf(const RI* rho, C* S, const W* tw, const Dims& d, const ScState* sc, const ConvItem* list,
                           int nitems, cudaStream_t s)
{
    const int bytes = fft::XMajor<L>::kSmemElems * (int)sizeof(W);
    static cudaError_t once = fft_smem(fft_xf_kernel<L, PLAN, RI, C, W>, bytes);
    if (once) return once;
    const int64_t nlines = (int64_t)((d.gy + 1) / 2) * d.gz;
    dim3 grid(ceil_div64(nlines, fft::Shape<L>::W), 1, nitems);
    fft_xf_kernel<L, PLAN, RI, C, W><<<grid, fft::Shape<L>::THREADS, bytes, s>>>(rho, S, tw, d, sc, list);
    return cudaSuccess;
}
template <int L, int PLAN, typename C, typename W, bool INV>
static cudaError_t pass_y(C* S, const W* tw, const Dims& d, const ScState* sc, const ConvItem* list, int nitems,
                          cudaStream_t s)
{
    const int bytes = fft::LMajor<L>::kSmemElems * (int)sizeof(W);
    static cudaError_t once = fft_smem(fft_y_kernel<L, PLAN, C, W, INV>, bytes);
    if (once) return once;
    dim3 grid(ceil_div64((int64_t)d.gz * d.nkxp, fft::Shape<L>::W), 1, nitems);
    fft_y_kernel<L, PLAN, C, W, INV><<<grid, fft::Shape<L>::THREADS, bytes, s>>>(S, tw, d, sc, list);
    return cudaSuccess;
}
template <int L, int PLAN, typename C, typename W>
static cudaError_t pass_z(C* S, const double* Ghat, const W* tw, const Dims& d, const ScState* sc, const ConvItem* list,
                          int nitems, cudaStream_t s)
{
    const int bytes = fft::LMajor<L>::kSmemElems * (int)sizeof(W);
    static cudaError_t once = fft_smem(fft_z_conv_kernel<L, PLAN, C, W>, bytes);
    if (once) return once;
    dim3 grid(ceil_div64((int64_t)d.ny * d.nkxp, fft::Shape<L>::W), 1, nitems);
    fft_z_conv_kernel<L, PLAN, C, W><<<grid, fft::Shape<L>::THREADS, bytes, s>>>(S, Ghat, tw, d, sc, list);
    return cudaSuccess;
}
template <int L, int PLAN, typename C, typename W>
static cudaError_t pass_xi(const C* S, typename CxT<C>::R* phi, const W* tw, const Dims& d, const ScState* sc,
                           const ConvItem* list, int nitems, cudaStream_t s)
{
    typedef typename CxT<C>::R RO;
    const int bytes = fft::XMajor<L>::kSmemElems * (int)sizeof(W);
    static cudaError_t once = fft_smem(fft_xi_kernel<L, PLAN, C, W, RO>, bytes);
    if (once) return once;
    const int64_t nlines = (int64_t)((d.gy + 1) / 2) * d.gz;
    dim3 grid(ceil_div64(nlines, fft::Shape<L>::W), 1, nitems);
    fft_xi_kernel<L, PLAN, C, W, RO><<<grid, fft::Shape<L>::THREADS, bytes, s>>>(S, phi, tw, d, sc, list);
    return cudaSuccess;
}

template <typename RI, typename C, typename W>
static cudaError_t convolve_t(const RI* rho, C* S, const double* Ghat, typename CxT<C>::R* phi, const Dims& d,
                              const W* tw_x, const W* tw_y, const W* tw_z, const ScState* sc, cudaStream_t s,
                              const ConvItem* list = nullptr, int nitems = 1)
{
    cudaError_t e = cudaSuccess;
#define SB2_XF(LL) case LL: e = d.plan ? pass_xf<LL, fft::plan_of<LL>(1), RI, C, W>(rho, S, tw_x, d, sc, list, nitems, s) \
                                   : pass_xf<LL, 0, RI, C, W>(rho, S, tw_x, d, sc, list, nitems, s); break;
#define SB2_YF(LL) case LL: e = d.plan ? pass_y<LL, fft::plan_of<LL>(1), C, W, false>(S, tw_y, d, sc, list, nitems, s) \
                                   : pass_y<LL, 0, C, W, false>(S, tw_y, d, sc, list, nitems, s); break;
#define SB2_ZC(LL) case LL: e = d.plan ? pass_z<LL, fft::plan_of<LL>(1), C, W>(S, Ghat, tw_z, d, sc, list, nitems, s) \
                                   : pass_z<LL, 0, C, W>(S, Ghat, tw_z, d, sc, list, nitems, s); break;
#define SB2_YI(LL) case LL: e = d.plan ? pass_y<LL, fft::plan_of<LL>(1), C, W, true>(S, tw_y, d, sc, list, nitems, s) \
                                   : pass_y<LL, 0, C, W, true>(S, tw_y, d, sc, list, nitems, s); break;
#define SB2_XI(LL) case LL: e = d.plan ? pass_xi<LL, fft::plan_of<LL>(1), C, W>(S, phi, tw_x, d, sc, list, nitems, s) \
                                   : pass_xi<LL, 0, C, W>(S, phi, tw_x, d, sc, list, nitems, s); break;
    switch (d.nx) { SB2_FFT_LENGTHS(SB2_XF) default: return cudaErrorInvalidValue; }
    if (e) return e;
    switch (d.ny) { SB2_FFT_LENGTHS(SB2_YF) default: return cudaErrorInvalidValue; }
    if (e) return e;
    switch (d.nz) { SB2_FFT_LENGTHS(SB2_ZC) default: return cudaErrorInvalidValue; }
    if (e) return e;
    switch (d.ny) { SB2_FFT_LENGTHS(SB2_YI) default: return cudaErrorInvalidValue; }
    if (e) return e;
    switch (d.nx) { SB2_FFT_LENGTHS(SB2_XI) default: return cudaErrorInvalidValue; }
    if (e) return e;
#undef SB2_XF
#undef SB2_YF
#undef SB2_ZC
#undef SB2_YI
#undef SB2_XI
    return cudaGetLastError();
}

// rho -> phi through the five line passes (FP64).
cudaError_t launch_convolve(const double* rho, double2* S, const double* Ghat, double* phi, const Dims& d,
                            const double2* tw_x, const double2* tw_y, const double2* tw_z, const ScState* sc,
                            cudaStream_t s)
{
    return convolve_t<double, double2, double2>(rho, S, Ghat, phi, d, tw_x, tw_y, tw_z, sc, s);
}

// Mixed precision: rho (FP32, or FP64 where the charge is exchanged between
// ranks) -> phi in FP32 with an FP32 spectrum; butterflies in FP32 (float2
// twiddles rounded from long double) or FP64 (double2 twiddles).
cudaError_t launch_convolve_mixed(const MixedConv& m, float2* S, const double* Ghat, float* phi, const Dims& d,
                                  const ScState* sc, cudaStream_t s)
{
    if (m.fp32_butterflies) {
        if (m.rho32)
            return convolve_t<float, float2, float2>(m.rho32, S, Ghat, phi, d, m.tw32[0], m.tw32[1], m.tw32[2], sc, s);
        return convolve_t<double, float2, float2>(m.rho64, S, Ghat, phi, d, m.tw32[0], m.tw32[1], m.tw32[2], sc, s);
    }
    if (m.rho32)
        return convolve_t<float, float2, double2>(m.rho32, S, Ghat, phi, d, m.tw64[0], m.tw64[1], m.tw64[2], sc, s);
    return convolve_t<double, float2, double2>(m.rho64, S, Ghat, phi, d, m.tw64[0], m.tw64[1], m.tw64[2], sc, s);
}

cudaError_t launch_convolve_list(int mode, const ConvItem* items, int nitems, const Dims& d, const double2* const* tw64,
                                 const float2* const* tw32, cudaStream_t s)
{
    switch (mode) {
    case 0:
        return convolve_t<double, double2, double2>(nullptr, nullptr, nullptr, nullptr, d, tw64[0], tw64[1], tw64[2],
                                                    nullptr, s, items, nitems);
    case 1: // FP32 charge, FP32 butterflies
        return convolve_t<float, float2, float2>(nullptr, nullptr, nullptr, nullptr, d, tw32[0], tw32[1], tw32[2],
                                                 nullptr, s, items, nitems);
    case 2: // FP64 charge, FP32 butterflies
        return convolve_t<double, float2, float2>(nullptr, nullptr, nullptr, nullptr, d, tw32[0], tw32[1], tw32[2],
                                                  nullptr, s, items, nitems);
    case 3: // FP32 charge, FP64 butterflies
        return convolve_t<float, float2, double2>(nullptr, nullptr, nullptr, nullptr, d, tw64[0], tw64[1], tw64[2],
                                                  nullptr, s, items, nitems);
    default: // FP64 charge, FP64 butterflies, FP32 spectrum
        return convolve_t<double, float2, double2>(nullptr, nullptr, nullptr, nullptr, d, tw64[0], tw64[1], tw64[2],
                                                   nullptr, s, items, nitems);
    }
}

cudaError_t launch_efield(const double* phi, double2* E, int gx, int gy, int gz, const ScState* sc, cudaStream_t s)
{
    int64_t total = (int64_t)gy * gz * 32; // one warp per x row
    int nb = (int)std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 16);
    efield_kernel<double, double2><<<nb, 256, 0, s>>>(phi, E, gx, gy, gz, sc, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_efield_f32(const float* phi, float4* E, int gx, int gy, int gz, const ScState* sc, cudaStream_t s)
{
    int64_t total = (int64_t)gy * gz * 32; // one warp per x row
    int nb = (int)std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 16);
    efield_kernel<float, float4><<<nb, 256, 0, s>>>(phi, E, gx, gy, gz, sc, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_efield_list(bool f32, const ConvItem* items, int nitems, int gx, int gy, int gz, cudaStream_t s)
{
    int64_t total = (int64_t)gy * gz * 32; // one warp per x row
    int nb = (int)std::min<int64_t>((total + 255) / 256, std::max<int64_t>(1, (int64_t)sm_count() * 16 / nitems));
    if (f32)
        efield_kernel<float, float4><<<dim3(nb, nitems), 256, 0, s>>>(nullptr, nullptr, gx, gy, gz, nullptr, items);
    else
        efield_kernel<double, double2><<<dim3(nb, nitems), 256, 0, s>>>(nullptr, nullptr, gx, gy, gz, nullptr, items);
    return cudaGetLastError();
}

} // namespace sb2
