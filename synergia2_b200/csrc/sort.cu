// Cell-ordered working copy of a bunch for the space-charge step.
//
// Unsorted particles make the CIC deposit one FP64 atomic per particle and
// corner (L2 atomic bound) and make the kick's field gathers touch a
// different cache line per thread (L1 wavefront bound).  During a propagate
// call the particles therefore live in a working copy ordered by the cell of
// their deposit stencil, rebuilt before each deposit by a counting sort:
//   key       cell (iz*gy + iy)*gx + ix of the stencil's lower corner;
//             G for live particles outside the grid, G+1 for lost ones
//   histogram warp-aggregated atomics on key counts
//   scan      exclusive prefix sum of the counts (three small kernels)
//   scatter   every column, the mask, the discard flag and the original
//             index move to offset[key] + rank, a tile at a time through
//             shared memory (runs of equal keys leave as coalesced stores)
// The caller's arrays are untouched while the bunch lives in the working
// copy; they are brought back up to date (the working copy scattered back to
// the original order) when the caller next reads or writes them.  The order within a cell
// depends on atomic arrival order; every per-particle result is independent
// of it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "sb2_kernels.h"

namespace sb2 {

__device__ __forceinline__ int cell_key(double x, double y, double z, const ScState& sc, int gx, int gy, int gz)
{ // collective/utils.h:9-18
    double sx = (x - sc.left[0]) * sc.ih[0] - 0.5;
    double sy = (y - sc.left[1]) * sc.ih[1] - 0.5;
    double sz = (z - sc.left[2]) * sc.ih[2] - 0.5;
    int ix = (int)floor(sx), iy = (int)floor(sy), iz = (int)floor(sz);
    const int G = gx * gy * gz;
    if (ix < 0 || ix >= gx || iy < 0 || iy >= gy || iz < 0 || iz >= gz) return G;
    return (iz * gy + iy) * gx + ix;
}

// block vb of vg blocks of one bunch's histogram; a warp takes 64
// consecutive particles per iteration, both loads of a lane in flight
__device__ __forceinline__ void sort_hist_body(const double* __restrict__ parts, int64_t stride,
                                               const uint8_t* __restrict__ masks, int64_t n,
                                               const ScState* __restrict__ scp, int gx, int gy, int gz,
                                               int32_t* counts, int vb, int vg)
{
    const ScState& sc = *scp;
    const int G = gx * gy * gz;
    const int lane = threadIdx.x & 31;
    const int64_t wstride = (int64_t)vg * blockDim.x * 2;
    for (int64_t wb = (vb * (int64_t)blockDim.x + threadIdx.x - lane) * 2; wb < n; wb += wstride) {
        double x[2], y[2], z[2];
        int m[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int64_t i = wb + u * 32 + lane;
            m[u] = -1;
            if (i < n) {
                m[u] = masks[i];
                x[u] = parts[i];
                y[u] = parts[i + 2 * stride];
                z[u] = parts[i + 4 * stride];
            }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            int key = -1;
            if (m[u] >= 0) key = (!m[u] || !sc.valid) ? G + 1 : cell_key(x[u], y[u], z[u], sc, gx, gy, gz);
            const unsigned grp = __match_any_sync(0xffffffffu, key);
            if (key >= 0 && lane == __ffs(grp) - 1) atomicAdd(&counts[key], __popc(grp));
        }
    }
}

__global__ void __launch_bounds__(256, 6) sort_hist_kernel(const double* __restrict__ parts, int64_t stride,
                                                        const uint8_t* __restrict__ masks, int64_t n,
                                                        const ScState* __restrict__ scp, int gx, int gy, int gz,
                                                        int32_t* counts)
{
    sort_hist_body(parts, stride, masks, n, scp, gx, gy, gz, counts, blockIdx.x, gridDim.x);
}

// exclusive scan: per-block (1024 values), then block sums, then add
constexpr int kScanBlock = 1024;

__device__ __forceinline__ void scan_block_body(const int32_t* __restrict__ in, int32_t* out, int n,
                                                int32_t* block_sums, int blk)
{
    __shared__ int32_t s[kScanBlock];
    __shared__ int32_t warp_tot[8];
    const int base = blk * kScanBlock;
    for (int k = threadIdx.x; k < kScanBlock; k += blockDim.x) s[k] = (base + k < n) ? in[base + k] : 0;
    __syncthreads();
    // each thread owns 4 consecutive values
    const int t = threadIdx.x;
    int32_t v0 = s[4 * t], v1 = s[4 * t + 1], v2 = s[4 * t + 2], v3 = s[4 * t + 3];
    int32_t tot = v0 + v1 + v2 + v3;
    const int lane = t & 31, w = t >> 5;
    int32_t inc = tot;
    for (int o = 1; o < 32; o <<= 1) {
        int32_t u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) warp_tot[w] = inc;
    __syncthreads();
    int32_t woff = 0;
    for (int k = 0; k < w; ++k) woff += warp_tot[k];
    int32_t ex = woff + inc - tot;
    s[4 * t] = ex;
    s[4 * t + 1] = ex + v0;
    s[4 * t + 2] = ex + v0 + v1;
    s[4 * t + 3] = ex + v0 + v1 + v2;
    __syncthreads();
    for (int k = threadIdx.x; k < kScanBlock; k += blockDim.x)
        if (base + k < n) out[base + k] = s[k];
    if (threadIdx.x == blockDim.x - 1) {
        int32_t all = 0;
        for (int k = 0; k < 8; ++k) all += warp_tot[k];
        block_sums[blk] = all;
    }
}

__global__ void __launch_bounds__(256) scan_block_kernel(const int32_t* __restrict__ in, int32_t* out, int n,
                                                         int32_t* block_sums)
{
    scan_block_body(in, out, n, block_sums, blockIdx.x);
}

__device__ __forceinline__ void scan_sums_body(int32_t* sums, int nb)
{
    // single block: sequential per-thread chunks, then a block scan of the
    // chunk totals
    __shared__ int32_t tot[1024];
    const int per = (nb + 1023) / 1024;
    const int b = threadIdx.x * per;
    int32_t acc = 0;
    for (int k = 0; k < per && b + k < nb; ++k) acc += sums[b + k];
    tot[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        int32_t u = (threadIdx.x >= (unsigned)o) ? tot[threadIdx.x - o] : 0;
        __syncthreads();
        tot[threadIdx.x] += u;
        __syncthreads();
    }
    int32_t run = tot[threadIdx.x] - acc; // exclusive
    for (int k = 0; k < per && b + k < nb; ++k) {
        int32_t v = sums[b + k];
        sums[b + k] = run;
        run += v;
    }
}

__global__ void __launch_bounds__(1024) scan_sums_kernel(int32_t* sums, int nb) { scan_sums_body(sums, nb); }

__global__ void scan_add_kernel(int32_t* out, int n, const int32_t* __restrict__ sums)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += sums[i / kScanBlock];
}

// Scatter through a CTA-local grouping.  A CTA takes tiles of kTile
// consecutive particles; the tile's keys go into a shared-memory hash table
// (key -> count, each particle's rank inside its key), each distinct key of
// the tile reserves its run of destinations with one global atomic, and the
// tile is then moved array by array through shared memory so that a warp's
// stores cover whole runs of consecutive destinations (a nearly ordered
// bunch keeps most of a tile's particles in a few cells) instead of one
// scattered 8-byte store per lane.  The lanes of a warp with the same key
// make one table insertion.
constexpr int kTileThreads = 256;
constexpr int kTile = 1024;
constexpr int kTable = 2048; // hash slots (power of two)
constexpr int kEmpty = -2;

// open addressing with linear probing; returns the slot, and the first of
// `count` consecutive ranks inside its key (arrival order of the shared
// atomics)
__device__ __forceinline__ int table_insert_n(int* t_key, int* t_cnt, int key, int count, int& rank)
{
    const unsigned h = (unsigned)key * 2654435761u; // multiplicative hashing (Knuth)
    int e = (int)(h >> 21) & (kTable - 1);
    for (int probe = 0; probe < kTable; ++probe) {
        const int old = atomicCAS(&t_key[e], kEmpty, key);
        if (old == kEmpty || old == key) {
            rank = atomicAdd(&t_cnt[e], count);
            return e;
        }
        e = (e + 1) & (kTable - 1);
    }
    rank = 0;
    return -1; // unreachable: the table has more slots than a tile has keys
}

// The tile's arrays come into shared memory by asynchronous 16-byte copies
// (cp.async), each while the previous one is stored (two buffers); the
// first array's copy is in flight during the grouping.  After its
// reservation a table slot's key is replaced by the run's first
// destination.  The copies of the last tile are rounded up to 16 bytes: the
// working copy's arrays hold a multiple of 32 particles.
__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}

// block vb of vg blocks of one bunch's scatter.  cursor holds the exclusive
// scan of the key counts; each distinct key of a tile reserves its run of
// destinations by advancing cursor[key] atomically.
__device__ __forceinline__ void sort_scatter_piped_body(
    const double* __restrict__ src, const uint8_t* __restrict__ m_src, const uint8_t* __restrict__ d_src,
    const int32_t* __restrict__ p_src, double* dst, uint8_t* m_dst, uint8_t* d_dst, int32_t* p_dst, int64_t n,
    int64_t stride, const ScState* __restrict__ scp, int gx, int gy, int gz, int32_t* cursor, int vb, int vg)
{
    __shared__ int t_key[kTable]; // key; after the reservation, the run's first destination
    __shared__ int t_cnt[kTable];
    __shared__ int t_off[kTable]; // local exclusive offsets
    __shared__ short s_src[kTile];
    __shared__ int s_dst[kTile];
    __shared__ __align__(16) double s_buf[2][kTile];
    __shared__ int s_wsum[kTileThreads / 32];
    const ScState& sc = *scp;
    const int G = gx * gy * gz;
    constexpr int PPT = kTile / kTileThreads;
    // copies of array a of the tile at `base` (tn particles; the lengths
    // rounded up to 16 bytes: the arrays hold a multiple of 32 particles)
    auto issue = [&](int a, int64_t base, int tn) {
        unsigned char* b = (unsigned char*)s_buf[a & 1];
        if (a < 7) {
            const double* c = src + a * stride + base;
            for (int k = threadIdx.x; k < (tn + 1) / 2; k += kTileThreads) cp_async16(b + 16 * k, c + 2 * k);
        } else if (a < 9) {
            const uint8_t* c = (a == 7 ? m_src : d_src) + base;
            for (int k = threadIdx.x; k < (tn + 15) / 16; k += kTileThreads) cp_async16(b + 16 * k, c + 16 * k);
        } else {
            const int32_t* c = p_src + base;
            for (int k = threadIdx.x; k < (tn + 3) / 4; k += kTileThreads) cp_async16(b + 16 * k, c + 4 * k);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    for (int e = threadIdx.x; e < kTable; e += kTileThreads) {
        t_key[e] = kEmpty;
        t_cnt[e] = 0;
    }
    __syncthreads();
    for (int64_t base = (int64_t)vb * kTile; base < n; base += (int64_t)vg * kTile) {
        const int tn = (int)min((int64_t)kTile, n - base);
        issue(0, base, tn);
        int ent[PPT], rnk[PPT];
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
            const int l = q * kTileThreads + threadIdx.x;
            ent[q] = -1;
            int key = -1;
            if (l < tn) {
                const int64_t i = base + l;
                key = (!m_src[i] || !sc.valid) ? G + 1
                                               : cell_key(src[i], src[i + 2 * stride], src[i + 4 * stride], sc, gx, gy, gz);
            }
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            const int lead = __ffs(peers) - 1;
            unsigned below;
            asm("mov.u32 %0, %%lanemask_lt;" : "=r"(below));
            int e = -1, r0 = 0;
            if (key >= 0 && (int)(threadIdx.x & 31) == lead) e = table_insert_n(t_key, t_cnt, key, __popc(peers), r0);
            e = __shfl_sync(0xffffffffu, e, lead);
            r0 = __shfl_sync(0xffffffffu, r0, lead);
            if (key >= 0) {
                ent[q] = e;
                rnk[q] = r0 + __popc(peers & below);
            }
        }
        __syncthreads();
        constexpr int EPT = kTable / kTileThreads;
        int c[EPT], tot = 0;
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            c[k] = t_cnt[threadIdx.x * EPT + k];
            tot += c[k];
        }
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        int inc = tot;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        if (lane == 31) s_wsum[w] = inc;
        // one global reservation per distinct key, a thread's atomics all in flight
        int g[EPT];
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const int e = threadIdx.x * EPT + k;
            g[k] = c[k] ? atomicAdd(&cursor[t_key[e]], c[k]) : 0;
        }
        __syncthreads();
        int run = inc - tot;
        for (int k = 0; k < w; ++k) run += s_wsum[k];
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const int e = threadIdx.x * EPT + k;
            t_off[e] = run;
            if (c[k]) t_key[e] = g[k];
            run += c[k];
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
            if (ent[q] < 0) continue;
            const int slot = t_off[ent[q]] + rnk[q];
            s_src[slot] = (short)(q * kTileThreads + threadIdx.x);
            s_dst[slot] = t_key[ent[q]] + rnk[q];
        }
        // array by array, the next one's copies in flight during the stores
        for (int a = 0; a < 10; ++a) {
            if (a + 1 < 10) {
                issue(a + 1, base, tn);
                asm volatile("cp.async.wait_group 1;" ::: "memory");
            } else {
                asm volatile("cp.async.wait_group 0;" ::: "memory");
            }
            __syncthreads();
            const unsigned char* b = (const unsigned char*)s_buf[a & 1];
            for (int j = threadIdx.x; j < tn; j += kTileThreads) {
                const int l = s_src[j];
                const int64_t d = s_dst[j];
                if (a < 7)
                    dst[d + a * stride] = ((const double*)b)[l];
                else if (a == 7)
                    m_dst[d] = b[l];
                else if (a == 8)
                    d_dst[d] = b[l];
                else
                    p_dst[d] = ((const int32_t*)b)[l];
            }
            __syncthreads();
        }
        for (int e = threadIdx.x; e < kTable; e += kTileThreads) {
            t_key[e] = kEmpty;
            t_cnt[e] = 0;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kTileThreads) sort_scatter_piped_kernel(
    const double* __restrict__ src, const uint8_t* __restrict__ m_src, const uint8_t* __restrict__ d_src,
    const int32_t* __restrict__ p_src, double* dst, uint8_t* m_dst, uint8_t* d_dst, int32_t* p_dst, int64_t n,
    int64_t stride, const ScState* __restrict__ scp, int gx, int gy, int gz, int32_t* cursor)
{
    sort_scatter_piped_body(src, m_src, d_src, p_src, dst, m_dst, d_dst, p_dst, n, stride, scp, gx, gy, gz, cursor,
                            blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// The counting sort of many bunches at once (a batch in lockstep): every
// kernel of the sort takes a list of SortItem, and the blocks of one launch
// are split among the items in proportion to their work (item i owns blocks
// [first[i], first[i+1]) of each kernel).
// ---------------------------------------------------------------------------
struct SortView {
    int G, m, nb;
    int32_t *counts, *offsets, *bsums;
};
__host__ __device__ __forceinline__ SortView sort_view(const SortItem& it)
{
    SortView v;
    v.G = it.gx * it.gy * it.gz;
    v.m = v.G + 2;
    v.nb = (v.m + kScanBlock - 1) / kScanBlock;
    v.counts = it.scratch;
    v.offsets = v.counts + v.m;
    v.bsums = v.offsets + v.m;
    return v;
}

__device__ __forceinline__ int sort_item_of(const int* __restrict__ first, int nitems)
{
    int lo = 0, hi = nitems;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (first[mid] <= (int)blockIdx.x)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// grid (x, nitems): item blockIdx.y clears its counts
__global__ void sort_zero_list_kernel(const SortItem* __restrict__ items)
{
    const SortView v = sort_view(items[blockIdx.y]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < v.m; i += gridDim.x * blockDim.x) v.counts[i] = 0;
}

__global__ void __launch_bounds__(256, 6) sort_hist_list_kernel(const SortItem* __restrict__ items,
                                                             const int* __restrict__ first, int nitems)
{
    const int k = sort_item_of(first, nitems);
    const SortItem& it = items[k];
    sort_hist_body(it.sb.parts, it.sb.stride, it.sb.masks, it.sb.n, it.sc, it.gx, it.gy, it.gz, sort_view(it).counts,
                   (int)blockIdx.x - first[k], first[k + 1] - first[k]);
}

__global__ void __launch_bounds__(256) scan_block_list_kernel(const SortItem* __restrict__ items,
                                                              const int* __restrict__ first, int nitems)
{
    const int k = sort_item_of(first, nitems);
    const SortView v = sort_view(items[k]);
    scan_block_body(v.counts, v.offsets, v.m, v.bsums, (int)blockIdx.x - first[k]);
}

// one block per item
__global__ void __launch_bounds__(1024) scan_sums_list_kernel(const SortItem* __restrict__ items)
{
    const SortView v = sort_view(items[blockIdx.x]);
    scan_sums_body(v.bsums, v.nb);
}

__global__ void scan_add_list_kernel(const SortItem* __restrict__ items, const int* __restrict__ first, int nitems)
{
    const int k = sort_item_of(first, nitems);
    const SortView v = sort_view(items[k]);
    const int i = ((int)blockIdx.x - first[k]) * blockDim.x + threadIdx.x;
    if (i < v.m) v.offsets[i] += v.bsums[i / kScanBlock];
}

__global__ void __launch_bounds__(kTileThreads, 4) sort_scatter_list_kernel(const SortItem* __restrict__ items,
                                                                        const int* __restrict__ first, int nitems)
{
    const int k = sort_item_of(first, nitems);
    const SortItem& it = items[k];
    const SortView v = sort_view(it);
    const SortBuffers& sb = it.sb;
    sort_scatter_piped_body(sb.parts, sb.masks, sb.discards, sb.perm, sb.parts2, sb.masks2, sb.discards2, sb.perm2,
                            sb.n, sb.stride, it.sc, it.gx, it.gy, it.gz, v.offsets,
                            (int)blockIdx.x - first[k], first[k + 1] - first[k]);
}

// the block partitions of the list launches: first holds 4 arrays of
// nitems + 1 entries (histogram, block scan, scan add, scatter)
void sort_list_plan(const SortItem* items, int nitems, int* first, int* nblocks)
{
    const int stride = nitems + 1;
    for (int a = 0; a < 4; ++a) first[a * stride] = 0;
    for (int i = 0; i < nitems; ++i) {
        const SortView v = sort_view(items[i]);
        const int64_t n = items[i].sb.n;
        const int64_t tiles = (n + kTile - 1) / kTile;
        const int b[4] = {(int)std::max<int64_t>(1, (n + 4095) / 4096), v.nb, (v.m + 255) / 256,
                          (int)std::max<int64_t>(1, (tiles + 1) / 2)};
        for (int a = 0; a < 4; ++a) first[a * stride + i + 1] = first[a * stride + i] + b[a];
    }
    for (int a = 0; a < 4; ++a) nblocks[a] = first[a * stride + nitems];
}

cudaError_t launch_cell_sort_list(const SortItem* items, const int* first, int nitems, const int* nblocks,
                                  int max_m, cudaStream_t s)
{
    const int stride = nitems + 1;
    const int zb = std::max(1, std::min(64, (max_m + 255) / 256));
    sort_zero_list_kernel<<<dim3(zb, nitems), 256, 0, s>>>(items);
    sort_hist_list_kernel<<<nblocks[0], 256, 0, s>>>(items, first, nitems);
    scan_block_list_kernel<<<nblocks[1], 256, 0, s>>>(items, first + stride, nitems);
    scan_sums_list_kernel<<<nitems, 1024, 0, s>>>(items);
    scan_add_list_kernel<<<nblocks[2], 256, 0, s>>>(items, first + 2 * stride, nitems);
    sort_scatter_list_kernel<<<nblocks[3], kTileThreads, 0, s>>>(items, first + 3 * stride, nitems);
    return cudaGetLastError();
}

// working copy <- caller arrays (identity order)
__global__ void sort_gather_in_kernel(const double* __restrict__ ups, int64_t ustride, const uint8_t* __restrict__ um,
                                      const uint8_t* __restrict__ ud, double* w, uint8_t* wm, uint8_t* wd, int32_t* wp,
                                      int64_t n, int64_t wstride)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        for (int j = 0; j < 7; ++j) w[i + j * wstride] = ups[i + j * ustride];
        wm[i] = um[i];
        wd[i] = ud ? ud[i] : 0;
        wp[i] = (int32_t)i;
    }
}

// working copy <- caller arrays in the order of the working copy the bunch
// last left (perm: slot -> caller index, kept): nearly cell-ordered for the
// last domain, so the first sort after it is a cheap re-sort
__global__ void sort_gather_perm_kernel(const double* __restrict__ ups, int64_t ustride,
                                        const uint8_t* __restrict__ um, const uint8_t* __restrict__ ud, double* w,
                                        uint8_t* wm, uint8_t* wd, const int32_t* __restrict__ wp, int64_t n,
                                        int64_t wstride)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = wp[j];
        for (int c = 0; c < 7; ++c) w[j + c * wstride] = ups[i + c * ustride];
        wm[j] = um[i];
        wd[j] = ud ? ud[i] : 0;
    }
}

// caller arrays <- working copy, back in the original order: invert the
// permutation (4-byte scattered writes), then gather so that the wide
// writes to the caller's columns are coalesced
__global__ void sort_invert_kernel(const int32_t* __restrict__ wp, int32_t* inv, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        inv[wp[i]] = (int32_t)i;
}

__global__ void sort_scatter_out_kernel(const double* __restrict__ w, const uint8_t* __restrict__ wm,
                                        const uint8_t* __restrict__ wd, const int32_t* __restrict__ inv, double* ups,
                                        int64_t ustride, uint8_t* um, uint8_t* ud, int64_t n, int64_t wstride)
{
    for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < n; o += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = inv[o];
        for (int j = 0; j < 7; ++j) ups[o + j * ustride] = w[i + j * wstride];
        um[o] = wm[i];
        if (ud) ud[o] = wd[i];
    }
}

static int sm_count_s()
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

size_t sort_scratch_ints(int64_t G)
{ // counts, offsets (advanced in place by the scatter's reservations), block sums
    const int64_t m = G + 2;
    return (size_t)(2 * m + (m + kScanBlock - 1) / kScanBlock + 8);
}

cudaError_t launch_cell_sort(const SortBuffers& sb, int32_t* scratch, const ScState* sc, int gx, int gy, int gz,
                             cudaStream_t s)
{
    const int64_t G = (int64_t)gx * gy * gz;
    const int m = (int)(G + 2);
    int32_t* counts = scratch;
    int32_t* offsets = counts + m;
    int32_t* bsums = offsets + m;
    const int nb = (m + kScanBlock - 1) / kScanBlock;
    cudaError_t e;
    if ((e = cudaMemsetAsync(counts, 0, sizeof(int32_t) * m, s))) return e;
    const int grid = sm_count_s() * 8;
    sort_hist_kernel<<<sm_count_s() * 6, 256, 0, s>>>(sb.parts, sb.stride, sb.masks, sb.n, sc, gx, gy, gz, counts);
    scan_block_kernel<<<nb, 256, 0, s>>>(counts, offsets, m, bsums);
    scan_sums_kernel<<<1, 1024, 0, s>>>(bsums, nb);
    scan_add_kernel<<<(m + 255) / 256, 256, 0, s>>>(offsets, m, bsums);
    // each distinct key of a tile reserves its run by advancing offsets[key]
    sort_scatter_piped_kernel<<<grid, kTileThreads, 0, s>>>(sb.parts, sb.masks, sb.discards, sb.perm, sb.parts2,
                                                            sb.masks2, sb.discards2, sb.perm2, sb.n, sb.stride, sc, gx,
                                                            gy, gz, offsets);
    return cudaGetLastError();
}

cudaError_t launch_sort_gather_perm(const double* ups, int64_t ustride, const uint8_t* um, const uint8_t* ud,
                                    const SortBuffers& sb, cudaStream_t s)
{
    sort_gather_perm_kernel<<<sm_count_s() * 8, 256, 0, s>>>(ups, ustride, um, ud, sb.parts, sb.masks, sb.discards,
                                                               sb.perm, sb.n, sb.stride);
    return cudaGetLastError();
}

cudaError_t launch_sort_gather_in(const double* ups, int64_t ustride, const uint8_t* um, const uint8_t* ud,
                                  const SortBuffers& sb, cudaStream_t s)
{
    sort_gather_in_kernel<<<sm_count_s() * 8, 256, 0, s>>>(ups, ustride, um, ud, sb.parts, sb.masks, sb.discards,
                                                             sb.perm, sb.n, sb.stride);
    return cudaGetLastError();
}

// one array back in the caller's order: out[o] = w[inv[o]]
template <typename T>
__global__ void sort_scatter_out_col_kernel(const T* __restrict__ w, const int32_t* __restrict__ inv, T* out, int64_t n)
{
    for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < n; o += (int64_t)gridDim.x * blockDim.x)
        out[o] = w[inv[o]];
}

cudaError_t launch_sort_invert(const SortBuffers& sb, cudaStream_t s)
{
    sort_invert_kernel<<<sm_count_s() * 8, 256, 0, s>>>(sb.perm, sb.perm2, sb.n);
    return cudaGetLastError();
}

cudaError_t launch_sort_scatter_out_col(const SortBuffers& sb, int col, double* out, cudaStream_t s)
{
    sort_scatter_out_col_kernel<double><<<sm_count_s() * 8, 256, 0, s>>>(sb.parts + col * sb.stride, sb.perm2, out,
                                                                          sb.n);
    return cudaGetLastError();
}

cudaError_t launch_sort_scatter_out_bytes(const uint8_t* w, const SortBuffers& sb, uint8_t* out, cudaStream_t s)
{
    sort_scatter_out_col_kernel<uint8_t><<<sm_count_s() * 8, 256, 0, s>>>(w, sb.perm2, out, sb.n);
    return cudaGetLastError();
}

cudaError_t launch_sort_scatter_out(const SortBuffers& sb, double* ups, int64_t ustride, uint8_t* um, uint8_t* ud,
                                    cudaStream_t s)
{
    // perm2 is free outside a sort: it holds the inverse permutation here
    sort_invert_kernel<<<sm_count_s() * 8, 256, 0, s>>>(sb.perm, sb.perm2, sb.n);
    sort_scatter_out_kernel<<<sm_count_s() * 8, 256, 0, s>>>(sb.parts, sb.masks, sb.discards, sb.perm2, ups, ustride,
                                                               um, ud, sb.n, sb.stride);
    return cudaGetLastError();
}

} // namespace sb2
