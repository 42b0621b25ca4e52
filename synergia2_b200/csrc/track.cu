// Exact FP64 particle passes (the drop-in), moments, population, launchers.
// The pass kernels themselves are in track_impl.cuh.
#define SB2_FAST_MAPS 0
#define SB2_TRACK_NS exact
#include "track_impl.cuh"

namespace sb2 {

cudaError_t launch_track_fast(const TrackParams& p, const TrackTune& t, cudaStream_t s); // track_fast.cu
cudaError_t launch_track_list_fast(int choice, const TrackParams* const* items, const int* first, int nitems, int nblocks,
                                   int max_ops, cudaStream_t s);

// Masked sums for diagnostics: mean (6) or central second moments (21 lower
// triangle) per block, core_diagnostics.cc:105-111,174-186.
__global__ void __launch_bounds__(256) moments_kernel(const double* parts, int64_t stride,
                                                      const uint8_t* masks, int64_t n,
                                                      const double* mean, double* partials)
{
    __shared__ double s_red[8][28];
    double acc[27];
    for (int j = 0; j < 27; ++j) acc[j] = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (!masks[i]) continue;
        double v[6];
        for (int j = 0; j < 6; ++j) v[j] = parts[i + j * stride];
        for (int j = 0; j < 6; ++j) acc[j] += v[j];
        if (mean) {
            int t = 6;
            for (int j = 0; j < 6; ++j) {
                double dj = v[j] - mean[j];
                for (int k = 0; k <= j; ++k) acc[t++] += dj * (v[k] - mean[k]);
            }
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int j = 0; j < 27; ++j) {
        double v = acc[j];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) s_red[w][j] = v;
    }
    __syncthreads();
    if (threadIdx.x < 27) {
        double v = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v += s_red[k][threadIdx.x];
        partials[blockIdx.x * 27 + threadIdx.x] = v;
    }
}

// Counter-based normal generator: Philox-4x32-10 (Salmon et al., SC'11)
// keyed by the seed, counter = (particle, column pair); Box-Muller.
__device__ __forceinline__ void philox4x32(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
        uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

__global__ void populate_kernel(double* parts, int64_t stride, uint8_t* masks, int64_t n,
                                double s0, double s1, double s2, double s3, double s4, double s5,
                                uint64_t seed)
{
    const double sig[6] = {s0, s1, s2, s3, s4, s5};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        for (int pr = 0; pr < 3; ++pr) {
            uint32_t c[4] = {(uint32_t)i, (uint32_t)(i >> 32), (uint32_t)pr, 0x5b200u};
            philox4x32(c, (uint32_t)seed, (uint32_t)(seed >> 32));
            uint64_t a = ((uint64_t)c[0] << 32) | c[1];
            uint64_t b = ((uint64_t)c[2] << 32) | c[3];
            double u1 = ((a >> 11) + 0.5) * (1.0 / 9007199254740992.0);
            double u2 = ((b >> 11) + 0.5) * (1.0 / 9007199254740992.0);
            double r = sqrt(-2.0 * log(u1));
            double sn, cs;
            sincospi(2.0 * u2, &sn, &cs);
            parts[i + (2 * pr) * stride] = sig[2 * pr] * r * cs;
            parts[i + (2 * pr + 1) * stride] = sig[2 * pr + 1] * r * sn;
        }
        parts[i + 6 * stride] = (double)i;
        masks[i] = 1;
    }
}

// ---------------------------------------------------------------------------
// launchers (called from host.cc)
// ---------------------------------------------------------------------------
static int sm_count_cached()
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    return sms;
}

TrackTune track_tune_defaults()
{
    TrackTune t;
    t.light_shape = 3;
    t.full_occ = 2;
    t.full_ppt = 1;
    t.quad_variant = 1;
    t.ctas_per_sm = 8;
    const char* e = getenv("SB2_TRACK_LIGHT");
    if (e && e[0] == '2' && e[1] == 'p') t.light_shape = 2;
    if (e && e[0] == '2' && e[1] == 0) t.light_shape = 0;
    if (e && e[0] == '1') t.light_shape = 1;
    e = getenv("SB2_TRACK_FULL_OCC");
    if (e && atoi(e) == 3) t.full_occ = 3;
    e = getenv("SB2_TRACK_FULL_PPT");
    if (e && atoi(e) == 2) t.full_ppt = 2;
    e = getenv("SB2_TRACK_QUAD");
    if (e && e[0] == '0') t.quad_variant = 0;
    e = getenv("SB2_TRACK_CTAS_PER_SM");
    if (e && atoi(e) >= 1 && atoi(e) <= kMaxCtasPerSm) t.ctas_per_sm = atoi(e);
    return t;
}

int track_grid_blocks(int ctas_per_sm)
{
    return sm_count_cached() * std::max(1, std::min(ctas_per_sm, kMaxCtasPerSm));
}

int track_grid_blocks()
{
    static int per = track_tune_defaults().ctas_per_sm;
    return track_grid_blocks(per);
}

cudaError_t launch_track(const TrackParams& p, const TrackTune& t, cudaStream_t s)
{
    return p.fast_maps ? launch_track_fast(p, t, s) : exact::launch_pass(p, t, s);
}

int track_pass_choice(const TrackParams& p, const TrackTune& t) { return exact::pass_choice(p, t); }

int track_pass_tile(int choice)
{ // particles a block takes per iteration
    return exact::kTrackThreads * ((choice == 2 || choice == 3 || choice == 5 || choice == 7) ? 2 : 1);
}

cudaError_t launch_track_list(int choice, bool fast_maps, const TrackParams* const* items, const int* first, int nitems,
                              int nblocks, int max_ops, cudaStream_t s)
{
    return fast_maps ? launch_track_list_fast(choice, items, first, nitems, nblocks, max_ops, s)
                     : exact::launch_pass_list(choice, items, first, nitems, nblocks, max_ops, s);
}

cudaError_t launch_moments(const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                           const double* mean, double* partials, int nblocks, cudaStream_t s)
{
    moments_kernel<<<nblocks, 256, 0, s>>>(parts, stride, masks, n, mean, partials);
    return cudaGetLastError();
}

cudaError_t launch_populate(double* parts, int64_t stride, uint8_t* masks, int64_t n, const double* sig,
                            uint64_t seed, cudaStream_t s)
{
    int nb = track_grid_blocks();
    populate_kernel<<<nb, 256, 0, s>>>(parts, stride, masks, n, sig[0], sig[1], sig[2], sig[3], sig[4],
                                       sig[5], seed);
    return cudaGetLastError();
}

} // namespace sb2
