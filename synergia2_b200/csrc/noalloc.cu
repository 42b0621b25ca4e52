// sb2_sc3d_apply_noalloc: the space-charge kick of sb2_sc3d_apply with every
// workspace taken from one fixed, file-scope device array instead of device
// allocations.
//
// Who needs it: hosts that own every byte of device memory themselves (a
// simulation framework with its own pool, an embedded or real-time caller
// with a fixed budget) and must not have a library call cudaMalloc or
// cudaFree behind their back -- those calls synchronise the device, fail
// inside some allocator regimes, and make the footprint unpredictable.  Such
// a caller passes its own particle arrays and gets the kick done in place;
// the grids, spectra and field live in `g_sc_scratch` below, which every GPU
// that loads this library holds for the life of the process.
//
// Limits and rules:
//   * grids up to kNoAllocMaxCells = 65,536 cells (gx*gy*gz, e.g. 32x32x64)
//     with every doubled dimension <= 128; larger grids are rejected with
//     SB2_ERR_INVALID and a message naming the limit;
//   * the first call on a device resolves the array's device address with
//     cudaGetSymbolAddress while that device is current -- make that first
//     call before any stream capture;
//   * all calls share the one array and it keeps the last call's contents;
//     everything that must start at zero is cleared on each call, and calls
//     whose work overlaps on the GPU (different streams or host threads
//     without ordering) race on it.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "sb2_kernels.h"

namespace sb2 {
namespace {

constexpr int64_t kNoAllocMaxCells = 65536;
constexpr int kNoAllocMaxDoubled = 128;
constexpr int kNoAllocMaxPartials = 2048; // particle-pass CTAs (moment partials)
constexpr size_t kNoAllocBytes = (size_t)12 << 20; // 12 MiB

__device__ __align__(256) unsigned char g_sc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
// device address of g_sc_scratch per device, looked up on the first call on
// that device (atomic: host threads may make their first calls at once)
std::atomic<void*> g_scratch_ptr[kMaxDevices];

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

struct Layout {
    size_t state, counters, ap_counts, partials, tw_x, tw_y, tw_z, rho, phi, E, ghat, S, total;
};

Layout layout_for(const Dims& d)
{
    Layout L{};
    size_t o = 0;
    auto take = [&](size_t bytes) {
        size_t at = o;
        o = align256(o + bytes);
        return at;
    };
    const size_t cells = (size_t)d.gx * d.gy * d.gz;
    L.state = take(sizeof(ScState));
    L.counters = take(sizeof(BunchCounters));
    L.ap_counts = take(sizeof(int32_t) * kMaxSlotsPerPass);
    L.partials = take(sizeof(double) * 6 * kNoAllocMaxPartials);
    L.tw_x = take(sizeof(double2) * d.nx);
    L.tw_y = take(sizeof(double2) * d.ny);
    L.tw_z = take(sizeof(double2) * d.nz);
    L.rho = take(sizeof(double) * cells);
    L.phi = take(sizeof(double) * cells);
    L.E = take(sizeof(double2) * 2 * cells);
    L.ghat = take(sizeof(double) * (size_t)(d.nx / 2 + 1) * (d.ny / 2 + 1) * (d.nz / 2 + 1));
    L.S = take(sizeof(double2) * (size_t)d.nz * d.ny * d.nkxp);
    L.total = o;
    return L;
}

int ilog2i(int v)
{
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}

void fill_twiddles(double2* h, int L)
{ // exp(-2 pi i k / L), k < L
    for (int k = 0; k < L; ++k) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * k / L;
        h[k] = make_double2((double)std::cos(a), (double)std::sin(a));
    }
}

int fail(int code, const std::string& m)
{
    set_last_error(m);
    return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
    cudaGetLastError();
    return fail(SB2_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

} // namespace
} // namespace sb2

using namespace sb2;

extern "C" sb2_status sb2_sc3d_apply_noalloc(const sb2_sc3d_options* opts, double* parts, int64_t stride,
                                             const uint8_t* masks, int64_t n, int32_t n_total, double real_num,
                                             int32_t charge, double mass, double value, int32_t kind,
                                             double time_step, void* stream)
{
    if (!opts || (n > 0 && (!parts || !masks)) || n < 0 || stride < n)
        return fail(SB2_ERR_INVALID, "sb2_sc3d_apply_noalloc: bad particle arguments");
    std::string msg;
    int rc = check_sc_options(*opts, &msg);
    if (rc != SB2_OK) return fail(rc, msg);
    const sb2_sc3d_options& o = *opts;
    if (o.precision != SB2_PRECISION_FP64)
        return fail(SB2_ERR_UNSUPPORTED, "sb2_sc3d_apply_noalloc: only the FP64 path runs without allocation");
    Dims d{};
    d.gx = o.shape[0];
    d.gy = o.shape[1];
    d.gz = o.shape[2];
    d.nx = o.doubled_shape[0];
    d.ny = o.doubled_shape[1];
    d.nz = o.doubled_shape[2];
    d.nkx = d.nx / 2 + 1;
    d.nkxp = (d.nkx + 1) & ~1;
    d.lx = ilog2i(d.nx);
    d.ly = ilog2i(d.ny);
    d.lz = ilog2i(d.nz);
    if ((int64_t)d.gx * d.gy * d.gz > kNoAllocMaxCells || d.nx > kNoAllocMaxDoubled || d.ny > kNoAllocMaxDoubled ||
        d.nz > kNoAllocMaxDoubled)
        return fail(SB2_ERR_INVALID, "sb2_sc3d_apply_noalloc: grid exceeds the fixed workspace (at most 65536 cells "
                                     "and doubled dimensions <= 128)");
    Layout lay = layout_for(d);
    // Guard only: with at most 65,536 cells and doubled dimensions <= 128 the
    // layout stays below 8 MiB (the spectrum, 2gz * 2gy * (gx+2) complex
    // values, is the largest part at about 4.3 MiB), so no accepted grid
    // reaches this check.
    if (lay.total > kNoAllocBytes)
        return fail(SB2_ERR_INVALID, "sb2_sc3d_apply_noalloc: grid exceeds the 12 MiB fixed workspace");
    // one launch shape for both particle passes, so the moment partials the
    // first pass writes are the ones the domain kernel reduces
    const TrackTune tune = track_tune_defaults();
    const int nblocks = track_grid_blocks(tune.ctas_per_sm);
    if (nblocks > kNoAllocMaxPartials)
        return fail(SB2_ERR_UNSUPPORTED, "sb2_sc3d_apply_noalloc: device has more SMs than the workspace allows");
    double gamma, beta, pref;
    rc = ref_kinematics(charge, mass, value, kind, &gamma, &beta, &pref, &msg);
    if (rc != SB2_OK) return fail(rc, msg);

    // per-device address of the static workspace (set-up on first use)
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return fail(SB2_ERR_UNSUPPORTED, "sb2_sc3d_apply_noalloc: device ordinal");
    void* sym = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (!sym) {
        e = cudaGetSymbolAddress(&sym, g_sc_scratch);
        if (e) return cuda_fail(e, "cudaGetSymbolAddress");
        g_scratch_ptr[dev].store(sym, std::memory_order_release); // every thread finds the same address
    }
    unsigned char* base = (unsigned char*)sym;
    cudaStream_t s = (cudaStream_t)stream;
    ScState* state = (ScState*)(base + lay.state);
    BunchCounters* counters = (BunchCounters*)(base + lay.counters);
    int32_t* ap_counts = (int32_t*)(base + lay.ap_counts);
    double* partials = (double*)(base + lay.partials);
    double2* tw_x = (double2*)(base + lay.tw_x);
    double2* tw_y = (double2*)(base + lay.tw_y);
    double2* tw_z = (double2*)(base + lay.tw_z);
    double* rho = (double*)(base + lay.rho);
    double* phi = (double*)(base + lay.phi);
    double2* E = (double2*)(base + lay.E);
    double* ghat = (double*)(base + lay.ghat);
    double2* S = (double2*)(base + lay.S);
    const size_t cells = (size_t)d.gx * d.gy * d.gz;

    // inputs staged from the host stack (pageable copies are staged before
    // cudaMemcpyAsync returns)
    double2 tw[3][kNoAllocMaxDoubled];
    fill_twiddles(tw[0], d.nx);
    fill_twiddles(tw[1], d.ny);
    fill_twiddles(tw[2], d.nz);
    BunchCounters c{};
    c.n_valid = n_total;
    c.n_total = n_total;
    c.real_num = real_num;
    if ((e = cudaMemcpyAsync(tw_x, tw[0], sizeof(double2) * d.nx, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(tw_y, tw[1], sizeof(double2) * d.ny, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(tw_z, tw[2], sizeof(double2) * d.nz, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(counters, &c, sizeof(c), cudaMemcpyHostToDevice, s)))
        return cuda_fail(e, "workspace upload");
    // state left by the previous call is cleared
    if ((e = cudaMemsetAsync(state, 0, sizeof(ScState), s)) ||
        (e = cudaMemsetAsync(ap_counts, 0, sizeof(int32_t) * kMaxSlotsPerPass, s)) ||
        (e = cudaMemsetAsync(partials, 0, sizeof(double) * 6 * kNoAllocMaxPartials, s)) ||
        (e = cudaMemsetAsync(E, 0, sizeof(double2) * 2 * cells, s)))
        return cuda_fail(e, "workspace clear");

    TrackParams tp; // ~25 KB on the caller's stack; nothing is allocated
    std::memset(&tp, 0, sizeof(tp));
    tp.parts = parts;
    tp.stride = stride;
    tp.masks = const_cast<uint8_t*>(masks);
    tp.discards = nullptr;
    tp.n = n;
    tp.ap_counts = ap_counts;
    tp.moment_partials = partials;
    tp.sc = state;
    tp.efield = E;
    tp.gx = d.gx;
    tp.gy = d.gy;
    tp.gz = d.gz;
    tp.nops = 1;
    tp.ops[0].kind = OP_MOMENTS;
    if (!o.domain_fixed && (e = launch_track(tp, tune, s))) return cuda_fail(e, "moments pass");

    DomainParams dp;
    std::memset(&dp, 0, sizeof(dp));
    dp.counters = counters;
    dp.ap_counts = ap_counts;
    dp.moment_partials = partials;
    dp.n_partials = nblocks;
    dp.compute_domain = 1;
    dp.sc = state;
    for (int i = 0; i < 3; ++i) {
        dp.g[i] = o.shape[i];
        dp.dg[i] = o.doubled_shape[i];
        dp.fixed_size[i] = o.size[i];
        dp.fixed_offset[i] = o.offset[i];
    }
    dp.domain_fixed = o.domain_fixed;
    dp.grid_entire_period = o.grid_entire_period;
    dp.green_linear = o.green_fn == SB2_GREEN_LINEAR;
    dp.n_sigma = o.n_sigma;
    dp.z_period = o.z_period;
    dp.kick_scale = o.kick_scale;
    dp.charge = charge;
    dp.pref = pref;
    dp.gamma = gamma;
    dp.beta = beta;
    dp.time_step = time_step;
    if ((e = launch_book_domain(dp, s))) return cuda_fail(e, "domain");
    if ((e = cudaMemsetAsync(rho, 0, sizeof(double) * cells, s))) return cuda_fail(e, "rho clear");
    if ((e = launch_deposit(parts, stride, masks, n, state, rho, d.gx, d.gy, d.gz, s))) return cuda_fail(e, "deposit");
    if ((e = launch_green(state, ghat, d, o.green_fn == SB2_GREEN_LINEAR, tw_x, tw_y, tw_z, s)))
        return cuda_fail(e, "green");
    if ((e = launch_convolve(rho, S, ghat, phi, d, tw_x, tw_y, tw_z, state, s))) return cuda_fail(e, "convolve");
    if ((e = launch_efield(phi, E, d.gx, d.gy, d.gz, state, s))) return cuda_fail(e, "efield");
    tp.ops[0].kind = OP_SC_KICK;
    tp.ops[0].d[0] = pref; // reference momentum and mass of the kick
    tp.ops[0].d[1] = mass;
    if ((e = launch_track(tp, tune, s))) return cuda_fail(e, "kick pass");

    ScState st;
    if ((e = cudaMemcpyAsync(&st, state, sizeof(st), cudaMemcpyDeviceToHost, s)) || (e = cudaStreamSynchronize(s)))
        return cuda_fail(e, "sync");
    if (st.error == 1)
        return fail(SB2_ERR_RUNTIME, "Space_charge_3d_open_hockney_eigen::update_domain: all three spatial "
                                     "dimensions have neglible extent");
    return SB2_OK;
}
