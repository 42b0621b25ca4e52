// Kernel parameter blocks and launchers shared by the host runtime and the
// .cu translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

#include "../../include/sb2.h"

#include "sb2_ops.h"

namespace sb2 {

struct TrackParams {
    double* parts;
    int64_t stride;
    uint8_t* masks;
    uint8_t* discards;
    int64_t n;
    int32_t* ap_counts;         // discard counter per aperture slot
    double* moment_partials;    // [gridDim.x][6]
    const ScState* sc;          // space-charge state (kick)
    const double2* efield;      // (gz,gy,gx) cells x {ex,ey | ez,0}, FP64 path
    const float4* efield32;     // (gz,gy,gx) cells x {ex,ey,ez,0}, mixed path (used when set)
    int32_t gx, gy, gz;
    int32_t nops;
    int32_t write_discards;
    int32_t slot_base;          // aperture slots of this launch: slot_base + [0, kMaxOpsPerPass)
    int32_t fast_maps;          // 1: FMA-contracted maps of the mixed-precision path (track_fast.cu)
    double* loss_buf;           // lost-particle records [loss_cap][8] (null: off)
    int32_t* loss_count;        // records appended (device)
    int32_t loss_cap;
    MapOp ops[kMaxOpsPerPass];
};

struct DomainParams {
    BunchCounters* counters;
    int32_t* ap_counts;
    double* elem_charge; // per lattice element, may be null
    PassBook book;
    const double* moment_partials;
    int32_t n_partials;
    int32_t compute_domain; // 0: bookkeeping only
    ScState* sc;
    // options
    int32_t g[3], dg[3];
    int32_t domain_fixed, grid_entire_period, green_linear;
    double n_sigma, z_period, kick_scale;
    double fixed_size[3], fixed_offset[3];
    // bunch
    int32_t charge;
    double pref, gamma, beta;
    double time_step;
    // bunch split over ranks: [6 moment sums][discards per slot] summed over
    // the ranks (null for a whole bunch); counters then hold the local
    // n_valid and the global n_total / real_num
    const double* xchg;
    // per-step count records (PassBook::op_record), may be null.  With
    // rec_cursor the records go to step_records[*rec_cursor] (pinned host
    // memory written by the device; op_record only flags the operators that
    // end a step), and the cursor advances; up to rec_cap records.
    BunchCounters* step_records;
    int32_t* rec_cursor;
    int32_t rec_cap;
};

struct Dims {
    int gx, gy, gz;    // original grid
    int nx, ny, nz;    // doubled grid
    int nkx, nkxp;     // nx/2+1, padded row pitch of S
    int lx, ly, lz;    // log2 of nx, ny, nz
    int plan;          // FFT radix plan of the line passes (fft.cuh): 0 radix 8 first, 1 the remainder first
};

// Working copy of a bunch ordered by deposit cell (sort.cu), double-buffered.
struct SortBuffers {
    double* parts;
    uint8_t* masks;
    uint8_t* discards;
    int32_t* perm;   // original index of each working-copy particle
    double* parts2;
    uint8_t* masks2;
    uint8_t* discards2;
    int32_t* perm2;
    int64_t n, stride;
};

// One bunch of a counting sort over many bunches (sort.cu, batch in
// lockstep): its working copy, domain, grid and scratch (sort_scratch_ints).
struct SortItem {
    SortBuffers sb;
    const ScState* sc;
    int32_t* scratch;
    int gx, gy, gz;
};

// Launch shape of the particle passes: the autotuner's search space
// (host.cc, Propagator::autotune).
struct TrackTune {
    int32_t light_shape;  // light passes: 1 one particle per thread with the next tile prefetched,
                          // 2 two per thread with prefetch, 0 two per thread without, 3 one per
                          // thread with the next tile prefetched into shared memory (cp.async)
    int32_t full_occ;     // full passes: 2 (128 registers, TRACK_FULL_WIDE) or 3 CTAs/SM (80, TRACK_FULL)
    int32_t full_ppt;     // particles per thread of the 2-CTA full variant (1 or 2)
    int32_t quad_variant; // passes whose only integrator is the quadrupole run TRACK_QUAD with 1 (1) or
                          // 2 (2) particles per thread, or the full variant (0)
    int32_t ctas_per_sm;  // grid of the grid-stride particle passes, 1..12 CTAs per SM
};
// measured defaults, overridden by SB2_TRACK_LIGHT, SB2_TRACK_FULL_OCC,
// SB2_TRACK_FULL_PPT, SB2_TRACK_QUAD, SB2_TRACK_CTAS_PER_SM
TrackTune track_tune_defaults();
constexpr int kMaxCtasPerSm = 12;

// track.cu
int track_grid_blocks();                // grid at the default CTAs per SM
int track_grid_blocks(int ctas_per_sm); // SM count x ctas_per_sm
cudaError_t launch_track(const TrackParams& p, const TrackTune& t, cudaStream_t s);
// work lists (a batch in lockstep): the kernel a pass runs, the particles a
// block of it takes per iteration, and one launch of many bunches' passes
// with the same kernel (items in device memory, item i on blocks
// [first[i], first[i+1]) of nblocks; max_ops the largest op count of an
// item)
int track_pass_choice(const TrackParams& p, const TrackTune& t);
int track_pass_tile(int choice);
cudaError_t launch_track_list(int choice, bool fast_maps, const TrackParams* const* items, const int* first,
                              int nitems, int nblocks, int max_ops, cudaStream_t s);
cudaError_t launch_moments(const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                           const double* mean, double* partials, int nblocks, cudaStream_t s);
cudaError_t launch_populate(double* parts, int64_t stride, uint8_t* masks, int64_t n, const double* sig,
                            uint64_t seed, cudaStream_t s);
// Work-list items of the space-charge kernels (a batch in lockstep): one
// per bunch; the grid kernels' items share a grid shape.
struct ZeroItem {
    void* ptr;
    int64_t bytes; // a multiple of 8
};
struct DepositItem {
    const double* parts;
    int64_t stride;
    const uint8_t* masks;
    int64_t n;
    const ScState* sc;
    void* rho; // double, or float for the FP32 charge grid
};
struct ConvItem {
    const void* rho; // charge density (double or float)
    void* S;         // spectrum (double2 or float2)
    double* ghat;    // Green function octant
    void* phi;       // potential (double or float)
    void* E;         // field (double2 pairs or float4)
    const ScState* sc;
};

// sc3d.cu
cudaError_t launch_book_domain(const DomainParams& p, cudaStream_t s);
cudaError_t launch_book_domain_list(const DomainParams* items, int nitems, cudaStream_t s);
cudaError_t launch_zero_list(const ZeroItem* items, int nitems, cudaStream_t s);
// the deposit of many bunches: item i on blocks [first[i], first[i+1]),
// deposit_list_blocks(n) blocks for a bunch of n particles
int deposit_list_blocks(int64_t n);
cudaError_t launch_deposit_list(bool f32, const DepositItem* items, const int* first, int nitems, int nblocks, int gx,
                                int gy, int gz, cudaStream_t s);
// Green function, convolution (mode 0: FP64; 1..4: mixed with FP32 / FP64
// charge and FP32 / FP64 butterflies as MixedConv) and field of nitems
// bunches with the grid shape d
cudaError_t launch_green_list(const ConvItem* items, int nitems, const Dims& d, int linear, const double2* tw_x,
                              const double2* tw_y, const double2* tw_z, cudaStream_t s);
cudaError_t launch_convolve_list(int mode, const ConvItem* items, int nitems, const Dims& d, const double2* const* tw64,
                                 const float2* const* tw32, cudaStream_t s);
cudaError_t launch_efield_list(bool f32, const ConvItem* items, int nitems, int gx, int gy, int gz, cudaStream_t s);
// sharded bunch: moment sums and per-slot discards into xchg (to be summed
// over the ranks), and the global n_total from a summed local count
cudaError_t launch_shard_pack(const DomainParams& p, int nslots, double* xchg, cudaStream_t s);
cudaError_t launch_shard_count(const BunchCounters* c, double* xchg, cudaStream_t s);
cudaError_t launch_shard_total(BunchCounters* c, const double* xchg, cudaStream_t s);
cudaError_t launch_deposit(const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                           const ScState* sc, double* rho, int gx, int gy, int gz, cudaStream_t s);
// with an explicit chunk: 4 or 8 particles per thread of the tile deposit,
// 0 the warp-group deposit (FP64 grid only); the default chunk comes from
// SB2_DEPOSIT / SB2_DEPOSIT_K (4 unless set)
int deposit_default_chunk();
cudaError_t launch_deposit_k(int chunk, const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                             const ScState* sc, double* rho, int gx, int gy, int gz, cudaStream_t s);
cudaError_t launch_deposit_f32_k(int chunk, const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                                 const ScState* sc, float* rho, int gx, int gy, int gz, cudaStream_t s);
// the same deposit into an FP32 charge grid (the tiles' sums are exact; only
// the merge of neighbouring tiles rounds to FP32)
cudaError_t launch_deposit_f32(const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                               const ScState* sc, float* rho, int gx, int gy, int gz, cudaStream_t s);
cudaError_t launch_green(const ScState* sc, double* G, const Dims& d, int linear, const double2* tw_x,
                         const double2* tw_y, const double2* tw_z, cudaStream_t s);
cudaError_t launch_convolve(const double* rho, double2* S, const double* Ghat, double* phi, const Dims& d,
                            const double2* tw_x, const double2* tw_y, const double2* tw_z, const ScState* sc,
                            cudaStream_t s);
cudaError_t launch_efield(const double* phi, double2* E, int gx, int gy, int gz, const ScState* sc, cudaStream_t s);
// inputs of the mixed-precision convolution: the charge density in FP32
// (rho32) or FP64 (rho64, the other null), the twiddles of the x, y, z
// lengths in both precisions, and the butterflies' precision
struct MixedConv {
    const float* rho32;
    const double* rho64;
    const double2* tw64[3];
    const float2* tw32[3];
    int32_t fp32_butterflies;
};
cudaError_t launch_convolve_mixed(const MixedConv& m, float2* S, const double* Ghat, float* phi, const Dims& d,
                                  const ScState* sc, cudaStream_t s);
cudaError_t launch_efield_f32(const float* phi, float4* E, int gx, int gy, int gz, const ScState* sc, cudaStream_t s);
// sort.cu
size_t sort_scratch_ints(int64_t G);
void sort_list_plan(const SortItem* items, int nitems, int* first, int* nblocks);
cudaError_t launch_cell_sort_list(const SortItem* items, const int* first, int nitems, const int* nblocks,
                                  int max_m, cudaStream_t s);
cudaError_t launch_cell_sort(const SortBuffers& sb, int32_t* scratch, const ScState* sc, int gx, int gy, int gz,
                             cudaStream_t s);
// the inverse permutation into perm2, then one array at a time back in the
// caller's order (pipelined check-out)
cudaError_t launch_sort_invert(const SortBuffers& sb, cudaStream_t s);
cudaError_t launch_sort_scatter_out_col(const SortBuffers& sb, int col, double* out, cudaStream_t s);
cudaError_t launch_sort_scatter_out_bytes(const uint8_t* w, const SortBuffers& sb, uint8_t* out, cudaStream_t s);
cudaError_t launch_sort_gather_perm(const double* ups, int64_t ustride, const uint8_t* um, const uint8_t* ud,
                                    const SortBuffers& sb, cudaStream_t s);
cudaError_t launch_sort_gather_in(const double* ups, int64_t ustride, const uint8_t* um, const uint8_t* ud,
                                  const SortBuffers& sb, cudaStream_t s);
cudaError_t launch_sort_scatter_out(const SortBuffers& sb, double* ups, int64_t ustride, uint8_t* um, uint8_t* ud,
                                    cudaStream_t s);
// diag.cu: per-turn bunch diagnostics appended to a device record array
constexpr int kDiagRecord = 97;
cudaError_t launch_count_valid(const uint8_t* masks, int64_t n, BunchCounters* c, cudaStream_t s);
// blocks x 256 threads, each 8 x iters dependent-free FP64 FMAs; out holds
// blocks x 256 doubles
cudaError_t launch_fp64_probe(double* out, int blocks, int iters, cudaStream_t s);
cudaError_t launch_diagnostics(const double* parts, int64_t stride, const uint8_t* masks, int64_t n,
                               const BunchCounters* counters, double* partials, int nb, double* tmp, double* records,
                               int32_t* count, int capacity, cudaStream_t s);
// host.cc
int check_sc_options(const sb2_sc3d_options& o, std::string* msg);
int ref_kinematics(int charge, double mass, double value, int kind, double* gamma, double* beta, double* p,
                   std::string* msg);
void set_last_error(const std::string& m);

} // namespace sb2
