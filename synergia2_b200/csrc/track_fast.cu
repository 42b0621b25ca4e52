// FP64 particle passes with fused multiply-adds and the folded drift
// (mixed-precision path); see track_impl.cuh.
#define SB2_FAST_MAPS 1
#define SB2_TRACK_NS fast
#include "track_impl.cuh"

namespace sb2 {

cudaError_t launch_track_fast(const TrackParams& p, const TrackTune& t, cudaStream_t s)
{
    return fast::launch_pass(p, t, s);
}

cudaError_t launch_track_list_fast(int choice, const TrackParams* const* items, const int* first, int nitems, int nblocks,
                                   int max_ops, cudaStream_t s)
{
    return fast::launch_pass_list(choice, items, first, nitems, nblocks, max_ops, s);
}

} // namespace sb2
