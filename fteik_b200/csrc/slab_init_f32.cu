/*
 * slab_init_f32.cu -- the initialisation sweeps of the FP32 3D solve.
 * Compiled without multiply-add contraction: the near-source spherical
 * stencil runs in FP64 and rounds as the FP64 CPU algorithm does; the FP32
 * plane-wave stencil of these sweeps (noinit_v, or noinit_f32 in the staged
 * walk) rounds every operation once by itself, so it is the same either
 * way.
 */
#include "row3d_impl.cuh"

namespace fk3rw {
int launch_init_f32(const fk3tw::Params &P, int zring, cudaStream_t st, int blocks_per_sm, const int *pairs,
                    bool staged)
{
    if (pairs) return launch_slab_kernel<float, true, false, 2>(P, pairs, zring, st, 0, blocks_per_sm);
    if (staged) return launch_slab_kernel<float, true, false, 1, true>(P, nullptr, zring, st, 0, blocks_per_sm);
    return launch_slab_kernel<float, true, false, 1>(P, nullptr, zring, st, 0, blocks_per_sm);
}
} // namespace fk3rw
