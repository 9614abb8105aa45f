// step_shifted.cu -- FP32 instantiations of the fused step for the shifted
// storage forms: populations stored as d_i = f_i - w_i*rho_ref in float
// (SCLBM_FP32_SHIFTED) or half (SCLBM_FP16_SHIFTED), arithmetic in float.
// Compiled with the default contraction rules (FMA allowed).
#include "fused_step.cuh"

namespace sclbm {

cudaError_t launch_fused2_f32(const Fused2Args<float, float> &a, int variant, int tx,
                              cudaStream_t s)
{
    return launch_fused2_any<float, float>(a, variant, tx, s);
}
cudaError_t launch_fused2_f16(const Fused2Args<__half, float> &a, int variant, int tx,
                              cudaStream_t s)
{
    return launch_fused2_any<__half, float>(a, variant, tx, s);
}
cudaError_t launch_fused1_f32(const Fused1Args<float, float> &a, cudaStream_t s)
{
    k_fused1<float, float><<<grid_for(a.N, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_fused1_f16(const Fused1Args<__half, float> &a, cudaStream_t s)
{
    k_fused1<__half, float><<<grid_for(a.N, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_density_f32(const uint8_t *mask, const float *f0, const float *f1, float *r0,
                               float *r1, size_t N, cudaStream_t s)
{
    k_density2<float, float><<<grid_for(N, 256), 256, 0, s>>>(mask, f0, f1, r0, r1, N);
    return cudaGetLastError();
}
cudaError_t launch_density_f16(const uint8_t *mask, const __half *f0, const __half *f1,
                               float *r0, float *r1, size_t N, cudaStream_t s)
{
    k_density2<__half, float><<<grid_for(N, 256), 256, 0, s>>>(mask, f0, f1, r0, r1, N);
    return cudaGetLastError();
}

} // namespace sclbm

#include "batch_kernel.cuh"
namespace sclbm {
cudaError_t launch_batch_f32(const Fused2Args<float, float> *doms, const TileRef *tiles,
                             int ntiles, int parity, int grid, int flags, int body, cudaStream_t s)
{
    if (body == BODY_AHEAD)
        return launch_batch_t<float, float, true>(doms, tiles, ntiles, parity, grid, flags, s);
    if (body == BODY_COMPACT)
        return launch_batch_t<float, float, false, true>(doms, tiles, ntiles, parity, grid, flags, s);
    if (body == BODY_UNIFORM)
        return launch_batch_t<float, float, false, false, KF_UNIFORM>(doms, tiles, ntiles, parity, grid,
                                                                 flags, s);
    if (body == BODY_HALF)
        return launch_batch_half_t<float, float>(doms, tiles, ntiles, parity, grid, flags, s);
    if (body == BODY_WARP)
        return launch_batch_warp_t<float, float>(doms, tiles, ntiles, parity, grid, flags, s);
    return launch_batch_t<float, float>(doms, tiles, ntiles, parity, grid, flags, s);
}
cudaError_t launch_batch_f16(const Fused2Args<__half, float> *doms, const TileRef *tiles,
                             int ntiles, int parity, int grid, int flags, int body, cudaStream_t s)
{
    if (body == BODY_AHEAD)
        return launch_batch_t<__half, float, true>(doms, tiles, ntiles, parity, grid, flags, s);
    if (body == BODY_COMPACT)
        return launch_batch_t<__half, float, false, true>(doms, tiles, ntiles, parity, grid, flags, s);
    if (body == BODY_UNIFORM)
        return launch_batch_t<__half, float, false, false, KF_UNIFORM>(doms, tiles, ntiles, parity, grid,
                                                                 flags, s);
    if (body == BODY_HALF)
        return launch_batch_half_t<__half, float>(doms, tiles, ntiles, parity, grid, flags, s);
    if (body == BODY_WARP)
        return launch_batch_warp_t<__half, float>(doms, tiles, ntiles, parity, grid, flags, s);
    return launch_batch_t<__half, float>(doms, tiles, ntiles, parity, grid, flags, s);
}
int batch_blocks_per_sm_fp64();
int batch_blocks_per_sm(sclbm_precision p, int body)
{
    switch (p) {
    case SCLBM_FP64: return batch_blocks_per_sm_fp64();
    case SCLBM_FP32_SHIFTED:
        return body == BODY_AHEAD     ? batch_blocks_per_sm_t<float, float, true>()
               : body == BODY_COMPACT ? batch_blocks_per_sm_t<float, float, false, true>()
               : body == BODY_UNIFORM ? batch_blocks_per_sm_t<float, float, false, false, KF_UNIFORM>()
               : body == BODY_HALF    ? batch_half_blocks_per_sm_t<float, float>()
               : body == BODY_WARP    ? batch_warp_blocks_per_sm_t<float, float>()
                                      : batch_blocks_per_sm_t<float, float>();
    default:
        return body == BODY_AHEAD     ? batch_blocks_per_sm_t<__half, float, true>()
               : body == BODY_COMPACT ? batch_blocks_per_sm_t<__half, float, false, true>()
               : body == BODY_UNIFORM ? batch_blocks_per_sm_t<__half, float, false, false, KF_UNIFORM>()
               : body == BODY_HALF    ? batch_half_blocks_per_sm_t<__half, float>()
               : body == BODY_WARP    ? batch_warp_blocks_per_sm_t<__half, float>()
                                      : batch_blocks_per_sm_t<__half, float>();
    }
}
} // namespace sclbm

#include "fused_ring.cuh"
namespace sclbm {
// FP32: 10.8 KB per stage with halo boxes (9.8 KB without); FP16: 6.3 KB
// (5.3 KB).  Without halo boxes four FP32 stages leave room for five CTAs per
// SM instead of four.
cudaError_t launch_ring2_f32(const Fused2Args<float, float> &a, int stages, int rows, cudaStream_t s,
                             bool edge)
{
    if (edge) return launch_ring2_any<float, float, 4, KF_UNIFORM, false>(a, rows, s);
    if (stages < 0) return launch_ring2_any<float, float, 2>(a, rows, s);
    if (stages > 0) return launch_ring2_any<float, float, 4>(a, rows, s);
    return launch_ring2_any<float, float, 3>(a, rows, s);
}
cudaError_t launch_ring2_f16(const Fused2Args<__half, float> &a, int stages, int rows, cudaStream_t s,
                             bool edge)
{
    // FP16 keeps its halo boxes: its registers set its residency, and its
    // 2-byte elements are below the smallest asynchronous element copy
    if (edge) return launch_ring2_any<__half, float, 4>(a, rows, s);
    if (stages < 0) return launch_ring2_any<__half, float, 4>(a, rows, s);
    if (stages > 0) return launch_ring2_any<__half, float, 6>(a, rows, s);
    return launch_ring2_any<__half, float, 5>(a, rows, s);
}
// batches: the single-domain depths, uniform solid form; strips 128 or 64
// columns wide
constexpr int RING_BATCH_R32 = 3, RING_BATCH_R16 = 5;
cudaError_t launch_batch_ring_f32(const Fused2Args<float, float> *doms, const RingMaps *maps,
                                  const RingUnit *units, int nunits, int parity, int grid, int flags,
                                  unsigned *counters, int width, cudaStream_t s)
{
    if (width == 64)
        return launch_batch_ring<float, float, RING_BATCH_R32, KF_UNIFORM, 64>(doms, maps, units, nunits,
                                                                               parity, grid, flags, counters, s);
    return launch_batch_ring<float, float, RING_BATCH_R32, KF_UNIFORM, 128>(doms, maps, units, nunits,
                                                                            parity, grid, flags, counters, s);
}
cudaError_t launch_batch_ring_f16(const Fused2Args<__half, float> *doms, const RingMaps *maps,
                                  const RingUnit *units, int nunits, int parity, int grid, int flags,
                                  unsigned *counters, int width, cudaStream_t s)
{
    if (width == 64)
        return launch_batch_ring<__half, float, RING_BATCH_R16, KF_UNIFORM, 64>(doms, maps, units, nunits,
                                                                                parity, grid, flags, counters, s);
    return launch_batch_ring<__half, float, RING_BATCH_R16, KF_UNIFORM, 128>(doms, maps, units, nunits,
                                                                             parity, grid, flags, counters, s);
}
int batch_ring_prepare_shifted(sclbm_precision p, int width, int *per_sm)
{
    cudaError_t e;
    if (p == SCLBM_FP32_SHIFTED)
        e = width == 64 ? batch_ring_prepare<float, float, RING_BATCH_R32, KF_UNIFORM, 64>(per_sm)
                        : batch_ring_prepare<float, float, RING_BATCH_R32, KF_UNIFORM, 128>(per_sm);
    else
        e = width == 64 ? batch_ring_prepare<__half, float, RING_BATCH_R16, KF_UNIFORM, 64>(per_sm)
                        : batch_ring_prepare<__half, float, RING_BATCH_R16, KF_UNIFORM, 128>(per_sm);
    return e == cudaSuccess ? 0 : cuda_fail(e, "ring batch set-up");
}
int ring_maps_of(const Fused2Args<float, float> &a, int width, RingMaps *m)
{
    const cudaError_t e = width == 64 ? ring_maps<float, float, RING_BATCH_R32, 64>(a, *m)
                                      : ring_maps<float, float, RING_BATCH_R32, 128>(a, *m);
    return e == cudaSuccess ? 0 : 1;
}
int ring_maps_of(const Fused2Args<__half, float> &a, int width, RingMaps *m)
{
    const cudaError_t e = width == 64 ? ring_maps<__half, float, RING_BATCH_R16, 64>(a, *m)
                                      : ring_maps<__half, float, RING_BATCH_R16, 128>(a, *m);
    return e == cudaSuccess ? 0 : 1;
}
} // namespace sclbm

#include "fused_async.cuh"
namespace sclbm {
cudaError_t launch_fused2_async_f32(const Fused2Args<float, float> &a, cudaStream_t s, bool uniform)
{
    if (uniform) return launch_fused2_async_t<float, float, 128, 4, KF_UNIFORM>(a, s);
    return launch_fused2_async_t<float, float, 128, 4>(a, s);
}
cudaError_t launch_batch2_async_f32(const Fused2Args<float, float> *doms, const BandTile *tiles,
                                    int ntiles, int grid, int parity, cudaStream_t s)
{
    return launch_batch2_async_t<float, float, 128, 4>(doms, tiles, ntiles, grid, parity, s);
}
int async_resident_f32() { return async_resident_ctas<float, float, 128, 4>(); }
} // namespace sclbm
