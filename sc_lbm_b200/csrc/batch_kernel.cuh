// batch_kernel.cuh -- the batched persistent kernel: one launch walks a tile
// list drawn from many domains, each tile running the fused single-pass body
// (fused2_tile).  Instantiated per storage type in the translation unit whose
// floating-point contraction rules that type needs (FP64 in ops_fp64.cu,
// compiled with -fmad=false; FP32/FP16 in step_shifted.cu).
#pragma once
#include "fused_step.cuh"

namespace sclbm {

constexpr int BATCH_TX = 128;

struct TileRef {
    int dom, xb, yb, pad;
};

// doms holds two argument blocks per domain (buffer parity 0 and 1)
template <typename S, typename T>
__global__ void __launch_bounds__(BATCH_TX)
    k_batch2(const Fused2Args<S, T> *__restrict__ doms, const TileRef *__restrict__ tiles,
             int ntiles, int parity)
{
    __shared__ T s_rho[2][4][BATCH_TX];
    __shared__ uint8_t s_m[4][BATCH_TX];
    for (int i = blockIdx.x; i < ntiles; i += gridDim.x) {
        const TileRef tr = tiles[i];
        const Fused2Args<S, T> a = doms[2 * tr.dom + parity];
        fused2_tile<S, T, BATCH_TX, false, KF_FORCE | KF_SOLID>(a, tr.xb, tr.yb, s_rho, s_m);
        __syncthreads(); // the shared ring is reused by the next tile
    }
}

template <typename S, typename T>
inline cudaError_t launch_batch_t(const Fused2Args<S, T> *doms, const TileRef *tiles, int ntiles,
                                  int parity, int grid, cudaStream_t s)
{
    k_batch2<S, T><<<grid, BATCH_TX, 0, s>>>(doms, tiles, ntiles, parity);
    return cudaGetLastError();
}

template <typename S, typename T> inline int batch_blocks_per_sm_t()
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch2<S, T>, BATCH_TX, 0) != cudaSuccess)
        return 1;
    return n;
}

cudaError_t launch_batch_fp64(const Fused2Args<double, double> *doms, const TileRef *tiles,
                              int ntiles, int parity, int grid, cudaStream_t s);
cudaError_t launch_batch_f32(const Fused2Args<float, float> *doms, const TileRef *tiles,
                             int ntiles, int parity, int grid, cudaStream_t s);
cudaError_t launch_batch_f16(const Fused2Args<__half, float> *doms, const TileRef *tiles,
                             int ntiles, int parity, int grid, cudaStream_t s);
int batch_blocks_per_sm(sclbm_precision p);

} // namespace sclbm
