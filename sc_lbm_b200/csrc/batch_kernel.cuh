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

// doms holds two argument blocks per domain (buffer parity 0 and 1).  The
// block of the current tile's domain is copied into shared memory, so the tile
// body reads its fields from there instead of holding the whole block in
// registers.
// Five resident CTAs per SM (102 registers): the tile loop and the shared
// argument block leave the six-CTA cap of the single-domain kernel spilling,
// and on the 512-domain ensemble the five-CTA form ran 13 % faster.  FP64:
// three CTAs per SM (168 registers, no spills; uncapped it took 174 and ran
// two).
template <typename S, typename T, int FLAGS = KF_FORCE | KF_SOLID, bool AHEAD = false,
          bool COMPACT = false>
__global__ void __launch_bounds__(BATCH_TX, (sizeof(T) == 8 ? 3 : 5))
    k_batch2(const Fused2Args<S, T> *__restrict__ doms, const TileRef *__restrict__ tiles,
             int ntiles, int parity)
{
    __shared__ V2<T> s_rho[4][BATCH_TX];
    __shared__ uint8_t s_m[4][BATCH_TX];
    __shared__ __align__(16) Fused2Args<S, T> sa;
    static_assert(sizeof(Fused2Args<S, T>) % 4 == 0, "argument block copied as words");
    int loaded = -1;
    for (int i = blockIdx.x; i < ntiles; i += gridDim.x) {
        const TileRef tr = tiles[i];
        const int key = 2 * tr.dom + parity;
        if (key != loaded) { // uniform over the CTA
            const uint32_t *src = reinterpret_cast<const uint32_t *>(doms + key);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&sa);
            for (int w = threadIdx.x; w < (int)(sizeof(sa) / 4); w += BATCH_TX) dst[w] = src[w];
            __syncthreads();
            loaded = key;
        }
        // alternate march directions of a domain's row bands (see fused2_tile)
        const bool down = ((tr.yb / sa.tile_y) & 1) != 0;
        if constexpr (COMPACT && (FLAGS & KF_SOLID) != 0) {
            __shared__ CompactSmem<S, T, BATCH_TX> cs;
            fused2_tile_compact<S, T, BATCH_TX, FLAGS>(sa, tr.xb, tr.yb, s_rho, s_m, cs, down);
        } else {
            fused2_tile<S, T, BATCH_TX, false, FLAGS, false, AHEAD>(sa, tr.xb, tr.yb, s_rho, s_m,
                                                                    down);
        }
        __syncthreads(); // the shared ring and block are reused by the next tile
    }
}

// Two 64-column tiles side by side in each 128-thread CTA: threads 0-63 run
// tiles 2c, 2c + 2g, ... and threads 64-127 tiles 2c + 1, 2c + 1 + 2g, ... of
// the 64-column tile list (g = gridDim.x), each half with its own density
// ring, argument block and named barrier, so the halves never wait on each
// other.  Narrow domains leave fewer idle lanes than with 128-column tiles
// (the ensemble's widths 64..512: 88 % of the lanes busy against 81 %).
constexpr int HALF_TX = BATCH_TX / 2;
// the tile loop of half h (named barrier 1 + h)
template <typename S, typename T, int FLAGS, int BAR>
__device__ __forceinline__ void batch_half_loop(const Fused2Args<S, T> *__restrict__ doms,
                                                const TileRef *__restrict__ tiles, int ntiles,
                                                int parity, V2<T> (&s_rho)[4][HALF_TX],
                                                uint8_t (&s_m)[4][HALF_TX], Fused2Args<S, T> &sa)
{
    const int lt = threadIdx.x % HALF_TX;
    int loaded = -1;
    for (int i = 2 * blockIdx.x + (BAR - 1); i < ntiles; i += 2 * gridDim.x) {
        const TileRef tr = tiles[i];
        const int key = 2 * tr.dom + parity;
        if (key != loaded) { // uniform over the half
            const uint32_t *src = reinterpret_cast<const uint32_t *>(doms + key);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&sa);
            for (int w = lt; w < (int)(sizeof(Fused2Args<S, T>) / 4); w += HALF_TX) dst[w] = src[w];
            tile_sync<HALF_TX, BAR>();
            loaded = key;
        }
        const bool down = ((tr.yb / sa.tile_y) & 1) != 0;
        fused2_tile<S, T, HALF_TX, false, FLAGS, false, false, false, BAR>(sa, tr.xb, tr.yb, s_rho, s_m,
                                                                           down);
        tile_sync<HALF_TX, BAR>(); // the half's ring and block are reused by its next tile
    }
}

template <typename S, typename T, int FLAGS>
__global__ void __launch_bounds__(BATCH_TX, (sizeof(T) == 8 ? 3 : 5))
    k_batch2_half(const Fused2Args<S, T> *__restrict__ doms, const TileRef *__restrict__ tiles,
                  int ntiles, int parity)
{
    __shared__ V2<T> s_rho[2][4][HALF_TX];
    __shared__ uint8_t s_m[2][4][HALF_TX];
    __shared__ __align__(16) Fused2Args<S, T> sa[2];
    static_assert(sizeof(Fused2Args<S, T>) % 4 == 0, "argument block copied as words");
    if (threadIdx.x < HALF_TX)
        batch_half_loop<S, T, FLAGS, 1>(doms, tiles, ntiles, parity, s_rho[0], s_m[0], sa[0]);
    else
        batch_half_loop<S, T, FLAGS, 2>(doms, tiles, ntiles, parity, s_rho[1], s_m[1], sa[1]);
}

// One-warp tiles: each warp of a 128-thread CTA walks its own 32-column tiles
// (tiles 4c + w, 4c + w + 4g, ...) with its own density ring and argument
// block; the row loop needs only warp synchronisation, so warps never wait on
// one another (the ensemble's widths 64..512: 89 % of the lanes busy).
constexpr int WARP_TX = 32;
template <typename S, typename T, int FLAGS>
__global__ void __launch_bounds__(BATCH_TX, (sizeof(T) == 8 ? 3 : 5))
    k_batch2_warp(const Fused2Args<S, T> *__restrict__ doms, const TileRef *__restrict__ tiles,
                  int ntiles, int parity)
{
    constexpr int NW = BATCH_TX / WARP_TX;
    __shared__ V2<T> s_rho[NW][4][WARP_TX];
    __shared__ uint8_t s_m[NW][4][WARP_TX];
    __shared__ __align__(16) Fused2Args<S, T> sa[NW];
    static_assert(sizeof(Fused2Args<S, T>) % 4 == 0, "argument block copied as words");
    const int w = threadIdx.x / WARP_TX, lane = threadIdx.x % WARP_TX;
    int loaded = -1;
    for (int i = NW * blockIdx.x + w; i < ntiles; i += NW * gridDim.x) {
        const TileRef tr = tiles[i];
        const int key = 2 * tr.dom + parity;
        if (key != loaded) {
            const uint32_t *src = reinterpret_cast<const uint32_t *>(doms + key);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&sa[w]);
            for (int k = lane; k < (int)(sizeof(Fused2Args<S, T>) / 4); k += WARP_TX) dst[k] = src[k];
            __syncwarp();
            loaded = key;
        }
        const bool down = ((tr.yb / sa[w].tile_y) & 1) != 0;
        fused2_tile<S, T, WARP_TX, false, FLAGS, false, false, false, SYNC_WARP>(
            sa[w], tr.xb, tr.yb, s_rho[w], s_m[w], down);
        __syncwarp(); // the warp's ring and block are reused by its next tile
    }
}

template <typename S, typename T>
inline cudaError_t launch_batch_warp_t(const Fused2Args<S, T> *doms, const TileRef *tiles,
                                       int ntiles, int parity, int grid, int flags, cudaStream_t s)
{
    if (flags & KF_SOLID)
        k_batch2_warp<S, T, KF_FORCE | KF_SOLID | KF_UNIFORM><<<grid, BATCH_TX, 0, s>>>(doms, tiles,
                                                                                      ntiles, parity);
    else
        k_batch2_warp<S, T, KF_FORCE><<<grid, BATCH_TX, 0, s>>>(doms, tiles, ntiles, parity);
    return cudaGetLastError();
}

template <typename S, typename T> inline int batch_warp_blocks_per_sm_t()
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, k_batch2_warp<S, T, KF_FORCE | KF_SOLID | KF_UNIFORM>, BATCH_TX, 0) != cudaSuccess)
        return 1;
    return n;
}

template <typename S, typename T>
inline cudaError_t launch_batch_half_t(const Fused2Args<S, T> *doms, const TileRef *tiles,
                                       int ntiles, int parity, int grid, int flags, cudaStream_t s)
{
    if (flags & KF_SOLID)
        k_batch2_half<S, T, KF_FORCE | KF_SOLID | KF_UNIFORM><<<grid, BATCH_TX, 0, s>>>(doms, tiles,
                                                                                      ntiles, parity);
    else
        k_batch2_half<S, T, KF_FORCE><<<grid, BATCH_TX, 0, s>>>(doms, tiles, ntiles, parity);
    return cudaGetLastError();
}

template <typename S, typename T> inline int batch_half_blocks_per_sm_t()
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, k_batch2_half<S, T, KF_FORCE | KF_SOLID | KF_UNIFORM>, BATCH_TX, 0) != cudaSuccess)
        return 1;
    return n;
}

// flags: KF_FORCE / KF_SOLID when any domain of the batch has a volume force /
// a solid node (the body drops what no domain needs)
template <typename S, typename T, bool AHEAD = false, bool COMPACT = false, int UNI = 0>
inline cudaError_t launch_batch_t(const Fused2Args<S, T> *doms, const TileRef *tiles, int ntiles,
                                  int parity, int grid, int flags, cudaStream_t s)
{
    // batches with solid nodes run the force + solid body (the force vector is
    // zero where no force is set); it compiled leaner than the solid-only one
    if (AHEAD || (flags & KF_SOLID))
        k_batch2<S, T, KF_FORCE | KF_SOLID | UNI, AHEAD, COMPACT><<<grid, BATCH_TX, 0, s>>>(
            doms, tiles, ntiles, parity);
    else if (flags == KF_FORCE)
        k_batch2<S, T, KF_FORCE><<<grid, BATCH_TX, 0, s>>>(doms, tiles, ntiles, parity);
    else
        k_batch2<S, T, 0><<<grid, BATCH_TX, 0, s>>>(doms, tiles, ntiles, parity);
    return cudaGetLastError();
}

template <typename S, typename T, bool AHEAD = false, bool COMPACT = false, int UNI = 0>
inline int batch_blocks_per_sm_t()
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, k_batch2<S, T, KF_FORCE | KF_SOLID | UNI, AHEAD, COMPACT>, BATCH_TX, 0) !=
        cudaSuccess)
        return 1;
    return n;
}

// tile body of the FP32-arithmetic batches (ignored for FP64)
enum BatchBody {
    BODY_TILE = 0,
    BODY_AHEAD = 1,
    BODY_COMPACT = 2,
    BODY_UNIFORM = 3,
    BODY_HALF = 4, // two 64-column tiles per CTA (k_batch2_half), its own tile list
    BODY_WARP = 5, // one 32-column tile per warp (k_batch2_warp), its own tile list
    BODY_COUNT = 6
};
cudaError_t launch_batch_fp64(const Fused2Args<double, double> *doms, const TileRef *tiles,
                              int ntiles, int parity, int grid, int flags, cudaStream_t s);
cudaError_t launch_batch_f32(const Fused2Args<float, float> *doms, const TileRef *tiles,
                             int ntiles, int parity, int grid, int flags, int body, cudaStream_t s);
cudaError_t launch_batch_f16(const Fused2Args<__half, float> *doms, const TileRef *tiles,
                             int ntiles, int parity, int grid, int flags, int body, cudaStream_t s);
int batch_blocks_per_sm(sclbm_precision p, int body = BODY_TILE);

} // namespace sclbm
