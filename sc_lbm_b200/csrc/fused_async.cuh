// fused_async.cuh -- variant of the fused step whose population rows are
// staged through a shared-memory ring by asynchronous global->shared copies
// (cp.async / LDGSTS), with a band decomposition of the lattice.
//
// Work decomposition.  The lattice is cut into column strips of TX columns
// (one thread per column, all threads interior) and row bands; CTA (s, b)
// owns strip s, band b.  The bands split every strip at the same rows and
// neighbouring strips have consecutive CTA indices, so the CTAs of one band
// walk the same rows at the same time: a strip's halo columns and the sectors
// its pushes share with the next strip are touched by both within a few rows
// (L2 hits, whole-sector writes).  The number of bands is chosen so that all
// CTAs are resident at once.
//
// Pipeline.  For a segment of rows [y0, y1), local row lr (0 = the halo row
// below, nrow+1 = the halo row above) lives in ring stage lr % R.  Before the
// row loop, rows 0..R-2 are requested; iteration lr waits for row lr, reduces
// it to the densities of both components (shared density ring, one
// __syncthreads), collides row lr-1 from its populations still in the ring,
// pushes the results to global memory, and finally requests row lr+R-1 into
// the stage that row lr-1 just vacated.  Each thread copies and reads only its
// own column (threads 0 and ncol-1 also the halo columns), so the population
// ring needs no barrier; R-1 rows per thread are in flight while it computes.
#pragma once
#include <cuda_pipeline.h>

#include "fused_step.cuh"

namespace sclbm {

template <typename S, typename T, int TX, int R> struct AsyncLayout {
    static constexpr int P = TX + 2; // columns including the two halo columns
    static constexpr size_t pops = size_t(R) * 18 * P * sizeof(S);
    static constexpr size_t rho = size_t(2) * 4 * P * sizeof(T);
    static constexpr size_t bytes = pops + rho + 4 * P;
};

template <typename S, typename T, int TX, int R>
__device__ __forceinline__ void async_copy_node(S *pops, int stage, int col,
                                                const Fused2Args<S, T> &a, uint32_t node)
{
    constexpr int P = TX + 2;
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int i = 0; i < 9; ++i)
            __pipeline_memcpy_async(pops + ((stage * 2 + k) * 9 + i) * P + col,
                                    a.fin[k] + (size_t)i * a.N + node, sizeof(S));
}

template <typename S, typename T, int TX, int R>
__device__ __forceinline__ void async_density(const S *pops, int stage, int col, uint8_t m,
                                              V2<T> *rho, uint8_t *msk, int slot)
{
    constexpr int P = TX + 2;
    T r[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        T s = T(0); // 0.0 + f0 + ... + f8, src/fluid.cpp:177-181
#pragma unroll
        for (int i = 0; i < 9; ++i) s += T(pops[((stage * 2 + k) * 9 + i) * P + col]);
        r[k] = m ? s : T(0);
    }
    rho[slot * P + col] = Vec2<T>::make(r[0], r[1]);
    msk[slot * P + col] = m;
}

// Rows [y0, y1) of the strip starting at column xb.
template <typename S, typename T, int TX, int R, int FLAGS>
__device__ __forceinline__ void async_segment(const Fused2Args<S, T> &a, const int xb,
                                              const int y0, const int y1, unsigned char *smem)
{
    using L = AsyncLayout<S, T, TX, R>;
    constexpr int P = L::P;
    constexpr bool SOLID = (FLAGS & KF_SOLID) != 0;
    S *pops = reinterpret_cast<S *>(smem);
    V2<T> *rho = reinterpret_cast<V2<T> *>(smem + L::pops);
    static_assert(L::pops % sizeof(V2<T>) == 0, "density ring alignment");
    uint8_t *msk = smem + L::pops + L::rho;

    const int t = threadIdx.x;
    const int nx = a.nx, ny = a.ny;
    const int ncol = min(TX, nx - xb);
    const int nrow = y1 - y0;
    const bool act = t < ncol;
    const bool hl = act && t == 0, hr = act && t == ncol - 1;
    const int x = act ? xb + t : 0;
    const int xl = wrap1(x - 1, nx), xr = wrap1(x + 1, nx);
    const int xhl = wrap1(xb - 1, nx), xhr = wrap1(xb + ncol, nx);
    const int last = nrow + 1;

    int issue_stage = 0;
    auto issue = [&](int lr) {
        if (act && lr <= last) {
            const uint32_t row = (uint32_t)wrap1(y0 - 1 + lr, ny) * (uint32_t)nx;
            async_copy_node<S, T, TX, R>(pops, issue_stage, t + 1, a, row + x);
            if (hl) async_copy_node<S, T, TX, R>(pops, issue_stage, 0, a, row + xhl);
            if (hr) async_copy_node<S, T, TX, R>(pops, issue_stage, ncol + 1, a, row + xhr);
        }
        __pipeline_commit();
        issue_stage = issue_stage + 1 == R ? 0 : issue_stage + 1;
    };
#pragma unroll
    for (int q = 0; q < R - 1; ++q) issue(q);

    uint8_t mn = 1, mnl = 1, mnr = 1; // masks of the next row (loaded one row ahead)
    if (SOLID && act) {
        const uint32_t row = (uint32_t)wrap1(y0 - 1, ny) * (uint32_t)nx;
        mn = a.mask[row + x];
        if (hl) mnl = a.mask[row + xhl];
        if (hr) mnr = a.mask[row + xhr];
    }
    int stage = 0;      // ring stage of row lr
    int cstage = R - 1; // ring stage of row lr-1
    for (int lr = 0; lr <= last; ++lr) {
        const int slot = lr & 3;
        const uint8_t m = mn, ml = mnl, mr = mnr;
        if (SOLID && act && lr < last) {
            const uint32_t row = (uint32_t)wrap1(y0 + lr, ny) * (uint32_t)nx;
            mn = a.mask[row + x];
            if (hl) mnl = a.mask[row + xhl];
            if (hr) mnr = a.mask[row + xhr];
        }
        __pipeline_wait_prior(R - 2);
        if (act) {
            async_density<S, T, TX, R>(pops, stage, t + 1, m, rho, msk, slot);
            if (hl) async_density<S, T, TX, R>(pops, stage, 0, ml, rho, msk, slot);
            if (hr) async_density<S, T, TX, R>(pops, stage, ncol + 1, mr, rho, msk, slot);
        }
        __syncthreads();
        if (act && lr >= 2) {
            const int yc = wrap1(y0 + lr - 2, ny);
            const int sm = (lr - 2) & 3, sc = (lr - 1) & 3, sp = slot;
            const RingPops<S, T, P> f{pops + cstage * 18 * P + t + 1};
            const Stencil<T> st{{rho + sm * P, rho + sc * P, rho + sp * P},
                                {msk + sm * P, msk + sc * P, msk + sp * P}, t + 1};
            const Nbr n = make_nbr(nx, x, xl, xr, yc, wrap1(yc - 1, ny), wrap1(yc + 1, ny));
            collide_push<S, T, FLAGS, true>(a, f, st, n); // 64-bit offsets: any lattice size
        }
        // row lr-1's stage is free again: request row lr+R-1 into it
        issue(lr + R - 1);
        cstage = stage;
        stage = stage + 1 == R ? 0 : stage + 1;
    }
    __pipeline_wait_prior(0);
    __syncthreads(); // the rings are reused by the next segment
}

// Grid (strips, bands): CTA (s, b) owns strip s, rows [b*ny/B, (b+1)*ny/B).
template <typename S, typename T, int TX, int R, int FLAGS>
__global__ void __launch_bounds__(TX) k_fused2_async(const __grid_constant__ Fused2Args<S, T> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int y0 = (int)((long long)a.ny * blockIdx.y / gridDim.y);
    const int y1 = (int)((long long)a.ny * (blockIdx.y + 1) / gridDim.y);
    if (y1 > y0) async_segment<S, T, TX, R, FLAGS>(a, blockIdx.x * TX, y0, y1, smem);
}

// Batched form: a list of (domain, strip, row band) tiles, neighbouring strips
// of a band adjacent in the list; CTA i takes tiles i, i + grid, ...
struct BandTile {
    int dom, xb, y0, y1;
};

template <typename S, typename T, int TX, int R, int FLAGS>
__global__ void __launch_bounds__(TX)
    k_batch2_async(const Fused2Args<S, T> *__restrict__ doms, const BandTile *__restrict__ tiles,
                   int ntiles, int parity)
{
    extern __shared__ __align__(16) unsigned char smem[];
    // argument block of the current tile's domain, read from shared memory
    __shared__ __align__(16) Fused2Args<S, T> sa;
    static_assert(sizeof(Fused2Args<S, T>) % 4 == 0, "argument block copied as words");
    int loaded = -1;
    for (int i = blockIdx.x; i < ntiles; i += gridDim.x) {
        const BandTile tl = tiles[i];
        const int key = 2 * tl.dom + parity;
        if (key != loaded) { // uniform over the CTA; the previous segment ended in a barrier
            const uint32_t *src = reinterpret_cast<const uint32_t *>(doms + key);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&sa);
            for (int w = threadIdx.x; w < (int)(sizeof(sa) / 4); w += TX) dst[w] = src[w];
            __syncthreads();
            loaded = key;
        }
        async_segment<S, T, TX, R, FLAGS>(sa, tl.xb, tl.y0, tl.y1, smem);
    }
}

// resident CTAs per SM for a kernel with the ring's dynamic shared memory
template <typename K> inline int resident_ctas(K kernel, int threads, size_t smem)
{
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess)
        return 0;
    return n;
}

template <typename S, typename T, int TX, int R, int FLAGS>
inline cudaError_t launch_fused2_async_f(const Fused2Args<S, T> &a, cudaStream_t s)
{
    using L = AsyncLayout<S, T, TX, R>;
    static int per_sm = resident_ctas(k_fused2_async<S, T, TX, R, FLAGS>, TX, L::bytes);
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int nstrips = (a.nx + TX - 1) / TX;
    // as many bands as fit resident beside each other, at least 4 rows each
    int nbands = std::max(1, per_sm * sm_count() / nstrips);
    nbands = std::max(1, std::min(nbands, a.ny / 4));
    k_fused2_async<S, T, TX, R, FLAGS><<<dim3(nstrips, nbands), TX, L::bytes, s>>>(a);
    return cudaGetLastError();
}

// UNI = KF_UNIFORM: lattices with solid nodes run the uniform solid form
template <typename S, typename T, int TX, int R, int UNI = 0>
inline cudaError_t launch_fused2_async_t(const Fused2Args<S, T> &a, cudaStream_t s)
{
    switch (kernel_flags(a)) {
    case 0: return launch_fused2_async_f<S, T, TX, R, 0>(a, s);
    case KF_FORCE: return launch_fused2_async_f<S, T, TX, R, KF_FORCE>(a, s);
    case KF_SOLID: return launch_fused2_async_f<S, T, TX, R, KF_SOLID | UNI>(a, s);
    default: return launch_fused2_async_f<S, T, TX, R, KF_FORCE | KF_SOLID | UNI>(a, s);
    }
}

// the batched kernel always runs the general body (force and solids handled)
template <typename S, typename T, int TX, int R> inline int async_resident_ctas()
{
    using L = AsyncLayout<S, T, TX, R>;
    static int per_sm =
        resident_ctas(k_batch2_async<S, T, TX, R, KF_FORCE | KF_SOLID>, TX, L::bytes);
    return per_sm * sm_count();
}

template <typename S, typename T, int TX, int R>
inline cudaError_t launch_batch2_async_t(const Fused2Args<S, T> *doms, const BandTile *tiles,
                                         int ntiles, int grid, int parity, cudaStream_t s)
{
    using L = AsyncLayout<S, T, TX, R>;
    if (async_resident_ctas<S, T, TX, R>() < 1) return cudaErrorInvalidConfiguration;
    k_batch2_async<S, T, TX, R, KF_FORCE | KF_SOLID><<<grid, TX, L::bytes, s>>>(doms, tiles, ntiles,
                                                                               parity);
    return cudaGetLastError();
}

} // namespace sclbm
