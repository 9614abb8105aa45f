// fused_ring.cuh -- the fused two-component step with its population rows
// streamed into a shared-memory ring by the TMA engine (cp.async.bulk.tensor:
// one 3-D box per component and row -- the row segment of all nine
// directions -- completion counted in bytes on an mbarrier per ring stage).
//
// Why.  The register-tile kernel (fused_step.cuh) keeps at most one row of
// loads in flight per warp, and the registers that hold them cap residency;
// its FP32 and FP16 forms wait on load latency.  Here the bytes in flight do
// not live in registers: each CTA keeps R whole population rows on their way
// into shared memory while its threads reduce one row and collide the one
// before it.  Two tensor copies per row replace eighteen per-thread loads
// and their address arithmetic (eighteen 1-D bulk copies per row, one per
// population array, were measured slower than the register tile: the copy
// engine's per-copy cost dominated at 300-1000 bytes a copy).
//
// Work decomposition.  A CTA of RING_W threads owns a strip of RING_W interior
// columns and a band of rows (16 to 32 as the caller chooses: several waves
// of CTAs, which the block scheduler balances where bands hold different
// numbers of fluid nodes).  Neighbouring bands march in opposite directions, so the two halo
// rows that a pair of bands shares are read by both near the same time and
// the second read often hits L2.
//
// Ring.  Row j of a band (j = 0 .. nrow+1, halo rows included) lands in stage
// j % R: per component a box of 9 directions x P = RING_W + 2A elements,
// lattice columns xb - A .. xb + RING_W + A - 1, where A elements make 16 bytes
// (a box's first column must start on a 16-byte boundary: nx must be a
// multiple of A).  Columns outside the lattice arrive as zeros; where a strip
// touches the lattice's left or right edge, the periodic halo column comes
// from a second, A-column box at the other edge (or, in the form without
// halo boxes, from element copies into a small edge buffer one row ahead).
// Iteration j waits for row j, reads each thread's column into registers and
// reduces it to both components' densities (density ring in shared memory,
// one __syncthreads); the stage is then free and is refilled at once with row
// j + R, so all R stages are in flight while the CTA computes; finally row
// j - 1 is collided from registers and pushed straight to global memory (the
// scattered push of collide_push, half-way bounce-back included).  The
// arithmetic per node is the register tile's (collide_push), so both kernels
// write the same bytes.
//
// Waits are bounded: a stage that does not fill within RING_WAIT_LIMIT polls
// sets *a.status and the CTA skips the rest of its band (no hang); the
// domain's monitor reports the flag.
#pragma once
#include <cuda.h>

#include "fused_step.cuh"

namespace sclbm {

constexpr int RING_W = 128;              // interior columns per strip = threads per CTA
constexpr int RING_WAIT_LIMIT = 1 << 20; // polls of one stage before giving up (~1 s)

// elements per 16 bytes of storage type S
template <typename S> constexpr int ring_pad() { return 16 / (int)sizeof(S); }

// HB: each stage holds the halo boxes of strips at the lattice's left and
// right edges (the wrapped halo column).  Without them (4- and 8-byte storage
// only) a stage is 1 KB smaller and the halo lane of such a strip copies the
// wrapped column's populations of the next row into its own slot of a small
// edge buffer (two slots per halo lane: 36 elements).
template <typename S, typename T, int R, int W = RING_W, bool HB = true> struct RingLayout {
    static constexpr int A = ring_pad<S>();
    static constexpr int P = W + 2 * A; // box columns
    static constexpr int Q = W + 2;     // density ring columns
    // tensor-copy destinations start on 128-byte boundaries
    static constexpr size_t comp = (size_t(9) * P * sizeof(S) + 127) & ~size_t(127);
    static constexpr size_t halo = 256; // one A-column box of one component (144 bytes)
    static constexpr size_t stage = 2 * comp + (HB ? 4 * halo : 0); // components, then halos [side][k]
    static constexpr size_t pops = size_t(R) * stage;
    static constexpr size_t rho = size_t(4) * Q * sizeof(V2<T>);
    static constexpr size_t msk = size_t(4) * Q;
    static constexpr size_t edge_at = (pops + rho + msk + 15) & ~size_t(15);
    static constexpr size_t edge = HB ? 0 : size_t(2) * 2 * 18 * sizeof(S); // [slot][lane][k][i]
    static constexpr size_t bars = (edge_at + edge + 15) & ~size_t(15);
    static constexpr size_t bytes = bars + size_t(R) * 8 + 16 + 128; // + base alignment
    static constexpr uint32_t CE = (uint32_t)(comp / sizeof(S));     // component stride, elements
    static_assert(comp % 128 == 0 && stage % 128 == 0, "tensor-copy alignment");
    static_assert(size_t(9) * A * sizeof(S) <= halo, "halo box");
    static_assert(HB || sizeof(S) >= 4, "edge copies move 4 or 8 bytes");
};

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// one arrival that also announces the bytes the stage's copies will deliver
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return ok != 0;
}
// asynchronous copy of one 4- or 8-byte element from global into shared
// memory (cp.async); only the issuing thread waits on it and reads it
template <int B> __device__ __forceinline__ void cp_async_elem(uint32_t dst, const void *src)
{
    static_assert(B == 4 || B == 8, "cp.async.ca moves 4, 8 or 16 bytes");
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(dst), "l"(src), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// one 3-D box of a tiled tensor map into shared memory (dst 128-byte aligned),
// completing on mbarrier `bar`; coordinates in elements (x may be negative or
// past the end: those elements arrive as zeros); no multicast
__device__ __forceinline__ void tensor_g2s_3d(uint32_t dst, const void *map, int x, int y, int z,
                                              uint32_t bar)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
                 "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar)
                 : "memory");
}

// tiled tensor map over [dim[2]][dim[1]][dim[0]] (no swizzle, zero fill,
// 256-byte L2 promotion); 0 on success (tensor_map.cpp)
int encode_tensor_map(CUtensorMap *m, CUtensorMapDataType dt, unsigned rank, void *base,
                      const cuuint64_t *dim, const cuuint64_t *stride_bytes, const cuuint32_t *box,
                      const cuuint32_t *elem_strides);

// The four tensor maps of one launch: per component the row box (P x 1 x 9)
// and the halo box (A x 1 x 9) over the input populations [9][ny][nx].
struct RingMaps {
    CUtensorMap row[2], halo[2];
};

// resident CTAs per SM the register cap aims at (the ring's shared memory
// allows about as many): the register tile's figures, six for FP32
// arithmetic (five in the uniform solid form, which spills at 80 registers,
// and without halo boxes, whose smaller stages let a fifth CTA's shared
// memory fit), three for FP64
template <typename T, int FLAGS, bool HB = true> constexpr int ring_min_ctas()
{
    return sizeof(T) == 8 ? 3 : (((FLAGS & KF_UNIFORM) || !HB) ? 5 : 6);
}

// The shared-memory pieces of one CTA's ring.
template <typename S, typename T, int R, int W = RING_W, bool HB = true> struct RingShared {
    unsigned char *base; // 128-byte aligned: the R stages
    V2<T> *rho;          // density ring [4][Q]
    uint8_t *msk;        // mask ring [4][Q]
    S *edge;             // edge buffer (HB false)
    uint64_t *bars;      // one mbarrier per stage
    volatile int *abort_flag;
};

template <typename S, typename T, int R, int W = RING_W, bool HB = true>
__device__ __forceinline__ RingShared<S, T, R, W, HB> ring_shared(unsigned char *raw)
{
    using L = RingLayout<S, T, R, W, HB>;
    RingShared<S, T, R, W, HB> sh;
    sh.base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(raw) + 127) & ~uintptr_t(127));
    sh.rho = reinterpret_cast<V2<T> *>(sh.base + L::pops);
    sh.msk = sh.base + L::pops + L::rho;
    sh.edge = reinterpret_cast<S *>(sh.base + L::edge_at);
    sh.bars = reinterpret_cast<uint64_t *>(sh.base + L::bars);
    sh.abort_flag = reinterpret_cast<volatile int *>(sh.base + L::bars + R * 8);
    if (threadIdx.x == 0) {
        for (int s = 0; s < R; ++s) mbar_init(smem_addr(&sh.bars[s]), 1);
        *sh.abort_flag = 0;
        mbar_fence_init();
    }
    __syncthreads();
    return sh;
}

// One unit of work: strip [xb, xb + RING_W) of rows [y0, y0 + nrow) of the
// lattice of `a`, rows marched upward or (down) downward.  The ring rows of
// a CTA are numbered on across its units (g0, advanced here), so every
// stage's mbarrier phase follows from that count.  maps: row boxes of both
// components, then halo boxes.  Returns false once the CTA has given up on a
// bounded wait (*a.status is then set).
template <typename S, typename T, int FLAGS, int R, bool WIDE, int W = RING_W, bool HB = true>
__device__ __forceinline__ bool ring_unit(const Fused2Args<S, T> &a, const CUtensorMap *map_row0,
                                          const CUtensorMap *map_row1, const CUtensorMap *map_halo0,
                                          const CUtensorMap *map_halo1, const int xb, const int y0,
                                          const int nrow, const bool down,
                                          const RingShared<S, T, R, W, HB> &sh, uint32_t &g0)
{
    using L = RingLayout<S, T, R, W, HB>;
    constexpr int A = L::A, P = L::P, Q = L::Q;
    constexpr uint32_t CE = L::CE;
    constexpr bool SOLID = (FLAGS & KF_SOLID) != 0;
    unsigned char *const ring_smem = sh.base;
    V2<T> *const rho = sh.rho;
    uint8_t *const msk = sh.msk;
    uint64_t *const bars = sh.bars;
    volatile int *const abort_flag = sh.abort_flag;

    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nx = a.nx, ny = a.ny;
    const int ncol = min(W, nx - xb);
    const bool act = t < ncol;
    const int x = act ? xb + t : xb;
    const int xl = wrap1(x - 1, nx), xr = wrap1(x + 1, nx);
    // the densities of the two halo columns come from lanes 0 (left) and 1
    // (right) of warp HW, which run the same instructions side by side whether
    // or not their own columns hold nodes.  FP16 storage takes them to warp 1,
    // away from warp 0, which issues the row copies: its issue-bound rows then
    // wait less at the row barrier (4096^2: 49.1 -> 50.3 GLUPS all-fluid,
    // 37.4 -> 38.2 at 72 % fluid); FP32 storage ran 1.2 % slower that way
    // (41.1 -> 40.6) and keeps them in warp 0, as does FP64 (no change)
    constexpr int HW = (sizeof(S) == 2 && W >= 64) ? 1 : 0;
    const bool hal = warp == HW && lane <= 1, hl = hal && lane == 0;
    const int xh = hl ? wrap1(xb - 1, nx) : wrap1(xb + ncol, nx);
    const int last = nrow + 1;
    const uint32_t gbase = g0;
    // lattice row of ring row j (tile row -1 .. nrow in march order)
    auto gy = [&](int j) { return wrap1(y0 + (down ? nrow - j : j - 1), ny); };
    auto stage_of = [&](int j) { return (int)((gbase + (uint32_t)j) % (uint32_t)R); };
    auto phase_of = [&](int j) { return ((gbase + (uint32_t)j) / (uint32_t)R) & 1u; };

    // the halo column left (right) of the strip wraps around the lattice edge:
    // it comes from an A-column box at the other edge
    const bool wrap_l = xb == 0, wrap_r = xb + ncol == nx;
    const uint32_t box_bytes = 9u * (uint32_t)P * (uint32_t)sizeof(S);
    const uint32_t halo_bytes = 9u * (uint32_t)A * (uint32_t)sizeof(S);
    const uint32_t row_bytes =
        2u * (box_bytes + (HB && wrap_l ? halo_bytes : 0u) + (HB && wrap_r ? halo_bytes : 0u));
    auto stage_at = [&](int st) { return ring_smem + (size_t)st * L::stage; };
    // lane 0 of warp 0 requests row j: one box per component (+ halo boxes)
    auto issue = [&](int j) {
        if (lane != 0) return;
        const int st = stage_of(j);
        const uint32_t bar = smem_addr(&bars[st]);
        const uint32_t sb = smem_addr(stage_at(st));
        const int y = gy(j);
        mbar_expect_tx(bar, row_bytes);
        const CUtensorMap *rowm[2] = {map_row0, map_row1}, *halom[2] = {map_halo0, map_halo1};
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            tensor_g2s_3d(sb + k * (uint32_t)L::comp, rowm[k], xb - A, y, 0, bar);
            if (HB && wrap_l)
                tensor_g2s_3d(sb + 2 * (uint32_t)L::comp + (0 + k) * (uint32_t)L::halo, halom[k], nx - A, y,
                              0, bar);
            if (HB && wrap_r)
                tensor_g2s_3d(sb + 2 * (uint32_t)L::comp + (2 + k) * (uint32_t)L::halo, halom[k], 0, y, 0,
                              bar);
        }
    };
    auto wait_row = [&](int j) {
        const uint32_t bar = smem_addr(&bars[stage_of(j)]);
        const uint32_t par = phase_of(j);
        for (int it = 0; it < RING_WAIT_LIMIT; ++it)
            if (mbar_try_wait(bar, par)) return true;
        return false;
    };

    int issued = -1; // last row requested (warp 0's view)
    if (warp == 0)
        for (int j = 0; j < R && j <= last; ++j) {
            issue(j);
            issued = j;
        }

    // without halo boxes, a halo lane whose column wraps around the lattice
    // edge copies that column's populations of ring row j into its edge slot
    // j & 1 one row ahead; it alone waits on and reads its copies
    const bool edge = !HB && hal && (hl ? wrap_l : wrap_r);
    auto edge_slot = [&](int j) { return sh.edge + ((j & 1) * 2 + (hl ? 0 : 1)) * 18; };
    auto copy_edge = [&](int j) {
        if constexpr (!HB) {
            const uint32_t node = (uint32_t)gy(j) * (uint32_t)nx + (uint32_t)xh;
            const uint32_t dst = smem_addr(edge_slot(j));
#pragma unroll
            for (int k = 0; k < 2; ++k)
#pragma unroll
                for (int i = 0; i < 9; ++i)
                    cp_async_elem<(int)sizeof(S)>(dst + (uint32_t)((k * 9 + i) * sizeof(S)),
                                                  a.fin[k] + elem<WIDE>(i, a.N, node));
            cp_async_commit();
        }
    };
    if constexpr (!HB) {
        if (edge) copy_edge(0);
    }

    // masks of the next row, loaded one row ahead
    uint8_t mn = 1, mnh = 1;
    if (SOLID) {
        const size_t row = (size_t)gy(0) * (size_t)nx;
        if (act) mn = a.mask[row + x];
        if (hal) mnh = a.mask[row + xh];
    }
    bool aborted = false;
    int consumed = -1;

    // iteration j: row j from its stage into registers (cur) and its densities
    // into the ring; barrier; the stage is free, so request row j + R into it;
    // collide row j - 1 (prev) from the stencil rows j - 2, j - 1, j
    auto step_row = [&](const int j, T(&cur)[2][9], const T(&prev)[2][9]) {
        const uint8_t m = mn, mh = mnh;
        if (SOLID && j < last) {
            const size_t row = (size_t)gy(j + 1) * (size_t)nx;
            if (act) mn = a.mask[row + x];
            if (hal) mnh = a.mask[row + xh];
        }
        const int slot = j & 3;
        if (!aborted) {
            if (wait_row(j)) {
                consumed = j;
                const unsigned char *sg = stage_at(stage_of(j));
                const S *stg = reinterpret_cast<const S *>(sg);
                const S *hlp = reinterpret_cast<const S *>(sg + 2 * L::comp);            // [k][9][A]
                const S *hrp = reinterpret_cast<const S *>(sg + 2 * L::comp + 2 * L::halo);
                auto density = [&](const T(&f)[2][9], uint8_t mm, int q) {
                    T r[2];
                    node_density(f, r[0], r[1]);
                    if (SOLID && !mm) r[0] = r[1] = T(0);
                    rho[slot * Q + q] = Vec2<T>::make(r[0], r[1]);
                    msk[slot * Q + q] = SOLID ? mm : 1;
                };
                // f[k][i] from a box of component stride cs, direction stride ds
                auto load = [&](const S *p, uint32_t cs, int ds, int col, T(&f)[2][9]) {
#pragma unroll
                    for (int k = 0; k < 2; ++k)
#pragma unroll
                        for (int i = 0; i < 9; ++i) f[k][i] = T(p[k * cs + i * ds + col]);
                };
                constexpr uint32_t HE = (uint32_t)(L::halo / sizeof(S));
                if (act) {
                    load(stg, CE, P, A + t, cur);
                    density(cur, m, t + 1);
                }
                if (!HB && edge) {
                    cp_async_wait_all(); // row j's copies, issued one iteration ago
                    const S *e = edge_slot(j);
                    T h[2][9];
#pragma unroll
                    for (int k = 0; k < 2; ++k)
#pragma unroll
                        for (int i = 0; i < 9; ++i) h[k][i] = T(e[k * 9 + i]);
                    density(h, mh, hl ? 0 : ncol + 1);
                    if (j < last) copy_edge(j + 1);
                } else if (hal) {
                    // the halo column wrapped around a lattice edge comes
                    // from its own box, else from the row box
                    const bool wrap = HB && (hl ? wrap_l : wrap_r);
                    const S *hp = wrap ? (hl ? hlp : hrp) : stg;
                    const uint32_t hcs = wrap ? HE : CE;
                    const int hds = wrap ? A : P;
                    const int hcol = wrap ? (hl ? A - 1 : 0) : (hl ? A - 1 : A + ncol);
                    T h[2][9];
                    load(hp, hcs, hds, hcol, h);
                    density(h, mh, hl ? 0 : ncol + 1);
                }
            } else {
                *abort_flag = 1;
                if (a.status) atomicExch(a.status, 1);
            }
        }
        __syncthreads();
        aborted = *abort_flag != 0;
        if (aborted) return;
        // every thread has read row j's stage before the barrier
        if (warp == 0 && j + R <= last) {
            issue(j + R);
            issued = j + R;
        }
        if (act && j >= 2) {
            // rows below (sb), at (sc) and above (sa) the node of ring row j-1
            const int s_old = (j - 2) & 3, sc = (j - 1) & 3, s_new = slot;
            const int sb = down ? s_new : s_old, sa = down ? s_old : s_new;
            const int yc = gy(j - 1);
            const Stencil<T> st{{rho + sb * Q, rho + sc * Q, rho + sa * Q},
                                {msk + sb * Q, msk + sc * Q, msk + sa * Q}, t + 1};
            const Nbr n = make_nbr(nx, x, xl, xr, yc, wrap1(yc - 1, ny), wrap1(yc + 1, ny));
            collide_push<S, T, FLAGS, WIDE>(a, prev, st, n);
        }
    };
    T Ab[2][9], Bb[2][9];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int i = 0; i < 9; ++i) Ab[k][i] = Bb[k][i] = T(0);
    // two rows per trip so the register buffers swap roles instead of being copied
    for (int j = 0; j <= last; j += 2) {
        step_row(j, Ab, Bb);
        if (j + 1 <= last) step_row(j + 1, Bb, Ab);
    }
    if (aborted && warp == 0 && lane == 0) {
        // let the copies still in flight land before the CTA's shared memory is released
        for (int j = consumed + 1; j <= issued; ++j) (void)wait_row(j);
    }
    if constexpr (!HB) {
        if (edge) cp_async_wait_all(); // an edge copy still in flight after an abort
    }
    g0 = gbase + (uint32_t)(last + 1);
    return !aborted;
}

// One band of one strip per CTA; band b covers rows [b*ny/bands, (b+1)*ny/bands).
template <typename S, typename T, int FLAGS, int R, bool WIDE, bool HB>
__global__ void __launch_bounds__(RING_W, (ring_min_ctas<T, FLAGS, HB>()))
    k_ring2(const __grid_constant__ Fused2Args<S, T> a, const __grid_constant__ RingMaps maps, int bands)
{
    extern __shared__ __align__(128) unsigned char ring_raw[];
    const RingShared<S, T, R, RING_W, HB> sh = ring_shared<S, T, R, RING_W, HB>(ring_raw);
    if (threadIdx.x == 0) {
        asm volatile("prefetch.tensormap [%0];" ::"l"(&maps.row[0]) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&maps.row[1]) : "memory");
    }
    const int band = blockIdx.y;
    const int y0 = (int)((long long)band * a.ny / bands);
    const int nrow = (int)((long long)(band + 1) * a.ny / bands) - y0;
    uint32_t g = 0;
    (void)ring_unit<S, T, FLAGS, R, WIDE, RING_W, HB>(a, &maps.row[0], &maps.row[1], &maps.halo[0],
                                                      &maps.halo[1], blockIdx.x * RING_W, y0, nrow,
                                                      (band & 1) != 0, sh, g);
}

// A unit of the batched ring kernel: strip xb of rows [y0, y1) of domain dom;
// down: the march direction (alternating between a domain's bands).
struct RingUnit {
    int dom, xb, y0, y1, down, pad[3];
};

// Batched ring kernel: every CTA takes units from a shared counter (largest
// units first in the list) until the list is exhausted; the last CTA to finish
// resets the counters for the next launch (kernel boundaries order it).  No
// CTA waits on another.  doms and maps hold two entries per domain (buffer
// parity 0 and 1); the current unit's argument block is copied into shared
// memory.  counters: [0] the next unit, [1] CTAs finished.
template <typename S, typename T, int FLAGS, int R, int W>
__global__ void __launch_bounds__(W, (ring_min_ctas<T, FLAGS>() * (RING_W / W)))
    k_batch_ring(const Fused2Args<S, T> *__restrict__ doms, const RingMaps *__restrict__ maps,
                 const RingUnit *__restrict__ units, int nunits, int parity, unsigned *counters)
{
    extern __shared__ __align__(128) unsigned char ring_raw[];
    __shared__ __align__(16) Fused2Args<S, T> sa;
    __shared__ int s_next;
    static_assert(sizeof(Fused2Args<S, T>) % 4 == 0, "argument block copied as words");
    const RingShared<S, T, R, W> sh = ring_shared<S, T, R, W>(ring_raw);
    uint32_t g = 0;
    int loaded = -1;
    for (;;) {
        if (threadIdx.x == 0) s_next = (int)atomicAdd(&counters[0], 1u);
        __syncthreads();
        const int i = s_next;
        if (i >= nunits) break;
        const RingUnit u = units[i];
        const int key = 2 * u.dom + parity;
        if (key != loaded) { // uniform over the CTA
            const uint32_t *src = reinterpret_cast<const uint32_t *>(doms + key);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&sa);
            for (int w = threadIdx.x; w < (int)(sizeof(sa) / 4); w += W) dst[w] = src[w];
            __syncthreads();
            loaded = key;
        }
        const RingMaps *m = maps + key;
        const bool ok = ring_unit<S, T, FLAGS, R, false, W>(sa, &m->row[0], &m->row[1], &m->halo[0],
                                                          &m->halo[1], u.xb, u.y0, u.y1 - u.y0,
                                                          u.down != 0, sh, g);
        __syncthreads(); // the ring, s_next and the argument block are reused by the next unit
        if (!ok) break;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&counters[1], 1u) == gridDim.x - 1) { // the last CTA out
            counters[0] = 0;
            counters[1] = 0;
        }
    }
}

// tensor maps of the input populations of both components (host)
template <typename S, typename T, int R, int W = RING_W>
inline cudaError_t ring_maps(const Fused2Args<S, T> &a, RingMaps &m)
{
    using L = RingLayout<S, T, R, W>;
    const CUtensorMapDataType dt = sizeof(S) == 8   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                   : sizeof(S) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                                    : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    const cuuint64_t dim[3] = {(cuuint64_t)a.nx, (cuuint64_t)a.ny, 9};
    const cuuint64_t stride[2] = {(cuuint64_t)a.nx * sizeof(S), (cuuint64_t)a.N * sizeof(S)};
    const cuuint32_t row_box[3] = {(cuuint32_t)L::P, 1, 9}, halo_box[3] = {(cuuint32_t)L::A, 1, 9};
    const cuuint32_t es[3] = {1, 1, 1};
    for (int k = 0; k < 2; ++k) {
        int rc = encode_tensor_map(&m.row[k], dt, 3, (void *)a.fin[k], dim, stride, row_box, es);
        if (!rc) rc = encode_tensor_map(&m.halo[k], dt, 3, (void *)a.fin[k], dim, stride, halo_box, es);
        if (rc) return cudaErrorInvalidValue;
    }
    return cudaSuccess;
}

// rows: rows per band (0: RING_ROWS; the domain's default choice passes its
// own per-precision height).  Short bands give 4096^2 lattices several waves
// of CTAs, which lets the block scheduler even out bands whose fluid nodes,
// and so whose work, differ: on porous 4096^2 lattices one wave of tall bands
// ran 5-25 % slower than 32-row bands, 128-row bands 3-14 % slower (FP32 and
// FP64, disks of radius 8-20 at 60 % fluid and 2-8 at 72 %).
constexpr int RING_ROWS = 32;
template <typename S, typename T, int FLAGS, int R, bool WIDE, bool HB>
inline cudaError_t launch_ring2_f(const Fused2Args<S, T> &a, int rows, cudaStream_t s)
{
    using L = RingLayout<S, T, R, RING_W, HB>;
    auto kern = k_ring2<S, T, FLAGS, R, WIDE, HB>;
    static int per_sm = 0; // resident CTAs per SM of this instantiation (one device): >= 1 checked once
    if (per_sm == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::bytes);
        if (e != cudaSuccess) return e;
        int n = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, RING_W, L::bytes);
        if (e != cudaSuccess) return e;
        if (n < 1) return cudaErrorInvalidConfiguration;
        per_sm = n;
    }
    const int strips = (a.nx + RING_W - 1) / RING_W;
    const int r = rows > 0 ? rows : RING_ROWS;
    int bands = (a.ny + r - 1) / r;
    bands = std::min(bands, std::max(1, a.ny / 4)); // at least 4 rows a band
    bands = std::min(bands, 65535);                 // grid y limit
    RingMaps maps;
    const cudaError_t em = ring_maps<S, T, R>(a, maps);
    if (em != cudaSuccess) return em;
    kern<<<dim3(strips, bands), RING_W, L::bytes, s>>>(a, maps, bands);
    return cudaGetLastError();
}

// the ring needs rows that start on 16-byte boundaries: nx a multiple of
// 16 / sizeof(S) (buffers from cudaMalloc are 256-byte aligned)
template <typename S> inline bool ring_fits(int nx) { return nx % ring_pad<S>() == 0; }

// UNI: lattices with solid nodes run the uniform solid form (KF_UNIFORM);
// HB: halo boxes in the stages (else edge columns from global memory)
template <typename S, typename T, int R, int UNI = KF_UNIFORM, bool HB = true>
inline cudaError_t launch_ring2_any(const Fused2Args<S, T> &a, int rows, cudaStream_t s)
{
    if (!ring_fits<S>(a.nx) || a.nx < 1 || a.ny < 1) return cudaErrorInvalidValue;
    if (needs_wide_offsets(a.N))
        return launch_ring2_f<S, T, KF_FORCE | KF_SOLID | UNI, R, true, HB>(a, rows, s);
    switch (kernel_flags(a)) {
    case 0: return launch_ring2_f<S, T, 0, R, false, HB>(a, rows, s);
    case KF_FORCE: return launch_ring2_f<S, T, KF_FORCE, R, false, HB>(a, rows, s);
    case KF_SOLID: return launch_ring2_f<S, T, KF_SOLID | UNI, R, false, HB>(a, rows, s);
    default: return launch_ring2_f<S, T, KF_FORCE | KF_SOLID | UNI, R, false, HB>(a, rows, s);
    }
}

// ---------------------------------------------------------------- batches
// UNI: the uniform solid form for batches holding solid nodes (FP32/FP16)
template <typename S, typename T, int R, int UNI, int FLAGS, int W>
inline cudaError_t batch_ring_prepare_f(int *per_sm)
{
    using L = RingLayout<S, T, R, W>;
    auto kern = k_batch_ring<S, T, FLAGS, R, W>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::bytes);
    if (e != cudaSuccess) return e;
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, W, L::bytes);
    if (per_sm) *per_sm = n;
    return e;
}

// sets the shared-memory limit of every body the batch may run (outside any
// graph capture) and returns the resident CTAs per SM of the solid body
template <typename S, typename T, int R, int UNI, int W>
inline cudaError_t batch_ring_prepare(int *per_sm)
{
    cudaError_t e = batch_ring_prepare_f<S, T, R, UNI, 0, W>(nullptr);
    if (e == cudaSuccess) e = batch_ring_prepare_f<S, T, R, UNI, KF_FORCE, W>(nullptr);
    if (e == cudaSuccess) e = batch_ring_prepare_f<S, T, R, UNI, KF_FORCE | KF_SOLID | UNI, W>(per_sm);
    return e;
}

template <typename S, typename T, int R, int UNI, int W>
inline cudaError_t launch_batch_ring(const Fused2Args<S, T> *doms, const RingMaps *maps,
                                     const RingUnit *units, int nunits, int parity, int grid, int flags,
                                     unsigned *counters, cudaStream_t s)
{
    using L = RingLayout<S, T, R, W>;
    if (flags & KF_SOLID)
        k_batch_ring<S, T, KF_FORCE | KF_SOLID | UNI, R, W><<<grid, W, L::bytes, s>>>(
            doms, maps, units, nunits, parity, counters);
    else if (flags == KF_FORCE)
        k_batch_ring<S, T, KF_FORCE, R, W><<<grid, W, L::bytes, s>>>(doms, maps, units, nunits, parity,
                                                                      counters);
    else
        k_batch_ring<S, T, 0, R, W><<<grid, W, L::bytes, s>>>(doms, maps, units, nunits, parity, counters);
    return cudaGetLastError();
}

} // namespace sclbm
