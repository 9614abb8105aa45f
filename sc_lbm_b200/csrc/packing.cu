// packing.cu -- seeded porous media built on the device: the random
// sequential addition of non-overlapping disks of sclbm_geometry_add_random_disks
// (capi.cu), run in speculative batches so that the result is the host
// packer's, disk for disk, while the lattice-sized work (occupancy tests,
// occupancy marking, rasterisation into the mask) runs on the GPU.
//
// Why it can be batched: every trial draws exactly three numbers (radius,
// centre x, centre y) from the splitmix64 stream at indices 3t .. 3t + 2,
// accepted or not, so trial t's disk is known without running trials 0..t-1.
// Whether it is accepted depends on the disks accepted before it, and the
// loop's stopping rules (solid target, tries, consecutive misses) on the
// accept/reject sequence.  A batch of B trials is therefore:
//   1. device: each trial's disk and its test against the occupancy grid of
//      the disks accepted in earlier batches (the walls and existing solids
//      included) -- a warp per trial scans the disk's bounding box;
//   2. host: the trials in order, applying the stopping rules exactly as the
//      host packer does, and rejecting a trial that conflicts with a disk
//      accepted earlier in the same batch (the same cell-level test: a cell
//      of the lattice within r + 1.5 of both centres);
//   3. device: the accepted disks' occupancy marked for the next batch.
// Finally every accepted disk is rasterised into the domain's mask with the
// reference's integer circle (Ellipse::find_nodes with Lx = Ly = 2r + 1,
// src/geom_object/ellipse.cpp:12-34; add_circle, src/geometry.cpp:132-147)
// and the populations of the new solid nodes are zeroed in both buffers, the
// domain path's invariant.
#include <algorithm>
#include <cmath>
#include <vector>

#include "domain.h"

namespace sclbm {
namespace {

constexpr int PACK_BATCH = 8192; // trials per speculative batch

__host__ __device__ inline double pack_u01(uint64_t seed, uint64_t k)
{
    uint64_t z = k + seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// integer in [lo, hi] as the host packer draws it (truncation toward zero)
__host__ __device__ inline long long pack_int(uint64_t seed, uint64_t k, long long lo, long long hi)
{
    const double u = pack_u01(seed, k);
    const long long n = (long long)(u * (double)(hi - lo + 1));
    return lo + (hi - lo < n ? hi - lo : n);
}

struct Disk {
    long long r, xc, yc;
};

__host__ __device__ inline Disk pack_trial(uint64_t seed, long long t, int rmin, int rmax, long long nx,
                                           long long ny, int wall_rows)
{
    Disk d;
    d.r = pack_int(seed, 3 * (uint64_t)t, rmin, rmax);
    d.xc = pack_int(seed, 3 * (uint64_t)t + 1, d.r, nx - 1 - d.r);
    d.yc = pack_int(seed, 3 * (uint64_t)t + 2, d.r + wall_rows, ny - 1 - d.r - wall_rows);
    return d;
}

__host__ __device__ inline bool pack_inside(const Disk &d, long long nx, long long ny)
{
    return !(d.xc - d.r < 0 || d.yc - d.r < 0 || d.xc + d.r >= nx || d.yc + d.r >= ny);
}

// status: 0 outside the bounds, 1 hits the occupancy grid, 2 clear
__global__ void k_pack_trials(uint64_t seed, long long t0, int count, int rmin, int rmax, long long nx,
                              long long ny, int wall_rows, const uint8_t *__restrict__ occ,
                              int8_t *__restrict__ status)
{
    const int w = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= count) return; // whole warps leave together
    const Disk d = pack_trial(seed, t0 + w, rmin, rmax, nx, ny, wall_rows);
    if (!pack_inside(d, nx, ny)) {
        if (lane == 0) status[w] = 0;
        return;
    }
    const long long y0 = max(0LL, d.yc - d.r - 1), y1 = min(ny, d.yc + d.r + 2);
    const long long x0 = max(0LL, d.xc - d.r - 1), x1 = min(nx, d.xc + d.r + 2);
    const double lim = ((double)d.r + 1.5) * ((double)d.r + 1.5);
    const long long bw = x1 - x0, cells = bw * (y1 - y0);
    bool hit = false;
    for (long long c = lane; c < cells && !hit; c += 32) {
        const long long y = y0 + c / bw, x = x0 + c % bw;
        hit = (double)((y - d.yc) * (y - d.yc) + (x - d.xc) * (x - d.xc)) <= lim && occ[y * nx + x];
    }
    hit = __any_sync(0xffffffffu, hit);
    if (lane == 0) status[w] = hit ? 1 : 2;
}

// occupancy (cells within r + 1.5 of the centre) of the accepted disks; one
// block per disk
__global__ void k_pack_mark(const long long *__restrict__ disks, long long nx, long long ny,
                            uint8_t *__restrict__ occ)
{
    const long long r = disks[3 * blockIdx.x], xc = disks[3 * blockIdx.x + 1], yc = disks[3 * blockIdx.x + 2];
    const long long y0 = max(0LL, yc - r - 1), y1 = min(ny, yc + r + 2);
    const long long x0 = max(0LL, xc - r - 1), x1 = min(nx, xc + r + 2);
    const double lim = ((double)r + 1.5) * ((double)r + 1.5);
    const long long bw = x1 - x0, cells = bw * (y1 - y0);
    for (long long c = threadIdx.x; c < cells; c += blockDim.x) {
        const long long y = y0 + c / bw, x = x0 + c % bw;
        if ((double)((y - yc) * (y - yc) + (x - xc) * (x - xc)) <= lim) occ[y * nx + x] = 1;
    }
}

// Rasterise the circle of diameter D = 2r + 1 around (xc, yc) with the
// reference's integer ellipse test (Lx = Ly = D, odd, so no shrinking):
//   dx^2 Ly^2 / 4 + dy^2 Lx^2 / 4 <= Lx^2 Ly^2 / 16   (unsigned 64-bit, as
// size_t in the reference; a negative offset squares to the same value), set
// the node solid and zero its populations in both buffers of every component.
template <typename S>
__global__ void k_pack_raster(const long long *__restrict__ disks, long long nx, size_t N,
                              uint8_t *__restrict__ mask, S *__restrict__ a0, S *__restrict__ a1,
                              S *__restrict__ b0, S *__restrict__ b1)
{
    const long long r = disks[3 * blockIdx.x], xc = disks[3 * blockIdx.x + 1], yc = disks[3 * blockIdx.x + 2];
    const unsigned long long L = (unsigned long long)(2 * r + 1);
    const unsigned long long rhs = L * L * L * L / 16;
    const long long side = 2 * r + 1, cells = side * side;
    for (long long c = threadIdx.x; c < cells; c += blockDim.x) {
        const long long ix = xc - r + c % side, iy = yc - r + c / side;
        const unsigned long long dx = (unsigned long long)(ix - xc), dy = (unsigned long long)(iy - yc);
        if (dx * dx * L * L / 4 + dy * dy * L * L / 4 <= rhs) {
            const size_t node = (size_t)iy * (size_t)nx + (size_t)ix;
            mask[node] = 0;
            for (int i = 0; i < 9; ++i) {
                a0[i * N + node] = S(0.0f);
                b0[i * N + node] = S(0.0f);
                if (a1) {
                    a1[i * N + node] = S(0.0f);
                    b1[i * N + node] = S(0.0f);
                }
            }
        }
    }
}

__global__ void k_pack_occ_init(size_t N, const uint8_t *__restrict__ mask, uint8_t *__restrict__ occ,
                                unsigned long long *__restrict__ solids)
{
    unsigned long long n = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const uint8_t s = mask[i] == 0;
        occ[i] = s;
        n += s;
    }
    for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(solids, n);
}

// the cell-level conflict of two disks' occupancy regions (cells of the
// lattice within r + 1.5 of both centres)
bool pack_conflict(const Disk &a, const Disk &b, long long nx, long long ny)
{
    const long long dx = a.xc - b.xc, dy = a.yc - b.yc, reach = a.r + b.r + 3;
    if (dx > reach || -dx > reach || dy > reach || -dy > reach) return false;
    const long long y0 = std::max({0LL, a.yc - a.r - 1, b.yc - b.r - 1});
    const long long y1 = std::min({ny, a.yc + a.r + 2, b.yc + b.r + 2});
    const long long x0 = std::max({0LL, a.xc - a.r - 1, b.xc - b.r - 1});
    const long long x1 = std::min({nx, a.xc + a.r + 2, b.xc + b.r + 2});
    const double la = ((double)a.r + 1.5) * ((double)a.r + 1.5), lb = ((double)b.r + 1.5) * ((double)b.r + 1.5);
    for (long long y = y0; y < y1; ++y)
        for (long long x = x0; x < x1; ++x)
            if ((double)((y - a.yc) * (y - a.yc) + (x - a.xc) * (x - a.xc)) <= la &&
                (double)((y - b.yc) * (y - b.yc) + (x - b.xc) * (x - b.xc)) <= lb)
                return true;
    return false;
}

struct DevBuf {
    void *p = nullptr;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
};

} // namespace
} // namespace sclbm

using namespace sclbm;

extern "C" int sclbm_domain_add_random_disks(sclbm_domain *d, double porosity, int rmin, int rmax,
                                             uint64_t seed, int wall_rows, long max_tries, long max_misses,
                                             size_t *placed)
{
    if (!d) return set_error(SCLBM_E_INVALID_ARGUMENT, "null domain");
    if (rmin < 0 || rmax < rmin || !(porosity >= 0.0 && porosity <= 1.0) || wall_rows < 0)
        return set_error(SCLBM_E_INVALID_ARGUMENT, "bad disk parameters");
    const long long nx = (long long)d->nx, ny = (long long)d->ny;
    const size_t N = d->N;
    cudaStream_t s = stream();
    DevBuf occ, status, list, count;
    SCLBM_CUDA(cudaMalloc(&occ.p, N));
    SCLBM_CUDA(cudaMalloc(&status.p, PACK_BATCH));
    SCLBM_CUDA(cudaMalloc(&count.p, sizeof(unsigned long long)));
    SCLBM_CUDA(cudaMemsetAsync(count.p, 0, sizeof(unsigned long long), s));
    k_pack_occ_init<<<grid_for(N, 256), 256, 0, s>>>(N, d->d_mask, (uint8_t *)occ.p,
                                                    (unsigned long long *)count.p);
    SCLBM_LAUNCHED("packing: occupancy");
    unsigned long long nsolid = 0;
    SCLBM_CUDA(cudaMemcpyAsync(&nsolid, count.p, sizeof(nsolid), cudaMemcpyDeviceToHost, s));
    SCLBM_CUDA(cudaStreamSynchronize(s));

    // the loop of the host packer, over speculative batches of trials
    double solid = (double)nsolid;
    const double target = (1.0 - porosity) * (double)nx * (double)ny;
    long tries = 0, misses = 0;
    long long t0 = 0;
    std::vector<long long> all;      // r, xc, yc of every accepted disk, in order
    std::vector<int8_t> st(PACK_BATCH);
    size_t list_cap = 0;
    bool done = !(solid < target && tries < max_tries && misses < max_misses);
    while (!done) {
        const int B = PACK_BATCH;
        k_pack_trials<<<(B * 32 + 255) / 256, 256, 0, s>>>(seed, t0, B, rmin, rmax, nx, ny, wall_rows,
                                                           (const uint8_t *)occ.p, (int8_t *)status.p);
        SCLBM_LAUNCHED("packing: trials");
        SCLBM_CUDA(cudaMemcpyAsync(st.data(), status.p, B, cudaMemcpyDeviceToHost, s));
        SCLBM_CUDA(cudaStreamSynchronize(s));
        std::vector<Disk> batch; // accepted in this batch
        for (int w = 0; w < B; ++w) {
            if (!(solid < target && tries < max_tries && misses < max_misses)) {
                done = true;
                break;
            }
            ++tries;
            ++misses;
            if (st[w] != 2) continue;
            const Disk dk = pack_trial(seed, t0 + w, rmin, rmax, nx, ny, wall_rows);
            bool hit = false;
            for (const Disk &o : batch)
                if (pack_conflict(dk, o, nx, ny)) {
                    hit = true;
                    break;
                }
            if (hit) continue;
            batch.push_back(dk);
            misses = 0;
            solid += M_PI * (((double)dk.r + 0.5) * ((double)dk.r + 0.5));
        }
        t0 += B;
        if (batch.empty()) continue;
        const size_t first = all.size();
        for (const Disk &dk : batch) {
            all.push_back(dk.r);
            all.push_back(dk.xc);
            all.push_back(dk.yc);
        }
        if (!done) { // the next batch tests against these disks' occupancy
            if (all.size() > list_cap) {
                if (list.p) cudaFree(list.p);
                list.p = nullptr;
                list_cap = std::max(all.size() * 2, (size_t)3 * 4096);
                SCLBM_CUDA(cudaMalloc(&list.p, list_cap * sizeof(long long)));
            }
            SCLBM_CUDA(cudaMemcpyAsync((long long *)list.p + first, all.data() + first,
                                       (all.size() - first) * sizeof(long long), cudaMemcpyHostToDevice, s));
            k_pack_mark<<<(unsigned)batch.size(), 128, 0, s>>>((const long long *)list.p + first, nx, ny,
                                                              (uint8_t *)occ.p);
            SCLBM_LAUNCHED("packing: occupancy marks");
        }
    }
    const size_t ndisks = all.size() / 3;
    if (ndisks) {
        if (all.size() > list_cap) {
            if (list.p) cudaFree(list.p);
            list.p = nullptr;
            SCLBM_CUDA(cudaMalloc(&list.p, all.size() * sizeof(long long)));
        }
        SCLBM_CUDA(cudaMemcpyAsync(list.p, all.data(), all.size() * sizeof(long long), cudaMemcpyHostToDevice, s));
        void *a0 = d->buf[0][0], *a1 = d->ncomp > 1 ? d->buf[0][1] : nullptr;
        void *b0 = d->buf[1][0], *b1 = d->ncomp > 1 ? d->buf[1][1] : nullptr;
        const long long *dl = (const long long *)list.p;
        switch (d->prec) {
        case SCLBM_FP64:
            k_pack_raster<double><<<(unsigned)ndisks, 128, 0, s>>>(dl, nx, N, d->d_mask, (double *)a0,
                                                                  (double *)a1, (double *)b0, (double *)b1);
            break;
        case SCLBM_FP32_SHIFTED:
            k_pack_raster<float><<<(unsigned)ndisks, 128, 0, s>>>(dl, nx, N, d->d_mask, (float *)a0,
                                                                 (float *)a1, (float *)b0, (float *)b1);
            break;
        default:
            k_pack_raster<__half><<<(unsigned)ndisks, 128, 0, s>>>(dl, nx, N, d->d_mask, (__half *)a0,
                                                                  (__half *)a1, (__half *)b0, (__half *)b1);
            break;
        }
        SCLBM_LAUNCHED("packing: rasterisation");
        d->has_solid = true;
    }
    SCLBM_CUDA(cudaStreamSynchronize(s));
    if (placed) *placed = ndisks;
    return SCLBM_OK;
}

extern "C" int sclbm_domain_download_mask(sclbm_domain *d, int32_t *mask, size_t count)
{
    if (!d || !mask) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    if (count != d->N) return set_error(SCLBM_E_INVALID_ARGUMENT, "count must be nx*ny");
    std::vector<uint8_t> m(d->N);
    cudaStream_t s = stream();
    SCLBM_CUDA(cudaMemcpyAsync(m.data(), d->d_mask, d->N, cudaMemcpyDeviceToHost, s));
    SCLBM_CUDA(cudaStreamSynchronize(s));
    for (size_t i = 0; i < d->N; ++i) mask[i] = m[i];
    return SCLBM_OK;
}
