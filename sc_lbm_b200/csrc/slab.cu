// slab.cu -- halo rows of a slab domain, for lattices cut into row slabs
// across GPUs (or several slabs on one GPU).
//
// A slab owning global rows [y0, y1) is stepped as a periodic domain of
// y1 - y0 + 2H rows: H ghost rows copied from each neighbour slab above and
// below its own rows.  One fused step reads the densities of rows y-1..y+1
// and pushes into rows y-1..y+1, so the rows within two of the domain's edge
// are wrong after a step (they were computed from the periodic wrap of the
// slab, not of the lattice) and the owned rows are exact as long as H >= 2k
// for k steps between exchanges.  The exchange copies the first (last) H
// owned rows of every population array to the neighbour below (above), where
// they become its upper (lower) ghost rows.  Results are then bit-identical
// to stepping the whole lattice: every owned node sees the same inputs and
// runs the same arithmetic.  The reference's own MATLAB generator cuts its
// lattices the same way (one exchange of the crossing populations and a
// density row per step, tests/lbm/lbm_matlab/two_phase_flow/main_droplet.m).
//
// Halo buffers hold [component][direction][H rows][nx] values of the storage
// type, contiguous: one gather (pack) or scatter (unpack) launch per side.
#include <algorithm>
#include <cstdint>

#include "domain.h"

using namespace sclbm;

namespace {

template <typename W>
__global__ void k_halo(W *__restrict__ f0, W *__restrict__ f1, W *__restrict__ buf, size_t N,
                       size_t row0, size_t nx, size_t H, int ncomp, int unpack)
{
    const size_t per_dir = H * nx, per_comp = 9 * per_dir, total = (size_t)ncomp * per_comp;
    for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < total;
         j += (size_t)gridDim.x * blockDim.x) {
        const size_t c = j / per_comp, r = j - c * per_comp;
        const size_t i = r / per_dir, o = r - i * per_dir;
        W *f = c ? f1 : f0;
        const size_t e = i * N + row0 * nx + o;
        if (unpack) f[e] = buf[j];
        else buf[j] = f[e];
    }
}

int halo_copy(sclbm_domain *d, int rows, int side, void *buf, bool unpack)
{
    if (!d || !buf) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    if (side != 0 && side != 1) return set_error(SCLBM_E_INVALID_ARGUMENT, "side is 0 (below) or 1 (above)");
    const size_t H = (size_t)rows;
    if (rows < 1 || 3 * H > d->ny)
        return set_error(SCLBM_E_OUT_OF_RANGE, "halo rows must be >= 1 and at most a third of the slab's rows");
    // pack: the first (side 0) or last (side 1) H owned rows; unpack: the
    // ghost rows below (side 0) or above (side 1) the owned rows
    const size_t row0 = unpack ? (side ? d->ny - H : 0) : (side ? d->ny - 2 * H : H);
    const size_t total = (size_t)d->ncomp * 9 * H * d->nx;
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((total + threads - 1) / threads, 148 * 16);
    void *f0 = d->buf[d->parity][0], *f1 = d->ncomp > 1 ? d->buf[d->parity][1] : f0;
    cudaStream_t s = stream();
    switch (elem_size(d->prec)) {
    case 8:
        k_halo<uint64_t><<<blocks, threads, 0, s>>>((uint64_t *)f0, (uint64_t *)f1, (uint64_t *)buf,
                                                    d->N, row0, d->nx, H, d->ncomp, unpack);
        break;
    case 4:
        k_halo<uint32_t><<<blocks, threads, 0, s>>>((uint32_t *)f0, (uint32_t *)f1, (uint32_t *)buf,
                                                    d->N, row0, d->nx, H, d->ncomp, unpack);
        break;
    default:
        k_halo<uint16_t><<<blocks, threads, 0, s>>>((uint16_t *)f0, (uint16_t *)f1, (uint16_t *)buf,
                                                    d->N, row0, d->nx, H, d->ncomp, unpack);
        break;
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "halo copy");
    return SCLBM_OK;
}

// ------------------------------------------------------- per-step exchange
// One ghost row per side, exchanged after every step, nine values per
// component and column per side (the scheme above moves whole rows).  Which
// slab computed a population slot correctly depends on where it came from:
// slot (j, y, x) is pushed from the node upstream, (x, y) - c_j, when that node
// is fluid, and is the node's own bounce-back otherwise.  Lower cut of a slab
// (local row 0 = ghost row, row 1 = first owned row), after a step:
//   * row 1 lacks the three directions entering from below (2, 5, 6) where
//     the upstream node in row 0 is fluid -- the ghost row's collision saw a
//     wrong stencil; where it is solid the slot is row 1's own bounce-back;
//   * row 0 is right only in the directions pushed down from row 1 (4, 7, 8)
//     where their upstream node in row 1 is fluid.
// The slab below computed the rest: its top owned row (our row 0) in full,
// and in its upper ghost row (our row 1) the crossing pushes.  It sends
//   slots 0-5: its top row's directions 0, 1, 3, 2, 5, 6 (our row 0's);
//   slots 6-8: per pair (cross, bounce, shift) = (2, 4, 0), (5, 7, -1),
//     (6, 8, +1): at column x, where our row-1 node x is fluid, the crossing
//     value (cross, row 1, x); where it is solid, the bounce-back value
//     (bounce, row 0, x + shift), whose upstream node is exactly (x, row 1).
// The two are never both needed at one x, so nine values carry everything;
// the receiver writes a crossing value only where its upstream node in row 0
// is fluid (elsewhere the slot is its own bounce-back).  The upper cut mirrors
// it with directions 0, 1, 3, 4, 7, 8 and pairs (4, 2, 0), (7, 5, +1),
// (8, 6, -1).  Every slot then holds what one domain holding the whole lattice
// would hold: owned rows stay bit-identical.  Buffer [component][9][nx].
__constant__ int kRowUp[6] = {0, 1, 3, 2, 5, 6};   // the slab above's ghost row from our top row
__constant__ int kRowDown[6] = {0, 1, 3, 4, 7, 8}; // the slab below's ghost row from our bottom row
// pairs at the lower cut of the receiving slab: crossing into row 1, bounce-back in row 0
__constant__ int kLowCross[3] = {2, 5, 6}, kLowBounce[3] = {4, 7, 8}, kLowShift[3] = {0, -1, 1};
// pairs at the upper cut: crossing into row n, bounce-back in row n + 1
__constant__ int kUpCross[3] = {4, 7, 8}, kUpBounce[3] = {2, 5, 6}, kUpShift[3] = {0, 1, -1};
__constant__ int kCx[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};

// pack side 0 (to the slab below, which unpacks it at its upper cut): rows
// n_recv = our 0, n_recv + 1 = our 1;  pack side 1 (to the slab above, unpacked
// at its lower cut): its row 0 = our n, its row 1 = our n + 1.
template <typename W>
__global__ void k_halo_min(W *__restrict__ f0, W *__restrict__ f1, W *__restrict__ buf,
                           const uint8_t *__restrict__ mask, size_t N, size_t nx, size_t ny, int ncomp,
                           int side, int unpack)
{
    const size_t per_comp = 9 * nx, total = (size_t)ncomp * per_comp;
    const size_t n = ny - 2; // owned rows 1..n
    for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < total; j += (size_t)gridDim.x * blockDim.x) {
        const size_t c = j / per_comp, r = j - c * per_comp;
        const int slot = (int)(r / nx);
        const size_t x = r - (size_t)slot * nx;
        W *f = c ? f1 : f0;
        auto at = [&](int dir, size_t row, size_t col) { return (size_t)dir * N + row * nx + col; };
        auto wrapx = [&](long long v) { return (size_t)((v % (long long)nx + (long long)nx) % (long long)nx); };
        if (slot < 6) {
            // whole-row values: pack our boundary row, unpack into our ghost row
            size_t row;
            int dir;
            if (!unpack) {
                dir = side == 0 ? kRowDown[slot] : kRowUp[slot];
                row = side == 0 ? 1 : n;
            } else {
                dir = side == 0 ? kRowUp[slot] : kRowDown[slot];
                row = side == 0 ? 0 : n + 1;
            }
            if (unpack) f[at(dir, row, x)] = buf[j];
            else buf[j] = f[at(dir, row, x)];
            continue;
        }
        const int p = slot - 6;
        if (!unpack) {
            // the receiver's first row across the cut is our ghost row (side 0:
            // row 0, paired with our row 1; side 1: row n + 1, paired with row n)
            const size_t rx = side == 0 ? 0 : n + 1, rb = side == 0 ? 1 : n;
            const int cross = side == 0 ? kUpCross[p] : kLowCross[p];
            const int bounce = side == 0 ? kUpBounce[p] : kLowBounce[p];
            const int shift = side == 0 ? kUpShift[p] : kLowShift[p];
            buf[j] = mask[rx * nx + x] ? f[at(cross, rx, x)] : f[at(bounce, rb, wrapx((long long)x + shift))];
        } else {
            // side 0: lower cut (row 1 owned, row 0 ghost); side 1: upper cut
            const size_t ro = side == 0 ? 1 : n, rg = side == 0 ? 0 : n + 1;
            const int cross = side == 0 ? kLowCross[p] : kUpCross[p];
            const int bounce = side == 0 ? kLowBounce[p] : kUpBounce[p];
            const int shift = side == 0 ? kLowShift[p] : kUpShift[p];
            if (mask[ro * nx + x]) {
                // crossing value, unless the upstream node (in the ghost row) is solid
                if (mask[rg * nx + wrapx((long long)x - kCx[cross])]) f[at(cross, ro, x)] = buf[j];
            } else {
                f[at(bounce, rg, wrapx((long long)x + shift))] = buf[j];
            }
        }
    }
}

int halo_min_copy(sclbm_domain *d, int side, void *buf, bool unpack)
{
    if (!d || !buf) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    if (side != 0 && side != 1) return set_error(SCLBM_E_INVALID_ARGUMENT, "side is 0 (below) or 1 (above)");
    if (d->ny < 3) return set_error(SCLBM_E_OUT_OF_RANGE, "a slab needs one owned row and two ghost rows");
    const size_t total = (size_t)d->ncomp * 9 * d->nx;
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((total + threads - 1) / threads, 148 * 16);
    void *f0 = d->buf[d->parity][0], *f1 = d->ncomp > 1 ? d->buf[d->parity][1] : f0;
    cudaStream_t s = stream();
    switch (elem_size(d->prec)) {
    case 8:
        k_halo_min<uint64_t><<<blocks, threads, 0, s>>>((uint64_t *)f0, (uint64_t *)f1, (uint64_t *)buf,
                                                        d->d_mask, d->N, d->nx, d->ny, d->ncomp, side, unpack);
        break;
    case 4:
        k_halo_min<uint32_t><<<blocks, threads, 0, s>>>((uint32_t *)f0, (uint32_t *)f1, (uint32_t *)buf,
                                                        d->d_mask, d->N, d->nx, d->ny, d->ncomp, side, unpack);
        break;
    default:
        k_halo_min<uint16_t><<<blocks, threads, 0, s>>>((uint16_t *)f0, (uint16_t *)f1, (uint16_t *)buf,
                                                        d->d_mask, d->N, d->nx, d->ny, d->ncomp, side, unpack);
        break;
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "halo copy");
    return SCLBM_OK;
}

} // namespace

extern "C" size_t sclbm_domain_halo_min_bytes(const sclbm_domain *d)
{
    if (!d) return 0;
    return (size_t)d->ncomp * 9 * d->nx * elem_size(d->prec);
}

extern "C" int sclbm_domain_halo_min_pack(sclbm_domain *d, int side, void *dst)
{
    return halo_min_copy(d, side, dst, false);
}

extern "C" int sclbm_domain_halo_min_unpack(sclbm_domain *d, int side, const void *src)
{
    return halo_min_copy(d, side, const_cast<void *>(src), true);
}

extern "C" size_t sclbm_domain_halo_bytes(const sclbm_domain *d, int rows)
{
    if (!d || rows < 1) return 0;
    return (size_t)d->ncomp * 9 * (size_t)rows * d->nx * elem_size(d->prec);
}

extern "C" int sclbm_domain_halo_pack(sclbm_domain *d, int rows, int side, void *dst)
{
    return halo_copy(d, rows, side, dst, false);
}

extern "C" int sclbm_domain_halo_unpack(sclbm_domain *d, int rows, int side, const void *src)
{
    return halo_copy(d, rows, side, const_cast<void *>(src), true);
}
