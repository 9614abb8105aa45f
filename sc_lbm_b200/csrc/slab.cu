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

} // namespace

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
