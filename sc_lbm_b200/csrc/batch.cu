// batch.cu -- many independent two-component domains advanced together, one
// persistent launch per time step, the launches of a run captured once into a
// CUDA graph and replayed.  All domains of a batch share the storage precision
// and the buffer parity.  Two work decompositions:
//
//  * bands (FP64/FP32): every domain is cut into 128-column strips and row
//    bands of one common height, chosen as the smallest for which all
//    (domain, strip, band) tiles are resident at once; neighbouring strips of
//    a band are adjacent in the list so they walk the same rows together; the
//    pipelined single-pass body (fused_async.cuh) runs each tile;
//  * tile list: every tile (126 columns x tile_y rows) of every domain,
//    largest first; CTA b takes tiles b, b+grid, ... and runs the
//    register-tile body (batch_kernel.cuh).
// The automatic choice and the rows per tile come from the autotuned size-class
// table (tuning.h), weighted by the nodes of each class in the batch.
#include <algorithm>
#include <numeric>

#include "domain.h"
#include "batch_kernel.cuh"
#include "fused_async.cuh"
#include "fused_ring.cuh"
#include "tuning.h"


using namespace sclbm;

static constexpr int GRAPH_STEPS = 20; // launches per captured graph (even: parity returns)

struct sclbm_batch {
    std::vector<sclbm_domain *> doms;
    sclbm_precision prec = SCLBM_FP32_SHIFTED;
    void *d_args = nullptr;  // Fused2Args<S,T>[2*ndom] (parity 0, parity 1)
    TileRef *d_tiles = nullptr;
    TileRef *d_tiles_half = nullptr; // 64-column tiles of the two-tiles-per-CTA body
    int ntiles_half = 0;
    TileRef *d_tiles_warp = nullptr; // 32-column tiles of the one-tile-per-warp body
    int ntiles_warp = 0;
    BandTile *d_bands = nullptr; // (domain, strip, band) tiles of the pipelined kernel
    int nbands = 0, band_grid = 0, band_rows = 0;
    int ntiles = 0, grid = 0, parity = 0;
    int use_units = 1;
    int auto_units = 1; // tuned choice for variant 0
    int body = BODY_TILE; // tile-list body: 2 register tile, 5 load ahead, 6 compacted, 8 uniform
    int auto_body = BODY_TILE; // tile-list body of variant 0
    int grid_body[BODY_COUNT] = {};  // resident grid of each body
    int flags = 0;                 // KF_FORCE / KF_SOLID if any domain needs them
    cudaGraphExec_t graph[2] = {nullptr, nullptr}; // by starting parity
    cudaStream_t graph_stream = nullptr;
    // ring bodies (variant 11: 128-column strips, 12: 64-column strips): units
    // of (domain, strip, band), tensor maps per domain and parity, the work
    // counters; absent when a domain's rows do not start on 16-byte boundaries
    bool ring = false;
    int use_ring = 0;  // 0, or the strip width of the ring body in use
    int auto_ring = 0; // the ring body of variant 0
    RingUnit *d_units[2] = {nullptr, nullptr}; // [0] 128 wide, [1] 64 wide
    RingMaps *d_maps[2] = {nullptr, nullptr};
    unsigned *d_counters = nullptr;
    int nunits[2] = {0, 0}, ring_grid[2] = {0, 0};
};

// the tile list of the current body
static const TileRef *batch_tiles(const sclbm_batch *b)
{
    return b->body == BODY_HALF ? b->d_tiles_half : b->body == BODY_WARP ? b->d_tiles_warp : b->d_tiles;
}
static int batch_ntiles(const sclbm_batch *b)
{
    return b->body == BODY_HALF ? b->ntiles_half : b->body == BODY_WARP ? b->ntiles_warp : b->ntiles;
}

static cudaError_t batch_launch_any(sclbm_batch *b, int parity, cudaStream_t s)
{
    if (b->use_ring) {
        const int w = b->use_ring, r = w == 64 ? 1 : 0;
        switch (b->prec) {
        case SCLBM_FP64:
            return launch_batch_ring_fp64((const Fused2Args<double, double> *)b->d_args, b->d_maps[r],
                                          b->d_units[r], b->nunits[r], parity, b->ring_grid[r], b->flags,
                                          b->d_counters, w, s);
        case SCLBM_FP32_SHIFTED:
            return launch_batch_ring_f32((const Fused2Args<float, float> *)b->d_args, b->d_maps[r],
                                         b->d_units[r], b->nunits[r], parity, b->ring_grid[r], b->flags,
                                         b->d_counters, w, s);
        default:
            return launch_batch_ring_f16((const Fused2Args<__half, float> *)b->d_args, b->d_maps[r],
                                         b->d_units[r], b->nunits[r], parity, b->ring_grid[r], b->flags,
                                         b->d_counters, w, s);
        }
    }
    if (b->use_units && b->prec == SCLBM_FP64)
        return launch_batch2_async_fp64((const Fused2Args<double, double> *)b->d_args, b->d_bands,
                                        b->nbands, b->band_grid, parity, s);
    if (b->use_units && b->prec == SCLBM_FP32_SHIFTED)
        return launch_batch2_async_f32((const Fused2Args<float, float> *)b->d_args, b->d_bands,
                                       b->nbands, b->band_grid, parity, s);
    switch (b->prec) {
    case SCLBM_FP64:
        return launch_batch_fp64((const Fused2Args<double, double> *)b->d_args, b->d_tiles,
                                 b->ntiles, parity, b->grid, b->flags, s);
    case SCLBM_FP32_SHIFTED:
        return launch_batch_f32((const Fused2Args<float, float> *)b->d_args, batch_tiles(b),
                                batch_ntiles(b), parity, b->grid_body[b->body], b->flags, b->body, s);
    default:
        return launch_batch_f16((const Fused2Args<__half, float> *)b->d_args, batch_tiles(b),
                                batch_ntiles(b), parity, b->grid_body[b->body], b->flags, b->body, s);
    }
}

// Ring bodies: every domain cut into strips `width` columns wide and bands of
// about `rows` rows (a domain's bands alternate their march direction),
// largest units first; tensor maps of both parities of every domain.
template <typename S, typename T>
static int build_ring(sclbm_batch *b, const std::vector<Fused2Args<S, T>> &h, const std::vector<int> &rows,
                      int width)
{
    const int r = width == 64 ? 1 : 0;
    std::vector<RingUnit> units;
    std::vector<long> cost;
    for (int k = 0; k < (int)b->doms.size(); ++k) {
        const sclbm_domain *d = b->doms[k];
        const int nb = std::max(1, (int)((d->ny + rows[k] / 2) / rows[k]));
        for (int j = 0; j < nb; ++j) {
            const int y0 = (int)((long long)d->ny * j / nb), y1 = (int)((long long)d->ny * (j + 1) / nb);
            for (int xb = 0; xb < (int)d->nx; xb += width) {
                units.push_back(RingUnit{k, xb, y0, y1, j & 1, {0, 0, 0}});
                cost.push_back((long)std::min(width, (int)d->nx - xb) * (y1 - y0 + 2));
            }
        }
    }
    // Largest first at domain granularity: a domain's units stay together in
    // band-major order, so vertically neighbouring bands (opposite march
    // directions) start within a few claims of each other and the halo rows
    // they share are read from L2 the second time; domains are ordered by
    // their largest unit.
    std::vector<long> dom_cost(b->doms.size(), 0);
    for (size_t i = 0; i < units.size(); ++i)
        dom_cost[units[i].dom] = std::max(dom_cost[units[i].dom], cost[i]);
    std::vector<int> order(units.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int c) { return dom_cost[units[a].dom] > dom_cost[units[c].dom]; });
    std::vector<RingUnit> sorted(units.size());
    for (size_t i = 0; i < order.size(); ++i) sorted[i] = units[order[i]];
    std::vector<RingMaps> maps(h.size());
    for (size_t i = 0; i < h.size(); ++i)
        if (ring_maps_of(h[i], width, &maps[i])) return set_error(SCLBM_E_CUDA, "tensor map encoding");
    int per_sm = 0;
    int rc = batch_ring_prepare(b->prec, width, &per_sm);
    if (rc) return rc;
    b->nunits[r] = (int)sorted.size();
    b->ring_grid[r] = std::max(1, std::min(b->nunits[r], std::max(1, per_sm) * sm_count()));
    SCLBM_CUDA(cudaMalloc(&b->d_units[r], sorted.size() * sizeof(RingUnit)));
    SCLBM_CUDA(cudaMemcpy(b->d_units[r], sorted.data(), sorted.size() * sizeof(RingUnit),
                          cudaMemcpyHostToDevice));
    SCLBM_CUDA(cudaMalloc(&b->d_maps[r], maps.size() * sizeof(RingMaps)));
    SCLBM_CUDA(cudaMemcpy(b->d_maps[r], maps.data(), maps.size() * sizeof(RingMaps), cudaMemcpyHostToDevice));
    return SCLBM_OK;
}

template <typename S, typename T>
static int build_rings(sclbm_batch *b, const std::vector<Fused2Args<S, T>> &h, const std::vector<int> &rows)
{
    const int A = 16 / (int)sizeof(S);
    for (auto *d : b->doms)
        if (d->nx % A != 0) return SCLBM_OK; // no ring body for this batch
    int rc = build_ring<S, T>(b, h, rows, 128);
    if (!rc) rc = build_ring<S, T>(b, h, rows, 64);
    if (rc) return rc;
    SCLBM_CUDA(cudaMalloc(&b->d_counters, 2 * sizeof(unsigned)));
    SCLBM_CUDA(cudaMemset(b->d_counters, 0, 2 * sizeof(unsigned)));
    b->ring = true;
    return SCLBM_OK;
}

// rows per unit of the ring body (a unit reads two halo rows), unless the
// caller gives tile_y per domain or the tuned batch default sets them
constexpr int RING_BATCH_ROWS = 32;

template <typename S, typename T>
static int upload_args(sclbm_batch *b, const std::vector<int> &ty, const std::vector<int> &ring_rows)
{
    std::vector<Fused2Args<S, T>> h(2 * b->doms.size());
    for (size_t k = 0; k < b->doms.size(); ++k) {
        sclbm_domain *d = b->doms[k];
        const int par = d->parity, saved_ty = d->tile_y;
        d->tile_y = ty[k];
        for (int p = 0; p < 2; ++p) {
            d->parity = p;
            Fused2Args<double, double> a64;
            Fused2Args<float, float> a32;
            Fused2Args<__half, float> a16;
            domain_fused2_args(d, &a64, &a32, &a16);
            if constexpr (sizeof(S) == 8) h[2 * k + p] = a64;
            else if constexpr (sizeof(S) == 4) h[2 * k + p] = a32;
            else h[2 * k + p] = a16;
        }
        d->parity = par;
        d->tile_y = saved_ty;
    }
    SCLBM_CUDA(cudaMalloc(&b->d_args, h.size() * sizeof(Fused2Args<S, T>)));
    SCLBM_CUDA(cudaMemcpy(b->d_args, h.data(), h.size() * sizeof(Fused2Args<S, T>),
                          cudaMemcpyHostToDevice));
    return build_rings<S, T>(b, h, ring_rows);
}

extern "C" {

void sclbm_batch_destroy(sclbm_batch *b)
{
    if (!b) return;
    for (auto &g : b->graph)
        if (g) cudaGraphExecDestroy(g);
    if (b->d_args) cudaFree(b->d_args);
    if (b->d_tiles) cudaFree(b->d_tiles);
    if (b->d_tiles_half) cudaFree(b->d_tiles_half);
    if (b->d_tiles_warp) cudaFree(b->d_tiles_warp);
    if (b->d_bands) cudaFree(b->d_bands);
    for (int r = 0; r < 2; ++r) {
        if (b->d_units[r]) cudaFree(b->d_units[r]);
        if (b->d_maps[r]) cudaFree(b->d_maps[r]);
    }
    if (b->d_counters) cudaFree(b->d_counters);
    delete b;
}

int sclbm_batch_create(sclbm_domain *const *domains, int ndomains, const int *tile_y_per_domain,
                       sclbm_batch **out)
{
    if (!domains || ndomains < 1 || !out) return set_error(SCLBM_E_INVALID_ARGUMENT, "bad batch");
    int rc = ensure_device();
    if (rc) return rc;
    auto *b = new (std::nothrow) sclbm_batch();
    if (!b) return set_error(SCLBM_E_ALLOC, "host allocation failed");
    b->doms.assign(domains, domains + ndomains);
    if (!b->doms[0]) {
        delete b;
        return set_error(SCLBM_E_INVALID_ARGUMENT, "null domain in batch");
    }
    b->prec = b->doms[0]->prec;
    b->parity = b->doms[0]->parity;
    std::vector<int> ty(ndomains);
    double nodes_units = 0.0, nodes_tiles = 0.0;
    const SclbmTunedShape bd = tuned_batch_default(b->prec);
    const bool bd_list = bd.variant == 2 || bd.variant == 8 || bd.variant == 9 || bd.variant == 10;
    for (int k = 0; k < ndomains; ++k) {
        sclbm_domain *d = b->doms[k];
        if (!d || d->ncomp != 2 || d->prec != b->prec || d->parity != b->parity) {
            sclbm_batch_destroy(b);
            return set_error(SCLBM_E_INVALID_ARGUMENT,
                             "batch domains must be two-component, of one precision and in step");
        }
        if (needs_wide_offsets(d->N)) {
            sclbm_batch_destroy(b);
            return set_error(SCLBM_E_INVALID_ARGUMENT,
                             "batch domains must have fewer than 2^32/9 nodes (step larger ones alone)");
        }
        if (d->has_solid) b->flags |= KF_SOLID;
        if (d->p.force_on[0] || d->p.force_on[1]) b->flags |= KF_FORCE;
        const SclbmTunedShape ts = tuned_shape(d->nx, d->ny, b->prec);
        ty[k] = tile_y_per_domain && tile_y_per_domain[k] > 0 ? tile_y_per_domain[k]
                : (bd_list && bd.tile_y > 0 && d->has_solid ? bd.tile_y : ts.tile_y);
        (ts.variant == 3 ? nodes_units : nodes_tiles) += (double)d->nx * (double)d->ny;
    }
    // Small batches: tiles as tall as the table's (tuned on batches of ~4M
    // nodes) would leave most CTAs idle -- a batch of five 256^2 domains got 60
    // tiles of 64 rows for 740 resident CTAs.  Heights the caller did not set
    // are halved (down to 4 rows) until there are four tiles per resident CTA.
    {
        const long resident = (long)std::max(1, batch_blocks_per_sm(b->prec)) * sm_count();
        auto count = [&]() {
            long n = 0;
            for (int k = 0; k < ndomains; ++k)
                n += (long)((b->doms[k]->nx + BATCH_TX - 3) / (BATCH_TX - 2)) *
                     (long)((b->doms[k]->ny + ty[k] - 1) / ty[k]);
            return n;
        };
        const bool given = tile_y_per_domain != nullptr;
        while (!given && count() < 4 * resident) {
            bool changed = false;
            for (int k = 0; k < ndomains; ++k)
                if (ty[k] > 4) {
                    ty[k] = std::max(4, ty[k] / 2);
                    changed = true;
                }
            if (!changed) break;
        }
    }
    // tile lists of tiles `width` columns wide, largest tiles first
    auto tile_list = [&](int width) {
        const int w = width - 2;
        std::vector<TileRef> list;
        std::vector<long> cost;
        for (int k = 0; k < ndomains; ++k) {
            const sclbm_domain *d = b->doms[k];
            for (int yb = 0; yb < (int)d->ny; yb += ty[k])
                for (int xb = 0; xb < (int)d->nx; xb += w) {
                    list.push_back(TileRef{k, xb, yb, 0});
                    cost.push_back((long)std::min(w, (int)d->nx - xb) *
                                   (std::min(ty[k], (int)d->ny - yb) + 2));
                }
        }
        std::vector<int> order(list.size());
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return cost[a] > cost[c]; });
        std::vector<TileRef> sorted(list.size());
        for (size_t i = 0; i < order.size(); ++i) sorted[i] = list[order[i]];
        return sorted;
    };
    const std::vector<TileRef> sorted = tile_list(BATCH_TX);
    const std::vector<TileRef> halves = tile_list(HALF_TX);
    const std::vector<TileRef> warps = tile_list(WARP_TX);
    b->ntiles = (int)sorted.size();
    b->ntiles_half = (int)halves.size();
    b->ntiles_warp = (int)warps.size();
    int per_sm = batch_blocks_per_sm(b->prec);
    if (per_sm < 1) per_sm = 1;
    b->grid = std::max(1, std::min(b->ntiles, per_sm * sm_count()));
    for (int body = 0; body < BODY_COUNT; ++body) {
        const int pb = b->prec == SCLBM_FP64 ? per_sm : std::max(1, batch_blocks_per_sm(b->prec, body));
        const int units = body == BODY_HALF   ? (b->ntiles_half + 1) / 2
                          : body == BODY_WARP ? (b->ntiles_warp + BATCH_TX / WARP_TX - 1) / (BATCH_TX / WARP_TX)
                                              : b->ntiles;
        b->grid_body[body] = std::max(1, std::min(units, pb * sm_count()));
    }
    // rows per unit of the ring bodies: the caller's tile_y, else the tuned
    // batch default's, else RING_BATCH_ROWS
    std::vector<int> ring_rows(ndomains);
    for (int k = 0; k < ndomains; ++k)
        ring_rows[k] = tile_y_per_domain && tile_y_per_domain[k] > 0
                           ? tile_y_per_domain[k]
                           : ((bd.variant == 11 || bd.variant == 12) && bd.tile_y > 0 ? bd.tile_y : RING_BATCH_ROWS);
    if (!tile_y_per_domain) {
        // as for the tile lists: four units per resident CTA, units of at least 8 rows
        const long resident = (long)std::max(1, per_sm) * sm_count();
        auto units = [&]() {
            long n = 0;
            for (int k = 0; k < ndomains; ++k)
                n += (long)((b->doms[k]->nx + 127) / 128) *
                     std::max(1L, (long)((b->doms[k]->ny + ring_rows[k] / 2) / ring_rows[k]));
            return n;
        };
        while (units() < 4 * resident) {
            bool changed = false;
            for (int k = 0; k < ndomains; ++k)
                if (ring_rows[k] > 8) {
                    ring_rows[k] = std::max(8, ring_rows[k] / 2);
                    changed = true;
                }
            if (!changed) break;
        }
    }
    switch (b->prec) {
    case SCLBM_FP64: rc = upload_args<double, double>(b, ty, ring_rows); break;
    case SCLBM_FP32_SHIFTED: rc = upload_args<float, float>(b, ty, ring_rows); break;
    default: rc = upload_args<__half, float>(b, ty, ring_rows); break;
    }
    // pipelined kernel: the smallest band height whose (domain, strip, band)
    // tiles all fit resident at once, bands of one domain split its rows evenly.
    // Default: the tuned variant of the size classes holding most nodes (the
    // FP16 form has no band kernel)
    b->auto_units = b->prec != SCLBM_FP16_SHIFTED && nodes_units > nodes_tiles;
    // FP32/FP16 tile lists with solid nodes: the uniform solid body (512-domain
    // ensemble, FP32: 21.7 vs 19.6 GLUPS), on one-warp tiles for FP16 storage
    // (25.3 vs 23.5 GLUPS)
    b->auto_body = !(b->flags & KF_SOLID) || b->prec == SCLBM_FP64 ? BODY_TILE
                   : b->prec == SCLBM_FP16_SHIFTED                 ? BODY_WARP
                                                                   : BODY_UNIFORM;
    b->body = b->auto_body;
    b->use_units = b->auto_units;
    // Batches with solid nodes run the body that the autotuner's sweep of the
    // whole mixed 512-domain ensemble found fastest for the precision (the
    // tuned batch default); without one recorded, FP32/FP64 take the ring body
    // on 128-column strips (ensemble: FP32 24.5 vs 21.3 GLUPS for the uniform
    // tile list, FP64 12.0 vs 10.3) and FP16 its one-warp tile list.
    if (b->flags & KF_SOLID) {
        if ((bd.variant == 11 || bd.variant == 12) && b->ring) {
            b->auto_ring = bd.variant == 11 ? 128 : 64;
        } else if (bd.variant == 2 || bd.variant == 8 || bd.variant == 10 || bd.variant == 9) {
            if (b->prec != SCLBM_FP64)
                b->auto_body = bd.variant == 8 ? BODY_UNIFORM : bd.variant == 10 ? BODY_WARP
                               : bd.variant == 9 ? BODY_HALF : BODY_TILE;
            b->auto_units = 0;
        } else if (bd.variant == 3 && b->prec != SCLBM_FP16_SHIFTED) {
            b->auto_units = 1;
        } else if (bd.variant == 0) {
            b->auto_ring = b->ring && b->prec != SCLBM_FP16_SHIFTED ? 128 : 0;
        }
        b->body = b->auto_body;
        b->use_units = b->auto_units;
    }
    b->use_ring = b->auto_ring;
    std::vector<BandTile> bands;
    if (b->prec != SCLBM_FP16_SHIFTED) {
        const int res = std::max(1, b->prec == SCLBM_FP64 ? async_resident_fp64() : async_resident_f32());
        int H = 4;
        auto count = [&](int h) {
            long long n = 0;
            for (auto *d : b->doms)
                n += (long long)((d->nx + ASYNC_STRIP - 1) / ASYNC_STRIP) * ((d->ny + h - 1) / h);
            return n;
        };
        int max_ny = 1;
        for (auto *d : b->doms) max_ny = std::max(max_ny, (int)d->ny);
        while (count(H) > res && H < max_ny) ++H;
        b->band_rows = H;
        for (int k = 0; k < ndomains; ++k) {
            const sclbm_domain *d = b->doms[k];
            const int nb = (int)((d->ny + H - 1) / H), ns = (int)((d->nx + ASYNC_STRIP - 1) / ASYNC_STRIP);
            for (int j = 0; j < nb; ++j) {
                const int y0 = (int)((long long)d->ny * j / nb), y1 = (int)((long long)d->ny * (j + 1) / nb);
                for (int s = 0; s < ns; ++s) bands.push_back(BandTile{k, s * ASYNC_STRIP, y0, y1});
            }
        }
        b->nbands = (int)bands.size();
        b->band_grid = std::max(1, std::min(b->nbands, res));
        if (!rc && cudaMalloc(&b->d_bands, bands.size() * sizeof(BandTile)) != cudaSuccess)
            rc = set_error(SCLBM_E_CUDA, "band list allocation");
        if (!rc && cudaMemcpy(b->d_bands, bands.data(), bands.size() * sizeof(BandTile),
                              cudaMemcpyHostToDevice) != cudaSuccess)
            rc = set_error(SCLBM_E_CUDA, "band list upload");
    }
    if (!rc && cudaMalloc(&b->d_tiles, sorted.size() * sizeof(TileRef)) != cudaSuccess)
        rc = set_error(SCLBM_E_CUDA, "tile list allocation");
    if (!rc && cudaMemcpy(b->d_tiles, sorted.data(), sorted.size() * sizeof(TileRef),
                          cudaMemcpyHostToDevice) != cudaSuccess)
        rc = set_error(SCLBM_E_CUDA, "tile list upload");
    if (!rc && cudaMalloc(&b->d_tiles_warp, warps.size() * sizeof(TileRef)) != cudaSuccess)
        rc = set_error(SCLBM_E_CUDA, "tile list allocation");
    if (!rc && cudaMemcpy(b->d_tiles_warp, warps.data(), warps.size() * sizeof(TileRef),
                          cudaMemcpyHostToDevice) != cudaSuccess)
        rc = set_error(SCLBM_E_CUDA, "tile list upload");
    if (!rc && cudaMalloc(&b->d_tiles_half, halves.size() * sizeof(TileRef)) != cudaSuccess)
        rc = set_error(SCLBM_E_CUDA, "tile list allocation");
    if (!rc && cudaMemcpy(b->d_tiles_half, halves.data(), halves.size() * sizeof(TileRef),
                          cudaMemcpyHostToDevice) != cudaSuccess)
        rc = set_error(SCLBM_E_CUDA, "tile list upload");
    if (rc) {
        sclbm_batch_destroy(b);
        return rc;
    }
    *out = b;
    return SCLBM_OK;
}

int sclbm_batch_set_kernel(sclbm_batch *b, int variant)
{
    if (!b) return set_error(SCLBM_E_INVALID_ARGUMENT, "null batch");
    if (variant != 0 && variant != 2 && variant != 3 && variant != 5 && variant != 6 && variant != 8 &&
        variant != 9 && variant != 10 && variant != 11 && variant != 12)
        return set_error(SCLBM_E_INVALID_ARGUMENT, "variant is 0, 2, 3, 5, 6, 8, 9, 10, 11 or 12");
    if ((variant == 11 || variant == 12) && !b->ring)
        return set_error(SCLBM_E_INVALID_ARGUMENT,
                         "the ring body needs every domain's width to be a multiple of "
                         "16 bytes of storage (nx a multiple of 2, 4 or 8 for FP64, FP32, FP16)");
    if (variant == 3 && b->prec == SCLBM_FP16_SHIFTED)
        return set_error(SCLBM_E_INVALID_ARGUMENT, "the FP16 form uses the tile list (variant 2)");
    if ((variant == 5 || variant == 6 || (variant >= 8 && variant <= 10)) && b->prec == SCLBM_FP64)
        return set_error(SCLBM_E_INVALID_ARGUMENT,
                         "the load-ahead, compacted and uniform tile lists are for FP32/FP16 storage");
    b->use_ring = variant == 11 ? 128 : (variant == 12 ? 64 : (variant == 0 ? b->auto_ring : 0));
    b->use_units = variant == 3 || (variant == 0 && b->auto_units);
    b->body = variant == 5   ? BODY_AHEAD
              : variant == 6 ? BODY_COMPACT
              : variant == 8 ? BODY_UNIFORM
              : variant == 9 ? BODY_HALF
              : variant == 10 ? BODY_WARP
              : variant == 0 ? b->auto_body
                             : BODY_TILE;
    for (auto &g : b->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    return SCLBM_OK;
}

int sclbm_batch_info(const sclbm_batch *b, int *ntiles, int *grid_ctas)
{
    if (!b) return set_error(SCLBM_E_INVALID_ARGUMENT, "null batch");
    const int r = b->use_ring == 64 ? 1 : 0;
    if (ntiles) *ntiles = b->use_ring ? b->nunits[r] : (b->use_units ? b->ntiles : batch_ntiles(b));
    if (grid_ctas)
        *grid_ctas = b->use_ring    ? b->ring_grid[r]
                     : b->use_units ? b->band_grid
                                    : (b->prec == SCLBM_FP64 ? b->grid : b->grid_body[b->body]);
    return SCLBM_OK;
}

int sclbm_batch_step(sclbm_batch *b, int nsteps, int use_graph)
{
    if (!b) return set_error(SCLBM_E_INVALID_ARGUMENT, "null batch");
    if (nsteps < 0) return set_error(SCLBM_E_INVALID_ARGUMENT, "negative step count");
    for (auto *d : b->doms)
        if (d->parity != b->parity)
            return set_error(SCLBM_E_RUNTIME, "a batch domain was stepped outside the batch");
    cudaStream_t s = stream();
    if (use_graph && b->graph_stream != s) {
        for (auto &g : b->graph)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        b->graph_stream = s;
    }
    int done = 0;
    while (use_graph && nsteps - done >= GRAPH_STEPS) {
        cudaGraphExec_t &ge = b->graph[b->parity];
        if (!ge) {
            cudaGraph_t g;
            SCLBM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = cudaSuccess;
            for (int k = 0; k < GRAPH_STEPS && e == cudaSuccess; ++k)
                e = batch_launch_any(b, b->parity ^ (k & 1), s);
            cudaError_t e2 = cudaStreamEndCapture(s, &g);
            if (e != cudaSuccess) return cuda_fail(e, "batch capture");
            if (e2 != cudaSuccess) return cuda_fail(e2, "batch capture end");
            e = cudaGraphInstantiate(&ge, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
        }
        SCLBM_CUDA(cudaGraphLaunch(ge, s));
        done += GRAPH_STEPS; // even: parity unchanged
    }
    for (; done < nsteps; ++done) {
        cudaError_t e = batch_launch_any(b, b->parity, s);
        if (e != cudaSuccess) return cuda_fail(e, "batch step");
        b->parity ^= 1;
    }
    for (auto *d : b->doms) d->parity = b->parity;
    return SCLBM_OK;
}

} // extern "C"
