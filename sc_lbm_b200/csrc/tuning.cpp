// tuning.cpp -- lookup in the autotuned size-class table (host code).
#include <cmath>

#include "internal.h"
#include "tuning.h"
#include "sclbm_tuned_table.h"

static const SclbmTunedShape kDefault[3] = {{3, 16}, {2, 16}, {2, 32}};

bool tuned_table_present() { return SCLBM_TUNED_COUNT > 0; }

SclbmTunedShape tuned_batch_default(int precision)
{
    if (precision < 0 || precision > 2) return SclbmTunedShape{0, 0};
    return kSclbmBatchDefault[precision];
}

SclbmTunedShape tuned_shape(size_t nx, size_t ny, int precision, int *recommended)
{
    if (precision < 0 || precision > 2) precision = -1;
    if (SCLBM_TUNED_COUNT == 0) {
        if (recommended) *recommended = SCLBM_FP32_SHIFTED;
        return kDefault[precision < 0 ? SCLBM_FP32_SHIFTED : precision];
    }
    const SclbmTunedClass *best = nullptr;
    double best_d = 0.0;
    for (int k = 0; k < SCLBM_TUNED_COUNT; ++k) {
        const SclbmTunedClass &c = kSclbmTuned[k];
        if ((int)nx >= c.nx_lo && (int)nx < c.nx_hi && (int)ny >= c.ny_lo && (int)ny < c.ny_hi) {
            best = &c;
            break;
        }
        // distance to the class's geometric centre, in log size
        const double cx = std::sqrt((double)c.nx_lo * (double)(c.nx_hi - 1));
        const double cy = std::sqrt((double)c.ny_lo * (double)(c.ny_hi - 1));
        const double d = std::fabs(std::log((double)(nx ? nx : 1) / cx)) +
                         std::fabs(std::log((double)(ny ? ny : 1) / cy));
        if (!best || d < best_d) {
            best = &c;
            best_d = d;
        }
    }
    if (recommended) *recommended = best->precision;
    return best->shape[precision < 0 ? best->precision : precision];
}

extern "C" int sclbm_tuned_config(size_t nx, size_t ny, int precision, int *tile_y, int *variant,
                                  int *recommended)
{
    if (nx == 0 || ny == 0) return sclbm::set_error(SCLBM_E_INVALID_ARGUMENT, "empty lattice");
    if (precision > 2) return sclbm::set_error(SCLBM_E_INVALID_ARGUMENT, "unknown precision");
    int rec = 0;
    const SclbmTunedShape s = tuned_shape(nx, ny, precision, &rec);
    if (tile_y) *tile_y = s.tile_y;
    if (variant) *variant = s.variant;
    if (recommended) *recommended = rec;
    return SCLBM_OK;
}
