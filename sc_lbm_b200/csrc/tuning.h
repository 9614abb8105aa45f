// tuning.h -- launch shapes per domain size class, measured on B200 by
// sc_lbm_b200/autotune.py (results in sc_lbm_b200/tuning/b200.json; build.py
// turns them into the table sclbm_tuned_table.h compiled in here).
#pragma once
#include <cstddef>

struct SclbmTunedShape {
    int variant; // 2 tile list (register-tile body), 3 strips x bands (pipelined body)
    int tile_y;  // rows per tile of the tile-list kernel
};

struct SclbmTunedClass {
    int nx_lo, nx_hi, ny_lo, ny_hi; // half-open size ranges of the class
    int precision;                  // recommended storage (sclbm_precision)
    SclbmTunedShape shape[3];       // by storage precision
};

/// Shape for one domain: the table entry of its size class, or the nearest
/// class (log-distance of the sizes); defaults when the table is empty.
SclbmTunedShape tuned_shape(size_t nx, size_t ny, int precision, int *recommended = nullptr);
/// Whether a measured table was compiled in
bool tuned_table_present();
/// Batch body for batches with solid nodes that the autotuner's sweep of the
/// whole mixed ensemble found fastest for a storage precision: variant (11 or
/// 12 the ring bodies, 2/8/10 tile lists, 3 bands; 0 = none recorded: the
/// size-class table decides) and its rows per unit / tile (0 = default).
SclbmTunedShape tuned_batch_default(int precision);
