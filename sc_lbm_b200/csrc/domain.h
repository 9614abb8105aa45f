// domain.h -- internal layout of sclbm_domain / sclbm_batch.
#pragma once
#include "internal.h"

struct sclbm_domain {
    size_t nx = 0, ny = 0, N = 0;
    int ncomp = 2;
    sclbm_precision prec = SCLBM_FP64;
    sclbm_params p{};
    uint8_t *d_mask = nullptr;
    void *buf[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}}; // [parity][comp], 9N each
    int parity = 0;                                             // buf[parity] holds the state
    void *rho_tmp[2] = {nullptr, nullptr}; // density arrays of the two-pass variant
    double *staging = nullptr;             // N doubles, host<->device conversions
    double *partials = nullptr;            // per-CTA partial sums of the monitor
    int *d_status = nullptr;               // set by a kernel whose bounded wait ran out
    int partial_blocks = 0;
    int variant = 0;  // 0 single pass, 1 two pass
    int tile_y = 0;   // rows per tile (0: default)
    int tx = 128;     // threads per CTA
    bool has_solid = true; // the mask has solid nodes
    size_t bytes = 0; // device bytes held
};

namespace sclbm {
size_t elem_size(sclbm_precision p);
int domain_launch_step(sclbm_domain *d, cudaStream_t s);
int domain_default_tile_y(const sclbm_domain *d);
int domain_field_async(sclbm_domain *d, int comp, int what, double *host, cudaStream_t s);
// fill the kernel argument blocks for the current parity
void domain_fused2_args(const sclbm_domain *d, Fused2Args<double, double> *a64,
                        Fused2Args<float, float> *a32, Fused2Args<__half, float> *a16);
} // namespace sclbm
