// internal.h -- object layouts and launch entry points shared by the C-ABI
// translation units of libsclbm_b200.so.  Not installed; the public interface
// is include/sclbm.h.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/sclbm.h"

namespace sclbm {

// ------------------------------------------------------------------ errors
int set_error(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
#define SCLBM_CUDA(call)                                                                         \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) return ::sclbm::cuda_fail(e_, #call);                              \
    } while (0)
#define SCLBM_LAUNCHED(what)                                                                     \
    do {                                                                                         \
        cudaError_t e_ = cudaGetLastError();                                                     \
        if (e_ != cudaSuccess) return ::sclbm::cuda_fail(e_, what);                               \
    } while (0)

cudaStream_t stream();
int ensure_device();
int grid_for(size_t n, int block);  // grid-stride grid size (multiple of the SM count)
int sm_count();

// ------------------------------------------------------------- host geometry
int geom_add_walls(std::vector<int32_t> &g, size_t nx, size_t ny, size_t dH, const std::string &w);
// kind: 0 rectangle, 1 square, 2 ellipse, 3 circle
int geom_add_object(std::vector<int32_t> &g, size_t nx, size_t ny, int kind, size_t Lx,
                    size_t Ly, size_t xc, size_t yc);
int geom_add_array(std::vector<int32_t> &g, size_t nx, size_t ny, const std::string &type,
                   const size_t *p, size_t np, const size_t *bounds, size_t a, size_t b,
                   int by_numbers);

} // namespace sclbm

// ------------------------------------------------------------------ objects
struct sclbm_geometry {
    size_t nx = 0, ny = 0;
    std::vector<int32_t> mask; // 1 fluid, 0 solid (Geometry::geom)
    // lazily refreshed device copy (uint8)
    mutable uint8_t *d_mask = nullptr;
    mutable size_t d_count = 0;
    mutable bool dirty = true;
    mutable bool has_solid = true; // refreshed with the device copy
};

struct sclbm_fluid {
    size_t nx = 0, ny = 0, N = 0;
    double tau = 1.0, omega = 1.0, g_solid = 0.0, g_fluid = 0.0;
    double *d[11] = {nullptr}; // indexed by sclbm_field
    bool solid_set = false;
};

struct sclbm_lbm {
    size_t nx = 0, ny = 0, N = 0;
    double *d_tmp[2] = {nullptr, nullptr}; // temp_f_dist, temp_f_dist_spare
};

namespace sclbm {

// per-component physics constants of the fused kernels (compute type T)
template <typename T> struct CompParams {
    T omega, one_m_omega, inv_omega;
    T gf;      // -1.0 * G  (src/lbm.cpp:163)
    T gs_neg;  // -1.0 * Gs (src/fluid.cpp:157)
    T rho_ref; // shift of the stored populations
    T force[9];
    T force_sum; // sum_i force[i] (0 for the drivers' g/6 c_i forces)
    int force_on;
};

// The same constants of both components side by side (element 0: component
// 0, element 1: component 1), each pair aligned so that one 64-bit read feeds
// a packed FP32 instruction of the float-arithmetic collision.
template <typename T> struct PairParams {
    alignas(2 * sizeof(T)) T omega[2];
    alignas(2 * sizeof(T)) T one_m_omega[2];
    alignas(2 * sizeof(T)) T inv_omega[2];
    alignas(2 * sizeof(T)) T gf[2];
    alignas(2 * sizeof(T)) T gs_neg[2];
    alignas(2 * sizeof(T)) T rho_ref[2];
    alignas(2 * sizeof(T)) T force_sum[2];
    alignas(2 * sizeof(T)) T force[9][2];
};

template <typename T> inline void pair_params(PairParams<T> &pc, const CompParams<T> (&c)[2])
{
    for (int k = 0; k < 2; ++k) {
        pc.omega[k] = c[k].omega;
        pc.one_m_omega[k] = c[k].one_m_omega;
        pc.inv_omega[k] = c[k].inv_omega;
        pc.gf[k] = c[k].gf;
        pc.gs_neg[k] = c[k].gs_neg;
        pc.rho_ref[k] = c[k].rho_ref;
        pc.force_sum[k] = c[k].force_sum;
        for (int i = 0; i < 9; ++i) pc.force[i][k] = c[k].force[i];
    }
}

// arguments of the two-component fused kernel
template <typename S, typename T> struct Fused2Args {
    int nx, ny, tile_y;
    size_t N;
    const uint8_t *__restrict__ mask;
    const S *fin[2];
    S *fout[2];
    const double *fsx[2], *fsy[2];       // explicit solid force (FP64 path), or null
    const double *uex_old[2], *uey_old[2]; // kept u_eq for rho ~ 0 (FP64 path), or null
    const T *rho_in[2];                  // two-pass variant: density per node
    CompParams<T> c[2];
    PairParams<T> pc;                    // c[0], c[1] side by side (filled with c)
    int solid_from_mask;                 // derive Fs from the mask (domain path)
    int has_solid;                       // the mask has solid nodes (else all fluid)
    int solids_zero;                     // both buffers hold 0 at solid nodes: the kernels
                                         // neither read nor write them (domain path)
    int *status;                         // set to 1 by a kernel whose bounded wait ran out
                                         // (ring kernel), or null
    int row0, row_end;                   // register tile: step the rows [row0, row_end)
                                         // only (row_end 0: up to ny)
};

// arguments of the single-component fused kernel
template <typename S, typename T> struct Fused1Args {
    int nx, ny;
    size_t N;
    const uint8_t *__restrict__ mask;
    const S *fin;
    S *fout;
    CompParams<T> c;
};

// launchers implemented in the .cu files; return cudaError_t of the launch
cudaError_t launch_fused2_fp64(const Fused2Args<double, double> &a, int variant, int tx,
                               cudaStream_t s);
cudaError_t launch_fused1_fp64(const Fused1Args<double, double> &a, cudaStream_t s);
cudaError_t launch_fused2_f32(const Fused2Args<float, float> &a, int variant, int tx,
                              cudaStream_t s);
cudaError_t launch_fused1_f32(const Fused1Args<float, float> &a, cudaStream_t s);
cudaError_t launch_fused2_f16(const Fused2Args<__half, float> &a, int variant, int tx,
                              cudaStream_t s);
cudaError_t launch_fused1_f16(const Fused1Args<__half, float> &a, cudaStream_t s);
// pipelined single-pass kernels (fused_async.cuh): 128-column strips cut into
// row bands; the batched form walks a list of (domain, strip, band) tiles
struct BandTile;
// uniform: lattices with solid nodes run the uniform solid form (KF_UNIFORM)
cudaError_t launch_fused2_async_fp64(const Fused2Args<double, double> &a, cudaStream_t s,
                                     bool uniform = false);
cudaError_t launch_fused2_async_f32(const Fused2Args<float, float> &a, cudaStream_t s,
                                    bool uniform = false);
cudaError_t launch_batch2_async_fp64(const Fused2Args<double, double> *doms, const BandTile *tiles,
                                     int ntiles, int grid, int parity, cudaStream_t s);
cudaError_t launch_batch2_async_f32(const Fused2Args<float, float> *doms, const BandTile *tiles,
                                    int ntiles, int grid, int parity, cudaStream_t s);
// ring kernels (fused_ring.cuh): population rows streamed into shared memory
// by tensor copies; stages selects the ring depth (0 default, -1 fewer, +1
// more), rows the rows per band (0 default); cudaErrorInvalidValue when nx is
// not a multiple of 16 / sizeof(storage)
// edge: the default depth (stages -1 for FP64 and FP16, +1 for FP32)
// without halo boxes in the stages (lattice-edge columns from global memory)
cudaError_t launch_ring2_fp64(const Fused2Args<double, double> &a, int stages, int rows, cudaStream_t s,
                              bool edge = false);
cudaError_t launch_ring2_f32(const Fused2Args<float, float> &a, int stages, int rows, cudaStream_t s,
                             bool edge = false);
cudaError_t launch_ring2_f16(const Fused2Args<__half, float> &a, int stages, int rows, cudaStream_t s,
                             bool edge = false);
// batched ring kernel (fused_ring.cuh): maps and units are device arrays
// (RingMaps per domain and parity; RingUnit work list); counters: two
// device words, zero before the first launch
struct RingMaps;
struct RingUnit;
cudaError_t launch_batch_ring_fp64(const Fused2Args<double, double> *doms, const RingMaps *maps,
                                   const RingUnit *units, int nunits, int parity, int grid, int flags,
                                   unsigned *counters, int width, cudaStream_t s);
cudaError_t launch_batch_ring_f32(const Fused2Args<float, float> *doms, const RingMaps *maps,
                                  const RingUnit *units, int nunits, int parity, int grid, int flags,
                                  unsigned *counters, int width, cudaStream_t s);
cudaError_t launch_batch_ring_f16(const Fused2Args<__half, float> *doms, const RingMaps *maps,
                                  const RingUnit *units, int nunits, int parity, int grid, int flags,
                                  unsigned *counters, int width, cudaStream_t s);
// shared-memory limits and resident CTAs per SM of the batched ring kernel
// with strips `width` (128 or 64) columns wide
int batch_ring_prepare(sclbm_precision p, int width, int *per_sm);
// tensor maps of a domain's argument block for strips `width` columns wide
// (host); 0 on success
int ring_maps_of(const Fused2Args<double, double> &a, int width, RingMaps *m);
int ring_maps_of(const Fused2Args<float, float> &a, int width, RingMaps *m);
int ring_maps_of(const Fused2Args<__half, float> &a, int width, RingMaps *m);
int async_resident_fp64(); // CTAs of the batched kernel resident on the device
int async_resident_f32();
constexpr int ASYNC_STRIP = 128;
// density pass (kernel a): rho (or rho - rho_ref for shifted storage) per node,
// 0 at solid nodes; both components in one launch
cudaError_t launch_density_fp64(const uint8_t *mask, const double *f0, const double *f1,
                                double *r0, double *r1, size_t N, cudaStream_t s);
cudaError_t launch_density_f32(const uint8_t *mask, const float *f0, const float *f1, float *r0,
                               float *r1, size_t N, cudaStream_t s);
cudaError_t launch_density_f16(const uint8_t *mask, const __half *f0, const __half *f1,
                               float *r0, float *r1, size_t N, cudaStream_t s);

} // namespace sclbm
