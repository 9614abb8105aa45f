// domain.cu -- sclbm_domain: device-resident lattice in one of three storage
// forms, advanced by the fused kernels of fused_step.cuh.
//
//   SCLBM_FP64          f_i in double (bit-exact with the reference sequence)
//   SCLBM_FP32_SHIFTED  d_i = f_i - w_i*rho_ref in float, float arithmetic
//   SCLBM_FP16_SHIFTED  d_i in half, float arithmetic
//
// Host data always crosses the boundary as FP64 in the reference layout; the
// conversions to and from the storage form run on the device, one lattice
// direction at a time through an N-double staging buffer.  The mass/momentum
// monitor reduces in FP64 with a fixed reduction order (deterministic).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "domain.h"
#include "fused_step.cuh"

namespace sclbm {

size_t elem_size(sclbm_precision p) { return p == SCLBM_FP64 ? 8 : (p == SCLBM_FP32_SHIFTED ? 4 : 2); }

template <typename S> struct Conv;
template <> struct Conv<double> {
    static __device__ double to_f64(double v) { return v; }
    static __device__ double from_f64(double v) { return v; }
};
template <> struct Conv<float> {
    static __device__ double to_f64(float v) { return (double)v; }
    static __device__ float from_f64(double v) { return (float)v; }
};
template <> struct Conv<__half> {
    static __device__ double to_f64(__half v) { return (double)__half2float(v); }
    static __device__ __half from_f64(double v) { return __double2half(v); }
};

#define GRID_STRIDE(n, N)                                                                      \
    for (size_t n = blockIdx.x * (size_t)blockDim.x + threadIdx.x; n < (N);                    \
         n += (size_t)gridDim.x * blockDim.x)

// staging (FP64 f_i of direction i) -> storage; solid nodes store 0
template <typename S>
__global__ void k_upload_dir(size_t N, const uint8_t *__restrict__ mask,
                             const double *__restrict__ src, S *__restrict__ dst, double shift)
{
    GRID_STRIDE(n, N) { dst[n] = Conv<S>::from_f64(mask[n] ? src[n] - shift : 0.0); }
}

// Seeded initial state written on the device: f_i = rho/9 on fluid nodes (the
// reference initialisers' shape, src/lbm.cpp:11-48, src/fluid.cpp:64-104),
// rho = rho0 * (1 + amp * (2u - 1)) with u the splitmix64 uniform of
// (seed, node) -- the stream of the host generator sc_lbm_b200/workloads.py,
// operation for operation in round-to-nearest (no contraction), so the state
// equals the host-built one bit for bit; storage conversion as in
// k_upload_dir (shift[i] = w_i * rho_ref, 0 for the FP64 form).
struct InitShift {
    double s[9];
};

__device__ inline double splitmix_u01(unsigned long long seed, unsigned long long n)
{
    unsigned long long z = n + seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

template <typename S>
__global__ void k_init_noise(size_t N, const uint8_t *__restrict__ mask, S *__restrict__ f,
                             double rho0, double amp, unsigned long long seed, InitShift sh)
{
    GRID_STRIDE(n, N)
    {
        const double u = splitmix_u01(seed, n);
        const double r = __dmul_rn(rho0, __dadd_rn(1.0, __dmul_rn(amp, __dsub_rn(__dmul_rn(2.0, u), 1.0))));
        const double fi = __ddiv_rn(r, 9.0);
        const bool fluid = mask[n] != 0;
#pragma unroll
        for (int i = 0; i < 9; ++i) f[i * N + n] = Conv<S>::from_f64(fluid ? __dsub_rn(fi, sh.s[i]) : 0.0);
    }
}

// all nine populations of the solid nodes set to 0 (FP64 uploads)
__global__ void k_zero_solids(size_t N, const uint8_t *__restrict__ mask, double *__restrict__ f)
{
    GRID_STRIDE(n, N)
    {
        if (!mask[n]) {
#pragma unroll
            for (int i = 0; i < 9; ++i) f[i * N + n] = 0.0;
        }
    }
}

// storage -> staging (FP64 f_i); solid nodes read 0 in the shifted forms
template <typename S>
__global__ void k_download_dir(size_t N, const uint8_t *__restrict__ mask, const S *__restrict__ src,
                               double *__restrict__ dst, double shift)
{
    GRID_STRIDE(n, N) { dst[n] = mask[n] ? Conv<S>::to_f64(src[n]) + shift : 0.0; }
}

// density (Fluid::compute_density) of one component into staging; the FP64
// form sums every node like the reference, the shifted forms the fluid nodes
template <typename S>
__global__ void k_rho(size_t N, const uint8_t *__restrict__ mask, const S *__restrict__ f,
                      double *__restrict__ rho, double rho_ref, int shifted)
{
    GRID_STRIDE(n, N)
    {
        double r = 0.0;
        if (!shifted) {
#pragma unroll
            for (int i = 0; i < 9; ++i) r += Conv<S>::to_f64(f[i * N + n]);
        } else if (mask[n]) {
#pragma unroll
            for (int i = 0; i < 9; ++i) r += Conv<S>::to_f64(f[i * N + n]) + w_eq(i) * rho_ref;
        }
        rho[n] = r;
    }
}

// velocity (Fluid::compute_velocities): u = (sum_i f_i c_i)/rho on fluid nodes
template <typename S>
__global__ void k_velocity(size_t N, const uint8_t *__restrict__ mask, const S *__restrict__ f,
                           double *__restrict__ ux, double *__restrict__ uy, double rho_ref,
                           int shifted)
{
    GRID_STRIDE(n, N)
    {
        double r = 0.0, x = 0.0, y = 0.0;
        if (mask[n] == 1) {
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const double v = Conv<S>::to_f64(f[i * N + n]) + (shifted ? w_eq(i) * rho_ref : 0.0);
                r += v;
            }
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const double v = Conv<S>::to_f64(f[i * N + n]) + (shifted ? w_eq(i) * rho_ref : 0.0);
                x += v * double(cx(i));
                y += v * double(cy(i));
            }
            x /= r;
            y /= r;
        }
        ux[n] = x;
        uy[n] = y;
    }
}

// ----------------------------------------------------------- FP64 monitor
constexpr int MON_VALUES = 7; // m, jx, jy per component + non-finite count
constexpr int MON_STRIDE = 8;

template <typename S>
__global__ void __launch_bounds__(256) k_monitor(size_t N, int ncomp, const uint8_t *__restrict__ mask,
                                                 const S *__restrict__ f0, const S *__restrict__ f1,
                                                 double rr0, double rr1, int shifted,
                                                 double *__restrict__ partials)
{
    double acc[MON_VALUES] = {0, 0, 0, 0, 0, 0, 0};
    GRID_STRIDE(n, N)
    {
        if (!mask[n]) continue;
        for (int k = 0; k < ncomp; ++k) {
            const S *f = k ? f1 : f0;
            const double rr = k ? rr1 : rr0;
            double m = 0.0, jx = 0.0, jy = 0.0;
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const double d = Conv<S>::to_f64(f[i * N + n]);
                if (!isfinite(d)) acc[6] += 1.0;
                m += d + (shifted ? w_eq(i) * rr : 0.0);
                jx += d * double(cx(i));
                jy += d * double(cy(i));
            }
            acc[3 * k + 0] += m;
            acc[3 * k + 1] += jx;
            acc[3 * k + 2] += jy;
        }
    }
    __shared__ double s[MON_VALUES][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < MON_VALUES; ++v) {
        double x = acc[v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) s[v][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x < MON_VALUES) {
        double x = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += s[threadIdx.x][w];
        partials[(size_t)blockIdx.x * MON_STRIDE + threadIdx.x] = x;
    }
}

__global__ void __launch_bounds__(256) k_monitor_final(int nblocks, const double *__restrict__ partials,
                                                       double *__restrict__ out)
{
    __shared__ double s[MON_VALUES][256];
    for (int v = 0; v < MON_VALUES; ++v) {
        double x = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) x += partials[(size_t)b * MON_STRIDE + v];
        s[v][threadIdx.x] = x;
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int v = 0; v < MON_VALUES; ++v) s[v][threadIdx.x] += s[v][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < MON_VALUES) out[threadIdx.x] = s[threadIdx.x][0];
}

// ------------------------------------------------------------------ steps
int domain_default_tile_y(const sclbm_domain *d)
{
    if (d->tile_y > 0) return d->tile_y;
    // Measured on B200 at 4096x4096 (register-tile kernel, 128 threads): 16 rows
    // for FP32/FP64 storage, 32 for FP16.  With fewer than ~8 waves of tiles the
    // last partial wave costs a visible share, so the rows per tile are chosen
    // to minimise waves x (rows + 2 halo rows), the time model of one launch.
    const int W = d->tx - 2;
    const long tiles_x = (long)((d->nx + W - 1) / W);
    const long base = d->prec == SCLBM_FP16_SHIFTED ? 32 : 16;
    // resident 128-thread CTAs per SM: 6 for the FP32-arithmetic kernels (80
    // registers), 5 for their uniform solid form (96), 3 for FP64 (168), 4 for
    // its all-fluid form without a volume force (128)
    const bool uniform = d->has_solid && d->prec != SCLBM_FP64 && (d->variant == 0 || d->variant == 8);
    const bool plain = !d->has_solid && !d->p.force_on[0] && !d->p.force_on[1];
    const long per_sm = (d->prec == SCLBM_FP64 ? (plain ? 4 : 3) : (uniform ? 5 : 6)) * (128 / d->tx);
    const long R = per_sm * sm_count();
    auto tiles = [&](long ty) { return tiles_x * (((long)d->ny + ty - 1) / ty); };
    if (tiles(base) >= 8 * R) return (int)base;
    static const long cand[] = {4, 6, 8, 10, 12, 16, 20, 24, 32};
    long best = base, best_cost = -1;
    for (long ty : cand) {
        if (ty > std::max<long>(base, 4) && ty > (long)d->ny) continue;
        const long cost = ((tiles(ty) + R - 1) / R) * (ty + 2);
        if (best_cost < 0 || cost < best_cost || (cost == best_cost && ty > best)) {
            best = ty;
            best_cost = cost;
        }
    }
    return (int)best;
}

template <typename T> static void fill_comp(CompParams<T> &c, const sclbm_params &p, int k)
{
    const double omega = 1 / p.tau[k];
    c.omega = (T)omega;
    c.one_m_omega = (T)(1.0 - omega);
    c.inv_omega = (T)(1.0 / omega);
    c.gf = (T)(-1.0 * p.g_fluid[k]);
    c.gs_neg = (T)(-1.0 * p.g_solid[k]);
    c.rho_ref = (T)p.rho_ref[k];
    c.force_on = p.force_on[k];
    c.force_sum = (T)0;
    for (int i = 0; i < 9; ++i) {
        c.force[i] = (T)(p.force_on[k] ? p.force[k][i] : 0.0);
        c.force_sum += c.force[i];
    }
}

template <typename S, typename T>
static void fill2(const sclbm_domain *d, Fused2Args<S, T> &a)
{
    a = Fused2Args<S, T>{};
    a.nx = (int)d->nx;
    a.ny = (int)d->ny;
    a.N = d->N;
    a.tile_y = domain_default_tile_y(d);
    a.mask = d->d_mask;
    for (int k = 0; k < 2; ++k) {
        a.fin[k] = (const S *)d->buf[d->parity][k];
        a.fout[k] = (S *)d->buf[d->parity ^ 1][k];
        a.rho_in[k] = (const T *)d->rho_tmp[k];
        fill_comp<T>(a.c[k], d->p, k);
    }
    pair_params(a.pc, a.c);
    a.solid_from_mask = 1;
    a.has_solid = d->has_solid ? 1 : 0;
    a.solids_zero = 1; // creation, uploads and initialisers write 0 at solid nodes
    a.status = d->d_status;
}

void domain_fused2_args(const sclbm_domain *d, Fused2Args<double, double> *a64,
                        Fused2Args<float, float> *a32, Fused2Args<__half, float> *a16)
{
    if (a64) fill2(d, *a64);
    if (a32) fill2(d, *a32);
    if (a16) fill2(d, *a16);
}

// rows of the domain start on 16-byte boundaries (the ring kernel's copies)
static bool ring_row_aligned(const sclbm_domain *d)
{
    return d->nx % (16 / elem_size(d->prec)) == 0;
}

// Ring depth (stages: -1, 0, +1 = the depths of variants 12, 11, 13) and rows
// per band that variant 0 runs, the fastest measured on B200 at 4096 x 4096
// (GLUPS all-fluid / 72 % fluid):
//   FP64  2 stages, 16 rows: 20.3 / 15.3 (3 stages 19.8 / 14.9; register tile 18.5)
//   FP32  4 stages, 24 rows: 41.6 (16 rows 41.3, 32 rows 40.1; 3 stages 36.8;
//         5 stages 37.5; register tile 37.6) / 33.1 at 16 rows, 32.9 at 32
//   FP16  4 stages, 32 rows: 49.4 / 35.6 (5 stages 49.0 / 35.3; register tile
//         47.6 / 35.2); 50.3 / 38.2 since its halo columns are reduced by warp 1
struct RingChoice {
    int stages, rows;
};
static RingChoice ring_choice(const sclbm_domain *d)
{
    if (d->prec == SCLBM_FP64) return {-1, 16};
    if (d->prec == SCLBM_FP32_SHIFTED) return {1, 24};
    return {-1, 32};
}

// The ring's bands give at least three waves of its resident CTAs (four per
// SM for FP32/FP16 storage, three for FP64): on smaller lattices the last
// partial wave costs more than the ring gains (2048 x 1024 FP64 porous: 1.15
// waves, 11.9 GLUPS against 14.2 for the register tile), and the register
// tile, which sizes its tiles by the number of waves, is kept.
static bool ring_fills_device(const sclbm_domain *d)
{
    const long per_sm = d->prec == SCLBM_FP64 ? 3 : 4;
    const long rows = d->tile_y > 0 ? d->tile_y : ring_choice(d).rows;
    const long units = (long)((d->nx + 127) / 128) * (long)((d->ny + rows - 1) / rows);
    return units >= 3 * per_sm * sm_count();
}

template <typename S, typename T>
static cudaError_t step_one(const sclbm_domain *d, cudaStream_t s)
{
    if (d->ncomp == 1) {
        Fused1Args<S, T> a{};
        a.nx = (int)d->nx;
        a.ny = (int)d->ny;
        a.N = d->N;
        a.mask = d->d_mask;
        a.fin = (const S *)d->buf[d->parity][0];
        a.fout = (S *)d->buf[d->parity ^ 1][0];
        fill_comp<T>(a.c, d->p, 0);
        if constexpr (sizeof(S) == 8) return launch_fused1_fp64(a, s);
        else if constexpr (sizeof(S) == 4) return launch_fused1_f32(a, s);
        else return launch_fused1_f16(a, s);
    }
    Fused2Args<S, T> a;
    fill2(d, a);
    if (d->variant == 1) {
        cudaError_t e;
        if constexpr (sizeof(S) == 8)
            e = launch_density_fp64(d->d_mask, a.fin[0], a.fin[1], (double *)d->rho_tmp[0],
                                    (double *)d->rho_tmp[1], d->N, s);
        else if constexpr (sizeof(S) == 4)
            e = launch_density_f32(d->d_mask, a.fin[0], a.fin[1], (float *)d->rho_tmp[0],
                                   (float *)d->rho_tmp[1], d->N, s);
        else
            e = launch_density_f16(d->d_mask, a.fin[0], a.fin[1], (float *)d->rho_tmp[0],
                                   (float *)d->rho_tmp[1], d->N, s);
        if (e != cudaSuccess) return e;
    }
    // variant 0 picks the fastest measured form on B200: the ring kernel
    // (rows streamed into shared memory by tensor copies) at the depth and
    // band height of ring_choice on lattices whose rows start on 16-byte
    // boundaries and whose bands fill three waves; else the register tile,
    // in its uniform solid form where FP32/FP16 lattices have solid nodes.
    // 3 and 9 force the pipelined kernel; 11, 12, 13 the ring kernel with its
    // default, fewer and more stages (unaligned lattices: the register tile)
    if (d->variant == 0 && ring_row_aligned(d) && ring_fills_device(d)) {
        const RingChoice rc = ring_choice(d);
        const int rows = d->tile_y > 0 ? d->tile_y : rc.rows;
        if constexpr (sizeof(S) == 8) return launch_ring2_fp64(a, rc.stages, rows, s);
        else if constexpr (sizeof(S) == 4) return launch_ring2_f32(a, rc.stages, rows, s);
        else return launch_ring2_f16(a, rc.stages, rows, s);
    }
    if (d->variant == 14 && ring_row_aligned(d)) {
        // the default depth without halo boxes in the stages
        const RingChoice rc = ring_choice(d);
        const int rows = d->tile_y > 0 ? d->tile_y : rc.rows;
        if constexpr (sizeof(S) == 8) return launch_ring2_fp64(a, rc.stages, rows, s, true);
        else if constexpr (sizeof(S) == 4) return launch_ring2_f32(a, rc.stages, rows, s, true);
        else return launch_ring2_f16(a, rc.stages, rows, s, true);
    }
    if (d->variant >= 11 && d->variant <= 13 && ring_row_aligned(d)) {
        const int st = d->variant == 11 ? 0 : (d->variant == 12 ? -1 : 1);
        if constexpr (sizeof(S) == 8) return launch_ring2_fp64(a, st, d->tile_y, s);
        else if constexpr (sizeof(S) == 4) return launch_ring2_f32(a, st, d->tile_y, s);
        else return launch_ring2_f16(a, st, d->tile_y, s);
    }
    const bool pipelined = d->variant == 3 || d->variant == 9;
    if (pipelined) {
        const bool uni = d->variant == 9;
        if constexpr (sizeof(S) == 8) return launch_fused2_async_fp64(a, s, uni);
        else if constexpr (sizeof(S) == 4) return launch_fused2_async_f32(a, s, uni);
    }
    // variant 1: two pass; 4: register tile with L2 row prefetch; 8: register
    // tile with the uniform solid form; variant 2 (and the FP16 form):
    // register-tile single pass
    int v = d->variant == 1 || (d->variant >= 4 && d->variant <= 9) ? d->variant : 0;
    // variant 0 on an FP32/FP16 lattice with solid nodes: the uniform solid
    // form (4096^2 FP32 at 60 % fluid: 29.7 vs 24.0 GLUPS; FP16 36.3 vs 32.7;
    // FP64 runs it slower, 13.9 vs 15.4)
    if (d->variant == 0 && d->has_solid && sizeof(S) != 8) v = 8;
    if constexpr (sizeof(S) == 8) return launch_fused2_fp64(a, v, d->tx, s);
    else if constexpr (sizeof(S) == 4) return launch_fused2_f32(a, v, d->tx, s);
    else return launch_fused2_f16(a, v, d->tx, s);
}

int domain_launch_step(sclbm_domain *d, cudaStream_t s)
{
    cudaError_t e;
    switch (d->prec) {
    case SCLBM_FP64: e = step_one<double, double>(d, s); break;
    case SCLBM_FP32_SHIFTED: e = step_one<float, float>(d, s); break;
    default: e = step_one<__half, float>(d, s); break;
    }
    if (e != cudaSuccess) return cuda_fail(e, "fused step launch");
    d->parity ^= 1;
    return SCLBM_OK;
}

} // namespace sclbm

using namespace sclbm;

static int dom_alloc(sclbm_domain *d, void **p, size_t bytes)
{
    cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) return cuda_fail(e, "domain allocation");
    d->bytes += bytes;
    return SCLBM_OK;
}

extern "C" {

void sclbm_domain_destroy(sclbm_domain *d)
{
    if (!d) return;
    cudaStreamSynchronize(stream());
    for (auto &b : d->buf)
        for (auto *p : b)
            if (p) cudaFree(p);
    for (auto *p : d->rho_tmp)
        if (p) cudaFree(p);
    if (d->d_mask) cudaFree(d->d_mask);
    if (d->staging) cudaFree(d->staging);
    if (d->partials) cudaFree(d->partials);
    if (d->d_status) cudaFree(d->d_status);
    delete d;
}

int sclbm_domain_create(size_t nx, size_t ny, const int32_t *mask, const sclbm_params *p,
                        sclbm_precision precision, sclbm_domain **out)
{
    if (!out || !mask || !p) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    if (nx < 1 || ny < 1 || nx > (1u << 30) || ny > (1u << 30) || nx * ny > (size_t(1) << 34))
        return set_error(SCLBM_E_INVALID_ARGUMENT, "lattice size out of range");
    if (p->ncomp != 1 && p->ncomp != 2)
        return set_error(SCLBM_E_INVALID_ARGUMENT, "ncomp must be 1 or 2");
    if (precision < SCLBM_FP64 || precision > SCLBM_FP16_SHIFTED)
        return set_error(SCLBM_E_INVALID_ARGUMENT, "unknown precision");
    for (int k = 0; k < p->ncomp; ++k)
        if (!(p->tau[k] > 0.0) || !std::isfinite(p->tau[k]))
            return set_error(SCLBM_E_INVALID_ARGUMENT, "tau must be positive and finite");
    int rc = ensure_device();
    if (rc) return rc;
    const size_t N = nx * ny;
    std::vector<uint8_t> hm(N);
    for (size_t i = 0; i < N; ++i) {
        if (mask[i] != 0 && mask[i] != 1)
            return set_error(SCLBM_E_INVALID_ARGUMENT, "mask values must be 0 or 1");
        hm[i] = (uint8_t)mask[i];
    }
    auto *d = new (std::nothrow) sclbm_domain();
    if (!d) return set_error(SCLBM_E_ALLOC, "host allocation failed");
    d->nx = nx;
    d->ny = ny;
    d->N = N;
    d->ncomp = p->ncomp;
    d->prec = precision;
    d->has_solid = std::find(hm.begin(), hm.end(), (uint8_t)0) != hm.end();
    d->p = *p;
    if (precision == SCLBM_FP64) d->p.rho_ref[0] = d->p.rho_ref[1] = 0.0;
    const size_t es = elem_size(precision);
    cudaStream_t s = stream();
    if ((rc = dom_alloc(d, (void **)&d->d_mask, N))) goto fail;
    for (int par = 0; par < 2; ++par)
        for (int k = 0; k < d->ncomp; ++k) {
            if ((rc = dom_alloc(d, &d->buf[par][k], 9 * N * es))) goto fail;
            if (cudaMemsetAsync(d->buf[par][k], 0, 9 * N * es, s) != cudaSuccess) {
                rc = set_error(SCLBM_E_CUDA, "memset");
                goto fail;
            }
        }
    if ((rc = dom_alloc(d, (void **)&d->staging, 2 * N * sizeof(double)))) goto fail;
    d->partial_blocks = sm_count() * 4;
    if ((rc = dom_alloc(d, (void **)&d->partials, (size_t)(d->partial_blocks + 1) * 8 * sizeof(double))))
        goto fail;
    if ((rc = dom_alloc(d, (void **)&d->d_status, sizeof(int)))) goto fail;
    if (cudaMemsetAsync(d->d_status, 0, sizeof(int), s) != cudaSuccess) {
        rc = set_error(SCLBM_E_CUDA, "memset");
        goto fail;
    }
    if (cudaMemcpyAsync(d->d_mask, hm.data(), N, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        rc = set_error(SCLBM_E_CUDA, "mask upload");
        goto fail;
    }
    *out = d;
    return SCLBM_OK;
fail:
    sclbm_domain_destroy(d);
    return rc;
}

// One step of the rows [row0, row0 + nrows) only (register tile), into the
// other buffer; `finish` ends the step (flips the buffers) once every row has
// been stepped.  For overlapping a slab's halo exchange with the rows that do
// not need it (sc_lbm_b200/slabs.py).
int sclbm_domain_step_rows(sclbm_domain *d, int row0, int nrows, int finish)
{
    if (!d) return set_error(SCLBM_E_INVALID_ARGUMENT, "null domain");
    if (d->ncomp != 2) return set_error(SCLBM_E_INVALID_ARGUMENT, "row ranges are for two-component domains");
    if (row0 < 0 || nrows < 0 || (size_t)row0 + (size_t)nrows > d->ny)
        return set_error(SCLBM_E_OUT_OF_RANGE, "row range outside the domain");
    if (d->variant == 1) return set_error(SCLBM_E_INVALID_ARGUMENT, "row ranges need a single-pass variant");
    cudaStream_t s = stream();
    if (nrows > 0) {
        // the register tile (in its uniform solid form for shifted lattices with solid nodes)
        const int v = d->has_solid && d->prec != SCLBM_FP64 ? 8 : 2;
        cudaError_t e;
        switch (d->prec) {
        case SCLBM_FP64: {
            Fused2Args<double, double> a;
            fill2(d, a);
            a.row0 = row0;
            a.row_end = row0 + nrows;
            e = launch_fused2_fp64(a, v, 128, s);
            break;
        }
        case SCLBM_FP32_SHIFTED: {
            Fused2Args<float, float> a;
            fill2(d, a);
            a.row0 = row0;
            a.row_end = row0 + nrows;
            e = launch_fused2_f32(a, v, 128, s);
            break;
        }
        default: {
            Fused2Args<__half, float> a;
            fill2(d, a);
            a.row0 = row0;
            a.row_end = row0 + nrows;
            e = launch_fused2_f16(a, v, 128, s);
            break;
        }
        }
        if (e != cudaSuccess) return cuda_fail(e, "row-range step");
    }
    if (finish) d->parity ^= 1;
    return SCLBM_OK;
}

int sclbm_domain_set_kernel(sclbm_domain *d, int variant, int tile_y)
{
    if (!d) return set_error(SCLBM_E_INVALID_ARGUMENT, "null domain");
    if (variant < 0 || variant > 14 || variant == 10)
        return set_error(SCLBM_E_INVALID_ARGUMENT, "variant is 0..9 or 11..14");
    if (tile_y < 0 || tile_y > 4096) return set_error(SCLBM_E_INVALID_ARGUMENT, "bad tile_y");
    if (variant == 1 && !d->rho_tmp[0] && d->ncomp == 2) {
        const size_t es = d->prec == SCLBM_FP64 ? 8 : 4;
        for (int k = 0; k < 2; ++k) {
            int rc = dom_alloc(d, &d->rho_tmp[k], d->N * es);
            if (rc) return rc;
        }
    }
    d->variant = variant;
    d->tile_y = tile_y;
    return SCLBM_OK;
}

int sclbm_domain_set_threads(sclbm_domain *d, int tx)
{
    if (!d) return set_error(SCLBM_E_INVALID_ARGUMENT, "null domain");
    if (tx != 32 && tx != 64 && tx != 128)
        return set_error(SCLBM_E_INVALID_ARGUMENT, "threads per tile must be 32, 64 or 128");
    d->tx = tx;
    return SCLBM_OK;
}

size_t sclbm_domain_device_bytes(const sclbm_domain *d) { return d ? d->bytes : 0; }

static int check_comp(const sclbm_domain *d, int comp, size_t count, size_t want)
{
    if (!d) return set_error(SCLBM_E_INVALID_ARGUMENT, "null domain");
    if (comp < 0 || comp >= d->ncomp) return set_error(SCLBM_E_INVALID_ARGUMENT, "bad component");
    if (count != want) return set_error(SCLBM_E_INVALID_ARGUMENT, "count mismatch");
    return SCLBM_OK;
}

int sclbm_domain_upload_f(sclbm_domain *d, int comp, const double *f, size_t count)
{
    int rc = check_comp(d, comp, count, d ? 9 * d->N : 0);
    if (rc) return rc;
    if (!f) return set_error(SCLBM_E_INVALID_ARGUMENT, "null f");
    cudaStream_t s = stream();
    void *dst = d->buf[d->parity][comp];
    if (d->prec == SCLBM_FP64) {
        SCLBM_CUDA(cudaMemcpyAsync(dst, f, 9 * d->N * 8, cudaMemcpyHostToDevice, s));
        if (d->has_solid) {
            // solid nodes hold 0 in both buffers (what the reference's stream leaves
            // there after every step); the fused kernels rely on it
            k_zero_solids<<<grid_for(d->N, 256), 256, 0, s>>>(d->N, d->d_mask, (double *)dst);
            SCLBM_LAUNCHED("solid zeroing");
        }
    } else {
        const double rr = d->p.rho_ref[comp];
        for (int i = 0; i < 9; ++i) {
            SCLBM_CUDA(cudaMemcpyAsync(d->staging, f + i * d->N, d->N * 8, cudaMemcpyHostToDevice, s));
            if (d->prec == SCLBM_FP32_SHIFTED)
                k_upload_dir<float><<<grid_for(d->N, 256), 256, 0, s>>>(
                    d->N, d->d_mask, d->staging, (float *)dst + i * d->N, w_eq(i) * rr);
            else
                k_upload_dir<__half><<<grid_for(d->N, 256), 256, 0, s>>>(
                    d->N, d->d_mask, d->staging, (__half *)dst + i * d->N, w_eq(i) * rr);
            SCLBM_LAUNCHED("upload conversion");
        }
    }
    SCLBM_CUDA(cudaStreamSynchronize(s));
    return SCLBM_OK;
}

int sclbm_domain_init_noise(sclbm_domain *d, int comp, double rho0, double amp, uint64_t seed)
{
    int rc = check_comp(d, comp, 0, 0);
    if (rc) return rc;
    if (!std::isfinite(rho0) || !std::isfinite(amp))
        return set_error(SCLBM_E_INVALID_ARGUMENT, "non-finite density or amplitude");
    cudaStream_t s = stream();
    InitShift sh;
    for (int i = 0; i < 9; ++i) sh.s[i] = d->prec == SCLBM_FP64 ? 0.0 : w_eq(i) * d->p.rho_ref[comp];
    void *dst = d->buf[d->parity][comp];
    const int grid = grid_for(d->N, 256);
    switch (d->prec) {
    case SCLBM_FP64:
        k_init_noise<double><<<grid, 256, 0, s>>>(d->N, d->d_mask, (double *)dst, rho0, amp, seed, sh);
        break;
    case SCLBM_FP32_SHIFTED:
        k_init_noise<float><<<grid, 256, 0, s>>>(d->N, d->d_mask, (float *)dst, rho0, amp, seed, sh);
        break;
    default:
        k_init_noise<__half><<<grid, 256, 0, s>>>(d->N, d->d_mask, (__half *)dst, rho0, amp, seed, sh);
    }
    SCLBM_LAUNCHED("seeded initial state");
    SCLBM_CUDA(cudaStreamSynchronize(s));
    return SCLBM_OK;
}

int sclbm_domain_download_f(sclbm_domain *d, int comp, double *f, size_t count)
{
    int rc = check_comp(d, comp, count, d ? 9 * d->N : 0);
    if (rc) return rc;
    if (!f) return set_error(SCLBM_E_INVALID_ARGUMENT, "null f");
    cudaStream_t s = stream();
    const void *src = d->buf[d->parity][comp];
    if (d->prec == SCLBM_FP64) {
        SCLBM_CUDA(cudaMemcpyAsync(f, src, 9 * d->N * 8, cudaMemcpyDeviceToHost, s));
    } else {
        const double rr = d->p.rho_ref[comp];
        for (int i = 0; i < 9; ++i) {
            if (d->prec == SCLBM_FP32_SHIFTED)
                k_download_dir<float><<<grid_for(d->N, 256), 256, 0, s>>>(
                    d->N, d->d_mask, (const float *)src + i * d->N, d->staging, w_eq(i) * rr);
            else
                k_download_dir<__half><<<grid_for(d->N, 256), 256, 0, s>>>(
                    d->N, d->d_mask, (const __half *)src + i * d->N, d->staging, w_eq(i) * rr);
            SCLBM_LAUNCHED("download conversion");
            SCLBM_CUDA(cudaMemcpyAsync(f + i * d->N, d->staging, d->N * 8, cudaMemcpyDeviceToHost, s));
        }
    }
    SCLBM_CUDA(cudaStreamSynchronize(s));
    return SCLBM_OK;
}

// density of one component into the staging buffer (queued, not synchronised)
static int rho_to_staging(sclbm_domain *d, int comp, cudaStream_t s)
{
    const void *src = d->buf[d->parity][comp];
    const double rr = d->p.rho_ref[comp];
    const int g = grid_for(d->N, 256);
    switch (d->prec) {
    case SCLBM_FP64: k_rho<double><<<g, 256, 0, s>>>(d->N, d->d_mask, (const double *)src, d->staging, 0.0, 0); break;
    case SCLBM_FP32_SHIFTED: k_rho<float><<<g, 256, 0, s>>>(d->N, d->d_mask, (const float *)src, d->staging, rr, 1); break;
    default: k_rho<__half><<<g, 256, 0, s>>>(d->N, d->d_mask, (const __half *)src, d->staging, rr, 1); break;
    }
    SCLBM_LAUNCHED("density");
    return SCLBM_OK;
}

} // extern "C"

namespace sclbm {
// One output field of component comp as FP64 values copied into host (pinned)
// memory, queued on stream s and not synchronised: what = 0 density, 1 ux,
// 2 uy (N values, Fluid::compute_density / compute_velocities), 3 the nine
// population arrays (9N values, direction-major).  The staging buffer is
// reused across directions; stream order keeps each copy before the next
// conversion.
int domain_field_async(sclbm_domain *d, int comp, int what, double *host, cudaStream_t s)
{
    const size_t N = d->N;
    const int g = grid_for(N, 256);
    const void *src = d->buf[d->parity][comp];
    const double rr = d->p.rho_ref[comp];
    if (what == 0) {
        int rc = rho_to_staging(d, comp, s);
        if (rc) return rc;
        SCLBM_CUDA(cudaMemcpyAsync(host, d->staging, N * 8, cudaMemcpyDeviceToHost, s));
        return SCLBM_OK;
    }
    if (what == 1 || what == 2) {
        double *a = d->staging, *b = d->staging + N;
        switch (d->prec) {
        case SCLBM_FP64: k_velocity<double><<<g, 256, 0, s>>>(N, d->d_mask, (const double *)src, a, b, 0.0, 0); break;
        case SCLBM_FP32_SHIFTED: k_velocity<float><<<g, 256, 0, s>>>(N, d->d_mask, (const float *)src, a, b, rr, 1); break;
        default: k_velocity<__half><<<g, 256, 0, s>>>(N, d->d_mask, (const __half *)src, a, b, rr, 1); break;
        }
        SCLBM_LAUNCHED("velocity");
        SCLBM_CUDA(cudaMemcpyAsync(host, what == 1 ? a : b, N * 8, cudaMemcpyDeviceToHost, s));
        return SCLBM_OK;
    }
    for (int i = 0; i < 9; ++i) {
        if (d->prec == SCLBM_FP64) {
            SCLBM_CUDA(cudaMemcpyAsync(host + i * N, (const double *)src + i * N, N * 8,
                                       cudaMemcpyDeviceToHost, s));
            continue;
        }
        if (d->prec == SCLBM_FP32_SHIFTED)
            k_download_dir<float><<<g, 256, 0, s>>>(N, d->d_mask, (const float *)src + i * N,
                                                    d->staging, w_eq(i) * rr);
        else
            k_download_dir<__half><<<g, 256, 0, s>>>(N, d->d_mask, (const __half *)src + i * N,
                                                     d->staging, w_eq(i) * rr);
        SCLBM_LAUNCHED("download conversion");
        SCLBM_CUDA(cudaMemcpyAsync(host + i * N, d->staging, N * 8, cudaMemcpyDeviceToHost, s));
    }
    return SCLBM_OK;
}
} // namespace sclbm

extern "C" {

int sclbm_domain_download_rho(sclbm_domain *d, int comp, double *rho, size_t count)
{
    int rc = check_comp(d, comp, count, d ? d->N : 0);
    if (rc) return rc;
    if (!rho) return set_error(SCLBM_E_INVALID_ARGUMENT, "null rho");
    cudaStream_t s = stream();
    if ((rc = rho_to_staging(d, comp, s))) return rc;
    SCLBM_CUDA(cudaMemcpyAsync(rho, d->staging, d->N * 8, cudaMemcpyDeviceToHost, s));
    SCLBM_CUDA(cudaStreamSynchronize(s));
    return SCLBM_OK;
}

int sclbm_domain_download_velocity(sclbm_domain *d, int comp, double *ux, double *uy, size_t count)
{
    int rc = check_comp(d, comp, count, d ? d->N : 0);
    if (rc) return rc;
    if (!ux || !uy) return set_error(SCLBM_E_INVALID_ARGUMENT, "null output");
    cudaStream_t s = stream();
    const void *src = d->buf[d->parity][comp];
    const double rr = d->p.rho_ref[comp];
    const int g = grid_for(d->N, 256);
    double *a = d->staging, *b = d->staging + d->N;
    switch (d->prec) {
    case SCLBM_FP64: k_velocity<double><<<g, 256, 0, s>>>(d->N, d->d_mask, (const double *)src, a, b, 0.0, 0); break;
    case SCLBM_FP32_SHIFTED: k_velocity<float><<<g, 256, 0, s>>>(d->N, d->d_mask, (const float *)src, a, b, rr, 1); break;
    default: k_velocity<__half><<<g, 256, 0, s>>>(d->N, d->d_mask, (const __half *)src, a, b, rr, 1); break;
    }
    SCLBM_LAUNCHED("velocity");
    SCLBM_CUDA(cudaMemcpyAsync(ux, a, d->N * 8, cudaMemcpyDeviceToHost, s));
    SCLBM_CUDA(cudaMemcpyAsync(uy, b, d->N * 8, cudaMemcpyDeviceToHost, s));
    SCLBM_CUDA(cudaStreamSynchronize(s));
    return SCLBM_OK;
}

int sclbm_domain_step(sclbm_domain *d, int nsteps)
{
    if (!d) return set_error(SCLBM_E_INVALID_ARGUMENT, "null domain");
    if (nsteps < 0) return set_error(SCLBM_E_INVALID_ARGUMENT, "negative step count");
    if (d->variant == 1 && d->ncomp == 2 && !d->rho_tmp[0])
        return set_error(SCLBM_E_RUNTIME, "two-pass buffers missing");
    cudaStream_t s = stream();
    for (int k = 0; k < nsteps; ++k) {
        int rc = domain_launch_step(d, s);
        if (rc) return rc;
    }
    return SCLBM_OK;
}

int sclbm_domain_mass_momentum(sclbm_domain *d, double out[7])
{
    if (!d || !out) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    cudaStream_t s = stream();
    const int nb = d->partial_blocks;
    const void *f0 = d->buf[d->parity][0];
    const void *f1 = d->ncomp > 1 ? d->buf[d->parity][1] : f0;
    const double r0 = d->p.rho_ref[0], r1 = d->p.rho_ref[1];
    switch (d->prec) {
    case SCLBM_FP64: k_monitor<double><<<nb, 256, 0, s>>>(d->N, d->ncomp, d->d_mask, (const double *)f0, (const double *)f1, 0.0, 0.0, 0, d->partials); break;
    case SCLBM_FP32_SHIFTED: k_monitor<float><<<nb, 256, 0, s>>>(d->N, d->ncomp, d->d_mask, (const float *)f0, (const float *)f1, r0, r1, 1, d->partials); break;
    default: k_monitor<__half><<<nb, 256, 0, s>>>(d->N, d->ncomp, d->d_mask, (const __half *)f0, (const __half *)f1, r0, r1, 1, d->partials); break;
    }
    SCLBM_LAUNCHED("monitor");
    double *res = d->partials + (size_t)nb * MON_STRIDE;
    k_monitor_final<<<1, 256, 0, s>>>(nb, d->partials, res);
    SCLBM_LAUNCHED("monitor final");
    SCLBM_CUDA(cudaMemcpyAsync(out, res, 7 * sizeof(double), cudaMemcpyDeviceToHost, s));
    int status = 0;
    SCLBM_CUDA(cudaMemcpyAsync(&status, d->d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
    SCLBM_CUDA(cudaStreamSynchronize(s));
    if (status != 0)
        return set_error(SCLBM_E_RUNTIME, "a fused-step kernel gave up waiting for its row copies; "
                                          "the populations are not valid");
    if (out[6] != 0.0) return set_error(SCLBM_E_NONFINITE, "non-finite populations in the domain");
    return SCLBM_OK;
}

int sclbm_domain_run(sclbm_domain *d, const double *f1, const double *f2, int nsteps, double *rho1,
                     double *rho2)
{
    if (!d) return set_error(SCLBM_E_INVALID_ARGUMENT, "null domain");
    int rc = sclbm_domain_upload_f(d, 0, f1, 9 * d->N);
    if (!rc && d->ncomp > 1) rc = sclbm_domain_upload_f(d, 1, f2, 9 * d->N);
    if (!rc) rc = sclbm_domain_step(d, nsteps);
    if (!rc) rc = sclbm_domain_download_rho(d, 0, rho1, d->N);
    if (!rc && d->ncomp > 1) rc = sclbm_domain_download_rho(d, 1, rho2, d->N);
    return rc;
}

} // extern "C"
