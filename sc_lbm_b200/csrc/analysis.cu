// analysis.cu -- measurements of a device lattice, computed where the
// populations live instead of after a text round trip:
//
//  * the Laplace-law measurement of the reference's post-processing
//    (benchmarks/two_phase_two_components_flows/laplace_law/
//    compute_surface_tension.py:55-73): the pressure p = (rho_b + rho_d)/3 +
//    G rho_b rho_d / 3 at an inside and an outside node, and the droplet
//    radius from the extent of the interface band rho_d < rho_b,
//    rho_disp < rho_b <= rho_bulk (half the row extent and half the column
//    extent, averaged);
//  * velocity statistics of one component over fluid nodes (the largest
//    |u| -- spurious currents -- and the mean of the nonzero magnitudes,
//    scripts/benchmark_utils.py:55-63);
//  * the row profile of u_x (mean over each row's fluid nodes), the quantity
//    a channel flow is compared with the analytic parabola on
//    (scripts/benchmark_utils.py:8-52);
//  * the contact angle of a droplet resting on a flat solid
//    (benchmarks/two_phase_two_components_flows/contact_angles/
//    compute_contact_angles.py:45-106): the base from the two lowest rows of
//    the droplet-side interface band, the height from its row extent, and the
//    angle of the circular cap through them.
//
// Densities and velocities are the FP64 values of Fluid::compute_density /
// compute_velocities (shifted forms add w_i rho_ref back); every reduction is
// deterministic (integer atomics on indices and on the bit patterns of
// non-negative doubles, fixed-order block sums).
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "domain.h"
#include "fused_step.cuh"

using namespace sclbm;

namespace {

template <typename S> __device__ __forceinline__ double pop(const S *f, size_t i, size_t N, size_t n)
{
    if constexpr (sizeof(S) == 2) return (double)__half2float(f[i * N + n]);
    else return (double)f[i * N + n];
}

// density, momentum of one component at node n (FP64, the reference's sums)
template <typename S>
__device__ __forceinline__ void moments(const S *f, size_t N, size_t n, double rr, bool shifted,
                                        double &r, double &jx, double &jy)
{
    r = 0.0;
    jx = 0.0;
    jy = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) r = __dadd_rn(r, __dadd_rn(pop(f, i, N, n), shifted ? w_eq(i) * rr : 0.0));
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const double v = __dadd_rn(pop(f, i, N, n), shifted ? w_eq(i) * rr : 0.0);
        jx = __dadd_rn(jx, v * double(cx(i)));
        jy = __dadd_rn(jy, v * double(cy(i)));
    }
}

// p = 1/3 (rb + rd) + G/3 rb rd, evaluated in that order without contraction
__device__ __forceinline__ double pressure(double rb, double rd, double G)
{
    return __dadd_rn(__dmul_rn(1.0 / 3.0, __dadd_rn(rb, rd)), __dmul_rn(__dmul_rn(G / 3.0, rb), rd));
}

struct LaplaceOut {
    unsigned int ymin, ymax, xmin, xmax;
    unsigned long long band;
    double p_in, p_out;
};

template <typename S>
__global__ void k_laplace(size_t N, int nx, const uint8_t *__restrict__ mask, const S *__restrict__ fb,
                          const S *__restrict__ fd, double rrb, double rrd, int shifted, double G,
                          double rho_bulk, double rho_disp, size_t n_in, size_t n_out,
                          LaplaceOut *out)
{
    for (size_t n = blockIdx.x * (size_t)blockDim.x + threadIdx.x; n < N;
         n += (size_t)gridDim.x * blockDim.x) {
        double rb, rd, jx, jy;
        moments(fb, N, n, rrb, shifted, rb, jx, jy);
        moments(fd, N, n, rrd, shifted, rd, jx, jy);
        if (!mask[n]) rb = rd = 0.0; // the reference's solid nodes hold zero populations
        if (n == n_in) out->p_in = pressure(rb, rd, G);
        if (n == n_out) out->p_out = pressure(rb, rd, G);
        if (rd - rb < 0.0 && rb <= rho_bulk && rb > rho_disp) {
            const unsigned int y = (unsigned int)(n / nx), x = (unsigned int)(n % nx);
            atomicMin(&out->ymin, y);
            atomicMax(&out->ymax, y);
            atomicMin(&out->xmin, x);
            atomicMax(&out->xmax, x);
            atomicAdd(&out->band, 1ull);
        }
    }
}

// Contact-angle band (compute_contact_angles.py:46): nodes with
// rho_b - rho_d <= 0, rho_d <= rho_bulk and rho_b > rho_disp; per row the
// smallest and largest x of the band, and its first and last rows.
struct ContactOut {
    unsigned int ymin, ymax;
    unsigned long long band;
};

template <typename S>
__global__ void k_contact_band(size_t N, int nx, const uint8_t *__restrict__ mask,
                               const S *__restrict__ fb, const S *__restrict__ fd, double rrb,
                               double rrd, int shifted, double rho_bulk, double rho_disp,
                               unsigned int *__restrict__ row_xmin, unsigned int *__restrict__ row_xmax,
                               ContactOut *out)
{
    for (size_t n = blockIdx.x * (size_t)blockDim.x + threadIdx.x; n < N;
         n += (size_t)gridDim.x * blockDim.x) {
        double rb, rd, jx, jy;
        moments(fb, N, n, rrb, shifted, rb, jx, jy);
        moments(fd, N, n, rrd, shifted, rd, jx, jy);
        if (!mask[n]) rb = rd = 0.0;
        if (rb - rd <= 0.0 && rd <= rho_bulk && rb > rho_disp) {
            const unsigned int y = (unsigned int)(n / nx), x = (unsigned int)(n % nx);
            atomicMin(&row_xmin[y], x);
            atomicMax(&row_xmax[y], x);
            atomicMin(&out->ymin, y);
            atomicMax(&out->ymax, y);
            atomicAdd(&out->band, 1ull);
        }
    }
}

struct VelOut {
    unsigned long long umax_bits; // bit pattern of the largest |u| (>= 0: ordered as integers)
    unsigned long long nonzero;
};

template <typename S>
__global__ void k_velocity_stats(size_t N, const uint8_t *__restrict__ mask, const S *__restrict__ f,
                                 double rr, int shifted, double *__restrict__ block_sum, VelOut *out)
{
    __shared__ double red[256];
    double s = 0.0;
    unsigned long long nz = 0, mx = 0;
    for (size_t n = blockIdx.x * (size_t)blockDim.x + threadIdx.x; n < N;
         n += (size_t)gridDim.x * blockDim.x) {
        if (mask[n] != 1) continue;
        double r, jx, jy;
        moments(f, N, n, rr, shifted, r, jx, jy);
        const double ux = jx / r, uy = jy / r;
        const double m = sqrt(__dadd_rn(__dmul_rn(ux, ux), __dmul_rn(uy, uy)));
        if (m != 0.0) {
            s += m;
            ++nz;
        }
        const unsigned long long b = (unsigned long long)__double_as_longlong(m);
        if (b > mx) mx = b;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) block_sum[blockIdx.x] = red[0];
    atomicAdd(&out->nonzero, nz);
    atomicMax(&out->umax_bits, mx);
}

// one block per row: mean of u_x over the row's fluid nodes (fixed-order sum)
template <typename S>
__global__ void k_row_profile(int nx, size_t N, const uint8_t *__restrict__ mask,
                              const S *__restrict__ f, double rr, int shifted, int axis,
                              double *__restrict__ prof)
{
    __shared__ double red[256];
    __shared__ int cnt[256];
    const int y = blockIdx.x;
    double s = 0.0;
    int c = 0;
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
        const size_t n = (size_t)y * nx + x;
        if (mask[n] != 1) continue;
        double r, jx, jy;
        moments(f, N, n, rr, shifted, r, jx, jy);
        s += (axis == 0 ? jx : jy) / r;
        ++c;
    }
    red[threadIdx.x] = s;
    cnt[threadIdx.x] = c;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            red[threadIdx.x] += red[threadIdx.x + w];
            cnt[threadIdx.x] += cnt[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) prof[y] = cnt[0] ? red[0] / cnt[0] : 0.0;
}

template <typename Launch> int with_precision(const sclbm_domain *d, Launch &&l)
{
    switch (d->prec) {
    case SCLBM_FP64: l((const double *)nullptr); break;
    case SCLBM_FP32_SHIFTED: l((const float *)nullptr); break;
    default: l((const __half *)nullptr); break;
    }
    return SCLBM_OK;
}

constexpr int STAT_BLOCKS = 1184; // 8 per SM on 148 SMs

} // namespace

extern "C" int sclbm_domain_laplace_measure(sclbm_domain *d, int bulk, double G, double rho_bulk,
                                            double rho_disp, size_t x_in, size_t y_in, size_t x_out,
                                            size_t y_out, double out[5])
{
    if (!d || !out) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    if (d->ncomp != 2 || (bulk != 0 && bulk != 1))
        return set_error(SCLBM_E_INVALID_ARGUMENT, "a two-component domain and bulk = 0 or 1");
    if (x_in >= d->nx || x_out >= d->nx || y_in >= d->ny || y_out >= d->ny)
        return set_error(SCLBM_E_OUT_OF_RANGE, "pressure node outside the lattice");
    LaplaceOut h{0xffffffffu, 0u, 0xffffffffu, 0u, 0ull, 0.0, 0.0};
    LaplaceOut *dv = nullptr;
    SCLBM_CUDA(cudaMalloc(&dv, sizeof(LaplaceOut)));
    cudaStream_t s = stream();
    cudaError_t e = cudaMemcpyAsync(dv, &h, sizeof h, cudaMemcpyHostToDevice, s);
    const int drop = 1 - bulk;
    const bool shifted = d->prec != SCLBM_FP64;
    const size_t n_in = y_in * d->nx + x_in, n_out = y_out * d->nx + x_out;
    if (e == cudaSuccess) {
        with_precision(d, [&](auto tag) {
            using S = std::remove_const_t<std::remove_pointer_t<decltype(tag)>>;
            k_laplace<S><<<STAT_BLOCKS, 256, 0, s>>>(
                d->N, (int)d->nx, d->d_mask, (const S *)d->buf[d->parity][bulk],
                (const S *)d->buf[d->parity][drop], d->p.rho_ref[bulk], d->p.rho_ref[drop],
                shifted ? 1 : 0, G, rho_bulk, rho_disp, n_in, n_out, dv);
        });
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, dv, sizeof h, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(dv);
    if (e != cudaSuccess) return cuda_fail(e, "laplace measurement");
    const double Rr = h.band ? (double(h.ymax) - double(h.ymin)) / 2.0 : 0.0;
    const double Rc = h.band ? (double(h.xmax) - double(h.xmin)) / 2.0 : 0.0;
    out[0] = h.p_in - h.p_out;
    out[1] = 0.5 * (Rr + Rc);
    out[2] = Rr;
    out[3] = Rc;
    out[4] = (double)h.band;
    return SCLBM_OK;
}

extern "C" int sclbm_domain_contact_angle(sclbm_domain *d, int bulk, double rho_bulk,
                                          double rho_disp, double out[9])
{
    if (!d || !out) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    if (d->ncomp != 2 || (bulk != 0 && bulk != 1))
        return set_error(SCLBM_E_INVALID_ARGUMENT, "a two-component domain and bulk = 0 or 1");
    const size_t ny = d->ny;
    ContactOut h{0xffffffffu, 0u, 0ull};
    ContactOut *dv = nullptr;
    unsigned int *rows = nullptr; // [0, ny): smallest x per row, [ny, 2 ny): largest
    SCLBM_CUDA(cudaMalloc(&dv, sizeof(ContactOut)));
    cudaError_t e = cudaMalloc(&rows, 2 * ny * sizeof(unsigned int));
    if (e != cudaSuccess) {
        cudaFree(dv);
        return cuda_fail(e, "contact angle scratch");
    }
    cudaStream_t s = stream();
    e = cudaMemcpyAsync(dv, &h, sizeof h, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(rows, 0xff, ny * sizeof(unsigned int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(rows + ny, 0, ny * sizeof(unsigned int), s);
    const int drop = 1 - bulk;
    const bool shifted = d->prec != SCLBM_FP64;
    if (e == cudaSuccess) {
        with_precision(d, [&](auto tag) {
            using S = std::remove_const_t<std::remove_pointer_t<decltype(tag)>>;
            k_contact_band<S><<<STAT_BLOCKS, 256, 0, s>>>(
                d->N, (int)d->nx, d->d_mask, (const S *)d->buf[d->parity][bulk],
                (const S *)d->buf[d->parity][drop], d->p.rho_ref[bulk], d->p.rho_ref[drop],
                shifted ? 1 : 0, rho_bulk, rho_disp, rows, rows + ny, dv);
        });
        e = cudaGetLastError();
    }
    std::vector<unsigned int> hr(2 * ny);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, dv, sizeof h, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hr.data(), rows, 2 * ny * sizeof(unsigned int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(dv);
    cudaFree(rows);
    if (e != cudaSuccess) return cuda_fail(e, "contact angle");
    if (h.band == 0) return set_error(SCLBM_E_OUT_OF_RANGE, "contact angle: no interface nodes");
    // compute_contact_angles.py:48-106: the two lowest rows of the band give
    // each end of the base, extrapolated half a node below the lowest row
    const size_t y2 = h.ymin, y1 = y2 + 1;
    if (y1 >= ny || hr[y1] == 0xffffffffu)
        return set_error(SCLBM_E_OUT_OF_RANGE, "contact angle: no interface nodes above the lowest row");
    double xL1 = hr[y1], xL2 = hr[y2], xR1 = hr[ny + y1], xR2 = hr[ny + y2];
    const double yA = (double)y1, yB = (double)y2, yBase = (double)h.ymin - 0.5;
    if (xL1 == xL2) xL1 = xL1 - 1;
    if (xR1 == xR2) xR1 = xR1 - 1;
    const double slopeL = (yA - yB) / (xL1 - xL2), slopeR = (yA - yB) / (xR1 - xR2);
    const double interL = yB - slopeL * xL2, interR = yB - slopeR * xR2;
    const double xL = 1 / slopeL * (yBase - interL), xR = 1 / slopeR * (yBase - interR);
    const double L = xR - xL;
    const double H = (double)(h.ymax - h.ymin) + 0.5;
    const double R = (4 * H * H + L * L) / (8 * H);
    double theta = std::atan(L / (2 * (R - H))) * (180.0 / 3.141592653589793);
    if (theta < 0) theta += 180;
    out[0] = theta;
    out[1] = L;
    out[2] = H;
    out[3] = R;
    out[4] = xL;
    out[5] = xR;
    out[6] = (double)h.ymin;
    out[7] = (double)h.ymax;
    out[8] = (double)h.band;
    return SCLBM_OK;
}

extern "C" int sclbm_domain_velocity_stats(sclbm_domain *d, int comp, double out[3])
{
    if (!d || !out) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    if (comp < 0 || comp >= d->ncomp) return set_error(SCLBM_E_INVALID_ARGUMENT, "bad component");
    VelOut h{0ull, 0ull};
    VelOut *dv = nullptr;
    double *bs = nullptr;
    SCLBM_CUDA(cudaMalloc(&dv, sizeof(VelOut)));
    cudaError_t e = cudaMalloc(&bs, STAT_BLOCKS * sizeof(double));
    if (e != cudaSuccess) {
        cudaFree(dv);
        return cuda_fail(e, "velocity statistics scratch");
    }
    cudaStream_t s = stream();
    e = cudaMemcpyAsync(dv, &h, sizeof h, cudaMemcpyHostToDevice, s);
    const bool shifted = d->prec != SCLBM_FP64;
    if (e == cudaSuccess) {
        with_precision(d, [&](auto tag) {
            using S = std::remove_const_t<std::remove_pointer_t<decltype(tag)>>;
            k_velocity_stats<S><<<STAT_BLOCKS, 256, 0, s>>>(d->N, d->d_mask,
                                                            (const S *)d->buf[d->parity][comp],
                                                            d->p.rho_ref[comp], shifted ? 1 : 0, bs, dv);
        });
        e = cudaGetLastError();
    }
    std::vector<double> hb(STAT_BLOCKS);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, dv, sizeof h, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hb.data(), bs, STAT_BLOCKS * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(dv);
    cudaFree(bs);
    if (e != cudaSuccess) return cuda_fail(e, "velocity statistics");
    double sum = 0.0;
    for (double v : hb) sum += v;
    double umax;
    std::memcpy(&umax, &h.umax_bits, sizeof umax);
    out[0] = umax;
    out[1] = h.nonzero ? sum / (double)h.nonzero : 0.0;
    out[2] = (double)h.nonzero;
    return SCLBM_OK;
}

extern "C" int sclbm_domain_profile(sclbm_domain *d, int comp, int axis, double *prof, size_t count)
{
    if (!d || !prof) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    if (comp < 0 || comp >= d->ncomp) return set_error(SCLBM_E_INVALID_ARGUMENT, "bad component");
    if (axis != 0 && axis != 1) return set_error(SCLBM_E_INVALID_ARGUMENT, "axis is 0 (u_x) or 1 (u_y)");
    if (count != d->ny) return set_error(SCLBM_E_INVALID_ARGUMENT, "count must be ny");
    double *dp = nullptr;
    SCLBM_CUDA(cudaMalloc(&dp, d->ny * sizeof(double)));
    cudaStream_t s = stream();
    const bool shifted = d->prec != SCLBM_FP64;
    with_precision(d, [&](auto tag) {
        using S = std::remove_const_t<std::remove_pointer_t<decltype(tag)>>;
        k_row_profile<S><<<(unsigned)d->ny, 256, 0, s>>>((int)d->nx, d->N, d->d_mask,
                                                         (const S *)d->buf[d->parity][comp],
                                                         d->p.rho_ref[comp], shifted ? 1 : 0, axis, dp);
    });
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(prof, dp, d->ny * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(dp);
    if (e != cudaSuccess) return cuda_fail(e, "row profile");
    return SCLBM_OK;
}
