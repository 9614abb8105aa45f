// ops_fp64.cu -- per-operator FP64 kernels (one per reference method) and the
// FP64 instantiations of the fused step.  Compiled with -fmad=false: every
// product and sum is rounded separately, in the reference's order, so results
// are bit-identical to the serial reference (g++ on x86-64 has no FMA).
#include "fused_step.cuh"
#include "ops_fp64.h"

namespace sclbm {

#define GRID_STRIDE(n, N)                                                                      \
    for (size_t n = blockIdx.x * (size_t)blockDim.x + threadIdx.x; n < (N);                    \
         n += (size_t)gridDim.x * blockDim.x)

// Fluid::compute_density, src/fluid.cpp:175-183 (all nodes)
__global__ void k_density(size_t N, const double *__restrict__ f, double *__restrict__ rho)
{
    GRID_STRIDE(n, N)
    {
        double r = 0.0;
#pragma unroll
        for (int j = 0; j < 9; ++j) r += f[j * N + n];
        rho[n] = r;
    }
}

// Fluid::compute_velocities, src/fluid.cpp:186-200
__device__ __forceinline__ void velocity_node(size_t N, size_t n, bool fluid, const double *f,
                                              double rho, double &ux, double &uy)
{
    double x = 0.0, y = 0.0;
    if (fluid) {
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            x += f[j * N + n] * double(cx(j));
            y += f[j * N + n] * double(cy(j));
        }
        x /= rho;
        y /= rho;
    }
    ux = x;
    uy = y;
}

__global__ void k_velocities(size_t N, const uint8_t *__restrict__ g, const double *__restrict__ f,
                             const double *__restrict__ rho, double *__restrict__ ux,
                             double *__restrict__ uy)
{
    GRID_STRIDE(n, N)
    {
        double a, b;
        velocity_node(N, n, g[n] == 1, f, rho[n], a, b);
        ux[n] = a;
        uy[n] = b;
    }
}

__device__ __forceinline__ void store_feq(size_t N, size_t n, const double fe[9], double *feq)
{
#pragma unroll
    for (int i = 0; i < 9; ++i) feq[i * N + n] = fe[i];
}

// Fluid::compute_f_equilibrium(geom), src/fluid.cpp:210-243; with collide=1
// also LBM::collide(geom, fluid), src/lbm.cpp:275-288
__global__ void k_feq_single(size_t N, const uint8_t *__restrict__ g, double *__restrict__ f,
                             double *__restrict__ rho, double *__restrict__ ux,
                             double *__restrict__ uy, double *__restrict__ feq, double omega,
                             int collide)
{
    GRID_STRIDE(n, N)
    {
        double r = 0.0;
#pragma unroll
        for (int j = 0; j < 9; ++j) r += f[j * N + n];
        double a, b;
        velocity_node(N, n, g[n] == 1, f, r, a, b);
        rho[n] = r;
        ux[n] = a;
        uy[n] = b;
        double fe[9];
        feq_exact(r, a, b, fe);
        store_feq(N, n, fe, feq);
        if (collide) {
#pragma unroll
            for (int i = 0; i < 9; ++i) f[i * N + n] = (1.0 - omega) * f[i * N + n] + omega * fe[i];
        }
    }
}

// Fluid::compute_f_equilibrium(), src/fluid.cpp:246-278; with omega > 0 also the
// collision loop of LBM::collide(f1, f2), src/lbm.cpp:305-311
__global__ void k_feq_multi(size_t N, double *__restrict__ f, const double *__restrict__ rho,
                            const double *__restrict__ uex, const double *__restrict__ uey,
                            double *__restrict__ feq, double omega, int collide)
{
    GRID_STRIDE(n, N)
    {
        double fe[9];
        feq_exact(rho[n], uex[n], uey[n], fe);
        store_feq(N, n, fe, feq);
        if (collide) {
#pragma unroll
            for (int i = 0; i < 9; ++i) f[i * N + n] = (1.0 - omega) * f[i * N + n] + omega * fe[i];
        }
    }
}

// LBM::compute_solid_surface_force common sums, src/lbm.cpp:110-136
__global__ void k_solid_sums(int nx, int ny, const uint8_t *__restrict__ g, double *__restrict__ sx,
                             double *__restrict__ sy)
{
    const size_t N = (size_t)nx * ny;
    GRID_STRIDE(n, N)
    {
        double a = 0.0, b = 0.0;
        const int x = int(n % nx), y = int(n / nx);
        if (g[n] != 0) {
#pragma unroll
            for (int i = 1; i < 9; ++i) {
                const int xn = wrap1(x + cx(i), nx), yn = wrap1(y + cy(i), ny);
                if (g[(size_t)yn * nx + xn] == 0) {
                    a += w_sc(i) * cx(i);
                    b += w_sc(i) * cy(i);
                }
            }
        }
        sx[n] = a;
        sy[n] = b;
    }
}

// LBM::compute_fluid_repulsive_interactions, src/lbm.cpp:144-206
__global__ void k_repulsive(int nx, int ny, const uint8_t *__restrict__ g,
                            const double *__restrict__ psi1, const double *__restrict__ psi2,
                            double gf1, double gf2, double *__restrict__ f1x,
                            double *__restrict__ f1y, double *__restrict__ f2x,
                            double *__restrict__ f2y)
{
    const size_t N = (size_t)nx * ny;
    GRID_STRIDE(n, N)
    {
        double ax = 0.0, ay = 0.0, bx = 0.0, by = 0.0;
        if (g[n] != 0) {
            const int x = int(n % nx), y = int(n / nx);
#pragma unroll
            for (int i = 1; i < 9; ++i) {
                const int xn = wrap1(x + cx(i), nx), yn = wrap1(y + cy(i), ny);
                const size_t ij = (size_t)yn * nx + xn;
                if (g[ij] == 0) continue;
                const double wcx = w_sc(i) * cx(i), wcy = w_sc(i) * cy(i);
                ax += wcx * psi2[ij];
                ay += wcy * psi2[ij];
                bx += wcx * psi1[ij];
                by += wcy * psi1[ij];
            }
            ax *= gf1 * psi1[n];
            ay *= gf1 * psi1[n];
            bx *= gf2 * psi2[n];
            by *= gf2 * psi2[n];
        }
        f1x[n] = ax;
        f1y[n] = ay;
        f2x[n] = bx;
        f2y[n] = by;
    }
}

struct EqvelFluid {
    const double *f, *rho, *frx, *fry, *fsx, *fsy;
    double *ux, *uy, *uex, *uey;
    double omega, inv_omega;
};

// LBM::compute_equilibrium_velocities, src/lbm.cpp:209-272
__global__ void k_eqvel(size_t N, const uint8_t *__restrict__ g, EqvelFluid a, EqvelFluid b)
{
    GRID_STRIDE(n, N)
    {
        if (g[n] != 1) {
            a.ux[n] = a.uy[n] = b.ux[n] = b.uy[n] = 0.0;
            continue;
        }
        double p = 0.0, q = 0.0, r = 0.0, s = 0.0;
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            p += a.f[j * N + n] * double(cx(j));
            q += a.f[j * N + n] * double(cy(j));
            r += b.f[j * N + n] * double(cx(j));
            s += b.f[j * N + n] * double(cy(j));
        }
        a.ux[n] = p;
        a.uy[n] = q;
        b.ux[n] = r;
        b.uy[n] = s;
        const double ra = a.rho[n], rb = b.rho[n];
        const double ucx = (p * a.omega + r * b.omega) / (ra * a.omega + rb * b.omega);
        const double ucy = (q * a.omega + s * b.omega) / (ra * a.omega + rb * b.omega);
        if (!rho_is_zero(ra)) {
            a.uex[n] = ucx + a.frx[n] * a.inv_omega / ra + a.fsx[n] * a.inv_omega;
            a.uey[n] = ucy + a.fry[n] * a.inv_omega / ra + a.fsy[n] * a.inv_omega;
        }
        if (!rho_is_zero(rb)) {
            b.uex[n] = ucx + b.frx[n] * b.inv_omega / rb + b.fsx[n] * b.inv_omega;
            b.uey[n] = ucy + b.fry[n] * b.inv_omega / rb + b.fsy[n] * b.inv_omega;
        }
    }
}

struct ForceVec {
    double v[9];
};

// LBM::add_volume_force, src/lbm.cpp:315-340
__global__ void k_volume_force(size_t N, const uint8_t *__restrict__ g, double *__restrict__ f,
                               ForceVec F)
{
    GRID_STRIDE(n, N)
    {
        if (g[n] == 1) {
#pragma unroll
            for (int i = 0; i < 9; ++i) f[i * N + n] += F.v[i];
        }
    }
}

// LBM::stream, src/lbm.cpp:343-384, written in gather form: every destination
// slot is assigned exactly the value the reference pushes into it (zero at
// solid nodes, bounce-back where the upstream node is solid).
__global__ void k_stream(int nx, int ny, const uint8_t *__restrict__ g,
                         const double *__restrict__ f, double *__restrict__ out)
{
    const size_t N = (size_t)nx * ny;
    GRID_STRIDE(n, N)
    {
        if (g[n] != 1) {
#pragma unroll
            for (int i = 0; i < 9; ++i) out[i * N + n] = 0.0;
            continue;
        }
        const int x = int(n % nx), y = int(n / nx);
        out[n] = f[n];
#pragma unroll
        for (int i = 1; i < 9; ++i) {
            const int xs = wrap1(x - cx(i), nx), ys = wrap1(y - cy(i), ny);
            const size_t src = (size_t)ys * nx + xs;
            out[i * N + n] = g[src] == 1 ? f[i * N + src] : f[opp(i) * N + n];
        }
    }
}

// f = value on fluid nodes (Fluid::simple_ini, src/fluid.cpp:86-101)
__global__ void k_fill_fluid(size_t N, const uint8_t *__restrict__ g, double *__restrict__ f,
                             double v)
{
    GRID_STRIDE(n, N)
    {
        if (g[n] == 1) {
#pragma unroll
            for (int i = 0; i < 9; ++i) f[i * N + n] = v;
        }
    }
}

// LBM::initialize_droplet, src/lbm.cpp:11-48
__global__ void k_init_droplet(int nx, int ny, const uint8_t *__restrict__ g, double *fb,
                               double *fd, double rb, double rd, double rbd, double rdb, double xc,
                               double yc, double radius)
{
    const size_t N = (size_t)nx * ny;
    GRID_STRIDE(n, N)
    {
        const int xi = int(n % nx), yj = int(n / nx);
        if (g[n] == 0) continue;
        const bool in = (((double)xi - xc) * ((double)xi - xc) +
                         ((double)yj - yc) * ((double)yj - yc)) <= radius * radius;
        const double vb = (in ? rbd : rb) / 9.0, vd = (in ? rd : rdb) / 9.0;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            fb[i * N + n] = vb;
            fd[i * N + n] = vd;
        }
    }
}

// LBM::initialize_fluid_rectangle, src/lbm.cpp:51-99 (both passes; the caller
// has already checked that the rectangle indexes stay inside the lattice)
__global__ void k_init_rect(int nx, int ny, const uint8_t *__restrict__ g, double *fb, double *fd,
                            double rb, double rd, double rbd, double rdb, long long x0,
                            long long xf, long long y0, long long yf)
{
    const size_t N = (size_t)nx * ny;
    GRID_STRIDE(n, N)
    {
        if (g[n] == 0) continue;
        const long long xi = (long long)(n % nx), yj = (long long)(n / nx);
        // a rectangle node (xi', yj') touches linear index yj'*nx + xi'; xi' may
        // exceed nx and wrap into the next row exactly like the reference's
        // geom(xi, yj) = geom.at(yj*Nx + xi)
        bool in = false;
        for (long long yy = y0; yy <= yf && !in; ++yy) {
            const long long rem = (long long)n - yy * nx;
            if (rem >= x0 && rem <= xf) in = true;
        }
        (void)xi;
        (void)yj;
        const double vb = (in ? rbd : rb) / 9.0, vd = (in ? rd : rdb) / 9.0;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            fb[i * N + n] = vb;
            fd[i * N + n] = vd;
        }
    }
}

// ----------------------------------------------------------------- launchers
#define LAUNCH(kern, N, ...)                                                                   \
    do {                                                                                       \
        kern<<<grid_for((N), 256), 256, 0, s>>>(__VA_ARGS__);                                  \
        return cudaGetLastError();                                                             \
    } while (0)

cudaError_t op_density(size_t N, const double *f, double *rho, cudaStream_t s)
{
    LAUNCH(k_density, N, N, f, rho);
}
cudaError_t op_velocities(size_t N, const uint8_t *g, const double *f, const double *rho,
                          double *ux, double *uy, cudaStream_t s)
{
    LAUNCH(k_velocities, N, N, g, f, rho, ux, uy);
}
cudaError_t op_feq_single(size_t N, const uint8_t *g, double *f, double *rho, double *ux,
                          double *uy, double *feq, double omega, int collide, cudaStream_t s)
{
    LAUNCH(k_feq_single, N, N, g, f, rho, ux, uy, feq, omega, collide);
}
cudaError_t op_feq_multi(size_t N, double *f, const double *rho, const double *uex,
                         const double *uey, double *feq, double omega, int collide, cudaStream_t s)
{
    LAUNCH(k_feq_multi, N, N, f, rho, uex, uey, feq, omega, collide);
}
cudaError_t op_solid_sums(int nx, int ny, const uint8_t *g, double *sx, double *sy, cudaStream_t s)
{
    LAUNCH(k_solid_sums, (size_t)nx * ny, nx, ny, g, sx, sy);
}
cudaError_t op_repulsive(int nx, int ny, const uint8_t *g, const double *psi1, const double *psi2,
                         double gf1, double gf2, double *f1x, double *f1y, double *f2x,
                         double *f2y, cudaStream_t s)
{
    LAUNCH(k_repulsive, (size_t)nx * ny, nx, ny, g, psi1, psi2, gf1, gf2, f1x, f1y, f2x, f2y);
}
cudaError_t op_eqvel(size_t N, const uint8_t *g, const EqvelArgs &a, const EqvelArgs &b,
                     cudaStream_t s)
{
    EqvelFluid A{a.f, a.rho, a.frx, a.fry, a.fsx, a.fsy, a.ux, a.uy, a.uex, a.uey, a.omega,
                 1.0 / a.omega};
    EqvelFluid B{b.f, b.rho, b.frx, b.fry, b.fsx, b.fsy, b.ux, b.uy, b.uex, b.uey, b.omega,
                 1.0 / b.omega};
    LAUNCH(k_eqvel, N, N, g, A, B);
}
cudaError_t op_volume_force(size_t N, const uint8_t *g, double *f, const double *force9,
                            cudaStream_t s)
{
    ForceVec F;
    for (int i = 0; i < 9; ++i) F.v[i] = force9[i];
    LAUNCH(k_volume_force, N, N, g, f, F);
}
cudaError_t op_stream(int nx, int ny, const uint8_t *g, const double *f, double *out,
                      cudaStream_t s)
{
    LAUNCH(k_stream, (size_t)nx * ny, nx, ny, g, f, out);
}
cudaError_t op_fill_fluid(size_t N, const uint8_t *g, double *f, double v, cudaStream_t s)
{
    LAUNCH(k_fill_fluid, N, N, g, f, v);
}
cudaError_t op_init_droplet(int nx, int ny, const uint8_t *g, double *fb, double *fd, double rb,
                            double rd, double rbd, double rdb, double xc, double yc, double radius,
                            cudaStream_t s)
{
    LAUNCH(k_init_droplet, (size_t)nx * ny, nx, ny, g, fb, fd, rb, rd, rbd, rdb, xc, yc, radius);
}
cudaError_t op_init_rect(int nx, int ny, const uint8_t *g, double *fb, double *fd, double rb,
                         double rd, double rbd, double rdb, long long x0, long long xf,
                         long long y0, long long yf, cudaStream_t s)
{
    LAUNCH(k_init_rect, (size_t)nx * ny, nx, ny, g, fb, fd, rb, rd, rbd, rdb, x0, xf, y0, yf);
}

cudaError_t launch_fused2_fp64(const Fused2Args<double, double> &a, int variant, int tx,
                               cudaStream_t s)
{
    return launch_fused2_any<double, double>(a, variant, tx, s);
}
cudaError_t launch_fused1_fp64(const Fused1Args<double, double> &a, cudaStream_t s)
{
    k_fused1<double, double><<<grid_for(a.N, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_density_fp64(const uint8_t *mask, const double *f0, const double *f1,
                                double *r0, double *r1, size_t N, cudaStream_t s)
{
    k_density2<double, double><<<grid_for(N, 256), 256, 0, s>>>(mask, f0, f1, r0, r1, N);
    return cudaGetLastError();
}

} // namespace sclbm

// the FP64 batched kernel lives in this -fmad=false translation unit
#include "batch_kernel.cuh"
namespace sclbm {
cudaError_t launch_batch_fp64(const Fused2Args<double, double> *doms, const TileRef *tiles,
                              int ntiles, int parity, int grid, int flags, cudaStream_t s)
{
    return launch_batch_t<double, double>(doms, tiles, ntiles, parity, grid, flags, s);
}
int batch_blocks_per_sm_fp64() { return batch_blocks_per_sm_t<double, double>(); }
} // namespace sclbm

// pipelined persistent FP64 kernels (-fmad=false keeps them bit-exact)
#include "fused_async.cuh"
namespace sclbm {
cudaError_t launch_fused2_async_fp64(const Fused2Args<double, double> &a, cudaStream_t s,
                                     bool uniform)
{
    if (uniform) return launch_fused2_async_t<double, double, 128, 3, KF_UNIFORM>(a, s);
    return launch_fused2_async_t<double, double, 128, 3>(a, s);
}
cudaError_t launch_batch2_async_fp64(const Fused2Args<double, double> *doms, const BandTile *tiles,
                                     int ntiles, int grid, int parity, cudaStream_t s)
{
    return launch_batch2_async_t<double, double, 128, 3>(doms, tiles, ntiles, grid, parity, s);
}
int async_resident_fp64() { return async_resident_ctas<double, double, 128, 3>(); }
} // namespace sclbm

// ring kernel, FP64 storage (-fmad=false keeps it bit-exact): 19 KB per stage,
// three stages beside the three CTAs per SM that the registers allow; solid
// lanes branch around the collision as in the FP64 register tile
#include "fused_ring.cuh"
namespace sclbm {
cudaError_t launch_ring2_fp64(const Fused2Args<double, double> &a, int stages, int rows, cudaStream_t s,
                              bool edge)
{
    // FP64 keeps its halo boxes: its registers, not its stages, set its residency
    if (edge) return launch_ring2_any<double, double, 2, 0>(a, rows, s);
    if (stages < 0) return launch_ring2_any<double, double, 2, 0>(a, rows, s);
    if (stages > 0) return launch_ring2_any<double, double, 4, 0>(a, rows, s);
    return launch_ring2_any<double, double, 3, 0>(a, rows, s);
}
constexpr int RING_BATCH_R64 = 3;
cudaError_t launch_batch_ring_fp64(const Fused2Args<double, double> *doms, const RingMaps *maps,
                                   const RingUnit *units, int nunits, int parity, int grid, int flags,
                                   unsigned *counters, int width, cudaStream_t s)
{
    if (width == 64)
        return launch_batch_ring<double, double, RING_BATCH_R64, 0, 64>(doms, maps, units, nunits, parity,
                                                                         grid, flags, counters, s);
    return launch_batch_ring<double, double, RING_BATCH_R64, 0, 128>(doms, maps, units, nunits, parity,
                                                                      grid, flags, counters, s);
}
int batch_ring_prepare_shifted(sclbm_precision p, int width, int *per_sm);
int batch_ring_prepare(sclbm_precision p, int width, int *per_sm)
{
    if (p != SCLBM_FP64) return batch_ring_prepare_shifted(p, width, per_sm);
    const cudaError_t e = width == 64 ? batch_ring_prepare<double, double, RING_BATCH_R64, 0, 64>(per_sm)
                                      : batch_ring_prepare<double, double, RING_BATCH_R64, 0, 128>(per_sm);
    return e == cudaSuccess ? 0 : cuda_fail(e, "ring batch set-up");
}
int ring_maps_of(const Fused2Args<double, double> &a, int width, RingMaps *m)
{
    const cudaError_t e = width == 64 ? ring_maps<double, double, RING_BATCH_R64, 64>(a, *m)
                                      : ring_maps<double, double, RING_BATCH_R64, 128>(a, *m);
    return e == cudaSuccess ? 0 : 1;
}
} // namespace sclbm
