// ops_fp64.h -- launchers of the per-operator FP64 kernels (ops_fp64.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace sclbm {

struct EqvelArgs {
    const double *f, *rho, *frx, *fry, *fsx, *fsy;
    double *ux, *uy, *uex, *uey;
    double omega;
};

cudaError_t op_density(size_t N, const double *f, double *rho, cudaStream_t s);
cudaError_t op_velocities(size_t N, const uint8_t *g, const double *f, const double *rho,
                          double *ux, double *uy, cudaStream_t s);
cudaError_t op_feq_single(size_t N, const uint8_t *g, double *f, double *rho, double *ux,
                          double *uy, double *feq, double omega, int collide, cudaStream_t s);
cudaError_t op_feq_multi(size_t N, double *f, const double *rho, const double *uex,
                         const double *uey, double *feq, double omega, int collide,
                         cudaStream_t s);
cudaError_t op_solid_sums(int nx, int ny, const uint8_t *g, double *sx, double *sy,
                          cudaStream_t s);
cudaError_t op_repulsive(int nx, int ny, const uint8_t *g, const double *psi1, const double *psi2,
                         double gf1, double gf2, double *f1x, double *f1y, double *f2x,
                         double *f2y, cudaStream_t s);
cudaError_t op_eqvel(size_t N, const uint8_t *g, const EqvelArgs &a, const EqvelArgs &b,
                     cudaStream_t s);
cudaError_t op_volume_force(size_t N, const uint8_t *g, double *f, const double *force9,
                            cudaStream_t s);
cudaError_t op_stream(int nx, int ny, const uint8_t *g, const double *f, double *out,
                      cudaStream_t s);
cudaError_t op_fill_fluid(size_t N, const uint8_t *g, double *f, double v, cudaStream_t s);
cudaError_t op_init_droplet(int nx, int ny, const uint8_t *g, double *fb, double *fd, double rb,
                            double rd, double rbd, double rdb, double xc, double yc, double radius,
                            cudaStream_t s);
cudaError_t op_init_rect(int nx, int ny, const uint8_t *g, double *fb, double *fd, double rb,
                         double rd, double rbd, double rdb, long long x0, long long xf,
                         long long y0, long long yf, cudaStream_t s);

} // namespace sclbm
