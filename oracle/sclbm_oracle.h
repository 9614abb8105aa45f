/*
 * sclbm_oracle.h -- CPU oracle for the sc_lbm D2Q9 Shan-Chen step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (LBMFluids/sc_lbm, src/lbm.cpp, src/fluid.cpp, src/geometry.cpp,
 * src/geom_object/*.cpp, src/arrays/regular_array.cpp).  It is used by the
 * tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the
 * checker.  The product library never links, loads or calls it.
 *
 * Parity is pinned two ways (see tests/test_oracle_pin.py):
 *   - against outputs of the reference itself, compiled from its own sources
 *     into oracle/_ref by oracle/Makefile (bit-exact, every operator);
 *   - against the golden fixtures committed under tests/golden/, which were
 *     produced by that reference build (tests/golden/make_golden.py).
 *
 * Conventions (identical to the reference):
 *   mask  : uint8 per node, row-major [y*nx + x], 1 = fluid, 0 = solid
 *   f     : SoA, direction-major [i*N + y*nx + x], N = nx*ny, 9 directions
 *   fields: [y*nx + x]
 * Arithmetic is IEEE double in the reference's operation order; build with
 * -ffp-contract=off so no multiply-add is fused.
 */
#ifndef SCLBM_ORACLE_H
#define SCLBM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* error codes mirror the reference's exception types */
#define ORC_OK 0
#define ORC_INVALID_ARGUMENT 1 /* std::invalid_argument */
#define ORC_RUNTIME_ERROR 2    /* std::runtime_error */
#define ORC_OUT_OF_RANGE 3     /* std::out_of_range (vector::at) */
#define ORC_DOMAIN_ERROR 4     /* division by zero in the reference (UB) */

/* ---------------- Geometry (src/geometry.cpp) ---------------- */
int orc_geom_add_walls(uint8_t *g, size_t nx, size_t ny, size_t dH, const char *where);
int orc_geom_add_rectangle(uint8_t *g, size_t nx, size_t ny, size_t Lx, size_t Ly, size_t xc, size_t yc);
int orc_geom_add_square(uint8_t *g, size_t nx, size_t ny, size_t Ls, size_t xc, size_t yc);
int orc_geom_add_ellipse(uint8_t *g, size_t nx, size_t ny, size_t Lx, size_t Ly, size_t xc, size_t yc);
int orc_geom_add_circle(uint8_t *g, size_t nx, size_t ny, size_t D, size_t xc, size_t yc);
/* props: parameters of the object in the order of its add_ function;
 * bounds = {x_lo, x_hi, y_lo, y_hi}; by_numbers selects the overload */
int orc_geom_add_array(uint8_t *g, size_t nx, size_t ny, const char *type, const size_t *props,
                       size_t nprops, const size_t *bounds, size_t a, size_t b, int by_numbers);

/* ---------------- Fluid (src/fluid.cpp) ---------------- */
void orc_compute_density(size_t N, const double *f, double *rho);
void orc_compute_velocities(size_t N, const uint8_t *g, const double *f, const double *rho,
                            double *ux, double *uy);
/* compute_f_equilibrium(geom): density + velocities + feq from (ux,uy) */
void orc_feq_single(size_t N, const uint8_t *g, const double *f, double *rho, double *ux,
                    double *uy, double *feq);
/* compute_f_equilibrium(): feq from rho and (u_eq_x,u_eq_y) */
void orc_feq_multi(size_t N, const double *rho, const double *uex, const double *uey, double *feq);

/* ---------------- initialisers (src/lbm.cpp:11-99, src/fluid.cpp:64-104) ---------------- */
/* f_bulk / f_drop are 9N each; only fluid nodes are written */
void orc_init_droplet(size_t nx, size_t ny, const uint8_t *g, double *f_bulk, double *f_drop,
                      double rho_bulk, double rho_drop, double rho_b_in_d, double rho_d_in_b,
                      double xc, double yc, double radius);
int orc_init_rectangle(size_t nx, size_t ny, const uint8_t *g, double *f_bulk, double *f_drop,
                       double rho_bulk, double rho_drop, double rho_b_in_d, double rho_d_in_b,
                       double xc, double yc, double half_lx, double half_ly);
void orc_simple_ini(size_t N, const uint8_t *g, double *f, double rho0);

/* ---------------- LBM (src/lbm.cpp) ---------------- */
/* compute_solid_surface_force: common sums Fxs/Fys (before the -Gs factor) */
void orc_solid_sum(size_t nx, size_t ny, const uint8_t *g, double *sx, double *sy);
/* Fluid::add_surface_forces factor: out = (-1.0*Gs)*s */
void orc_surface_force(size_t N, double gs, const double *sx, const double *sy, double *fsx,
                       double *fsy);
void orc_repulsive(size_t nx, size_t ny, const uint8_t *g, const double *rho1, const double *rho2,
                   double G1, double G2, double *f1x, double *f1y, double *f2x, double *f2y);
void orc_eqvel(size_t nx, size_t ny, const uint8_t *g, double omega1, double omega2,
               const double *f1, const double *f2, const double *rho1, const double *rho2,
               const double *fr1x, const double *fr1y, const double *fr2x, const double *fr2y,
               const double *fs1x, const double *fs1y, const double *fs2x, const double *fs2y,
               double *ux1, double *uy1, double *ux2, double *uy2, double *uex1, double *uey1,
               double *uex2, double *uey2);
void orc_collide(size_t N, double omega, double *f, const double *feq);
void orc_volume_force(size_t N, const uint8_t *g, double *f, const double *force9);
/* stream with half-way bounce-back; tmp is 9N scratch, f receives the result */
void orc_stream(size_t nx, size_t ny, const uint8_t *g, double *f, double *tmp);

/* ---------------- whole time steps (driver sequences) ---------------- */
/* Per-component state for the two-component sequence, all arrays caller-owned. */
typedef struct {
    double *f, *feq, *rho, *ux, *uy, *uex, *uey, *frx, *fry;
    const double *fsx, *fsy; /* solid force (already multiplied by -Gs) */
    double omega, G;
} orc_component;

/* nsteps of: density x2, repulsive, eqvel, collide(f1,f2), [volume force], stream
 * (laplace_law.cpp:123-133, droplet_in_a_channel.cpp:145-156).  force_mode bit0:
 * add_volume_force(geom,c1,force) ; bit1: c2 ; 3: the two-fluid overload. */
void orc_run_two(size_t nx, size_t ny, const uint8_t *g, orc_component *c1, orc_component *c2,
                 const double *force9, int force_mode, int nsteps, double *tmp);
/* nsteps of: collide(geom,f), add_volume_force, stream (laminar_flow_x_dir.cpp:64-68) */
void orc_run_single(size_t nx, size_t ny, const uint8_t *g, double omega, double *f,
                    double *feq, double *rho, double *ux, double *uy, const double *force9,
                    int nsteps, double *tmp);

#ifdef __cplusplus
}
#endif
#endif
