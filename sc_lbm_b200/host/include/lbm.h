#ifndef LBM_H
#define LBM_H

// LBM: the step operators of the reference's include/lbm.h:23-135, each one a
// call into libsclbm_b200 (sm_100a kernels, FP64, the reference's operation
// order: results are bit-identical to the serial reference).  step() is an
// extension that runs the whole driver time step in one fused kernel.
#include "common.h"
#include "fluid.h"
#include "geometry.h"
#include "io_operations/lbm_io.h"
#include "utils.h"

struct sclbm_lbm;
class Fluid;

class LBM {
public:
    LBM() = delete;
    LBM(const Geometry &geom);
    LBM(const LBM &) = delete;
    LBM &operator=(const LBM &) = delete;
    ~LBM();

    void initialize_droplet(const Geometry &geom, Fluid &bulk, Fluid &droplet,
                            const double rho_bulk, const double rho_droplet,
                            const double rho_b_in_d, const double rho_d_in_b, const double xc,
                            const double yc, const double radius);
    void initialize_fluid_rectangle(const Geometry &geom, Fluid &bulk, Fluid &droplet,
                                    const double rho_bulk, const double rho_droplet,
                                    const double rho_b_in_d, const double rho_d_in_b,
                                    const double xc, const double yc, const double half_Lx,
                                    const double half_Ly);
    void compute_solid_surface_force(const Geometry &, Fluid &, Fluid &);
    void compute_fluid_repulsive_interactions(const Geometry &, Fluid &, Fluid &);
    void compute_equilibrium_velocities(Geometry &geom, Fluid &, Fluid &);
    void collide(const Geometry &geom, Fluid &);
    void collide(Fluid &, Fluid &);
    void add_volume_force(const Geometry &, Fluid &, const std::vector<double> &);
    void add_volume_force(const Geometry &, Fluid &, Fluid &, const std::vector<double> &);
    void stream(const Geometry &, Fluid &);
    void stream(const Geometry &, Fluid &, Fluid &);

    /// Extension: nsteps of compute_density x2, compute_fluid_repulsive_
    /// interactions, compute_equilibrium_velocities, collide, [add_volume_force
    /// with force1 on fluid_1 / force2 on fluid_2 when non-empty], stream, in one
    /// fused kernel per step.  Populations are bit-identical to calling the
    /// methods; rho, u, u_eq, F_repulsive and f_eq keep their previous values.
    void step(const Geometry &geom, Fluid &fluid_1, Fluid &fluid_2, int nsteps,
              const std::vector<double> &force1 = {}, const std::vector<double> &force2 = {});
    /// Extension: nsteps of collide(geom, f), [add_volume_force], stream.
    void step(const Geometry &geom, Fluid &fluid, int nsteps,
              const std::vector<double> &force = {});

private:
    size_t Nx = 0, Ny = 0, Ntot = 0, Ndir = 9;
    sclbm_lbm *h = nullptr;
};

#endif
