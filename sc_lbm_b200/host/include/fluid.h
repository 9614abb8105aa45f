#ifndef FLUID_H
#define FLUID_H

// Fluid: one component, with the interface of the reference's
// include/fluid.h:52-320.  The arrays live on the GPU (FP64, reference layout
// [i*N + y*Nx + x]); the std::vector objects the getters return are host
// mirrors, refreshed from the device when a getter is called.  A non-const
// getter hands out a writable mirror, so the next device operation uploads it
// first: drivers that write populations or forces in place keep working.  A
// reference obtained from a getter is a snapshot -- call the getter again
// after device operations to see their results.
#include "common.h"
#include "geometry.h"
#include "io_operations/lbm_io.h"
#include "rng.h"
#include "utils.h"

struct sclbm_fluid;
class LBM;

class Fluid {
public:
    Fluid(const std::string &s, const double speed, const double rel);
    Fluid(const std::string &s) : Fluid(s, 1. / 3, 1.0) {}
    Fluid() : Fluid("fluid", 1. / 3, 1.0) {}
    Fluid(const Fluid &) = delete;
    Fluid &operator=(const Fluid &) = delete;
    ~Fluid();

    // initialisation (src/fluid.cpp:43-168)
    void zero_density_ini(const Geometry &geom);
    void simple_ini(const Geometry &geom, const double rho_0, const bool mcmp = false);
    void initialize_randomly_perturbed_density(const Geometry &geom, const double rho_0, RNG &gen,
                                               const bool mcmp = false);
    void set_multicomponent_interactions(const double Gs);
    void initialize_interactions(const double Gs, const double Gf);
    void add_surface_forces(const std::vector<double>, const std::vector<double>);
    void initialize_fluid_repulsion(const double Gf);

    // macroscopic properties (src/fluid.cpp:175-278)
    void compute_density();
    void compute_velocities(const Geometry &geom);
    void compute_macroscopic(const Geometry &geom);
    void compute_f_equilibrium(const Geometry &geom);
    void compute_f_equilibrium();

    // getters (include/fluid.h:150-201)
    std::vector<double> &get_f_dist() { return mut(0); }
    std::vector<double> &get_f_eq_dist() { return mut(1); }
    std::vector<double> &get_fluid_solid_force_x() { return mut(9); }
    std::vector<double> &get_fluid_solid_force_y() { return mut(10); }
    std::vector<double> &get_repulsive_force_x() { return mut(7); }
    std::vector<double> &get_repulsive_force_y() { return mut(8); }
    std::vector<double> &get_rho() { return mut(2); }
    std::vector<double> &get_ux() { return mut(3); }
    std::vector<double> &get_uy() { return mut(4); }
    std::vector<double> &get_u_eq_x() { return mut(5); }
    std::vector<double> &get_u_eq_y() { return mut(6); }
    const std::vector<double> &get_f_dist() const { return view(0); }
    const std::vector<double> &get_f_eq_dist() const { return view(1); }
    const std::vector<double> &get_fluid_solid_force_x() const { return view(9); }
    const std::vector<double> &get_fluid_solid_force_y() const { return view(10); }
    const std::vector<double> &get_rho() const { return view(2); }
    const std::vector<double> &get_ux() const { return view(3); }
    const std::vector<double> &get_uy() const { return view(4); }
    const std::vector<double> &get_u_eq_x() const { return view(5); }
    const std::vector<double> &get_u_eq_y() const { return view(6); }

    size_t get_Nx() const { return Nx; }
    size_t get_Ny() const { return Ny; }
    double get_omega() const { return omega; }
    double get_repulsive_g_fluid() const { return Gfluid_repulsion; }
    std::vector<double> get_wrts() const { return {wrt0, wrt1, wrt2}; }

    /// Populations from fname_<dir>.txt, one row of Nx values per line
    void restart_from_file(const std::string &fname);

    // output (include/fluid.h:219-254)
    void write_density(const std::string &fname)
    {
        compute_density();
        write_var(view(2), fname);
    }
    void write_ux(const std::string &fname, const Geometry &geom)
    {
        compute_velocities(geom);
        write_var(view(3), fname);
    }
    void write_uy(const std::string &fname, const Geometry &geom)
    {
        compute_velocities(geom);
        write_var(view(4), fname);
    }
    void write_F_repulsive_x(const std::string &fname) { write_var(view(7), fname); }
    void write_F_repulsive_y(const std::string &fname) { write_var(view(8), fname); }
    void write_u_eq_x(const std::string &fname) { write_var(view(5), fname); }
    void write_u_eq_y(const std::string &fname) { write_var(view(6), fname); }
    void write_feq(const std::string &fname) const { write_var(view(1), fname, true); }
    void write_f(const std::string &fname) const { write_var(view(0), fname, true); }
    void save_state(const std::string &frho, const std::string &fux, const std::string &fuy,
                    const int step, const Geometry &geom);

    // ---- extensions of the B200 build ----
    /// The C-ABI handle, after pushing any host-side edits to the device
    sclbm_fluid *device() const;
    /// Mark the host mirrors stale (the device changed the arrays)
    void device_changed(unsigned fields) const;

private:
    std::string name;
    const size_t Ndir = 9;
    double cs2 = 0.0, tau = 0.0, nu = 0.0, omega = 0.0;
    double Gsolid = 0.0, Gfluid_repulsion = 0.0;
    double wrt0 = 4.0 / 9.0, wrt1 = 1.0 / 9.0, wrt2 = 1.0 / 36.0;
    size_t Nx = 0, Ny = 0, Ntot = 0;

    // host mirrors of the 11 device arrays (order of sclbm_field)
    mutable std::vector<double> mirror[11];
    mutable unsigned host_stale = 0; // device newer than the mirror
    mutable unsigned host_dirty = 0; // mirror newer than the device
    mutable sclbm_fluid *h = nullptr;
    bool solid_pushed = false;

    void ensure(const Geometry &geom); // device arrays sized for geom
    std::vector<double> &mut(int field);
    const std::vector<double> &view(int field) const;
    void write_var(const std::vector<double> &variable, const std::string &fname) const;
    void write_var(const std::vector<double> &variable, const std::string &fname,
                   const bool is_3D) const;
    friend class LBM;
};

#include "lbm.h"

#endif
