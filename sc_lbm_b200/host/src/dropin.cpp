// dropin.cpp -- the reference's Geometry / Fluid / LBM classes implemented over
// the C ABI of libsclbm_b200 (include/sclbm.h).  Status codes become the
// reference's exception types; Fluid keeps host mirrors of its device arrays
// (synchronised lazily, see fluid.h).
#include "sclbm.h"

#include "fluid.h"
#include "geometry.h"
#include "lbm.h"

namespace {

void check(int rc)
{
    if (rc == SCLBM_OK) return;
    char buf[1024];
    sclbm_last_error(buf, sizeof buf);
    switch (rc) {
    case SCLBM_E_INVALID_ARGUMENT: throw std::invalid_argument(buf);
    case SCLBM_E_OUT_OF_RANGE: throw std::out_of_range(buf);
    case SCLBM_E_RUNTIME: throw std::runtime_error(buf);
    default: throw std::runtime_error(std::string("sclbm: ") + buf);
    }
}

enum : unsigned {
    F = 1u << 0, FEQ = 1u << 1, RHO = 1u << 2, UX = 1u << 3, UY = 1u << 4, UEQX = 1u << 5,
    UEQY = 1u << 6, FRX = 1u << 7, FRY = 1u << 8
};

} // namespace

// ============================================================== Geometry
Geometry::Geometry() { check(sclbm_geometry_create(0, 0, &h)); }

Geometry::Geometry(const size_t Nx, const size_t Ny) : _Nx(Nx), _Ny(Ny)
{
    geom.resize(_Nx * _Ny, 1);
    check(sclbm_geometry_create(Nx, Ny, &h));
}

Geometry::Geometry(const Geometry &o) : geom(o.geom), _Nx(o._Nx), _Ny(o._Ny)
{
    check(sclbm_geometry_create(_Nx, _Ny, &h));
    check(sclbm_geometry_set_mask(h, _Nx, _Ny, geom.data()));
}

Geometry &Geometry::operator=(const Geometry &o)
{
    if (this != &o) {
        geom = o.geom;
        _Nx = o._Nx;
        _Ny = o._Ny;
        check(sclbm_geometry_set_mask(h, _Nx, _Ny, geom.data()));
    }
    return *this;
}

Geometry::~Geometry() { sclbm_geometry_destroy(h); }

void Geometry::pull()
{
    if (!geom.empty()) sclbm_geometry_get_mask(h, geom.data(), geom.size());
}

// every mutation runs in the library (bit-exact with src/geometry.cpp); the
// mirror is refreshed even when it throws, since the reference leaves the
// mask modified as far as it got
#define GEOM_OP(call)                                                                          \
    do {                                                                                       \
        const int rc_ = (call);                                                                \
        pull();                                                                                \
        check(rc_);                                                                            \
    } while (0)

void Geometry::add_walls(const size_t dH, const std::string &where)
{
    GEOM_OP(sclbm_geometry_add_walls(h, dH, where.c_str()));
}
void Geometry::add_rectangle(const size_t Lx, const size_t Ly, const size_t xc, const size_t yc)
{
    GEOM_OP(sclbm_geometry_add_rectangle(h, Lx, Ly, xc, yc));
}
void Geometry::add_square(const size_t Ls, const size_t xc, const size_t yc)
{
    GEOM_OP(sclbm_geometry_add_square(h, Ls, xc, yc));
}
void Geometry::add_ellipse(const size_t Lx, const size_t Ly, const size_t xc, const size_t yc)
{
    GEOM_OP(sclbm_geometry_add_ellipse(h, Lx, Ly, xc, yc));
}
void Geometry::add_circle(const size_t D, const size_t xc, const size_t yc)
{
    GEOM_OP(sclbm_geometry_add_circle(h, D, xc, yc));
}

void Geometry::check_object_bounds(const size_t Lx, const size_t Ly, const size_t xc,
                                   const size_t yc, const std::string &name) const
{
    if ((static_cast<int>(xc) - static_cast<int>(Lx) / 2) < 0 ||
        (static_cast<int>(yc) - static_cast<int>(Ly) / 2) < 0)
        throw std::runtime_error(name + " lower bounds do not fit the domain.");
    if ((xc + Lx / 2) >= _Nx || (yc + Ly / 2) >= _Ny)
        throw std::runtime_error(name + " upper bounds do not fit the domain.");
}

void Geometry::check_constructed_object(const std::vector<size_t> &obj, const std::string &name) const
{
    if (!obj.empty() && *std::max_element(obj.begin(), obj.end()) >= _Nx * _Ny)
        throw std::runtime_error("Constructed " + name + " upper bounds do not fit the domain.");
}

static std::vector<size_t> bounds4(const std::vector<std::vector<size_t>> &b)
{
    return {b.at(0).at(0), b.at(0).at(1), b.at(1).at(0), b.at(1).at(1)};
}

void Geometry::add_array(const std::vector<size_t> &props,
                         const std::vector<std::vector<size_t>> &array_bounds, const size_t dx,
                         const size_t dy, const std::string &object_type, const size_t)
{
    const std::vector<size_t> b = bounds4(array_bounds);
    GEOM_OP(sclbm_geometry_add_array_spacing(h, props.data(), props.size(), b.data(), dx, dy,
                                             object_type.c_str()));
}

void Geometry::add_array(const std::vector<size_t> &props,
                         const std::vector<std::vector<size_t>> &array_bounds,
                         const std::vector<size_t> &object_numbers, const std::string &object_type,
                         const size_t)
{
    const std::vector<size_t> b = bounds4(array_bounds);
    GEOM_OP(sclbm_geometry_add_array_numbers(h, props.data(), props.size(), b.data(),
                                             object_numbers.at(0), object_numbers.at(1),
                                             object_type.c_str()));
}

void Geometry::set_node_fluid(const size_t xi, const size_t yi)
{
    geom.at(yi * _Nx + xi) = 1;
    check(sclbm_geometry_set_node(h, xi, yi, 1));
}

void Geometry::set_node_solid(const size_t xi, const size_t yi)
{
    geom.at(yi * _Nx + xi) = 0;
    check(sclbm_geometry_set_node(h, xi, yi, 0));
}

void Geometry::read(const std::string &fname)
{
    LbmIO io(fname, " ", true, {0, 0, 0});
    const std::vector<std::vector<int>> v = io.read_vector<int>();
    _Nx = v.at(0).size();
    _Ny = v.size();
    geom = vector_2D_2_flat_vector(v);
    check(sclbm_geometry_set_mask(h, _Nx, _Ny, geom.data()));
}

void Geometry::write(const std::string &fname) const
{
    LbmIO io(fname, " ", true, {0, 0, 0});
    io.write_vector<int>(flat_vector_2_vector_2D(_Nx, _Ny, geom));
}

const sclbm_geometry *Geometry::handle() const { return h; }

// ================================================================= Fluid
Fluid::Fluid(const std::string &s, const double speed, const double rel)
    : name(s), cs2(speed), tau(rel)
{
    omega = 1 / tau; // include/fluid.h:62
    nu = cs2 * (tau - 0.5);
}

Fluid::~Fluid() { sclbm_fluid_destroy(h); }

static size_t field_size(int field, size_t N) { return field <= 1 ? 9 * N : N; }

void Fluid::ensure(const Geometry &geom)
{
    if (h && Nx == geom.Nx() && Ny == geom.Ny()) return;
    if (h) {
        sclbm_fluid_destroy(h);
        h = nullptr;
    }
    Nx = geom.Nx();
    Ny = geom.Ny();
    Ntot = Nx * Ny;
    check(sclbm_fluid_create(Nx, Ny, tau, &h));
    check(sclbm_fluid_set_interactions(h, Gsolid, Gfluid_repulsion));
    for (int k = 0; k < 9; ++k) mirror[k].assign(field_size(k, Ntot), 0.0);
    host_stale = host_dirty = 0;
    solid_pushed = false;
    if (mirror[9].size() >= Ntot && Ntot) host_dirty |= 1u << 9 | 1u << 10;
}

std::vector<double> &Fluid::mut(int field)
{
    view(field);
    host_dirty |= 1u << field;
    return mirror[field];
}

const std::vector<double> &Fluid::view(int field) const
{
    const unsigned bit = 1u << field;
    if (h && (host_stale & bit)) {
        mirror[field].resize(field_size(field, Ntot));
        check(sclbm_fluid_read(h, (sclbm_field)field, mirror[field].data(), mirror[field].size()));
        host_stale &= ~bit;
    }
    return mirror[field];
}

sclbm_fluid *Fluid::device() const
{
    if (!h) throw std::out_of_range("vector::_M_range_check: the fluid was not initialised "
                                    "(zero_density_ini / simple_ini)");
    for (int k = 0; k < 9; ++k) {
        const unsigned bit = 1u << k;
        if (!(host_dirty & bit)) continue;
        if (mirror[k].size() != field_size(k, Ntot))
            throw std::invalid_argument("a Fluid array was resized by the caller");
        check(sclbm_fluid_write(h, (sclbm_field)k, mirror[k].data(), mirror[k].size()));
        host_dirty &= ~bit;
    }
    if (host_dirty & (1u << 9 | 1u << 10)) {
        // F_solid: the reference reads its first N entries (append semantics,
        // src/fluid.cpp:154-160); shorter vectors leave it unset
        if (mirror[9].size() >= Ntot && mirror[10].size() >= Ntot) {
            check(sclbm_fluid_write(h, SCLBM_FIELD_FSOLID_X, mirror[9].data(), Ntot));
            check(sclbm_fluid_write(h, SCLBM_FIELD_FSOLID_Y, mirror[10].data(), Ntot));
        }
        host_dirty &= ~(1u << 9 | 1u << 10);
    }
    return h;
}

void Fluid::device_changed(unsigned fields) const { host_stale |= fields; }

void Fluid::zero_density_ini(const Geometry &geom) { ensure(geom); }

void Fluid::simple_ini(const Geometry &geom, const double rho_0, const bool)
{
    ensure(geom);
    check(sclbm_fluid_simple_ini(device(), geom.handle(), rho_0));
    device_changed(F);
}

void Fluid::initialize_randomly_perturbed_density(const Geometry &geom, const double rho_0,
                                                  RNG &gen, const bool)
{
    // src/fluid.cpp:107-151: x outer, y inner, one draw per fluid node
    ensure(geom);
    std::vector<double> &f = mut(0);
    const double rho_factor = static_cast<double>(Ndir);
    const double rand_max = rho_0 / 1000.0;
    for (size_t i = 0; i < Nx; ++i)
        for (size_t j = 0; j < Ny; ++j)
            if (geom(i, j) == 1) {
                const double rho_rand = rho_0 + gen.get_random(0.0, rand_max);
                for (size_t k = 0; k < Ndir; ++k) f.at(k * Nx * Ny + j * Nx + i) = rho_rand / rho_factor;
            }
}

void Fluid::set_multicomponent_interactions(const double Gs)
{
    std::cout << "This function is deprecated and will be removed in future releases" << std::endl;
    Gsolid = Gs;
    if (h) check(sclbm_fluid_set_interactions(h, Gsolid, Gfluid_repulsion));
}

void Fluid::initialize_interactions(const double Gs, const double Gf)
{
    Gsolid = Gs;
    initialize_fluid_repulsion(Gf);
}

void Fluid::initialize_fluid_repulsion(const double Gf)
{
    Gfluid_repulsion = Gf;
    if (h) check(sclbm_fluid_set_interactions(h, Gsolid, Gfluid_repulsion));
}

void Fluid::add_surface_forces(const std::vector<double> Fxs, const std::vector<double> Fys)
{
    for (double el : Fxs) mirror[9].push_back(-1.0 * Gsolid * el);
    for (double el : Fys) mirror[10].push_back(-1.0 * Gsolid * el);
    host_dirty |= 1u << 9 | 1u << 10;
}

void Fluid::compute_density()
{
    check(sclbm_fluid_compute_density(device()));
    device_changed(RHO);
}

void Fluid::compute_velocities(const Geometry &geom)
{
    check(sclbm_fluid_compute_velocities(device(), geom.handle()));
    device_changed(UX | UY);
}

void Fluid::compute_macroscopic(const Geometry &geom)
{
    compute_density();
    compute_velocities(geom);
}

void Fluid::compute_f_equilibrium(const Geometry &geom)
{
    check(sclbm_fluid_compute_f_equilibrium_geom(device(), geom.handle()));
    device_changed(FEQ | RHO | UX | UY);
}

void Fluid::compute_f_equilibrium()
{
    check(sclbm_fluid_compute_f_equilibrium(device()));
    device_changed(FEQ);
}

void Fluid::restart_from_file(const std::string &fname)
{
    std::vector<double> &f = mut(0);
    for (size_t id = 0; id < Ndir; ++id) {
        LbmIO io(fname + "_" + std::to_string(id) + ".txt", " ", true, {Ny, Nx, 0});
        const std::vector<std::vector<double>> v = io.read_vector<double>();
        for (size_t yj = 0; yj < Ny; ++yj)
            std::copy(v.at(yj).cbegin(), v.at(yj).cend(), f.begin() + (id * Ntot + yj * Nx));
    }
}

// rows of Nx values cut as src/fluid.cpp:303-343 cuts them (sclbm_write_rows)
void Fluid::write_var(const std::vector<double> &variable, const std::string &fname) const
{
    if (variable.size() < Nx * Ny) throw std::out_of_range("vector::_M_range_check: short variable");
    const int rc = sclbm_write_rows(fname.c_str(), variable.data(), Nx, Ny);
    if (rc == SCLBM_E_RUNTIME) {
        char buf[1024];
        sclbm_last_error(buf, sizeof buf);
        throw std::ios_base::failure(buf);
    }
    check(rc);
}

void Fluid::write_var(const std::vector<double> &variable, const std::string &fname, const bool) const
{
    std::vector<double> temp(Nx * Ny, -1.0);
    for (size_t i = 0; i < Ndir; ++i) {
        std::copy(variable.cbegin() + i * Nx * Ny, variable.cbegin() + (i + 1) * Nx * Ny, temp.begin());
        write_var(temp, fname + "_" + std::to_string(i) + ".txt");
    }
}

void Fluid::save_state(const std::string &frho, const std::string &fux, const std::string &fuy,
                       const int step, const Geometry &geom)
{
    compute_density();
    write_var(view(2), frho + "_" + std::to_string(step) + ".txt");
    compute_velocities(geom);
    write_var(view(3), fux + "_" + std::to_string(step) + ".txt");
    write_var(view(4), fuy + "_" + std::to_string(step) + ".txt");
}

// =================================================================== LBM
LBM::LBM(const Geometry &geom)
{
    Nx = geom.Nx();
    Ny = geom.Ny();
    Ntot = Nx * Ny;
    check(sclbm_lbm_create(geom.handle(), &h));
}

LBM::~LBM() { sclbm_lbm_destroy(h); }

void LBM::initialize_droplet(const Geometry &geom, Fluid &bulk, Fluid &droplet,
                             const double rho_bulk, const double rho_droplet,
                             const double rho_b_in_d, const double rho_d_in_b, const double xc,
                             const double yc, const double radius)
{
    check(sclbm_lbm_initialize_droplet(h, geom.handle(), bulk.device(), droplet.device(), rho_bulk,
                                       rho_droplet, rho_b_in_d, rho_d_in_b, xc, yc, radius));
    bulk.device_changed(F);
    droplet.device_changed(F);
}

void LBM::initialize_fluid_rectangle(const Geometry &geom, Fluid &bulk, Fluid &droplet,
                                     const double rho_bulk, const double rho_droplet,
                                     const double rho_b_in_d, const double rho_d_in_b,
                                     const double xc, const double yc, const double half_Lx,
                                     const double half_Ly)
{
    const int rc = sclbm_lbm_initialize_fluid_rectangle(h, geom.handle(), bulk.device(),
                                                        droplet.device(), rho_bulk, rho_droplet,
                                                        rho_b_in_d, rho_d_in_b, xc, yc, half_Lx,
                                                        half_Ly);
    bulk.device_changed(F);
    droplet.device_changed(F);
    check(rc);
}

void LBM::compute_solid_surface_force(const Geometry &geom, Fluid &f1, Fluid &f2)
{
    // src/lbm.cpp:102-141: common sums, then -Gs per fluid (append semantics)
    std::vector<double> Fxs(Ntot), Fys(Ntot);
    check(sclbm_lbm_solid_surface_sums(h, geom.handle(), Fxs.data(), Fys.data(), Ntot));
    f1.add_surface_forces(Fxs, Fys);
    f2.add_surface_forces(Fxs, Fys);
}

void LBM::compute_fluid_repulsive_interactions(const Geometry &geom, Fluid &f1, Fluid &f2)
{
    check(sclbm_lbm_fluid_repulsive_interactions(h, geom.handle(), f1.device(), f2.device()));
    f1.device_changed(FRX | FRY);
    f2.device_changed(FRX | FRY);
}

void LBM::compute_equilibrium_velocities(Geometry &geom, Fluid &f1, Fluid &f2)
{
    check(sclbm_lbm_equilibrium_velocities(h, geom.handle(), f1.device(), f2.device()));
    f1.device_changed(UX | UY | UEQX | UEQY);
    f2.device_changed(UX | UY | UEQX | UEQY);
}

void LBM::collide(const Geometry &geom, Fluid &f)
{
    check(sclbm_lbm_collide_single(h, geom.handle(), f.device()));
    f.device_changed(F | FEQ | RHO | UX | UY);
}

void LBM::collide(Fluid &f1, Fluid &f2)
{
    check(sclbm_lbm_collide(h, f1.device(), f2.device()));
    f1.device_changed(F | FEQ);
    f2.device_changed(F | FEQ);
}

void LBM::add_volume_force(const Geometry &geom, Fluid &f, const std::vector<double> &force)
{
    check(sclbm_lbm_add_volume_force_single(h, geom.handle(), f.device(), force.data(), force.size()));
    f.device_changed(F);
}

void LBM::add_volume_force(const Geometry &geom, Fluid &f1, Fluid &f2,
                           const std::vector<double> &force)
{
    check(sclbm_lbm_add_volume_force(h, geom.handle(), f1.device(), f2.device(), force.data(),
                                     force.size()));
    f1.device_changed(F);
    f2.device_changed(F);
}

void LBM::stream(const Geometry &geom, Fluid &f)
{
    check(sclbm_lbm_stream_single(h, geom.handle(), f.device()));
    f.device_changed(F);
}

void LBM::stream(const Geometry &geom, Fluid &f1, Fluid &f2)
{
    check(sclbm_lbm_stream(h, geom.handle(), f1.device(), f2.device()));
    f1.device_changed(F);
    f2.device_changed(F);
}

static const double *force_ptr(const std::vector<double> &v)
{
    if (v.empty()) return nullptr;
    if (v.size() < 9) throw std::out_of_range("vector::_M_range_check: a volume force needs 9 values");
    return v.data();
}

void LBM::step(const Geometry &geom, Fluid &f1, Fluid &f2, int nsteps,
               const std::vector<double> &force1, const std::vector<double> &force2)
{
    check(sclbm_lbm_step(h, geom.handle(), f1.device(), f2.device(), force_ptr(force1),
                         force_ptr(force2), nsteps));
    f1.device_changed(F);
    f2.device_changed(F);
}

void LBM::step(const Geometry &geom, Fluid &f, int nsteps, const std::vector<double> &force)
{
    check(sclbm_lbm_step_single(h, geom.handle(), f.device(), force_ptr(force), nsteps));
    f.device_changed(F);
}
