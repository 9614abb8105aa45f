// dropin_step.cpp -- C++ driver for the drop-in classes (sc_lbm_b200/host/include).
//
// Checks, on the GPU, that the fused LBM::step extension reproduces the
// reference drivers' per-method time step bit for bit, including around host
// edits made through the non-const getters between steps:
//   two components : laplace_law.cpp:123-133 sequence with a volume force on
//                    fluid 1 (droplet_in_a_channel.cpp:145-156 overloads)
//   one component  : laminar_flow_x_dir.cpp:64-68 sequence
// Writes fluid 1's density in the reference text format (write_density) and
// its populations as raw doubles, for the Python side to compare.
//
// usage: dropin_step <outdir>        exit 0 when every comparison is exact
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "geometry.h"
#include "lbm.h"

namespace {

int failures = 0;

void expect_equal(const std::string &what, const std::vector<double> &a, const std::vector<double> &b)
{
    size_t bad = 0;
    double worst = 0.0;
    if (a.size() != b.size()) {
        std::printf("%s: sizes %zu and %zu\n", what.c_str(), a.size(), b.size());
        ++failures;
        return;
    }
    for (size_t i = 0; i < a.size(); ++i)
        if (a[i] != b[i]) {
            ++bad;
            worst = std::max(worst, std::fabs(a[i] - b[i]));
        }
    std::printf("%s: %zu of %zu values differ (max %.3g)\n", what.c_str(), bad, a.size(), worst);
    if (bad) ++failures;
}

void build_porous(Geometry &g)
{
    g.add_walls(1, "x");
    g.add_circle(9, 30, 20);
    g.add_circle(13, 60, 28);
    g.add_circle(7, 80, 12);
    g.add_square(5, 15, 35);
}

struct TwoFluids {
    Fluid a{"water", 1. / 3, 0.7};
    Fluid b{"oil", 1. / 3, 1.3};
    TwoFluids(LBM &lbm, const Geometry &geom)
    {
        a.zero_density_ini(geom);
        b.zero_density_ini(geom);
        a.initialize_interactions(-0.2, 0.9);
        b.initialize_interactions(0.2, 0.9);
        lbm.initialize_droplet(geom, a, b, 2.0, 2.0, 0.06, 0.06, 48, 24, 10);
        lbm.compute_solid_surface_force(geom, a, b);
    }
};

// the same host-side edit on both copies: a few populations nudged in place
void edit(Fluid &f)
{
    std::vector<double> &v = f.get_f_dist();
    for (size_t k = 7; k < v.size(); k += 977) v[k] *= 1.0001;
}

void two_components(const std::string &outdir)
{
    Geometry geom(96, 48);
    build_porous(geom);
    LBM lbm(geom);
    TwoFluids ops(lbm, geom), fused(lbm, geom);
    const std::vector<double> force{0, 1e-5, 0, -1e-5, 0, 1e-5, -1e-5, -1e-5, 1e-5};

    for (int half = 0; half < 2; ++half) {
        for (int s = 0; s < 60; ++s) {
            ops.a.compute_density();
            ops.b.compute_density();
            lbm.compute_fluid_repulsive_interactions(geom, ops.a, ops.b);
            lbm.compute_equilibrium_velocities(geom, ops.a, ops.b);
            lbm.collide(ops.a, ops.b);
            lbm.add_volume_force(geom, ops.a, force);
            lbm.stream(geom, ops.a, ops.b);
        }
        lbm.step(geom, fused.a, fused.b, 60, force, {});
        if (half == 0) {
            edit(ops.a);
            edit(fused.a);
        }
    }
    const Fluid &ca = ops.a, &cb = ops.b, &fa = fused.a, &fb = fused.b;
    expect_equal("two components, fluid 1", ca.get_f_dist(), fa.get_f_dist());
    expect_equal("two components, fluid 2", cb.get_f_dist(), fb.get_f_dist());

    ops.a.write_density(outdir + "/rho1.txt");
    std::ofstream bin(outdir + "/f1.bin", std::ios::binary);
    const std::vector<double> &f = ca.get_f_dist();
    bin.write(reinterpret_cast<const char *>(f.data()), f.size() * sizeof(double));
}

void one_component()
{
    Geometry geom(200, 50);
    geom.add_walls(1, "x");
    LBM lbm(geom);
    Fluid ops("water", 1. / 3, 1.0), fused("water", 1. / 3, 1.0);
    ops.simple_ini(geom, 1.0);
    fused.simple_ini(geom, 1.0);
    const std::vector<double> force{0, 1e-6, 0, -1e-6, 0, 1e-6, -1e-6, -1e-6, 1e-6};
    for (int s = 0; s < 100; ++s) {
        lbm.collide(geom, ops);
        lbm.add_volume_force(geom, ops, force);
        lbm.stream(geom, ops);
    }
    lbm.step(geom, fused, 100, force);
    const Fluid &c = ops, &d = fused;
    expect_equal("one component", c.get_f_dist(), d.get_f_dist());
}

} // namespace

int main(int argc, char **argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <outdir>\n", argv[0]);
        return 2;
    }
    try {
        two_components(argv[1]);
        one_component();
    } catch (const std::exception &e) {
        std::printf("exception: %s\n", e.what());
        return 3;
    }
    return failures ? 1 : 0;
}
