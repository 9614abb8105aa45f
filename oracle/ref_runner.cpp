// ref_runner.cpp -- drives the UNMODIFIED reference library (LBMFluids/sc_lbm),
// compiled from its own sources by oracle/Makefile into oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY: it produces golden outputs to pin the C oracle
// (tests/golden/make_golden.py, tests/test_oracle_pin.py) and times the
// reference's serial step for bench.py's reference arm.  The call sequences
// are those of the reference drivers:
//   two components: laplace_law.cpp:123-133, droplet_in_a_channel.cpp:145-156
//   one component : laminar_flow_x_dir.cpp:64-68
//   per operator  : tests/lbm/lbm_tests.cpp:12-44 and :119-127
//
// usage: sclbm_ref_runner case <spec.txt>      (writes the path named by `out`)
//        sclbm_ref_runner bench <nx> <ny> <steps> <seed> [max_seconds min_steps]
//        sclbm_ref_runner text <f.bin> <nx> <ny> <prefix>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "geometry.h"
#include "lbm.h"

namespace {

struct Out {
    std::ofstream os;
    explicit Out(const std::string &p) : os(p, std::ios::binary) { os.write("SCLBMREF", 8); }
    void put(const std::string &name, const std::vector<double> &v)
    {
        char nm[48] = {0};
        std::strncpy(nm, name.c_str(), 47);
        os.write(nm, 48);
        int32_t dt = 0;
        int64_t n = (int64_t)v.size();
        os.write((const char *)&dt, 4);
        os.write((const char *)&n, 8);
        os.write((const char *)v.data(), n * 8);
    }
    void put(const std::string &name, const std::vector<int> &v)
    {
        char nm[48] = {0};
        std::strncpy(nm, name.c_str(), 47);
        os.write(nm, 48);
        int32_t dt = 1;
        int64_t n = (int64_t)v.size();
        os.write((const char *)&dt, 4);
        os.write((const char *)&n, 8);
        for (int x : v) {
            int32_t y = x;
            os.write((const char *)&y, 4);
        }
    }
};

void dump_fluid(Out &o, const std::string &p, Fluid &fl, bool mcmp)
{
    o.put(p + "f", fl.get_f_dist());
    o.put(p + "feq", fl.get_f_eq_dist());
    o.put(p + "rho", fl.get_rho());
    o.put(p + "ux", fl.get_ux());
    o.put(p + "uy", fl.get_uy());
    if (mcmp) {
        o.put(p + "uex", fl.get_u_eq_x());
        o.put(p + "uey", fl.get_u_eq_y());
        o.put(p + "frx", fl.get_repulsive_force_x());
        o.put(p + "fry", fl.get_repulsive_force_y());
        o.put(p + "fsx", fl.get_fluid_solid_force_x());
        o.put(p + "fsy", fl.get_fluid_solid_force_y());
    }
}

std::vector<double> read_doubles(const std::string &path, size_t n)
{
    std::vector<double> v(n);
    std::ifstream is(path, std::ios::binary);
    is.read((char *)v.data(), n * 8);
    if ((size_t)is.gcount() != n * 8) throw std::runtime_error("short init file " + path);
    return v;
}

int exception_code(const std::exception &e)
{
    if (dynamic_cast<const std::invalid_argument *>(&e)) return 1;
    if (dynamic_cast<const std::out_of_range *>(&e)) return 3;
    if (dynamic_cast<const std::runtime_error *>(&e)) return 2;
    return 9;
}

int run_case(const std::string &spec)
{
    std::ifstream in(spec);
    if (!in) {
        std::fprintf(stderr, "cannot open %s\n", spec.c_str());
        return 2;
    }
    size_t nx = 0, ny = 0;
    std::string mode = "mask", out_path, init_kind, init_file;
    std::vector<double> init_args;
    double tau[2] = {1.0, 1.0}, G[2] = {0, 0}, Gs[2] = {0, 0};
    int force_mode = 0, steps = 0;
    std::vector<double> force(9, 0.0);
    std::vector<std::string> geom_cmds;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string k;
        if (!(ls >> k) || k[0] == '#') continue;
        if (k == "size") ls >> nx >> ny;
        else if (k == "mode") ls >> mode;
        else if (k == "out") ls >> out_path;
        else if (k == "fluid1") ls >> tau[0] >> G[0] >> Gs[0];
        else if (k == "fluid2") ls >> tau[1] >> G[1] >> Gs[1];
        else if (k == "steps") ls >> steps;
        else if (k == "force") {
            ls >> force_mode;
            for (auto &x : force) ls >> x;
        } else if (k == "init") {
            ls >> init_kind;
            if (init_kind == "file") ls >> init_file;
            else {
                double a;
                while (ls >> a) init_args.push_back(a);
            }
        } else geom_cmds.push_back(line);
    }
    Out o(out_path);
    Geometry geom(nx, ny);
    int err = 0;
    try {
        for (const auto &c : geom_cmds) {
            std::istringstream ls(c);
            std::string k;
            ls >> k;
            if (k == "walls") {
                size_t dh;
                std::string d;
                ls >> dh >> d;
                geom.add_walls(dh, d);
            } else if (k == "rectangle") {
                size_t a, b, x, y;
                ls >> a >> b >> x >> y;
                geom.add_rectangle(a, b, x, y);
            } else if (k == "square") {
                size_t a, x, y;
                ls >> a >> x >> y;
                geom.add_square(a, x, y);
            } else if (k == "ellipse") {
                size_t a, b, x, y;
                ls >> a >> b >> x >> y;
                geom.add_ellipse(a, b, x, y);
            } else if (k == "circle") {
                size_t a, x, y;
                ls >> a >> x >> y;
                geom.add_circle(a, x, y);
            } else if (k == "array_n" || k == "array_d") {
                std::string t;
                size_t np;
                ls >> t >> np;
                std::vector<size_t> p(np);
                for (auto &x : p) ls >> x;
                size_t b0, b1, b2, b3, a, b;
                ls >> b0 >> b1 >> b2 >> b3 >> a >> b;
                if (k == "array_n") geom.add_array(p, {{b0, b1}, {b2, b3}}, {a, b}, t);
                else geom.add_array(p, {{b0, b1}, {b2, b3}}, a, b, t);
            } else if (k == "fluid_node") {
                size_t x, y;
                ls >> x >> y;
                geom.set_node_fluid(x, y);
            } else if (k == "solid_node") {
                size_t x, y;
                ls >> x >> y;
                geom.set_node_solid(x, y);
            }
        }
    } catch (const std::exception &e) {
        err = exception_code(e);
    }
    o.put("mask", geom.get_geom());
    o.put("error", std::vector<int>{err});
    if (mode == "mask" || err) return 0;

    const size_t N = nx * ny;
    LBM lbm(geom);
    if (mode == "single" || mode == "ops1") {
        Fluid fl("fluid", 1. / 3, tau[0]);
        if (init_kind == "simple") fl.simple_ini(geom, init_args.at(0));
        else {
            fl.simple_ini(geom, 1.0);
            fl.get_f_dist() = read_doubles(init_file, 9 * N);
        }
        if (mode == "ops1") { // lbm_tests.cpp:12-44
            lbm.collide(geom, fl);
            dump_fluid(o, "collide_", fl, false);
            lbm.add_volume_force(geom, fl, force);
            o.put("force_f", fl.get_f_dist());
            lbm.stream(geom, fl);
            o.put("stream_f", fl.get_f_dist());
            return 0;
        }
        const auto t0 = std::chrono::steady_clock::now();
        for (int s = 0; s < steps; ++s) {
            lbm.collide(geom, fl);
            if (force_mode) lbm.add_volume_force(geom, fl, force);
            lbm.stream(geom, fl);
        }
        // main-loop time only (the drivers' "Simulation time (main loop only)")
        o.put("loop_seconds", std::vector<double>{
                                  std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()});
        dump_fluid(o, "c1_", fl, false);
        fl.compute_macroscopic(geom);
        o.put("c1_rho_final", fl.get_rho());
        o.put("c1_ux_final", fl.get_ux());
        o.put("c1_uy_final", fl.get_uy());
        return 0;
    }
    // two components (droplet_tests.cpp:82-127 / laplace_law.cpp:95-133)
    Fluid a("water", 1. / 3, tau[0]), b("oil", 1. / 3, tau[1]);
    a.zero_density_ini(geom);
    b.zero_density_ini(geom);
    a.initialize_interactions(Gs[0], G[0]);
    b.initialize_interactions(Gs[1], G[1]);
    if (init_kind == "droplet")
        lbm.initialize_droplet(geom, a, b, init_args.at(0), init_args.at(1), init_args.at(2),
                               init_args.at(3), init_args.at(4), init_args.at(5), init_args.at(6));
    else if (init_kind == "rectangle")
        lbm.initialize_fluid_rectangle(geom, a, b, init_args.at(0), init_args.at(1),
                                       init_args.at(2), init_args.at(3), init_args.at(4),
                                       init_args.at(5), init_args.at(6), init_args.at(7));
    else {
        std::vector<double> v = read_doubles(init_file, 18 * N);
        a.get_f_dist().assign(v.begin(), v.begin() + 9 * N);
        b.get_f_dist().assign(v.begin() + 9 * N, v.end());
    }
    lbm.compute_solid_surface_force(geom, a, b);
    if (mode == "ops2") {
        a.compute_density();
        b.compute_density();
        o.put("density_c1_rho", a.get_rho());
        o.put("density_c2_rho", b.get_rho());
        lbm.compute_fluid_repulsive_interactions(geom, a, b);
        o.put("rep_c1_frx", a.get_repulsive_force_x());
        o.put("rep_c1_fry", a.get_repulsive_force_y());
        o.put("rep_c2_frx", b.get_repulsive_force_x());
        o.put("rep_c2_fry", b.get_repulsive_force_y());
        lbm.compute_equilibrium_velocities(geom, a, b);
        o.put("eqv_c1_ux", a.get_ux());
        o.put("eqv_c1_uy", a.get_uy());
        o.put("eqv_c2_ux", b.get_ux());
        o.put("eqv_c2_uy", b.get_uy());
        o.put("eqv_c1_uex", a.get_u_eq_x());
        o.put("eqv_c1_uey", a.get_u_eq_y());
        o.put("eqv_c2_uex", b.get_u_eq_x());
        o.put("eqv_c2_uey", b.get_u_eq_y());
        lbm.collide(a, b);
        o.put("collide_c1_f", a.get_f_dist());
        o.put("collide_c2_f", b.get_f_dist());
        o.put("collide_c1_feq", a.get_f_eq_dist());
        o.put("collide_c2_feq", b.get_f_eq_dist());
        lbm.add_volume_force(geom, a, b, force);
        o.put("force_c1_f", a.get_f_dist());
        o.put("force_c2_f", b.get_f_dist());
        lbm.stream(geom, a, b);
        o.put("stream_c1_f", a.get_f_dist());
        o.put("stream_c2_f", b.get_f_dist());
        return 0;
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (int s = 0; s < steps; ++s) {
        a.compute_density();
        b.compute_density();
        lbm.compute_fluid_repulsive_interactions(geom, a, b);
        lbm.compute_equilibrium_velocities(geom, a, b);
        lbm.collide(a, b);
        if (force_mode == 3) lbm.add_volume_force(geom, a, b, force);
        else if (force_mode == 1) lbm.add_volume_force(geom, a, force);
        else if (force_mode == 2) lbm.add_volume_force(geom, b, force);
        lbm.stream(geom, a, b);
    }
    o.put("loop_seconds", std::vector<double>{
                              std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()});
    dump_fluid(o, "c1_", a, true);
    dump_fluid(o, "c2_", b, true);
    a.compute_macroscopic(geom);
    b.compute_macroscopic(geom);
    o.put("c1_rho_final", a.get_rho());
    o.put("c1_ux_final", a.get_ux());
    o.put("c1_uy_final", a.get_uy());
    o.put("c2_rho_final", b.get_rho());
    o.put("c2_ux_final", b.get_ux());
    o.put("c2_uy_final", b.get_uy());
    return 0;
}

// Serial timing of the reference two-component step (spinodal-type periodic
// domain, rho = 1 +- 1% per component, G = 1.2, tau = 1), for the CPU baseline.
// Runs `steps` steps, or stops early once max_seconds (> 0) have passed and at
// least min_steps steps are done (large lattices take seconds per step).
int run_bench(size_t nx, size_t ny, int steps, unsigned seed, double max_seconds, int min_steps)
{
    Geometry geom(nx, ny);
    LBM lbm(geom);
    Fluid a("a"), b("b");
    a.zero_density_ini(geom);
    b.zero_density_ini(geom);
    a.initialize_interactions(0.0, 1.2);
    b.initialize_interactions(0.0, 1.2);
    const size_t N = nx * ny;
    uint64_t s = seed * 0x9E3779B97F4A7C15ull + 1;
    auto u01 = [&s]() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return (double)(s >> 11) * (1.0 / 9007199254740992.0);
    };
    for (Fluid *fl : {&a, &b}) {
        std::vector<double> &f = fl->get_f_dist();
        for (size_t i = 0; i < N; ++i) {
            double r = 1.0 + 0.02 * (u01() - 0.5);
            for (size_t d = 0; d < 9; ++d) f[d * N + i] = r / 9.0;
        }
    }
    lbm.compute_solid_surface_force(geom, a, b);
    std::vector<double> per_step;
    auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < steps; ++k) {
        auto ts = std::chrono::steady_clock::now();
        a.compute_density();
        b.compute_density();
        lbm.compute_fluid_repulsive_interactions(geom, a, b);
        lbm.compute_equilibrium_velocities(geom, a, b);
        lbm.collide(a, b);
        lbm.stream(geom, a, b);
        per_step.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count());
        if (max_seconds > 0.0 && k + 1 >= min_steps &&
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > max_seconds)
            break;
    }
    steps = (int)per_step.size();
    double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    double chk = 0.0;
    for (double x : a.get_f_dist()) chk += x;
    std::printf("{\"nx\": %zu, \"ny\": %zu, \"steps\": %d, \"seconds\": %.6f, \"mlups\": %.6f, "
                "\"checksum\": %.17g, \"step_seconds\": [",
                nx, ny, steps, dt, (double)N * steps / dt / 1e6, chk);
    for (size_t k = 0; k < per_step.size(); ++k) std::printf("%s%.6f", k ? ", " : "", per_step[k]);
    std::printf("]}\n");
    return 0;
}

// The reference's own text output of one all-fluid component whose
// populations are read from f.bin (9*nx*ny doubles): write_density,
// write_ux, write_uy and write_f with the given path prefix
// (src/fluid.cpp:303-353, include/fluid.h:219-251).
int run_text(const std::string &fbin, size_t nx, size_t ny, const std::string &prefix)
{
    Geometry geom(nx, ny);
    Fluid fl("fluid", 1. / 3, 1.0);
    fl.simple_ini(geom, 1.0);
    fl.get_f_dist() = read_doubles(fbin, 9 * nx * ny);
    fl.write_density(prefix + "_rho.txt");
    fl.write_ux(prefix + "_ux.txt", geom);
    fl.write_uy(prefix + "_uy.txt", geom);
    fl.write_f(prefix + "_f");
    return 0;
}

} // namespace

int main(int argc, char **argv)
{
    if (argc >= 3 && std::string(argv[1]) == "case") return run_case(argv[2]);
    if (argc >= 6 && std::string(argv[1]) == "text")
        return run_text(argv[2], std::strtoull(argv[3], 0, 10), std::strtoull(argv[4], 0, 10),
                        argv[5]);
    if (argc >= 5 && std::string(argv[1]) == "bench")
        return run_bench(std::strtoull(argv[2], 0, 10), std::strtoull(argv[3], 0, 10),
                         std::atoi(argv[4]), argc > 5 ? (unsigned)std::atoi(argv[5]) : 1u,
                         argc > 6 ? std::atof(argv[6]) : 0.0, argc > 7 ? std::atoi(argv[7]) : 1);
    std::fprintf(stderr, "usage: %s case <spec> | bench <nx> <ny> <steps> [seed [max_seconds min_steps]]\n",
                 argv[0]);
    return 2;
}
