// capi.cu -- the extern "C" boundary of libsclbm_b200.so (include/sclbm.h):
// object lifetimes, argument checks that reproduce the reference's exceptions
// as status codes, and the launches of the per-operator and fused kernels.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "domain.h"
#include "internal.h"
#include "ops_fp64.h"

namespace sclbm {

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;

int set_error(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    return set_error(SCLBM_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ------------------------------------------------------------ device, stream
static std::mutex g_mu;
static cudaStream_t g_user_stream = nullptr;
static cudaStream_t g_own_stream = nullptr;
static bool g_user_set = false;
static int g_sms = 0;
static int g_dev_checked = 0; // 0 unknown, 1 ok, -1 unusable

int ensure_device()
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_dev_checked == 1) return SCLBM_OK;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(SCLBM_E_NO_DEVICE, "no CUDA device available");
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess)
        return set_error(SCLBM_E_NO_DEVICE, "cannot query the CUDA device");
    if (p.major != 10)
        return set_error(SCLBM_E_NO_DEVICE, std::string("libsclbm_b200 is built for sm_100a; device is ") +
                                                p.name);
    g_sms = p.multiProcessorCount;
    if (!g_own_stream) {
        if (cudaStreamCreateWithFlags(&g_own_stream, cudaStreamNonBlocking) != cudaSuccess)
            return set_error(SCLBM_E_CUDA, "cannot create the library stream");
    }
    g_dev_checked = 1;
    return SCLBM_OK;
}

cudaStream_t stream() { return g_user_set ? g_user_stream : g_own_stream; }
int sm_count() { return g_sms > 0 ? g_sms : 148; }

int grid_for(size_t n, int block)
{
    size_t b = (n + block - 1) / block;
    size_t cap = (size_t)sm_count() * 32;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// -------------------------------------------------------------- geometry
// device copy of the mask (uint8), refreshed when the host mask changed
int geometry_device_mask(const sclbm_geometry *g, const uint8_t **out)
{
    if (!g) return set_error(SCLBM_E_INVALID_ARGUMENT, "null geometry");
    int rc = ensure_device();
    if (rc) return rc;
    const size_t N = g->nx * g->ny;
    if (g->dirty || g->d_count != N) {
        std::vector<uint8_t> h(N);
        for (size_t i = 0; i < N; ++i) {
            const int32_t v = g->mask[i];
            if (v != 0 && v != 1)
                return set_error(SCLBM_E_INVALID_ARGUMENT,
                                 "geometry node values must be 0 (solid) or 1 (fluid)");
            h[i] = (uint8_t)v;
        }
        if (g->d_count != N) {
            if (g->d_mask) cudaFree(g->d_mask);
            g->d_mask = nullptr;
            g->d_count = 0;
            SCLBM_CUDA(cudaMalloc(&g->d_mask, std::max<size_t>(N, 1)));
            g->d_count = N;
        }
        SCLBM_CUDA(cudaMemcpyAsync(g->d_mask, h.data(), N, cudaMemcpyHostToDevice, stream()));
        SCLBM_CUDA(cudaStreamSynchronize(stream()));
        g->dirty = false;
        g->has_solid = std::find(h.begin(), h.end(), (uint8_t)0) != h.end();
    }
    *out = g->d_mask;
    return SCLBM_OK;
}

} // namespace sclbm

using namespace sclbm;

#define CHECK_NULL(p)                                                                          \
    do {                                                                                       \
        if (!(p)) return set_error(SCLBM_E_INVALID_ARGUMENT, "null " #p);                      \
    } while (0)

extern "C" {

int sclbm_last_error(char *buf, size_t len)
{
    if (!buf || !len) return SCLBM_E_INVALID_ARGUMENT;
    std::snprintf(buf, len, "%s", g_last_error.c_str());
    return SCLBM_OK;
}

const char *sclbm_version(void) { return "sclbm_b200 0.1.0 sm_100a"; }

int sclbm_set_stream(void *s)
{
    int rc = ensure_device();
    if (rc) return rc;
    g_user_stream = (cudaStream_t)s;
    g_user_set = s != nullptr;
    return SCLBM_OK;
}

void *sclbm_get_stream(void) { return (void *)stream(); }

int sclbm_synchronize(void)
{
    int rc = ensure_device();
    if (rc) return rc;
    SCLBM_CUDA(cudaStreamSynchronize(stream()));
    return SCLBM_OK;
}

// ---------------------------------------------------------------- geometry
int sclbm_geometry_create(size_t nx, size_t ny, sclbm_geometry **out)
{
    CHECK_NULL(out);
    auto *g = new (std::nothrow) sclbm_geometry();
    if (!g) return set_error(SCLBM_E_ALLOC, "host allocation failed");
    g->nx = nx;
    g->ny = ny;
    g->mask.assign(nx * ny, 1);
    *out = g;
    return SCLBM_OK;
}

void sclbm_geometry_destroy(sclbm_geometry *g)
{
    if (!g) return;
    if (g->d_mask) cudaFree(g->d_mask);
    delete g;
}

int sclbm_geometry_dims(const sclbm_geometry *g, size_t *nx, size_t *ny)
{
    CHECK_NULL(g);
    if (nx) *nx = g->nx;
    if (ny) *ny = g->ny;
    return SCLBM_OK;
}

int sclbm_geometry_add_walls(sclbm_geometry *g, size_t dH, const char *where)
{
    CHECK_NULL(g);
    CHECK_NULL(where);
    g->dirty = true;
    return geom_add_walls(g->mask, g->nx, g->ny, dH, where);
}
int sclbm_geometry_add_rectangle(sclbm_geometry *g, size_t Lx, size_t Ly, size_t xc, size_t yc)
{
    CHECK_NULL(g);
    g->dirty = true;
    return geom_add_object(g->mask, g->nx, g->ny, 0, Lx, Ly, xc, yc);
}
int sclbm_geometry_add_square(sclbm_geometry *g, size_t Ls, size_t xc, size_t yc)
{
    CHECK_NULL(g);
    g->dirty = true;
    return geom_add_object(g->mask, g->nx, g->ny, 1, Ls, Ls, xc, yc);
}
int sclbm_geometry_add_ellipse(sclbm_geometry *g, size_t Lx, size_t Ly, size_t xc, size_t yc)
{
    CHECK_NULL(g);
    g->dirty = true;
    return geom_add_object(g->mask, g->nx, g->ny, 2, Lx, Ly, xc, yc);
}
int sclbm_geometry_add_circle(sclbm_geometry *g, size_t D, size_t xc, size_t yc)
{
    CHECK_NULL(g);
    g->dirty = true;
    return geom_add_object(g->mask, g->nx, g->ny, 3, D, D, xc, yc);
}
// Seeded random sequential addition of non-overlapping disks (the porous media
// of the drainage and ensemble configurations): draws from the splitmix64
// stream u_k = splitmix(seed, k) exactly as sc_lbm_b200/workloads.py's
// Stream/disk_mask do, keeps a one-node gap (occupancy window of radius
// r + 1.5), stops at the target solid fraction, after max_tries draws or after
// max_misses failed draws in a row, then adds the disks with add_circle
// (D = 2r + 1).  The existing solid nodes (walls) count as occupied.
namespace {
inline double splitmix_u01_host(uint64_t seed, uint64_t k)
{
    uint64_t z = k + seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}
} // namespace

int sclbm_geometry_add_random_disks(sclbm_geometry *g, double porosity, int rmin, int rmax,
                                    uint64_t seed, int wall_rows, long max_tries, long max_misses,
                                    size_t *placed)
{
    CHECK_NULL(g);
    if (rmin < 0 || rmax < rmin || !(porosity >= 0.0 && porosity <= 1.0) || wall_rows < 0)
        return set_error(SCLBM_E_INVALID_ARGUMENT, "bad disk parameters");
    const long nx = (long)g->nx, ny = (long)g->ny;
    std::vector<uint8_t> occ(g->mask.size());
    double solid = 0.0;
    long nsolid = 0;
    for (size_t i = 0; i < occ.size(); ++i) {
        occ[i] = g->mask[i] == 0;
        nsolid += occ[i];
    }
    solid = (double)nsolid;
    uint64_t k = 0;
    auto integer = [&](long lo, long hi) {
        const double u = splitmix_u01_host(seed, k++);
        const long n = (long)(u * (double)(hi - lo + 1)); // truncation toward zero
        return lo + std::min(hi - lo, n);
    };
    const double target = (1.0 - porosity) * (double)nx * (double)ny;
    std::vector<long> disks;
    long tries = 0, misses = 0;
    while (solid < target && tries < max_tries && misses < max_misses) {
        ++tries;
        ++misses;
        const long r = integer(rmin, rmax);
        const long xc = integer(r, nx - 1 - r);
        const long yc = integer(r + wall_rows, ny - 1 - r - wall_rows);
        if (xc - r < 0 || yc - r < 0 || xc + r >= nx || yc + r >= ny) continue;
        const long y0 = std::max(0L, yc - r - 1), y1 = std::min(ny, yc + r + 2);
        const long x0 = std::max(0L, xc - r - 1), x1 = std::min(nx, xc + r + 2);
        const double lim = ((double)r + 1.5) * ((double)r + 1.5);
        bool hit = false;
        for (long y = y0; y < y1 && !hit; ++y)
            for (long x = x0; x < x1; ++x)
                if ((double)((y - yc) * (y - yc) + (x - xc) * (x - xc)) <= lim && occ[y * nx + x]) {
                    hit = true;
                    break;
                }
        if (hit) continue;
        for (long y = y0; y < y1; ++y)
            for (long x = x0; x < x1; ++x)
                if ((double)((y - yc) * (y - yc) + (x - xc) * (x - xc)) <= lim) occ[y * nx + x] = 1;
        misses = 0;
        disks.push_back(r);
        disks.push_back(xc);
        disks.push_back(yc);
        solid += M_PI * (((double)r + 0.5) * ((double)r + 0.5));
    }
    g->dirty = true;
    for (size_t i = 0; i < disks.size(); i += 3) {
        const int rc = geom_add_object(g->mask, g->nx, g->ny, 3, 2 * disks[i] + 1, 2 * disks[i] + 1,
                                       disks[i + 1], disks[i + 2]);
        if (rc) return rc;
    }
    if (placed) *placed = disks.size() / 3;
    return SCLBM_OK;
}

int sclbm_geometry_add_array_spacing(sclbm_geometry *g, const size_t *props, size_t nprops,
                                     const size_t bounds[4], size_t dx, size_t dy,
                                     const char *type)
{
    CHECK_NULL(g);
    CHECK_NULL(bounds);
    CHECK_NULL(type);
    if (nprops && !props) return set_error(SCLBM_E_INVALID_ARGUMENT, "null props");
    g->dirty = true;
    return geom_add_array(g->mask, g->nx, g->ny, type, props, nprops, bounds, dx, dy, 0);
}
int sclbm_geometry_add_array_numbers(sclbm_geometry *g, const size_t *props, size_t nprops,
                                     const size_t bounds[4], size_t nobj_x, size_t nobj_y,
                                     const char *type)
{
    CHECK_NULL(g);
    CHECK_NULL(bounds);
    CHECK_NULL(type);
    if (nprops && !props) return set_error(SCLBM_E_INVALID_ARGUMENT, "null props");
    g->dirty = true;
    return geom_add_array(g->mask, g->nx, g->ny, type, props, nprops, bounds, nobj_x, nobj_y, 1);
}
int sclbm_geometry_set_node(sclbm_geometry *g, size_t x, size_t y, int fluid)
{
    CHECK_NULL(g);
    const size_t i = y * g->nx + x;
    if (i >= g->mask.size())
        return set_error(SCLBM_E_OUT_OF_RANGE, "vector::_M_range_check (node outside the geometry)");
    g->mask[i] = fluid ? 1 : 0;
    g->dirty = true;
    return SCLBM_OK;
}
int sclbm_geometry_get_mask(const sclbm_geometry *g, int32_t *mask, size_t count)
{
    CHECK_NULL(g);
    CHECK_NULL(mask);
    if (count != g->mask.size()) return set_error(SCLBM_E_INVALID_ARGUMENT, "count != nx*ny");
    std::memcpy(mask, g->mask.data(), count * sizeof(int32_t));
    return SCLBM_OK;
}
int sclbm_geometry_set_mask(sclbm_geometry *g, size_t nx, size_t ny, const int32_t *mask)
{
    CHECK_NULL(g);
    if ((nx * ny) != 0 && !mask) return set_error(SCLBM_E_INVALID_ARGUMENT, "null mask");
    g->nx = nx;
    g->ny = ny;
    g->mask.assign(mask, mask + nx * ny);
    g->dirty = true;
    return SCLBM_OK;
}

// ------------------------------------------------------------------ fluid
static size_t field_count(const sclbm_fluid *f, int field)
{
    return (field == SCLBM_FIELD_F || field == SCLBM_FIELD_FEQ) ? 9 * f->N : f->N;
}

int sclbm_fluid_create(size_t nx, size_t ny, double tau, sclbm_fluid **out)
{
    CHECK_NULL(out);
    int rc = ensure_device();
    if (rc) return rc;
    auto *f = new (std::nothrow) sclbm_fluid();
    if (!f) return set_error(SCLBM_E_ALLOC, "host allocation failed");
    f->nx = nx;
    f->ny = ny;
    f->N = nx * ny;
    f->tau = tau;
    f->omega = 1 / tau; // Fluid::Fluid, include/fluid.h:62
    for (int k = 0; k < 11; ++k) {
        const size_t n = std::max<size_t>(field_count(f, k), 1);
        cudaError_t e = cudaMalloc(&f->d[k], n * sizeof(double));
        if (e == cudaSuccess) e = cudaMemsetAsync(f->d[k], 0, n * sizeof(double), stream());
        if (e != cudaSuccess) {
            sclbm_fluid_destroy(f);
            return cuda_fail(e, "fluid allocation");
        }
    }
    *out = f;
    return SCLBM_OK;
}

void sclbm_fluid_destroy(sclbm_fluid *f)
{
    if (!f) return;
    for (auto *p : f->d)
        if (p) cudaFree(p);
    delete f;
}

int sclbm_fluid_set_interactions(sclbm_fluid *f, double g_solid, double g_fluid)
{
    CHECK_NULL(f);
    f->g_solid = g_solid;
    f->g_fluid = g_fluid;
    return SCLBM_OK;
}

int sclbm_fluid_get_params(const sclbm_fluid *f, double *omega, double *g_solid, double *g_fluid)
{
    CHECK_NULL(f);
    if (omega) *omega = f->omega;
    if (g_solid) *g_solid = f->g_solid;
    if (g_fluid) *g_fluid = f->g_fluid;
    return SCLBM_OK;
}

int sclbm_fluid_write(sclbm_fluid *f, sclbm_field field, const double *src, size_t count)
{
    CHECK_NULL(f);
    if ((int)field < 0 || (int)field > 10) return set_error(SCLBM_E_INVALID_ARGUMENT, "bad field");
    if (count != field_count(f, field))
        return set_error(SCLBM_E_INVALID_ARGUMENT, "field size mismatch");
    if (count && !src) return set_error(SCLBM_E_INVALID_ARGUMENT, "null source");
    SCLBM_CUDA(cudaMemcpyAsync(f->d[field], src, count * sizeof(double), cudaMemcpyHostToDevice,
                               stream()));
    SCLBM_CUDA(cudaStreamSynchronize(stream()));
    if (field == SCLBM_FIELD_FSOLID_X || field == SCLBM_FIELD_FSOLID_Y) f->solid_set = true;
    return SCLBM_OK;
}

int sclbm_fluid_read(sclbm_fluid *f, sclbm_field field, double *dst, size_t count)
{
    CHECK_NULL(f);
    if ((int)field < 0 || (int)field > 10) return set_error(SCLBM_E_INVALID_ARGUMENT, "bad field");
    if (count != field_count(f, field))
        return set_error(SCLBM_E_INVALID_ARGUMENT, "field size mismatch");
    if (count && !dst) return set_error(SCLBM_E_INVALID_ARGUMENT, "null destination");
    SCLBM_CUDA(cudaMemcpyAsync(dst, f->d[field], count * sizeof(double), cudaMemcpyDeviceToHost,
                               stream()));
    SCLBM_CUDA(cudaStreamSynchronize(stream()));
    return SCLBM_OK;
}

static int same_shape(const sclbm_fluid *f, const sclbm_geometry *g)
{
    if (f->nx != g->nx || f->ny != g->ny)
        return set_error(SCLBM_E_INVALID_ARGUMENT, "fluid and geometry sizes differ");
    return SCLBM_OK;
}

#define CUDA_LAUNCH(expr)                                                                      \
    do {                                                                                       \
        cudaError_t e_ = (expr);                                                               \
        if (e_ != cudaSuccess) return cuda_fail(e_, #expr);                                    \
    } while (0)

int sclbm_fluid_compute_density(sclbm_fluid *f)
{
    CHECK_NULL(f);
    CUDA_LAUNCH(op_density(f->N, f->d[SCLBM_FIELD_F], f->d[SCLBM_FIELD_RHO], stream()));
    return SCLBM_OK;
}

int sclbm_fluid_compute_velocities(sclbm_fluid *f, const sclbm_geometry *g)
{
    CHECK_NULL(f);
    const uint8_t *m;
    int rc = geometry_device_mask(g, &m);
    if (rc || (rc = same_shape(f, g))) return rc;
    CUDA_LAUNCH(op_velocities(f->N, m, f->d[SCLBM_FIELD_F], f->d[SCLBM_FIELD_RHO],
                              f->d[SCLBM_FIELD_UX], f->d[SCLBM_FIELD_UY], stream()));
    return SCLBM_OK;
}

int sclbm_fluid_compute_f_equilibrium_geom(sclbm_fluid *f, const sclbm_geometry *g)
{
    CHECK_NULL(f);
    const uint8_t *m;
    int rc = geometry_device_mask(g, &m);
    if (rc || (rc = same_shape(f, g))) return rc;
    CUDA_LAUNCH(op_feq_single(f->N, m, f->d[SCLBM_FIELD_F], f->d[SCLBM_FIELD_RHO],
                              f->d[SCLBM_FIELD_UX], f->d[SCLBM_FIELD_UY], f->d[SCLBM_FIELD_FEQ],
                              f->omega, 0, stream()));
    return SCLBM_OK;
}

int sclbm_fluid_compute_f_equilibrium(sclbm_fluid *f)
{
    CHECK_NULL(f);
    CUDA_LAUNCH(op_feq_multi(f->N, f->d[SCLBM_FIELD_F], f->d[SCLBM_FIELD_RHO],
                             f->d[SCLBM_FIELD_UEQ_X], f->d[SCLBM_FIELD_UEQ_Y],
                             f->d[SCLBM_FIELD_FEQ], f->omega, 0, stream()));
    return SCLBM_OK;
}

int sclbm_fluid_simple_ini(sclbm_fluid *f, const sclbm_geometry *g, double rho0)
{
    CHECK_NULL(f);
    const uint8_t *m;
    int rc = geometry_device_mask(g, &m);
    if (rc || (rc = same_shape(f, g))) return rc;
    const double rho_factor = 9.0; // static_cast<double>(Ndir), src/fluid.cpp:70
    CUDA_LAUNCH(op_fill_fluid(f->N, m, f->d[SCLBM_FIELD_F], rho0 / rho_factor, stream()));
    return SCLBM_OK;
}

// --------------------------------------------------------------------- LBM
int sclbm_lbm_create(const sclbm_geometry *g, sclbm_lbm **out)
{
    CHECK_NULL(g);
    CHECK_NULL(out);
    int rc = ensure_device();
    if (rc) return rc;
    auto *l = new (std::nothrow) sclbm_lbm();
    if (!l) return set_error(SCLBM_E_ALLOC, "host allocation failed");
    l->nx = g->nx;
    l->ny = g->ny;
    l->N = g->nx * g->ny;
    for (int k = 0; k < 2; ++k) {
        cudaError_t e = cudaMalloc(&l->d_tmp[k], std::max<size_t>(9 * l->N, 1) * sizeof(double));
        if (e != cudaSuccess) {
            sclbm_lbm_destroy(l);
            return cuda_fail(e, "stream buffer allocation");
        }
    }
    *out = l;
    return SCLBM_OK;
}

void sclbm_lbm_destroy(sclbm_lbm *l)
{
    if (!l) return;
    for (auto *p : l->d_tmp)
        if (p) cudaFree(p);
    delete l;
}

// common checks of the LBM entry points: device mask, matching shapes
static int lbm_prep(sclbm_lbm *l, const sclbm_geometry *g, const sclbm_fluid *f1,
                    const sclbm_fluid *f2, const uint8_t **m)
{
    CHECK_NULL(l);
    CHECK_NULL(f1);
    int rc = geometry_device_mask(g, m);
    if (rc) return rc;
    if (l->nx != g->nx || l->ny != g->ny)
        return set_error(SCLBM_E_INVALID_ARGUMENT, "LBM and geometry sizes differ");
    if ((rc = same_shape(f1, g))) return rc;
    if (f2 && (rc = same_shape(f2, g))) return rc;
    return SCLBM_OK;
}

int sclbm_lbm_initialize_droplet(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *bulk,
                                 sclbm_fluid *droplet, double rb, double rd, double rbd,
                                 double rdb, double xc, double yc, double radius)
{
    const uint8_t *m;
    CHECK_NULL(droplet);
    int rc = lbm_prep(l, g, bulk, droplet, &m);
    if (rc) return rc;
    CUDA_LAUNCH(op_init_droplet((int)g->nx, (int)g->ny, m, bulk->d[SCLBM_FIELD_F],
                                droplet->d[SCLBM_FIELD_F], rb, rd, rbd, rdb, xc, yc, radius,
                                stream()));
    return SCLBM_OK;
}

int sclbm_lbm_initialize_fluid_rectangle(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *bulk,
                                         sclbm_fluid *droplet, double rb, double rd, double rbd,
                                         double rdb, double xc, double yc, double half_lx,
                                         double half_ly)
{
    const uint8_t *m;
    CHECK_NULL(droplet);
    int rc = lbm_prep(l, g, bulk, droplet, &m);
    if (rc) return rc;
    // src/lbm.cpp:78-81: bounds truncated to int
    const long long x0 = (int)(xc - half_lx + 1), xf = (int)(xc + half_lx - 1);
    const long long y0 = (int)(yc - half_ly + 1), yf = (int)(yc + half_ly - 1);
    const long long N = (long long)(g->nx * g->ny), nx = (long long)g->nx;
    bool in_range = true;
    for (long long xi = x0; xi <= xf && in_range; ++xi)
        for (long long yj = y0; yj <= yf; ++yj) {
            const unsigned long long lin = (unsigned long long)(yj * nx + xi);
            if (lin >= (unsigned long long)N) {
                in_range = false;
                break;
            }
        }
    if (!in_range) {
        // the reference throws std::out_of_range from geom(xi, yj) part way
        // through; reproduce its partial update on the host
        const size_t n9 = 9 * (size_t)N;
        std::vector<double> fb(n9), fd(n9);
        SCLBM_CUDA(cudaMemcpyAsync(fb.data(), bulk->d[0], n9 * 8, cudaMemcpyDeviceToHost, stream()));
        SCLBM_CUDA(cudaMemcpyAsync(fd.data(), droplet->d[0], n9 * 8, cudaMemcpyDeviceToHost, stream()));
        SCLBM_CUDA(cudaStreamSynchronize(stream()));
        const auto &gm = g->mask;
        for (long long i = 0; i < N; ++i)
            if (gm[i] != 0)
                for (int d = 0; d < 9; ++d) {
                    fb[d * N + i] = rb / 9.0;
                    fd[d * N + i] = rdb / 9.0;
                }
        rc = SCLBM_OK;
        for (long long xi = x0; xi <= xf && !rc; ++xi)
            for (long long yj = y0; yj <= yf; ++yj) {
                const unsigned long long lin = (unsigned long long)(yj * nx + xi);
                if (lin >= (unsigned long long)N) {
                    rc = set_error(SCLBM_E_OUT_OF_RANGE,
                                   "vector::_M_range_check (rectangle outside the geometry)");
                    break;
                }
                if (gm[lin] == 0) continue;
                for (int d = 0; d < 9; ++d) {
                    fb[d * N + lin] = rbd / 9.0;
                    fd[d * N + lin] = rd / 9.0;
                }
            }
        SCLBM_CUDA(cudaMemcpyAsync(bulk->d[0], fb.data(), n9 * 8, cudaMemcpyHostToDevice, stream()));
        SCLBM_CUDA(cudaMemcpyAsync(droplet->d[0], fd.data(), n9 * 8, cudaMemcpyHostToDevice, stream()));
        SCLBM_CUDA(cudaStreamSynchronize(stream()));
        return rc;
    }
    CUDA_LAUNCH(op_init_rect((int)g->nx, (int)g->ny, m, bulk->d[SCLBM_FIELD_F],
                             droplet->d[SCLBM_FIELD_F], rb, rd, rbd, rdb, x0, xf, y0, yf,
                             stream()));
    return SCLBM_OK;
}

int sclbm_lbm_solid_surface_sums(sclbm_lbm *l, const sclbm_geometry *g, double *sx, double *sy,
                                 size_t count)
{
    CHECK_NULL(l);
    const uint8_t *m;
    int rc = geometry_device_mask(g, &m);
    if (rc) return rc;
    const size_t N = g->nx * g->ny;
    if (count != N || !sx || !sy) return set_error(SCLBM_E_INVALID_ARGUMENT, "bad output arrays");
    double *d = l->d_tmp[0];
    CUDA_LAUNCH(op_solid_sums((int)g->nx, (int)g->ny, m, d, d + N, stream()));
    SCLBM_CUDA(cudaMemcpyAsync(sx, d, N * 8, cudaMemcpyDeviceToHost, stream()));
    SCLBM_CUDA(cudaMemcpyAsync(sy, d + N, N * 8, cudaMemcpyDeviceToHost, stream()));
    SCLBM_CUDA(cudaStreamSynchronize(stream()));
    return SCLBM_OK;
}

int sclbm_lbm_fluid_repulsive_interactions(sclbm_lbm *l, const sclbm_geometry *g,
                                           sclbm_fluid *f1, sclbm_fluid *f2)
{
    const uint8_t *m;
    CHECK_NULL(f2);
    int rc = lbm_prep(l, g, f1, f2, &m);
    if (rc) return rc;
    CUDA_LAUNCH(op_repulsive((int)g->nx, (int)g->ny, m, f1->d[SCLBM_FIELD_RHO],
                             f2->d[SCLBM_FIELD_RHO], -1.0 * f1->g_fluid, -1.0 * f2->g_fluid,
                             f1->d[SCLBM_FIELD_FREP_X], f1->d[SCLBM_FIELD_FREP_Y],
                             f2->d[SCLBM_FIELD_FREP_X], f2->d[SCLBM_FIELD_FREP_Y], stream()));
    return SCLBM_OK;
}

static EqvelArgs eqv(sclbm_fluid *f)
{
    return EqvelArgs{f->d[SCLBM_FIELD_F],       f->d[SCLBM_FIELD_RHO],     f->d[SCLBM_FIELD_FREP_X],
                     f->d[SCLBM_FIELD_FREP_Y],  f->d[SCLBM_FIELD_FSOLID_X], f->d[SCLBM_FIELD_FSOLID_Y],
                     f->d[SCLBM_FIELD_UX],      f->d[SCLBM_FIELD_UY],      f->d[SCLBM_FIELD_UEQ_X],
                     f->d[SCLBM_FIELD_UEQ_Y],   f->omega};
}

static int need_solid(const sclbm_fluid *f1, const sclbm_fluid *f2)
{
    if (!f1->solid_set || (f2 && !f2->solid_set))
        return set_error(SCLBM_E_OUT_OF_RANGE,
                         "vector::_M_range_check: the fluid-solid force was never set "
                         "(call compute_solid_surface_force first)");
    return SCLBM_OK;
}

int sclbm_lbm_equilibrium_velocities(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f1,
                                     sclbm_fluid *f2)
{
    const uint8_t *m;
    CHECK_NULL(f2);
    int rc = lbm_prep(l, g, f1, f2, &m);
    if (rc || (rc = need_solid(f1, f2))) return rc;
    CUDA_LAUNCH(op_eqvel(f1->N, m, eqv(f1), eqv(f2), stream()));
    return SCLBM_OK;
}

int sclbm_lbm_collide_single(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f)
{
    const uint8_t *m;
    int rc = lbm_prep(l, g, f, nullptr, &m);
    if (rc) return rc;
    CUDA_LAUNCH(op_feq_single(f->N, m, f->d[SCLBM_FIELD_F], f->d[SCLBM_FIELD_RHO],
                              f->d[SCLBM_FIELD_UX], f->d[SCLBM_FIELD_UY], f->d[SCLBM_FIELD_FEQ],
                              f->omega, 1, stream()));
    return SCLBM_OK;
}

int sclbm_lbm_collide(sclbm_lbm *l, sclbm_fluid *f1, sclbm_fluid *f2)
{
    CHECK_NULL(l);
    CHECK_NULL(f1);
    CHECK_NULL(f2);
    if (f1->N != l->N || f2->N != l->N)
        return set_error(SCLBM_E_INVALID_ARGUMENT, "LBM and fluid sizes differ");
    for (sclbm_fluid *f : {f1, f2})
        CUDA_LAUNCH(op_feq_multi(f->N, f->d[SCLBM_FIELD_F], f->d[SCLBM_FIELD_RHO],
                                 f->d[SCLBM_FIELD_UEQ_X], f->d[SCLBM_FIELD_UEQ_Y],
                                 f->d[SCLBM_FIELD_FEQ], f->omega, 1, stream()));
    return SCLBM_OK;
}

static int check_force(const double *force, size_t count)
{
    if (!force || count < 9)
        return set_error(SCLBM_E_OUT_OF_RANGE, "vector::_M_range_check: volume force needs 9 "
                                               "values (one per lattice direction)");
    return SCLBM_OK;
}

int sclbm_lbm_add_volume_force_single(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f,
                                      const double *force, size_t count)
{
    const uint8_t *m;
    int rc = lbm_prep(l, g, f, nullptr, &m);
    if (rc || (rc = check_force(force, count))) return rc;
    CUDA_LAUNCH(op_volume_force(f->N, m, f->d[SCLBM_FIELD_F], force, stream()));
    return SCLBM_OK;
}

int sclbm_lbm_add_volume_force(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f1,
                               sclbm_fluid *f2, const double *force, size_t count)
{
    const uint8_t *m;
    CHECK_NULL(f2);
    int rc = lbm_prep(l, g, f1, f2, &m);
    if (rc || (rc = check_force(force, count))) return rc;
    CUDA_LAUNCH(op_volume_force(f1->N, m, f1->d[SCLBM_FIELD_F], force, stream()));
    CUDA_LAUNCH(op_volume_force(f2->N, m, f2->d[SCLBM_FIELD_F], force, stream()));
    return SCLBM_OK;
}

int sclbm_lbm_stream_single(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f)
{
    const uint8_t *m;
    int rc = lbm_prep(l, g, f, nullptr, &m);
    if (rc) return rc;
    CUDA_LAUNCH(op_stream((int)g->nx, (int)g->ny, m, f->d[SCLBM_FIELD_F], l->d_tmp[0], stream()));
    std::swap(f->d[SCLBM_FIELD_F], l->d_tmp[0]); // std::swap(temp_f_dist, f_dist), src/lbm.cpp:382
    return SCLBM_OK;
}

int sclbm_lbm_stream(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f1, sclbm_fluid *f2)
{
    const uint8_t *m;
    CHECK_NULL(f2);
    int rc = lbm_prep(l, g, f1, f2, &m);
    if (rc) return rc;
    CUDA_LAUNCH(op_stream((int)g->nx, (int)g->ny, m, f1->d[SCLBM_FIELD_F], l->d_tmp[0], stream()));
    CUDA_LAUNCH(op_stream((int)g->nx, (int)g->ny, m, f2->d[SCLBM_FIELD_F], l->d_tmp[1], stream()));
    std::swap(f1->d[SCLBM_FIELD_F], l->d_tmp[0]);
    std::swap(f2->d[SCLBM_FIELD_F], l->d_tmp[1]);
    return SCLBM_OK;
}

int sclbm_lbm_step(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f1, sclbm_fluid *f2,
                   const double *force1, const double *force2, int nsteps)
{
    const uint8_t *m;
    CHECK_NULL(f2);
    int rc = lbm_prep(l, g, f1, f2, &m);
    if (rc || (rc = need_solid(f1, f2))) return rc;
    if (nsteps < 0) return set_error(SCLBM_E_INVALID_ARGUMENT, "negative step count");
    Fused2Args<double, double> a{};
    a.nx = (int)g->nx;
    a.ny = (int)g->ny;
    a.N = g->nx * g->ny;
    a.tile_y = 32;
    a.mask = m;
    sclbm_fluid *fl[2] = {f1, f2};
    const double *frc[2] = {force1, force2};
    for (int k = 0; k < 2; ++k) {
        CompParams<double> &c = a.c[k];
        c.omega = fl[k]->omega;
        c.one_m_omega = 1.0 - fl[k]->omega;
        c.inv_omega = 1.0 / fl[k]->omega;
        c.gf = -1.0 * fl[k]->g_fluid;
        c.gs_neg = -1.0 * fl[k]->g_solid;
        c.rho_ref = 0.0;
        c.force_on = frc[k] != nullptr;
        for (int i = 0; i < 9; ++i) c.force[i] = frc[k] ? frc[k][i] : 0.0;
        a.fsx[k] = fl[k]->d[SCLBM_FIELD_FSOLID_X];
        a.fsy[k] = fl[k]->d[SCLBM_FIELD_FSOLID_Y];
        a.uex_old[k] = fl[k]->d[SCLBM_FIELD_UEQ_X];
        a.uey_old[k] = fl[k]->d[SCLBM_FIELD_UEQ_Y];
    }
    a.solid_from_mask = 0;
    a.has_solid = g->has_solid ? 1 : 0;
    a.solids_zero = 0; // caller-owned arrays: solid nodes are rewritten with zeros
    for (int s = 0; s < nsteps; ++s) {
        a.fin[0] = f1->d[SCLBM_FIELD_F];
        a.fin[1] = f2->d[SCLBM_FIELD_F];
        a.fout[0] = l->d_tmp[0];
        a.fout[1] = l->d_tmp[1];
        CUDA_LAUNCH(launch_fused2_async_fp64(a, stream()));
        std::swap(f1->d[SCLBM_FIELD_F], l->d_tmp[0]);
        std::swap(f2->d[SCLBM_FIELD_F], l->d_tmp[1]);
    }
    return SCLBM_OK;
}

int sclbm_lbm_step_single(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f,
                          const double *force, int nsteps)
{
    const uint8_t *m;
    int rc = lbm_prep(l, g, f, nullptr, &m);
    if (rc) return rc;
    if (nsteps < 0) return set_error(SCLBM_E_INVALID_ARGUMENT, "negative step count");
    Fused1Args<double, double> a{};
    a.nx = (int)g->nx;
    a.ny = (int)g->ny;
    a.N = g->nx * g->ny;
    a.mask = m;
    a.c.omega = f->omega;
    a.c.one_m_omega = 1.0 - f->omega;
    a.c.inv_omega = 1.0 / f->omega;
    a.c.force_on = force != nullptr;
    for (int i = 0; i < 9; ++i) a.c.force[i] = force ? force[i] : 0.0;
    for (int s = 0; s < nsteps; ++s) {
        a.fin = f->d[SCLBM_FIELD_F];
        a.fout = l->d_tmp[0];
        CUDA_LAUNCH(launch_fused1_fp64(a, stream()));
        std::swap(f->d[SCLBM_FIELD_F], l->d_tmp[0]);
    }
    return SCLBM_OK;
}

} // extern "C"
