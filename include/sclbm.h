/*
 * sclbm.h -- C ABI of libsclbm_b200.so, a B200 (sm_100a) implementation of the
 * sc_lbm D2Q9 Shan-Chen time step.
 *
 * The reference (LBMFluids/sc_lbm) has no FFI layer: its interface is the C++
 * classes Geometry / Fluid / LBM.  Every entry point below names the reference
 * member it replaces (file:line inside the reference project).  The C++
 * drop-in classes in sc_lbm_b200/host/include/{geometry,fluid,lbm}.h are thin
 * wrappers over these functions; FFI users (ctypes, cgo, JNI) bind them
 * directly.
 *
 * Conventions (identical to the reference):
 *   - a lattice is nx * ny nodes, row-major [y*nx + x]; N = nx*ny;
 *   - masks are int32 per node, 1 = fluid, 0 = solid (Geometry::geom);
 *   - populations are structure-of-arrays, direction-major [i*N + y*nx + x],
 *     9 directions with c_x = {0,1,0,-1,0,1,-1,-1,1}, c_y = {0,0,1,0,-1,1,1,-1,-1};
 *   - every function returns an int status (SCLBM_OK = 0); the C++ layer maps
 *     the codes to the reference's exception types.  sclbm_last_error() gives
 *     the message of the last failure on the calling thread;
 *   - all host pointers are plain host memory (pageable or pinned); device
 *     state lives inside the opaque handles.  Work is queued on the library
 *     stream (sclbm_set_stream); functions that return data to the host
 *     synchronise that stream.
 */
#ifndef SCLBM_H
#define SCLBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define SCLBM_OK 0
#define SCLBM_E_INVALID_ARGUMENT 1 /* std::invalid_argument in the reference */
#define SCLBM_E_RUNTIME 2          /* std::runtime_error */
#define SCLBM_E_OUT_OF_RANGE 3     /* std::out_of_range (vector::at) */
#define SCLBM_E_DOMAIN 4           /* inputs on which the reference divides by zero */
#define SCLBM_E_CUDA 5             /* CUDA runtime failure */
#define SCLBM_E_NO_DEVICE 6        /* no usable CUDA device */
#define SCLBM_E_NONFINITE 7        /* monitor found NaN/Inf populations */
#define SCLBM_E_ALLOC 8            /* device allocation failed */

/* Message of the last failure on this thread (always NUL-terminated). */
int sclbm_last_error(char *buf, size_t len);
/* Library version string, e.g. "sclbm_b200 0.1.0 sm_100a". */
const char *sclbm_version(void);
/* Queue all following work on `cuda_stream` (a cudaStream_t; NULL = the
 * library's own non-blocking stream). */
int sclbm_set_stream(void *cuda_stream);
/* The cudaStream_t in use, as a pointer. */
void *sclbm_get_stream(void);
/* Wait for all queued work. */
int sclbm_synchronize(void);

/* ---------------------------------------------------------------- geometry
 * Host-side solid mask, bit-exact with the reference Geometry
 * (include/geometry.h:37-286, src/geometry.cpp). A device copy is made
 * lazily when an operator first needs it and refreshed after any change. */
typedef struct sclbm_geometry sclbm_geometry;

/* Geometry::Geometry(Nx, Ny), include/geometry.h:58-59 (all fluid) */
int sclbm_geometry_create(size_t nx, size_t ny, sclbm_geometry **out);
void sclbm_geometry_destroy(sclbm_geometry *g);
int sclbm_geometry_dims(const sclbm_geometry *g, size_t *nx, size_t *ny);
/* Geometry::add_walls, src/geometry.cpp:34-69 ; where = "x" or "y" */
int sclbm_geometry_add_walls(sclbm_geometry *g, size_t dH, const char *where);
/* Geometry::add_rectangle, src/geometry.cpp:76-92 */
int sclbm_geometry_add_rectangle(sclbm_geometry *g, size_t Lx, size_t Ly, size_t xc, size_t yc);
/* Geometry::add_square, src/geometry.cpp:95-110 */
int sclbm_geometry_add_square(sclbm_geometry *g, size_t Ls, size_t xc, size_t yc);
/* Geometry::add_ellipse, src/geometry.cpp:113-129 */
int sclbm_geometry_add_ellipse(sclbm_geometry *g, size_t Lx, size_t Ly, size_t xc, size_t yc);
/* Geometry::add_circle, src/geometry.cpp:132-147 */
int sclbm_geometry_add_circle(sclbm_geometry *g, size_t D, size_t xc, size_t yc);
/* Geometry::add_array (displacement overload), src/geometry.cpp:182-198.
 * bounds = {x_lo, x_hi, y_lo, y_hi}; type is rectangle/square/ellipse/circle. */
int sclbm_geometry_add_array_spacing(sclbm_geometry *g, const size_t *props, size_t nprops,
                                     const size_t bounds[4], size_t dx, size_t dy,
                                     const char *type);
/* Geometry::add_array (object-number overload), src/geometry.cpp:201-217 */
int sclbm_geometry_add_array_numbers(sclbm_geometry *g, const size_t *props, size_t nprops,
                                     const size_t bounds[4], size_t nobj_x, size_t nobj_y,
                                     const char *type);
/* Seeded porous medium: non-overlapping disks (add_circle, D = 2r + 1, r in
 * [rmin, rmax]) placed by random sequential addition with a one-node gap
 * until the fluid fraction reaches `porosity`, or max_tries draws were made,
 * or max_misses draws in a row found no room; disk centres keep wall_rows
 * rows clear of the top and bottom.  Existing solid nodes count as occupied.
 * The draws are the splitmix64 stream of sc_lbm_b200/workloads.py, so a seed
 * gives the same medium as its disk_mask.  No reference counterpart (the
 * reference's drivers place objects by hand or in regular arrays). */
int sclbm_geometry_add_random_disks(sclbm_geometry *g, double porosity, int rmin, int rmax,
                                    uint64_t seed, int wall_rows, long max_tries, long max_misses,
                                    size_t *placed);
/* Geometry::set_node_fluid / set_node_solid, include/geometry.h:200-210 */
int sclbm_geometry_set_node(sclbm_geometry *g, size_t x, size_t y, int fluid);
/* Geometry::get_geom, include/geometry.h:262 (count must be nx*ny) */
int sclbm_geometry_get_mask(const sclbm_geometry *g, int32_t *mask, size_t count);
/* Replace the whole mask (Geometry::read's effect, src/geometry.cpp:247-264) */
int sclbm_geometry_set_mask(sclbm_geometry *g, size_t nx, size_t ny, const int32_t *mask);

/* ------------------------------------------------------------------- fluid
 * FP64 device state of one component: every array of the reference Fluid
 * (include/fluid.h:285-309). */
typedef struct sclbm_fluid sclbm_fluid;

typedef enum {
    SCLBM_FIELD_F = 0,        /* f_dist, 9N      include/fluid.h:296 */
    SCLBM_FIELD_FEQ = 1,      /* f_eq_dist, 9N   :298 */
    SCLBM_FIELD_RHO = 2,      /* rho, N          :303 */
    SCLBM_FIELD_UX = 3,       /* ux, N           :305 */
    SCLBM_FIELD_UY = 4,       /* uy, N           :306 */
    SCLBM_FIELD_UEQ_X = 5,    /* u_eq_x, N       :308 */
    SCLBM_FIELD_UEQ_Y = 6,    /* u_eq_y, N       :309 */
    SCLBM_FIELD_FREP_X = 7,   /* F_repulsive_x   :300 */
    SCLBM_FIELD_FREP_Y = 8,   /* F_repulsive_y   :301 */
    SCLBM_FIELD_FSOLID_X = 9, /* F_solid_x       :286 */
    SCLBM_FIELD_FSOLID_Y = 10 /* F_solid_y       :287 */
} sclbm_field;

/* Fluid(name, cs2, tau) + zero_density_ini: include/fluid.h:60-62,
 * src/fluid.cpp:43-61.  omega = 1/tau.  All arrays zero; F_solid unset. */
int sclbm_fluid_create(size_t nx, size_t ny, double tau, sclbm_fluid **out);
void sclbm_fluid_destroy(sclbm_fluid *f);
/* Gsolid and Gfluid_repulsion, include/fluid.h:110-114 / src/fluid.cpp:163-168 */
int sclbm_fluid_set_interactions(sclbm_fluid *f, double g_solid, double g_fluid);
int sclbm_fluid_get_params(const sclbm_fluid *f, double *omega, double *g_solid, double *g_fluid);
/* Copy a field host -> device / device -> host (count = 9N or N). Writing
 * SCLBM_FIELD_FSOLID_X/Y marks the solid force as set (Fluid::add_surface_forces). */
int sclbm_fluid_write(sclbm_fluid *f, sclbm_field field, const double *src, size_t count);
int sclbm_fluid_read(sclbm_fluid *f, sclbm_field field, double *dst, size_t count);
/* Fluid::compute_density, src/fluid.cpp:175-183 */
int sclbm_fluid_compute_density(sclbm_fluid *f);
/* Fluid::compute_velocities, src/fluid.cpp:186-200 */
int sclbm_fluid_compute_velocities(sclbm_fluid *f, const sclbm_geometry *g);
/* Fluid::compute_f_equilibrium(geom), src/fluid.cpp:210-243 (incl. macroscopic) */
int sclbm_fluid_compute_f_equilibrium_geom(sclbm_fluid *f, const sclbm_geometry *g);
/* Fluid::compute_f_equilibrium(), src/fluid.cpp:246-278 */
int sclbm_fluid_compute_f_equilibrium(sclbm_fluid *f);
/* Fluid::simple_ini, src/fluid.cpp:64-104: f = rho0/9 on fluid nodes */
int sclbm_fluid_simple_ini(sclbm_fluid *f, const sclbm_geometry *g, double rho0);

/* --------------------------------------------------------------------- LBM
 * The step operators of class LBM (include/lbm.h:23-135). Each call launches
 * sm_100a kernels with the reference's exact FP64 operation order. */
typedef struct sclbm_lbm sclbm_lbm;

/* LBM::LBM(const Geometry&), include/lbm.h:30-37 (allocates the stream buffer) */
int sclbm_lbm_create(const sclbm_geometry *g, sclbm_lbm **out);
void sclbm_lbm_destroy(sclbm_lbm *l);
/* LBM::initialize_droplet, src/lbm.cpp:11-48 */
int sclbm_lbm_initialize_droplet(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *bulk,
                                 sclbm_fluid *droplet, double rho_bulk, double rho_droplet,
                                 double rho_b_in_d, double rho_d_in_b, double xc, double yc,
                                 double radius);
/* LBM::initialize_fluid_rectangle, src/lbm.cpp:51-99 */
int sclbm_lbm_initialize_fluid_rectangle(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *bulk,
                                         sclbm_fluid *droplet, double rho_bulk,
                                         double rho_droplet, double rho_b_in_d,
                                         double rho_d_in_b, double xc, double yc, double half_lx,
                                         double half_ly);
/* The common sums of LBM::compute_solid_surface_force, src/lbm.cpp:102-136,
 * returned to the host (N each); the C++ layer then applies
 * Fluid::add_surface_forces (src/fluid.cpp:154-160) to both fluids. */
int sclbm_lbm_solid_surface_sums(sclbm_lbm *l, const sclbm_geometry *g, double *sx, double *sy,
                                 size_t count);
/* LBM::compute_fluid_repulsive_interactions, src/lbm.cpp:144-206 */
int sclbm_lbm_fluid_repulsive_interactions(sclbm_lbm *l, const sclbm_geometry *g,
                                           sclbm_fluid *f1, sclbm_fluid *f2);
/* LBM::compute_equilibrium_velocities, src/lbm.cpp:209-272 (ux/uy receive
 * momentum, like the reference). Fails with SCLBM_E_OUT_OF_RANGE when a
 * fluid's solid force was never set, as the reference's .at() does. */
int sclbm_lbm_equilibrium_velocities(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f1,
                                     sclbm_fluid *f2);
/* LBM::collide(geom, fluid), src/lbm.cpp:275-288 */
int sclbm_lbm_collide_single(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f);
/* LBM::collide(fluid1, fluid2), src/lbm.cpp:291-312 */
int sclbm_lbm_collide(sclbm_lbm *l, sclbm_fluid *f1, sclbm_fluid *f2);
/* LBM::add_volume_force (single fluid), src/lbm.cpp:315-325; count >= 9 */
int sclbm_lbm_add_volume_force_single(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f,
                                      const double *force, size_t count);
/* LBM::add_volume_force (two fluids), src/lbm.cpp:328-340 */
int sclbm_lbm_add_volume_force(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f1,
                               sclbm_fluid *f2, const double *force, size_t count);
/* LBM::stream(geom, fluid), src/lbm.cpp:343-384 */
int sclbm_lbm_stream_single(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f);
/* LBM::stream(geom, fluid1, fluid2), src/lbm.cpp:387-435 */
int sclbm_lbm_stream(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f1, sclbm_fluid *f2);

/* Fused FP64 time steps on fluid objects: each step equals the driver
 * sequence compute_density x2, compute_fluid_repulsive_interactions,
 * compute_equilibrium_velocities, collide(f1,f2), add_volume_force (force1 on
 * f1 and/or force2 on f2 when non-NULL, 9 values each), stream
 * (laplace_law.cpp:123-133, droplet_in_a_channel.cpp:145-156).  Populations
 * are bit-identical to that sequence; the intermediate fields (rho, ux, uy,
 * u_eq, F_repulsive, f_eq) are left as they were. */
int sclbm_lbm_step(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f1, sclbm_fluid *f2,
                   const double *force1, const double *force2, int nsteps);
/* Fused single-component steps: collide(geom,f), [add_volume_force], stream
 * (laminar_flow_x_dir.cpp:64-68). */
int sclbm_lbm_step_single(sclbm_lbm *l, const sclbm_geometry *g, sclbm_fluid *f,
                          const double *force, int nsteps);

/* ------------------------------------------------------------------ domain
 * Self-contained device domain for production runs: the mask plus one or two
 * components in a chosen storage precision, advanced by the fused
 * single-pass kernel.  No reference counterpart; it runs the same step as
 * sclbm_lbm_step with the solid force derived from the mask
 * (LBM::compute_solid_surface_force). */
typedef enum {
    SCLBM_FP64 = 0,         /* double storage and arithmetic (bit-exact path) */
    SCLBM_FP32_SHIFTED = 1, /* float storage of f_i - w_i*rho_ref, float arithmetic */
    SCLBM_FP16_SHIFTED = 2  /* half storage of f_i - w_i*rho_ref, float arithmetic */
} sclbm_precision;

typedef struct {
    int ncomp;          /* 1 or 2 components */
    double tau[2];      /* relaxation time per component (omega = 1/tau) */
    double g_fluid[2];  /* Gfluid_repulsion per component */
    double g_solid[2];  /* Gsolid per component */
    double rho_ref[2];  /* reference density for the shifted storage */
    int force_on[2];    /* add force[k] after collision on component k */
    double force[2][9]; /* volume force per direction (src/lbm.cpp:315-340) */
} sclbm_params;

typedef struct sclbm_domain sclbm_domain;

int sclbm_domain_create(size_t nx, size_t ny, const int32_t *mask, const sclbm_params *p,
                        sclbm_precision precision, sclbm_domain **out);
void sclbm_domain_destroy(sclbm_domain *d);
/* populations of component comp in reference layout (FP64, 9N values) */
int sclbm_domain_upload_f(sclbm_domain *d, int comp, const double *f, size_t count);
int sclbm_domain_download_f(sclbm_domain *d, int comp, double *f, size_t count);
/* Seeded initial state written on the device, for lattices whose FP64
 * populations are too large to build on the host: f_i = rho/9 on fluid nodes
 * and 0 on solids (the shape of LBM::initialize_droplet, src/lbm.cpp:11-48,
 * and Fluid::simple_ini, src/fluid.cpp:64-104), rho = rho0*(1 + amp*(2u-1)),
 * u in [0,1) the splitmix64 uniform of (seed, node index).  Equal bit for bit
 * to uploading the same state built on the host (sc_lbm_b200/workloads.py
 * draws the same stream).  Replaces building the state through get_f_dist();
 * no reference counterpart (the reference's perturbed init,
 * src/fluid.cpp:107-151, is unseeded). */
int sclbm_domain_init_noise(sclbm_domain *d, int comp, double rho0, double amp, uint64_t seed);
/* Seeded porous medium built on the device: the non-overlapping disks of
 * sclbm_geometry_add_random_disks with the same arguments, placed against the
 * domain's current mask (walls and earlier solids) and rasterised into it
 * with the reference's integer circle (Geometry::add_circle,
 * src/geometry.cpp:132-147; Ellipse::find_nodes,
 * src/geom_object/ellipse.cpp:12-34): the resulting mask equals the host
 * geometry's node for node.  Populations of the new solid nodes are zeroed.
 * Call it before uploading or initialising populations.  Synchronises the
 * library stream; *placed (may be NULL) = disks placed.  No reference
 * counterpart (the reference's drivers place objects by hand). */
int sclbm_domain_add_random_disks(sclbm_domain *d, double porosity, int rmin, int rmax, uint64_t seed,
                                  int wall_rows, long max_tries, long max_misses, size_t *placed);
/* The device mask (1 fluid, 0 solid; count must be nx*ny). */
int sclbm_domain_download_mask(sclbm_domain *d, int32_t *mask, size_t count);
/* density (Fluid::compute_density) and velocity (Fluid::compute_velocities) */
int sclbm_domain_download_rho(sclbm_domain *d, int comp, double *rho, size_t count);
int sclbm_domain_download_velocity(sclbm_domain *d, int comp, double *ux, double *uy,
                                   size_t count);
/* advance nsteps time steps (queued on the library stream, not synchronised) */
int sclbm_domain_step(sclbm_domain *d, int nsteps);
/* Per component: total mass, x and y momentum over fluid nodes, reduced in
 * FP64 (out[3*comp + 0..2]); out[6] = number of non-finite populations. */
int sclbm_domain_mass_momentum(sclbm_domain *d, double out[7]);
/* Kernel selection (all variants give identical results):
 *   0 = automatic (default): the fastest measured form -- the ring kernel
 *       on lattices whose rows start on 16-byte boundaries and whose bands
 *       fill three waves of the GPU (FP64: the depth of 12 and 16-row bands;
 *       FP32: the depth of 13 and 24-row bands; FP16: the depth of 12 and
 *       32-row bands), else 8 for FP32/FP16 storage with solid nodes, 2
 *       otherwise;
 *   1 = two pass (density kernel, then the fused kernel reading it);
 *   2 = single pass, one tile per CTA, population rows held in registers;
 *   3 = single pass, population rows staged through a shared-memory ring by
 *       asynchronous copies, lattice cut into strips x row bands that are all
 *       resident at once (FP64 and FP32 storage; FP16 uses 2);
 *   4 = variant 2 with the row segments of each tile prefetched into L2 two
 *       rows ahead (cp.async.bulk.prefetch), 128 threads per tile;
 *   5 = variant 2 with the loads of row r+1 issued before row r is reduced
 *       (a third row buffer in registers), 128 threads per tile;
 *   6 = variant 2 with each row's collision done by consecutive threads on
 *       its fluid nodes only (populations staged in shared memory), for
 *       lattices with solid nodes (all-fluid lattices run variant 2);
 *   7 = variant 2 with 64-bit element offsets (what lattices of 2^32/9 nodes
 *       and more always run; the other variants use 32-bit offsets);
 *   8 = variant 2 with solid lanes running the collision beside the fluid
 *       ones and storing zeros into their own slots (no branch around the
 *       collision; every slot written each step);
 *   9 = variant 3 with the solid form of variant 8 (FP64 and FP32 storage;
 *       FP16 runs variant 2);
 *  11 = the ring kernel: 128-column strips x 32-row bands, population rows
 *       streamed into a shared-memory ring by TMA tensor copies (one box of
 *       nine directions per component and row) and collided from registers;
 *       12 and 13 the same with one stage fewer / more.  Needs rows that
 *       start on 16-byte boundaries (nx a multiple of 2, 4, 8 for FP64,
 *       FP32, FP16); other lattices run variant 2.
 *  14 = FP32 storage: the ring kernel at the default depth and band height
 *       without the halo boxes in each stage (the wrapped halo column of a
 *       strip at the lattice edge is copied from global memory one row ahead
 *       by asynchronous element copies), which makes room for five resident
 *       CTAs per SM instead of four; FP64 and FP16 run their default ring.
 * tile_y = rows per tile of variants 1, 2 and 4-8, rows per band of 11-14
 * (0 keeps the default). */
int sclbm_domain_set_kernel(sclbm_domain *d, int variant, int tile_y);
/* Threads per tile of the register-tile kernel (variants 1, 2, and 8 with
 * 32 or 128): 32 (one-warp tiles, no CTA barrier), 64 or 128. */
int sclbm_domain_set_threads(sclbm_domain *d, int tx);
/* Device bytes held by the domain. */
size_t sclbm_domain_device_bytes(const sclbm_domain *d);
/* Allocation-free form of sclbm_domain_mass_momentum.  No counterpart in the
 * reference.  For callers that may not allocate device memory -- a host
 * program that gives the library a fixed arena and forbids further
 * cudaMalloc, or code running where allocation is not permitted -- it works
 * on buffers the caller already owns: f0/f1 are device pointers to the
 * populations in the domain layout (9N values of the storage type of
 * `precision`, deviations from w_i*rho_ref[k] for the shifted forms), mask a
 * device pointer to N bytes (1 fluid, 0 solid).  Its scratch is a fixed
 * file-scope device array (about 128 KB, held on every GPU that loads the
 * library until exit), which limits the lattice to 2^27 nodes (e.g.
 * 16384 x 8192); larger lattices return SCLBM_E_INVALID_ARGUMENT.  The first
 * call on a device looks up the array's device address and loads the
 * monitor's kernels for all three precisions, so make one call on each
 * device before entering a region where nothing may be allocated or loaded.
 * All calls share the array and it keeps the last call's partial sums; calls
 * that overlap on the GPU race.  Work runs on `cuda_stream` (NULL = the
 * default stream), which is synchronised before out[7] (as
 * sclbm_domain_mass_momentum) is returned; so it must not be called while
 * that stream is being captured into a CUDA graph: a capturing stream is
 * refused with SCLBM_E_INVALID_ARGUMENT before anything is enqueued, and the
 * capture is left intact.  A non-finite population returns SCLBM_E_NONFINITE
 * (out[6] holds the count). */
int sclbm_mass_momentum_noalloc(const void *f0, const void *f1, const uint8_t *mask, size_t nx,
                                size_t ny, int ncomp, int precision, const double *rho_ref,
                                void *cuda_stream, double out[7]);
/* One end-to-end call: upload both components' populations from host memory,
 * advance nsteps, return the densities to host memory. f2/rho2 are ignored
 * for one component. */
int sclbm_domain_run(sclbm_domain *d, const double *f1, const double *f2, int nsteps,
                     double *rho1, double *rho2);

/* ------------------------------------------------------------------ output
 * Files of a device lattice.  Text in the reference's format (Fluid::write_var
 * through LbmIO::write_vector, src/fluid.cpp:303-353,
 * include/io_operations/lbm_io.h:106-116): one line per lattice row, each
 * value printed with 6 significant digits (%g) and followed by a space, rows
 * cut exactly as write_var cuts them.  `what`: 0 density (write_density),
 * 1 ux, 2 uy (write_ux / write_uy: momentum over density on fluid nodes),
 * 3 populations into nine files <path>_<i>.txt (write_f).  Fluid::save_state
 * (src/fluid.cpp:355-363) is what 0, 1 and 2 with "<name>_<step>.txt" paths.
 * async = 1 queues the device-to-host copy on the library stream and returns;
 * a worker thread formats and writes once the copy is done, while later steps
 * run; sclbm_io_wait() joins all such writers and returns the first failure. */
int sclbm_domain_write_text(sclbm_domain *d, int comp, int what, const char *path, int async);
int sclbm_io_wait(void);
/* Fluid::restart_from_file, src/fluid.cpp:285-298: populations from the nine
 * text files <prefix>_<i>.txt (ny rows of nx values each), uploaded as comp. */
int sclbm_domain_read_text_f(sclbm_domain *d, int comp, const char *prefix);
/* Host-only: write nx*ny values as write_var does / read them back (no device). */
int sclbm_write_rows(const char *path, const double *v, size_t nx, size_t ny);
int sclbm_read_rows(const char *path, double *v, size_t nx, size_t ny);
/* Exact binary checkpoint of the stored populations (any storage precision)
 * with the mask and sizes; load requires a domain of the same size, component
 * count, precision and mask, and continues the run bit for bit.  No reference
 * counterpart (the reference restarts only from its 6-digit text files). */
int sclbm_domain_checkpoint_save(sclbm_domain *d, const char *path);
int sclbm_domain_checkpoint_load(sclbm_domain *d, const char *path);

/* ---------------------------------------------------------------- analysis
 * Measurements computed on the device from the stored populations (FP64
 * densities and velocities as Fluid::compute_density / compute_velocities
 * give them); deterministic reductions.  No reference counterpart in the
 * library: they restate the reference's post-processing scripts. */
/* Laplace law, compute_surface_tension.py:55-73: out[0] = p(x_in, y_in) -
 * p(x_out, y_out) with p = (rho_b + rho_d)/3 + G rho_b rho_d / 3 (bulk
 * component `bulk`, droplet the other); out[1] = radius = the mean of half the
 * row extent (out[2]) and half the column extent (out[3]) of the nodes with
 * rho_d < rho_b and rho_disp < rho_b <= rho_bulk; out[4] = their number. */
int sclbm_domain_laplace_measure(sclbm_domain *d, int bulk, double G, double rho_bulk,
                                 double rho_disp, size_t x_in, size_t y_in, size_t x_out,
                                 size_t y_out, double out[5]);
/* Over the fluid nodes of component comp: out[0] = max |u| (spurious
 * currents, vel_mag of scripts/benchmark_utils.py:55-58), out[1] = mean of
 * the nonzero |u| (ave, :60-63), out[2] = number of nonzero |u|. */
int sclbm_domain_velocity_stats(sclbm_domain *d, int comp, double out[3]);
/* Row profile: prof[y] = mean of u_x (axis 0) or u_y (axis 1) over the fluid
 * nodes of row y (0 for a row without fluid); count must be ny.  The channel
 * profile compared with scripts/benchmark_utils.py:8-52. */
int sclbm_domain_profile(sclbm_domain *d, int comp, int axis, double *prof, size_t count);
/* Contact angle of a droplet (component 1 - bulk) resting on a flat solid,
 * as benchmarks/two_phase_two_components_flows/contact_angles/
 * compute_contact_angles.py:45-106 measures it from the density files: the
 * band rho_b - rho_d <= 0, rho_d <= rho_bulk, rho_b > rho_disp; the smallest
 * and largest x of its two lowest rows extrapolated half a node below the
 * lowest row give the base ends xL (out[4]) and xR (out[5]), L = xR - xL
 * (out[1]); H = row extent + 0.5 (out[2]); R = (4 H^2 + L^2) / (8 H)
 * (out[3]); out[0] = atan(L / (2 (R - H))) in degrees, in [0, 180).
 * out[6], out[7] = lowest and highest band row, out[8] = band nodes.
 * SCLBM_E_OUT_OF_RANGE when the band is empty or its lowest row is the only
 * one (the script's reductions over empty arrays). */
int sclbm_domain_contact_angle(sclbm_domain *d, int bulk, double rho_bulk, double rho_disp,
                               double out[9]);

/* ------------------------------------------------------------- slab halos
 * A lattice cut into row slabs (one per GPU, or several on one GPU): a slab
 * owning global rows [y0, y1) is a domain of y1 - y0 + 2 H rows whose first and
 * last H rows are ghost copies of the neighbouring slabs' rows (the lattice's
 * periodic wrap decides the neighbours).  k steps between exchanges need
 * H >= 2 k; owned rows then stay bit-identical to stepping the whole lattice.
 * The slab decomposition of tests/lbm/lbm_matlab/two_phase_flow/main_droplet.m
 * (:162-465) with whole population rows as the halo.  Buffers are device
 * memory of sclbm_domain_halo_bytes(d, H) bytes, laid out [component][direction]
 * [H rows][nx] in the storage type; the copies are queued on the library
 * stream.
 *   pack side 0: the first H owned rows (for the slab below), side 1: the
 *   last H owned rows (for the slab above);
 *   unpack side 0: into the H ghost rows below the owned rows, side 1: into
 *   the H ghost rows above.
 * SCLBM_E_OUT_OF_RANGE when H < 1 or 3 H > ny. */
size_t sclbm_domain_halo_bytes(const sclbm_domain *d, int rows);
int sclbm_domain_halo_pack(sclbm_domain *d, int rows, int side, void *dst);
int sclbm_domain_halo_unpack(sclbm_domain *d, int rows, int side, const void *src);
/* Per-step exchange with one ghost row per side (the domain is the slab's
 * owned rows plus one ghost row below and one above; exchange after every
 * step): nine values per component and column per side instead of whole
 * rows -- the six populations of the row next to the cut that the neighbour
 * cannot compute itself, and the three that crossed the cut.  Owned rows stay
 * bit-identical to one domain holding the whole lattice.  The buffer holds
 * sclbm_domain_halo_min_bytes(d) bytes, [component][9][nx] of the storage
 * type.  pack side 0 goes to the slab below (it unpacks it as side 1), side
 * 1 to the slab above (unpacked as side 0).  The reference's MATLAB slab
 * generator exchanges the crossing populations and a density row
 * (tests/lbm/lbm_matlab/two_phase_flow/main_droplet.m:300-465); a density row
 * instead of the six populations would change the order of the ghost
 * density's sum and with it the last bits. */
size_t sclbm_domain_halo_min_bytes(const sclbm_domain *d);
int sclbm_domain_halo_min_pack(sclbm_domain *d, int side, void *dst);
int sclbm_domain_halo_min_unpack(sclbm_domain *d, int side, const void *src);
/* One step of the domain rows [row0, row0 + nrows) only (register tile, into
 * the other buffer); finish = 1 ends the step (swaps the buffers) once every
 * row has been stepped.  A slab steps the rows that need no halo (all but
 * the three at each cut) while its exchange is in flight, then the rest.
 * Two-component domains. */
int sclbm_domain_step_rows(sclbm_domain *d, int row0, int nrows, int finish);

/* ------------------------------------------------------------------- batch
 * Many independent domains of one precision advanced together: one launch
 * per time step walks a tile list drawn from all domains, and the launch
 * sequence of a run is captured in a CUDA graph. */
typedef struct sclbm_batch sclbm_batch;

/* tile_y_per_domain may be NULL: rows per tile then come from the tuned table
 * (sclbm_tuned_config) for each domain's size class */
int sclbm_batch_create(sclbm_domain *const *domains, int ndomains, const int *tile_y_per_domain,
                       sclbm_batch **out);
void sclbm_batch_destroy(sclbm_batch *b);
/* Work decomposition (same results either way): 0 = automatic (batches with
 * solid nodes: the body the autotuner's mixed-ensemble sweep found fastest
 * for the precision -- the ring body 11 with 16-row units for FP64, 24 for
 * FP32 and 32 for FP16; other batches: the tuned variant of the size
 * class holding most of the batch's nodes); 11 = ring body: persistent CTAs
 * take (domain, 128-column strip, band) units from a work counter (each
 * domain's units together, domains largest first) and run the ring pipeline
 * of domain variant 11 (rows per unit: tile_y_per_domain,
 * else the tuned default); 12 = the same on 64-column strips (11, 12: every
 * domain's rows on 16-byte boundaries); 2 = tile
 * list, tile_y rows per tile, register-tile body; 3 = 128-column strips x
 * row bands of one common height, pipelined body (FP64 and FP32 storage);
 * 5 = tile list with the load-ahead body, 6 = tile list with the compacted
 * fluid-lane body, 8 = tile list with the uniform solid body (domain variant
 * 8), 9 = the uniform body on 64-column tiles, two side by side per CTA
 * (fewer idle lanes on narrow domains), 10 = the uniform body on one-warp
 * 32-column tiles, each warp walking its own tiles (no CTA barrier) (5, 6, 8,
 * 9 and 10: FP32 and FP16 storage).  The automatic tile list of FP32 and FP16 batches holding solid
 * nodes runs the uniform body. */
int sclbm_batch_set_kernel(sclbm_batch *b, int variant);
/* advance every domain nsteps; use_graph = 1 replays a captured CUDA graph */
int sclbm_batch_step(sclbm_batch *b, int nsteps, int use_graph);
int sclbm_batch_info(const sclbm_batch *b, int *ntiles, int *grid_ctas);

/* Tuned launch shape for an nx x ny two-component domain stored at
 * `precision` (sclbm_precision; -1 = the recommended one), from the table
 * that sc_lbm_b200/autotune.py measured on B200 and the build compiled in.
 * Sizes outside the table take the nearest size class.  *recommended is the
 * fastest storage whose density error against FP64 stayed within 1e-5 for
 * that class.  Host-only lookup (no device needed).  No reference
 * counterpart: the reference has no batched or tuned path.  Any output
 * pointer may be NULL. */
int sclbm_tuned_config(size_t nx, size_t ny, int precision, int *tile_y, int *variant,
                       int *recommended);

#ifdef __cplusplus
}
#endif
#endif
