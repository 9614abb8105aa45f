/*
 * sclbm_oracle.c -- CPU oracle (test infrastructure only; see sclbm_oracle.h).
 *
 * Each function restates one reference routine of LBMFluids/sc_lbm in plain C
 * and cites the file:line it follows.  Operation order is kept exactly so the
 * results are bit-identical to the reference's serial build (g++ -O3 on
 * x86-64, no FMA).  Compile with -ffp-contract=off.
 */
#include "sclbm_oracle.h"

#include <ctype.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* D2Q9 lattice: include/lbm.h:118-128, include/fluid.h:279-283 */
static const int CX[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
static const int CY[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
static const int BB[8] = {3, 4, 1, 2, 7, 8, 5, 6}; /* bb_rules, include/lbm.h:124 */
static const double W_SC[9] = {0.0, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9,
                               1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36}; /* lbm.h:118-122 */
#define WRT0 (4.0 / 9.0) /* fluid.h:282 */
#define WRT1 (1.0 / 9.0)
#define WRT2 (1.0 / 36.0)
#define FEQ1 3.0 /* fluid.h:283 */
#define FEQ2 4.5
#define FEQ3 1.5

/* periodic neighbour, src/lbm.cpp:120-129 */
static inline size_t wrap_x(size_t xi, int c, size_t nx)
{
    long v = (long)xi + c;
    if (c > 0) return v < (long)nx ? (size_t)v : 0;
    return v >= 0 ? (size_t)v : nx - 1;
}

/* ======================= Geometry ======================= */

/* Geometry::add_walls, src/geometry.cpp:34-69 */
int orc_geom_add_walls(uint8_t *g, size_t nx, size_t ny, size_t dH, const char *where)
{
    if (strcmp(where, "y") == 0) {
        if (dH > nx) return ORC_RUNTIME_ERROR;
        for (size_t iy = 0; iy < ny; iy++)
            for (size_t ix = 0; ix < dH; ix++) {
                g[iy * nx + ix] = 0;
                g[iy * nx + (nx - 1) - ix] = 0;
            }
    } else if (strcmp(where, "x") == 0) {
        if (dH > ny) return ORC_RUNTIME_ERROR;
        for (size_t iy = 0; iy < dH; iy++) {
            memset(g + iy * nx, 0, nx);
            memset(g + (ny - 1 - iy) * nx, 0, nx);
        }
    } else {
        return ORC_INVALID_ARGUMENT;
    }
    /* vector_2D_2_flat_vector reads vec2D.at(0): an empty domain throws */
    if (ny == 0) return ORC_OUT_OF_RANGE;
    return ORC_OK;
}

/* Geometry::check_object_bounds, src/geometry.cpp:150-162 */
static int check_object_bounds(size_t nx, size_t ny, size_t Lx, size_t Ly, size_t xc, size_t yc)
{
    if (((int)xc - (int)Lx / 2) < 0 || ((int)yc - (int)Ly / 2) < 0) return ORC_RUNTIME_ERROR;
    if ((xc + Lx / 2) >= nx || (yc + Ly / 2) >= ny) return ORC_RUNTIME_ERROR;
    return ORC_OK;
}

typedef struct {
    size_t *xy; /* pairs */
    size_t n, cap;
} nodelist;

static int nl_push(nodelist *l, size_t x, size_t y)
{
    if (l->n == l->cap) {
        size_t nc = l->cap ? 2 * l->cap : 64;
        size_t *p = (size_t *)realloc(l->xy, 2 * nc * sizeof(size_t));
        if (!p) return -1;
        l->xy = p;
        l->cap = nc;
    }
    l->xy[2 * l->n] = x;
    l->xy[2 * l->n + 1] = y;
    l->n++;
    return 0;
}

/* Rectangle::find_nodes, src/geom_object/rectangle.cpp:12-31 (even sizes shrink by 1) */
static int rect_nodes(size_t Lx, size_t Ly, size_t xc, size_t yc, nodelist *out)
{
    if (!(Lx % 2)) Lx--;
    if (!(Ly % 2)) Ly--;
    size_t x0 = xc - Lx / 2, y0 = yc - Ly / 2, xf = xc + Lx / 2, yf = yc + Ly / 2;
    for (size_t ix = x0; ix <= xf; ix++) {
        for (size_t iy = y0; iy <= yf; iy++) {
            if (nl_push(out, ix, iy)) return ORC_DOMAIN_ERROR;
            if (iy == (size_t)-1) break;
        }
        if (ix == (size_t)-1) break;
    }
    return ORC_OK;
}

/* Ellipse::find_nodes, src/geom_object/ellipse.cpp:12-34 (unsigned integer test) */
static int ellipse_nodes(size_t Lx, size_t Ly, size_t xc, size_t yc, nodelist *out)
{
    if (!(Lx % 2)) Lx--;
    if (!(Ly % 2)) Ly--;
    size_t x0 = xc - Lx / 2, y0 = yc - Ly / 2, xf = xc + Lx / 2, yf = yc + Ly / 2;
    for (size_t ix = x0; ix <= xf; ix++) {
        for (size_t iy = y0; iy <= yf; iy++) {
            size_t dx = ix - xc, dy = iy - yc;
            if ((dx * dx * Ly * Ly / 4 + dy * dy * Lx * Lx / 4) <= Lx * Lx * Ly * Ly / 16)
                if (nl_push(out, ix, iy)) return ORC_DOMAIN_ERROR;
            if (iy == (size_t)-1) break;
        }
        if (ix == (size_t)-1) break;
    }
    return ORC_OK;
}

/* Geometry::add_rectangle/add_square/add_ellipse/add_circle, src/geometry.cpp:76-147 */
static int add_object(uint8_t *g, size_t nx, size_t ny, int ellipse, size_t Lx, size_t Ly,
                      size_t xc, size_t yc)
{
    int rc = check_object_bounds(nx, ny, Lx, Ly, xc, yc);
    if (rc) return rc;
    nodelist l = {0};
    rc = ellipse ? ellipse_nodes(Lx, Ly, xc, yc, &l) : rect_nodes(Lx, Ly, xc, yc, &l);
    if (rc) {
        free(l.xy);
        return rc;
    }
    /* check_constructed_object, src/geometry.cpp:167-175 */
    for (size_t k = 0; k < l.n; k++)
        if (l.xy[2 * k + 1] * nx + l.xy[2 * k] >= nx * ny) {
            free(l.xy);
            return ORC_RUNTIME_ERROR;
        }
    for (size_t k = 0; k < l.n; k++) g[l.xy[2 * k + 1] * nx + l.xy[2 * k]] = 0;
    free(l.xy);
    return ORC_OK;
}

int orc_geom_add_rectangle(uint8_t *g, size_t nx, size_t ny, size_t Lx, size_t Ly, size_t xc,
                           size_t yc)
{
    return add_object(g, nx, ny, 0, Lx, Ly, xc, yc);
}
int orc_geom_add_square(uint8_t *g, size_t nx, size_t ny, size_t Ls, size_t xc, size_t yc)
{
    return add_object(g, nx, ny, 0, Ls, Ls, xc, yc);
}
int orc_geom_add_ellipse(uint8_t *g, size_t nx, size_t ny, size_t Lx, size_t Ly, size_t xc,
                         size_t yc)
{
    return add_object(g, nx, ny, 1, Lx, Ly, xc, yc);
}
int orc_geom_add_circle(uint8_t *g, size_t nx, size_t ny, size_t D, size_t xc, size_t yc)
{
    return add_object(g, nx, ny, 1, D, D, xc, yc);
}

/* Geometry::add_array (both overloads), src/geometry.cpp:182-240, with
 * RegularArray, src/arrays/regular_array.cpp:9-114 */
int orc_geom_add_array(uint8_t *g, size_t nx, size_t ny, const char *type, const size_t *p,
                       size_t np, const size_t *bounds, size_t a, size_t b, int by_numbers)
{
    char t[32];
    size_t k;
    for (k = 0; type[k] && k < sizeof(t) - 1; k++) t[k] = (char)tolower((unsigned char)type[k]);
    t[k] = 0;
    nodelist obj = {0};
    int rc;
    if (strcmp(t, "rectangle") == 0 && np >= 4) rc = rect_nodes(p[0], p[1], p[2], p[3], &obj);
    else if (strcmp(t, "square") == 0 && np >= 3) rc = rect_nodes(p[0], p[0], p[1], p[2], &obj);
    else if (strcmp(t, "ellipse") == 0 && np >= 4) rc = ellipse_nodes(p[0], p[1], p[2], p[3], &obj);
    else if (strcmp(t, "circle") == 0 && np >= 3) rc = ellipse_nodes(p[0], p[0], p[1], p[2], &obj);
    else return ORC_INVALID_ARGUMENT;
    if (rc) {
        free(obj.xy);
        return rc;
    }
    /* find_object_bounds, regular_array.cpp:9-38 */
    size_t xmin = (size_t)-1, xmax = 0, ymin = (size_t)-1, ymax = 0;
    for (k = 0; k < obj.n; k++) {
        size_t x = obj.xy[2 * k], y = obj.xy[2 * k + 1];
        if (x < xmin) xmin = x;
        if (x > xmax) xmax = x;
        if (y < ymin) ymin = y;
        if (y > ymax) ymax = y;
    }
    /* compute_object_size / compute_array_dimensions, regular_array.cpp:69-93 */
    size_t olx = xmax - xmin + 1, oly = ymax - ymin + 1;
    size_t alx = bounds[1] - bounds[0] - olx + 1, aly = bounds[3] - bounds[2] - oly + 1;
    size_t dx, dy, cnx, cny;
    if (by_numbers) { /* compute_displacements, regular_array.cpp:56-66 */
        cnx = a;
        cny = b;
        if (cnx - 1 == 0 || cny - 1 == 0) {
            free(obj.xy);
            return ORC_DOMAIN_ERROR;
        }
        dx = (alx + olx) / (cnx - 1) - olx;
        dy = (aly + oly) / (cny - 1) - oly;
    } else { /* compute_numbers, regular_array.cpp:42-53 */
        dx = a;
        dy = b;
        if (dx + olx == 0 || dy + oly == 0) {
            free(obj.xy);
            return ORC_DOMAIN_ERROR;
        }
        cnx = alx / (dx + olx) + 1;
        cny = aly / (dy + oly) + 1;
    }
    if (cnx > 100000000 || cny > 100000000 || (double)cnx * (double)cny * obj.n > 4e8) {
        free(obj.xy);
        return ORC_DOMAIN_ERROR; /* the reference would exhaust memory here */
    }
    /* RegularArray::find_nodes, regular_array.cpp:94-114; then geom.at(node) = 0 */
    size_t xs = xmax - xmin + dx + 1, ys = ymax - ymin + dy + 1;
    for (k = 0; k < obj.n; k++)
        for (size_t xi = 0; xi < cnx; ++xi)
            for (size_t yi = 0; yi < cny; ++yi) {
                size_t xp = obj.xy[2 * k] + xs * xi, yp = obj.xy[2 * k + 1] + ys * yi;
                size_t lin = yp * nx + xp;
                if (lin >= nx * ny) {
                    free(obj.xy);
                    return ORC_OUT_OF_RANGE;
                }
                g[lin] = 0;
            }
    free(obj.xy);
    return ORC_OK;
}

/* ======================= Fluid ======================= */

/* Fluid::compute_density, src/fluid.cpp:175-183 */
void orc_compute_density(size_t N, const double *f, double *rho)
{
    for (size_t i = 0; i < N; ++i) {
        double r = 0.0;
        for (size_t j = 0; j < 9; ++j) r += f[j * N + i];
        rho[i] = r;
    }
}

/* Fluid::compute_velocities, src/fluid.cpp:186-200 */
void orc_compute_velocities(size_t N, const uint8_t *g, const double *f, const double *rho,
                            double *ux, double *uy)
{
    for (size_t i = 0; i < N; ++i) {
        double x = 0.0, y = 0.0;
        if (g[i] == 1) {
            for (size_t j = 0; j < 9; ++j) {
                x += f[j * N + i] * (double)CX[j];
                y += f[j * N + i] * (double)CY[j];
            }
            x /= rho[i];
            y /= rho[i];
        }
        ux[i] = x;
        uy[i] = y;
    }
}

/* equilibrium formula shared by both overloads, src/fluid.cpp:219-241 / 254-276 */
static void feq_node(size_t N, size_t ai, double r, double ux, double uy, double *feq)
{
    double rt0 = WRT0 * r, rt1 = WRT1 * r, rt2 = WRT2 * r;
    double uxsq = ux * ux, uysq = uy * uy;
    double u5 = ux + uy, u6 = -ux + uy, u7 = -ux - uy, u8 = ux - uy;
    double usq = uxsq + uysq;
    feq[ai] = rt0 * (1.0 - FEQ3 * usq);
    feq[ai + N] = rt1 * (1.0 + FEQ1 * ux + FEQ2 * uxsq - FEQ3 * usq);
    feq[ai + 2 * N] = rt1 * (1.0 + FEQ1 * uy + FEQ2 * uysq - FEQ3 * usq);
    feq[ai + 3 * N] = rt1 * (1.0 - FEQ1 * ux + FEQ2 * uxsq - FEQ3 * usq);
    feq[ai + 4 * N] = rt1 * (1.0 - FEQ1 * uy + FEQ2 * uysq - FEQ3 * usq);
    feq[ai + 5 * N] = rt2 * (1.0 + FEQ1 * u5 + FEQ2 * u5 * u5 - FEQ3 * usq);
    feq[ai + 6 * N] = rt2 * (1.0 + FEQ1 * u6 + FEQ2 * u6 * u6 - FEQ3 * usq);
    feq[ai + 7 * N] = rt2 * (1.0 + FEQ1 * u7 + FEQ2 * u7 * u7 - FEQ3 * usq);
    feq[ai + 8 * N] = rt2 * (1.0 + FEQ1 * u8 + FEQ2 * u8 * u8 - FEQ3 * usq);
}

/* Fluid::compute_f_equilibrium(geom), src/fluid.cpp:210-243 */
void orc_feq_single(size_t N, const uint8_t *g, const double *f, double *rho, double *ux,
                    double *uy, double *feq)
{
    orc_compute_density(N, f, rho); /* compute_macroscopic, fluid.cpp:203-207 */
    orc_compute_velocities(N, g, f, rho, ux, uy);
    for (size_t ai = 0; ai < N; ++ai) feq_node(N, ai, rho[ai], ux[ai], uy[ai], feq);
}

/* Fluid::compute_f_equilibrium(), src/fluid.cpp:246-278 */
void orc_feq_multi(size_t N, const double *rho, const double *uex, const double *uey, double *feq)
{
    for (size_t ai = 0; ai < N; ++ai) feq_node(N, ai, rho[ai], uex[ai], uey[ai], feq);
}

/* ======================= initialisers ======================= */

/* LBM::initialize_droplet, src/lbm.cpp:11-48 (f = rho/9 on fluid nodes) */
void orc_init_droplet(size_t nx, size_t ny, const uint8_t *g, double *fb, double *fd,
                      double rho_bulk, double rho_drop, double rho_b_in_d, double rho_d_in_b,
                      double xc, double yc, double radius)
{
    size_t N = nx * ny;
    for (size_t ai = 0; ai < N; ++ai) {
        int xi = (int)(ai % nx);
        int yj = (int)(((ai - (size_t)xi) / nx) % ny);
        if (g[ai] == 0) continue;
        int inside = (((double)xi - xc) * ((double)xi - xc) + ((double)yj - yc) * ((double)yj - yc))
                     <= radius * radius;
        for (size_t dj = 0; dj < 9; ++dj) {
            fb[ai + dj * N] = (inside ? rho_b_in_d : rho_bulk) / 9.0;
            fd[ai + dj * N] = (inside ? rho_drop : rho_d_in_b) / 9.0;
        }
    }
}

/* LBM::initialize_fluid_rectangle, src/lbm.cpp:51-99 */
int orc_init_rectangle(size_t nx, size_t ny, const uint8_t *g, double *fb, double *fd,
                       double rho_bulk, double rho_drop, double rho_b_in_d, double rho_d_in_b,
                       double xc, double yc, double half_lx, double half_ly)
{
    size_t N = nx * ny;
    for (size_t ai = 0; ai < N; ++ai) {
        if (g[ai] == 0) continue;
        for (size_t dj = 0; dj < 9; ++dj) {
            fb[ai + dj * N] = rho_bulk / 9.0;
            fd[ai + dj * N] = rho_d_in_b / 9.0;
        }
    }
    int x0 = (int)(xc - half_lx + 1), xf = (int)(xc + half_lx - 1);
    int y0 = (int)(yc - half_ly + 1), yf = (int)(yc + half_ly - 1);
    for (int xi = x0; xi <= xf; ++xi)
        for (int yj = y0; yj <= yf; ++yj) {
            size_t lin = (size_t)yj * nx + (size_t)xi; /* geom(xi, yj) -> geom.at() */
            if (lin >= N) return ORC_OUT_OF_RANGE;
            if (g[lin] == 0) continue;
            for (size_t dj = 0; dj < 9; ++dj) {
                fb[dj * N + lin] = rho_b_in_d / 9.0;
                fd[dj * N + lin] = rho_drop / 9.0;
            }
        }
    return ORC_OK;
}

/* Fluid::simple_ini, src/fluid.cpp:64-104 (f = rho_0/9 on fluid nodes) */
void orc_simple_ini(size_t N, const uint8_t *g, double *f, double rho0)
{
    for (size_t i = 0; i < N; ++i)
        if (g[i] == 1)
            for (size_t k = 0; k < 9; ++k) f[k * N + i] = rho0 / 9.0;
}

/* ======================= LBM ======================= */

/* LBM::compute_solid_surface_force, src/lbm.cpp:102-141 (the shared sums) */
void orc_solid_sum(size_t nx, size_t ny, const uint8_t *g, double *sx, double *sy)
{
    size_t N = nx * ny;
    for (size_t ai = 0; ai < N; ++ai) {
        sx[ai] = 0.0;
        sy[ai] = 0.0;
        size_t xi = ai % nx, yj = ((ai - xi) / nx) % ny;
        if (g[ai] == 0) continue;
        for (size_t dj = 1; dj < 9; ++dj) {
            size_t in = wrap_x(xi, CX[dj], nx), jn = wrap_x(yj, CY[dj], ny);
            if (g[jn * nx + in] == 0) {
                sx[ai] += W_SC[dj] * CX[dj];
                sy[ai] += W_SC[dj] * CY[dj];
            }
        }
    }
}

/* Fluid::add_surface_forces, src/fluid.cpp:154-160 */
void orc_surface_force(size_t N, double gs, const double *sx, const double *sy, double *fsx,
                       double *fsy)
{
    for (size_t i = 0; i < N; ++i) {
        fsx[i] = -1.0 * gs * sx[i];
        fsy[i] = -1.0 * gs * sy[i];
    }
}

/* LBM::compute_fluid_repulsive_interactions, src/lbm.cpp:144-206 */
void orc_repulsive(size_t nx, size_t ny, const uint8_t *g, const double *psi1, const double *psi2,
                   double G1, double G2, double *f1x, double *f1y, double *f2x, double *f2y)
{
    size_t N = nx * ny;
    const double gf1 = -1.0 * G1, gf2 = -1.0 * G2;
    for (size_t ai = 0; ai < N; ++ai) {
        f1x[ai] = f1y[ai] = f2x[ai] = f2y[ai] = 0.0;
    }
    for (size_t ai = 0; ai < N; ++ai) {
        size_t xi = ai % nx, yj = ((ai - xi) / nx) % ny;
        if (g[ai] == 0) continue;
        for (size_t dj = 1; dj < 9; ++dj) {
            size_t in = wrap_x(xi, CX[dj], nx), jn = wrap_x(yj, CY[dj], ny);
            if (g[jn * nx + in] == 0) continue;
            size_t ij = jn * nx + in;
            f1x[ai] += W_SC[dj] * CX[dj] * psi2[ij];
            f1y[ai] += W_SC[dj] * CY[dj] * psi2[ij];
            f2x[ai] += W_SC[dj] * CX[dj] * psi1[ij];
            f2y[ai] += W_SC[dj] * CY[dj] * psi1[ij];
        }
        f1x[ai] *= gf1 * psi1[ai];
        f1y[ai] *= gf1 * psi1[ai];
        f2x[ai] *= gf2 * psi2[ai];
        f2y[ai] *= gf2 * psi2[ai];
    }
}

/* equal_floats(x, 0.0, 1e-16), include/utils.h:145-150 */
static inline int rho_is_zero(double r)
{
    double m = 1.0;
    if (m < fabs(r)) m = fabs(r);
    return fabs(r - 0.0) <= 1e-16 * m;
}

/* LBM::compute_equilibrium_velocities, src/lbm.cpp:209-272.  ux/uy receive the
 * momentum sums (not velocities), exactly like the reference. */
void orc_eqvel(size_t nx, size_t ny, const uint8_t *g, double omega1, double omega2,
               const double *f1, const double *f2, const double *rho1, const double *rho2,
               const double *fr1x, const double *fr1y, const double *fr2x, const double *fr2y,
               const double *fs1x, const double *fs1y, const double *fs2x, const double *fs2y,
               double *ux1, double *uy1, double *ux2, double *uy2, double *uex1, double *uey1,
               double *uex2, double *uey2)
{
    size_t N = nx * ny;
    const double io1 = 1.0 / omega1, io2 = 1.0 / omega2;
    for (size_t i = 0; i < N; ++i) ux1[i] = uy1[i] = ux2[i] = uy2[i] = 0.0;
    for (size_t i = 0; i < N; ++i) {
        if (g[i] != 1) continue;
        double a = 0.0, b = 0.0, c = 0.0, d = 0.0;
        for (size_t j = 0; j < 9; ++j) {
            a += f1[j * N + i] * CX[j];
            b += f1[j * N + i] * CY[j];
            c += f2[j * N + i] * CX[j];
            d += f2[j * N + i] * CY[j];
        }
        ux1[i] = a;
        uy1[i] = b;
        ux2[i] = c;
        uy2[i] = d;
        double ucx = (a * omega1 + c * omega2) / (rho1[i] * omega1 + rho2[i] * omega2);
        double ucy = (b * omega1 + d * omega2) / (rho1[i] * omega1 + rho2[i] * omega2);
        if (!rho_is_zero(rho1[i])) {
            uex1[i] = ucx + fr1x[i] * io1 / rho1[i] + fs1x[i] * io1;
            uey1[i] = ucy + fr1y[i] * io1 / rho1[i] + fs1y[i] * io1;
        }
        if (!rho_is_zero(rho2[i])) {
            uex2[i] = ucx + fr2x[i] * io2 / rho2[i] + fs2x[i] * io2;
            uey2[i] = ucy + fr2y[i] * io2 / rho2[i] + fs2y[i] * io2;
        }
    }
}

/* LBM::collide loops, src/lbm.cpp:283-287 and 306-311 */
void orc_collide(size_t N, double omega, double *f, const double *feq)
{
    for (size_t k = 0; k < 9 * N; ++k) f[k] = (1.0 - omega) * f[k] + omega * feq[k];
}

/* LBM::add_volume_force, src/lbm.cpp:315-340 */
void orc_volume_force(size_t N, const uint8_t *g, double *f, const double *force9)
{
    for (size_t ai = 0; ai < N; ++ai)
        if (g[ai] == 1)
            for (size_t dj = 0; dj < 9; ++dj) f[ai + dj * N] += force9[dj];
}

/* LBM::stream, src/lbm.cpp:343-384: push from fluid nodes to fluid neighbours,
 * half-way bounce-back into bb(dj) at the node itself, solids end up zero. */
void orc_stream(size_t nx, size_t ny, const uint8_t *g, double *f, double *tmp)
{
    size_t N = nx * ny;
    memset(tmp, 0, 9 * N * sizeof(double));
    for (size_t ai = 0; ai < N; ++ai) {
        size_t xi = ai % nx, yj = ((ai - xi) / nx) % ny;
        if (g[ai] != 1) continue;
        tmp[ai] = f[ai];
        for (size_t dj = 1; dj < 9; ++dj) {
            size_t is = wrap_x(xi, CX[dj], nx), js = wrap_x(yj, CY[dj], ny);
            size_t ini = dj * N + yj * nx + xi;
            if (g[js * nx + is] == 1)
                tmp[dj * N + js * nx + is] = f[ini];
            else
                tmp[(size_t)BB[dj - 1] * N + yj * nx + xi] = f[ini];
        }
    }
    memcpy(f, tmp, 9 * N * sizeof(double));
}

/* Time loops of the drivers: laplace_law.cpp:123-133 (two components) */
void orc_run_two(size_t nx, size_t ny, const uint8_t *g, orc_component *c1, orc_component *c2,
                 const double *force9, int force_mode, int nsteps, double *tmp)
{
    size_t N = nx * ny;
    for (int s = 0; s < nsteps; ++s) {
        orc_compute_density(N, c1->f, c1->rho);
        orc_compute_density(N, c2->f, c2->rho);
        orc_repulsive(nx, ny, g, c1->rho, c2->rho, c1->G, c2->G, c1->frx, c1->fry, c2->frx,
                      c2->fry);
        orc_eqvel(nx, ny, g, c1->omega, c2->omega, c1->f, c2->f, c1->rho, c2->rho, c1->frx,
                  c1->fry, c2->frx, c2->fry, c1->fsx, c1->fsy, c2->fsx, c2->fsy, c1->ux, c1->uy,
                  c2->ux, c2->uy, c1->uex, c1->uey, c2->uex, c2->uey);
        orc_feq_multi(N, c1->rho, c1->uex, c1->uey, c1->feq);
        orc_feq_multi(N, c2->rho, c2->uex, c2->uey, c2->feq);
        /* collide(f1,f2) interleaves the two fluids per element; the values are
         * independent so component order does not matter */
        orc_collide(N, c1->omega, c1->f, c1->feq);
        orc_collide(N, c2->omega, c2->f, c2->feq);
        if (force9 && (force_mode & 1)) orc_volume_force(N, g, c1->f, force9);
        if (force9 && (force_mode & 2)) orc_volume_force(N, g, c2->f, force9);
        orc_stream(nx, ny, g, c1->f, tmp);
        orc_stream(nx, ny, g, c2->f, tmp);
    }
}

/* laminar_flow_x_dir.cpp:64-68 (one component) */
void orc_run_single(size_t nx, size_t ny, const uint8_t *g, double omega, double *f,
                    double *feq, double *rho, double *ux, double *uy, const double *force9,
                    int nsteps, double *tmp)
{
    size_t N = nx * ny;
    for (int s = 0; s < nsteps; ++s) {
        orc_feq_single(N, g, f, rho, ux, uy, feq);
        orc_collide(N, omega, f, feq);
        if (force9) orc_volume_force(N, g, f, force9);
        orc_stream(nx, ny, g, f, tmp);
    }
}
