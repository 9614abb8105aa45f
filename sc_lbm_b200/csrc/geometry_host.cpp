// geometry_host.cpp -- host construction of the solid mask, bit-exact with the
// reference Geometry (src/geometry.cpp, src/geom_object/{rectangle,ellipse}.cpp,
// src/arrays/regular_array.cpp).  Sizes are unsigned 64-bit exactly like the
// reference's size_t arithmetic, including its wrap-around for objects that
// reach past the lattice, and an error leaves the mask modified exactly as far
// as the reference got before throwing.
#include <algorithm>
#include <cctype>
#include <cstring>

#include "internal.h"

namespace sclbm {
namespace {

using Nodes = std::vector<std::pair<size_t, size_t>>;

// Rectangle::find_nodes, rectangle.cpp:12-31 -- an even extent shrinks by one
// so the object is symmetric about its centre; x outer, y inner.
int rectangle_nodes(size_t lx, size_t ly, size_t xc, size_t yc, Nodes &out)
{
    if (lx % 2 == 0) --lx;
    if (ly % 2 == 0) --ly;
    const size_t x0 = xc - lx / 2, x1 = xc + lx / 2, y0 = yc - ly / 2, y1 = yc + ly / 2;
    for (size_t ix = x0; ix <= x1; ++ix) {
        for (size_t iy = y0; iy <= y1; ++iy) {
            if (out.size() > (size_t(1) << 31)) return SCLBM_E_DOMAIN;
            out.emplace_back(ix, iy);
            if (iy == SIZE_MAX) break;
        }
        if (ix == SIZE_MAX) break;
    }
    return SCLBM_OK;
}

// Ellipse::find_nodes, ellipse.cpp:12-34 -- integer test
//   dx^2*Ly^2/4 + dy^2*Lx^2/4 <= Lx^2*Ly^2/16 with unsigned wrap-around
int ellipse_nodes(size_t lx, size_t ly, size_t xc, size_t yc, Nodes &out)
{
    if (lx % 2 == 0) --lx;
    if (ly % 2 == 0) --ly;
    const size_t x0 = xc - lx / 2, x1 = xc + lx / 2, y0 = yc - ly / 2, y1 = yc + ly / 2;
    const size_t rhs = lx * lx * ly * ly / 16;
    for (size_t ix = x0; ix <= x1; ++ix) {
        const size_t dx = ix - xc;
        const size_t ax = dx * dx * ly * ly / 4;
        for (size_t iy = y0; iy <= y1; ++iy) {
            const size_t dy = iy - yc;
            if (ax + dy * dy * lx * lx / 4 <= rhs) {
                if (out.size() > (size_t(1) << 31)) return SCLBM_E_DOMAIN;
                out.emplace_back(ix, iy);
            }
            if (iy == SIZE_MAX) break;
        }
        if (ix == SIZE_MAX) break;
    }
    return SCLBM_OK;
}

} // namespace

// Geometry::add_walls, geometry.cpp:34-69
int geom_add_walls(std::vector<int32_t> &g, size_t nx, size_t ny, size_t dH, const std::string &w)
{
    if (w == "y") {
        if (dH > nx) return set_error(SCLBM_E_RUNTIME, "Wall thickness larger than domain width (x)");
        for (size_t iy = 0; iy < ny; ++iy)
            for (size_t ix = 0; ix < dH; ++ix) {
                g[iy * nx + ix] = 0;
                g[iy * nx + (nx - 1 - ix)] = 0;
            }
    } else if (w == "x") {
        if (dH > ny)
            return set_error(SCLBM_E_RUNTIME, "Wall thickness larger than domain height (y)");
        for (size_t iy = 0; iy < dH; ++iy) {
            std::fill(g.begin() + iy * nx, g.begin() + (iy + 1) * nx, 0);
            std::fill(g.begin() + (ny - 1 - iy) * nx, g.begin() + (ny - iy) * nx, 0);
        }
    } else {
        return set_error(SCLBM_E_INVALID_ARGUMENT, "No options for position argument: " + w);
    }
    if (ny == 0) return set_error(SCLBM_E_OUT_OF_RANGE, "vector::_M_range_check (empty geometry)");
    return SCLBM_OK;
}

// add_rectangle / add_square / add_ellipse / add_circle, geometry.cpp:76-147,
// with check_object_bounds (:150-162) and check_constructed_object (:167-175)
int geom_add_object(std::vector<int32_t> &g, size_t nx, size_t ny, int kind, size_t lx,
                    size_t ly, size_t xc, size_t yc)
{
    static const char *names[4] = {"Rectangle", "Square", "Ellipse", "Circle"};
    const char *name = names[kind & 3];
    const bool ellipse = kind >= 2;
    if ((int(xc) - int(lx) / 2) < 0 || (int(yc) - int(ly) / 2) < 0)
        return set_error(SCLBM_E_RUNTIME, std::string(name) + " lower bounds do not fit the domain.");
    if ((xc + lx / 2) >= nx || (yc + ly / 2) >= ny)
        return set_error(SCLBM_E_RUNTIME, std::string(name) + " upper bounds do not fit the domain.");
    Nodes nodes;
    int rc = ellipse ? ellipse_nodes(lx, ly, xc, yc, nodes) : rectangle_nodes(lx, ly, xc, yc, nodes);
    if (rc) return set_error(rc, "object too large");
    for (const auto &p : nodes)
        if (p.second * nx + p.first >= nx * ny)
            return set_error(SCLBM_E_RUNTIME,
                             std::string("Constructed ") + name + " upper bounds do not fit the domain.");
    for (const auto &p : nodes) g[p.second * nx + p.first] = 0;
    return SCLBM_OK;
}

// Geometry::add_array, geometry.cpp:182-240 with RegularArray,
// regular_array.cpp:9-114
int geom_add_array(std::vector<int32_t> &g, size_t nx, size_t ny, const std::string &type,
                   const size_t *p, size_t np, const size_t *bounds, size_t a, size_t b,
                   int by_numbers)
{
    std::string t = type;
    std::transform(t.begin(), t.end(), t.begin(), [](unsigned char c) { return std::tolower(c); });
    Nodes obj;
    int rc;
    if (t == "rectangle" && np >= 4) rc = rectangle_nodes(p[0], p[1], p[2], p[3], obj);
    else if (t == "square" && np >= 3) rc = rectangle_nodes(p[0], p[0], p[1], p[2], obj);
    else if (t == "ellipse" && np >= 4) rc = ellipse_nodes(p[0], p[1], p[2], p[3], obj);
    else if (t == "circle" && np >= 3) rc = ellipse_nodes(p[0], p[0], p[1], p[2], obj);
    else
        return set_error(SCLBM_E_INVALID_ARGUMENT,
                         "Non-existing object type. Valid types are: rectangle, square, ellipse, "
                         "and circle.");
    if (rc) return set_error(rc, "object too large");
    // bounding box of the object (find_object_bounds)
    size_t xmin = SIZE_MAX, xmax = 0, ymin = SIZE_MAX, ymax = 0;
    for (const auto &q : obj) {
        xmin = std::min(xmin, q.first);
        xmax = std::max(xmax, q.first);
        ymin = std::min(ymin, q.second);
        ymax = std::max(ymax, q.second);
    }
    const size_t olx = xmax - xmin + 1, oly = ymax - ymin + 1;
    const size_t alx = bounds[1] - bounds[0] - olx + 1, aly = bounds[3] - bounds[2] - oly + 1;
    size_t dx, dy, cnx, cny;
    if (by_numbers) { // compute_displacements
        cnx = a;
        cny = b;
        if (cnx - 1 == 0 || cny - 1 == 0)
            return set_error(SCLBM_E_DOMAIN, "one object per direction divides by zero");
        dx = (alx + olx) / (cnx - 1) - olx;
        dy = (aly + oly) / (cny - 1) - oly;
    } else { // compute_numbers
        dx = a;
        dy = b;
        if (dx + olx == 0 || dy + oly == 0) return set_error(SCLBM_E_DOMAIN, "zero object pitch");
        cnx = alx / (dx + olx) + 1;
        cny = aly / (dy + oly) + 1;
    }
    if (cnx > 100000000 || cny > 100000000 || double(cnx) * double(cny) * obj.size() > 4e8)
        return set_error(SCLBM_E_DOMAIN, "array too large");
    const size_t xs = xmax - xmin + dx + 1, ys = ymax - ymin + dy + 1;
    for (const auto &q : obj)
        for (size_t xi = 0; xi < cnx; ++xi)
            for (size_t yi = 0; yi < cny; ++yi) {
                const size_t lin = (q.second + ys * yi) * nx + (q.first + xs * xi);
                if (lin >= nx * ny)
                    return set_error(SCLBM_E_OUT_OF_RANGE, "vector::_M_range_check (array node "
                                                           "outside the geometry)");
                g[lin] = 0;
            }
    return SCLBM_OK;
}

} // namespace sclbm
