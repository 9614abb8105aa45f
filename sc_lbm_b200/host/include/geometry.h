#ifndef GEOMETRY_H
#define GEOMETRY_H

// Geometry: the solid mask (1 fluid, 0 solid), row-major [y*Nx + x], with the
// interface of the reference's include/geometry.h:37-286.  Construction runs
// on the host (bit-exact with the reference, same exceptions); a device copy
// for the sm_100a kernels is refreshed lazily after every change.
#include "common.h"
#include "io_operations/lbm_io.h"
#include "utils.h"

struct sclbm_geometry;

class Geometry {
public:
    Geometry();
    Geometry(const size_t Nx, const size_t Ny);
    Geometry(const Geometry &other);
    Geometry &operator=(const Geometry &other);
    ~Geometry();

    /// Pair of solid walls of thickness dH: "y" = first/last columns, "x" = rows
    void add_walls(const size_t dH = 1, const std::string &where = "y");

    void add_rectangle(const size_t Lx, const size_t Ly, const size_t xc, const size_t yc);
    void add_square(const size_t Ls, const size_t xc, const size_t yc);
    void add_ellipse(const size_t Lx, const size_t Ly, const size_t xc, const size_t yc);
    void add_circle(const size_t D, const size_t xc, const size_t yc);

    /// Throws std::runtime_error when an object of the given extent around
    /// (xc, yc) would leave the domain (even extents shrink by one node).
    void check_object_bounds(const size_t Lx, const size_t Ly, const size_t xc, const size_t yc,
                             const std::string &name) const;
    /// Throws std::runtime_error when a node index lies past the domain.
    void check_constructed_object(const std::vector<size_t> &obj, const std::string &name) const;

    /// Regular array of built-in objects given the spacing between them
    void add_array(const std::vector<size_t> &object_properties,
                   const std::vector<std::vector<size_t>> &array_bounds, const size_t dx,
                   const size_t dy, const std::string &object_type, const size_t alpha = 0);
    /// Regular array of built-in objects given their numbers in x and y
    void add_array(const std::vector<size_t> &object_properties,
                   const std::vector<std::vector<size_t>> &array_bounds,
                   const std::vector<size_t> &object_numbers, const std::string &object_type,
                   const size_t alpha = 0);

    void set_node_fluid(const size_t xi, const size_t yi);
    void set_node_solid(const size_t xi, const size_t yi);

    /// Text mask: one row of Nx integers per line
    void read(const std::string &fname);
    void write(const std::string &fname) const;

    const int operator()(const size_t xi, const size_t yi) const { return geom.at(yi * _Nx + xi); }
    const int operator()(const size_t ind) const { return geom.at(ind); }

    size_t Nx() const { return _Nx; }
    size_t Ny() const { return _Ny; }
    const std::vector<int> &get_geom() const { return geom; }

    /// The C-ABI handle (device copy of the mask) used by Fluid and LBM
    const sclbm_geometry *handle() const;

private:
    std::vector<int> geom;
    size_t _Nx = 0, _Ny = 0;
    mutable sclbm_geometry *h = nullptr; // created on first use, kept in sync
    void pull();                         // host mask <- handle after a change
};

#endif
