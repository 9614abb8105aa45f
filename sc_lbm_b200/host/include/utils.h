#ifndef UTILS_H
#define UTILS_H

// Index and comparison helpers with the names and behaviour of the reference's
// include/utils.h:18-150 (drivers and tests use them directly).
#include "common.h"

/// (x, y) subscripts to linear indices y*Nx + x
template <typename T> std::vector<T> sub2ind(const std::vector<std::vector<T>> &subs, const size_t Nx)
{
    std::vector<T> lin(subs.size());
    for (size_t i = 0; i < subs.size(); ++i) lin.at(i) = subs[i].at(1) * Nx + subs[i].at(0);
    return lin;
}

/// Row-major flat vector to nested vector: Nrow rows of Ncol values
template <typename T>
std::vector<std::vector<T>> flat_vector_2_vector_2D(const size_t Ncol, const size_t Nrow,
                                                    const std::vector<T> &flat_vec)
{
    std::vector<std::vector<T>> out(Nrow, std::vector<T>(Ncol));
    for (size_t r = 0; r < Nrow; ++r)
        for (size_t c = 0; c < Ncol; ++c) out.at(r).at(c) = flat_vec.at(Ncol * r + c);
    return out;
}

/// Nested vector to row-major flat vector (row length from the first row)
template <typename T> std::vector<T> vector_2D_2_flat_vector(const std::vector<std::vector<T>> &v)
{
    const size_t ncol = v.at(0).size();
    std::vector<T> out(v.size() * ncol);
    for (size_t r = 0; r < v.size(); ++r) std::copy(v[r].begin(), v[r].end(), out.begin() + r * ncol);
    return out;
}

/// Lower-case copy of a string
inline std::string str_to_lower(std::string s)
{
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return std::tolower(c); });
    return s;
}

/// Print a collection on one line after an optional prefix
template <typename T> inline void print_elements(const T &coll, const std::string &optstr = "")
{
    std::cout << optstr;
    for (const auto &e : coll) std::cout << e << ' ';
    std::cout << std::endl;
}

/// |a - b| <= tol * max(1, |a|, |b|)
template <typename T> bool equal_floats(T num1, T num2, T tol)
{
    T m = 1.0;
    if (m < std::fabs(num1)) m = std::fabs(num1);
    if (m < std::fabs(num2)) m = std::fabs(num2);
    return std::fabs(num1 - num2) <= tol * m;
}

#endif
