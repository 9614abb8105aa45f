#ifndef LBM_IO_H
#define LBM_IO_H

// Space-delimited text matrices, the file format of the reference's
// include/io_operations/lbm_io.h:51-116: one row per line, every value
// followed by the delimiter, default stream precision (6 significant digits).
#include "../common.h"

class LbmIO {
public:
    LbmIO() = default;
    LbmIO(const std::string &name, const std::string &delim, const bool sflag,
          const std::vector<size_t> &dims)
        : fname(name), delim(delim), single_file(sflag), dimensions(dims)
    {
    }

    /// Read all whitespace-separated values, one vector per line
    template <typename T> std::vector<std::vector<T>> read_vector() const
    {
        std::ifstream in(fname);
        if (!in.is_open()) {
            std::cerr << "Error opening file " << fname << std::endl;
            throw std::ios_base::failure(std::strerror(errno));
        }
        std::vector<std::vector<T>> out;
        std::string line;
        while (std::getline(in, line)) {
            std::istringstream row(line);
            std::vector<T> v;
            T x;
            while (row >> x) v.push_back(x);
            out.push_back(v);
        }
        return out;
    }

    /// Write one line per row (truncates the file)
    template <typename T> void write_vector(const std::vector<std::vector<T>> &data) const
    {
        std::ofstream out(fname, std::ios_base::out | std::ios_base::trunc);
        if (!out.is_open()) {
            std::cerr << "Error opening file " << fname << std::endl;
            throw std::ios_base::failure(std::strerror(errno));
        }
        for (const auto &row : data) {
            std::copy(row.begin(), row.end(), std::ostream_iterator<T>(out, delim.c_str()));
            out << '\n';
        }
    }

private:
    std::string fname = {"dflt_lbm_io_file.txt"};
    std::string delim = {" "};
    bool single_file = true;
    std::vector<size_t> dimensions = {0, 0, 0};
};

#endif
