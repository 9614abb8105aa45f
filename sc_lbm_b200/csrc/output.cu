// output.cu -- files of a device lattice: the reference's text formats and an
// exact binary checkpoint.
//
// Text (Fluid::write_var, src/fluid.cpp:303-343, written through
// LbmIO::write_vector, include/io_operations/lbm_io.h:106-116): one line per
// lattice row, every value printed with the stream defaults (6 significant
// digits, the %g style) and followed by a space.  The rows are cut the way
// write_var cuts them, including its corner cases: a 1 x 1 lattice gives an
// empty file, and with nx == 1 the value before the last one is dropped.
// Populations go to nine files <prefix>_<i>.txt (write_var's 3-D overload,
// :346-353) and are read back by the same layout (Fluid::restart_from_file,
// :285-298).
//
// Device fields are computed on the library stream and copied into pinned host
// memory; the formatting and the file writes then run either in the calling
// thread or, asynchronously, in a worker thread that waits on an event, so the
// GPU keeps stepping while the text is written.
//
// Checkpoint: a header (magic, version, precision, sizes), the mask, then the
// stored populations of every component byte for byte (FP64, FP32 or FP16
// storage as held on the device): a reload continues the run bit for bit.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "domain.h"

using namespace sclbm;

namespace {

// write_var's rows of v (nx * ny values), as text
std::string reference_rows(const double *v, size_t nx, size_t ny)
{
    const size_t N = nx * ny;
    std::vector<std::vector<double>> rows;
    std::vector<double> row(nx, -1.0);
    size_t ind = 0;
    for (size_t i = 0; i < N; ++i) {
        if (i == 0) {
            row[ind++] = v[i];
            continue;
        }
        if (i == N - 1) {
            row[nx - 1] = v[i];
            rows.push_back(row);
            continue;
        }
        if (ind > 0 && ind < nx) {
            row[ind++] = v[i];
        } else {
            ind = 0;
            rows.push_back(row);
            std::fill(row.begin(), row.end(), -1.0);
            row[ind++] = v[i];
        }
    }
    std::string out;
    out.reserve(rows.size() * (nx * 12 + 1));
    char buf[64];
    for (const auto &r : rows) {
        for (double x : r) {
            const int n = std::snprintf(buf, sizeof buf, "%.6g ", x);
            out.append(buf, (size_t)n);
        }
        out.push_back('\n');
    }
    return out;
}

int write_file(const std::string &path, const std::string &text)
{
    std::FILE *fp = std::fopen(path.c_str(), "wb");
    if (!fp) return set_error(SCLBM_E_RUNTIME, "cannot open " + path + ": " + std::strerror(errno));
    const size_t n = std::fwrite(text.data(), 1, text.size(), fp);
    const bool bad = std::fclose(fp) != 0 || n != text.size();
    if (bad) return set_error(SCLBM_E_RUNTIME, "cannot write " + path);
    return SCLBM_OK;
}

// rows of whitespace-separated numbers (LbmIO::read_vector), ny rows of nx
int read_rows(const std::string &path, double *v, size_t nx, size_t ny)
{
    std::ifstream in(path);
    if (!in) return set_error(SCLBM_E_RUNTIME, "cannot open " + path + ": " + std::strerror(errno));
    std::string line;
    size_t y = 0;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::vector<double> r;
        double x;
        while (ls >> x) r.push_back(x);
        if (y < ny) {
            if (r.size() != nx)
                return set_error(SCLBM_E_OUT_OF_RANGE,
                                 path + ": row " + std::to_string(y) + " has " +
                                     std::to_string(r.size()) + " values, expected " +
                                     std::to_string(nx));
            std::copy(r.begin(), r.end(), v + y * nx);
        }
        ++y;
    }
    if (y < ny)
        return set_error(SCLBM_E_OUT_OF_RANGE, path + ": " + std::to_string(y) + " rows, expected " +
                                                   std::to_string(ny));
    return SCLBM_OK;
}

std::string dir_path(const char *prefix, int i) { return std::string(prefix) + "_" + std::to_string(i) + ".txt"; }

// formats and writes the fields held in `host` (N values, or 9N for what == 3)
int write_fields(const double *host, size_t nx, size_t ny, int what, const std::string &path)
{
    const size_t N = nx * ny;
    if (what != 3) return write_file(path, reference_rows(host, nx, ny));
    for (int i = 0; i < 9; ++i) {
        const int rc = write_file(dir_path(path.c_str(), i), reference_rows(host + i * N, nx, ny));
        if (rc) return rc;
    }
    return SCLBM_OK;
}

// asynchronous writers: joined by sclbm_io_wait, first failure kept
std::mutex g_io_mu;
std::vector<std::thread> g_io_threads;
int g_io_status = SCLBM_OK;
std::string g_io_message;

struct PinnedJob {
    double *host = nullptr;
    cudaEvent_t done = nullptr;
};

void release(PinnedJob &j)
{
    if (j.done) cudaEventDestroy(j.done);
    if (j.host) cudaFreeHost(j.host);
    j = PinnedJob{};
}

struct CkHeader {
    char magic[8];
    uint32_t version, precision;
    uint64_t nx, ny;
    uint32_t ncomp, elem;
};

} // namespace

extern "C" int sclbm_write_rows(const char *path, const double *v, size_t nx, size_t ny)
{
    if (!path || (!v && nx * ny != 0)) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    return write_file(path, reference_rows(v, nx, ny));
}

extern "C" int sclbm_read_rows(const char *path, double *v, size_t nx, size_t ny)
{
    if (!path || !v) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    return read_rows(path, v, nx, ny);
}

extern "C" int sclbm_domain_write_text(sclbm_domain *d, int comp, int what, const char *path,
                                       int async)
{
    if (!d || !path) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    if (comp < 0 || comp >= d->ncomp) return set_error(SCLBM_E_INVALID_ARGUMENT, "bad component");
    if (what < 0 || what > 3) return set_error(SCLBM_E_INVALID_ARGUMENT, "what is 0..3");
    const size_t count = (what == 3 ? 9 : 1) * d->N;
    cudaStream_t s = stream();
    PinnedJob job;
    cudaError_t e = cudaMallocHost(&job.host, count * sizeof(double));
    if (e != cudaSuccess) {
        job.host = nullptr;
        return cuda_fail(e, "pinned output buffer");
    }
    if ((e = cudaEventCreateWithFlags(&job.done, cudaEventDisableTiming)) != cudaSuccess) {
        job.done = nullptr;
        release(job);
        return cuda_fail(e, "output event");
    }
    int rc = domain_field_async(d, comp, what, job.host, s);
    if (!rc && (e = cudaEventRecord(job.done, s)) != cudaSuccess) rc = cuda_fail(e, "output event");
    if (rc) {
        cudaStreamSynchronize(s);
        release(job);
        return rc;
    }
    const size_t nx = d->nx, ny = d->ny;
    const std::string p(path);
    if (!async) {
        e = cudaEventSynchronize(job.done);
        rc = e == cudaSuccess ? write_fields(job.host, nx, ny, what, p) : cuda_fail(e, "output copy");
        release(job);
        return rc;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_io_mu);
    g_io_threads.emplace_back([job, nx, ny, what, p, dev]() mutable {
        cudaSetDevice(dev);
        int r = cudaEventSynchronize(job.done) == cudaSuccess ? SCLBM_OK : SCLBM_E_CUDA;
        std::string msg = r ? "asynchronous output copy failed" : "";
        if (!r) {
            r = write_fields(job.host, nx, ny, what, p);
            if (r) {
                char buf[512];
                sclbm_last_error(buf, sizeof buf);
                msg = buf;
            }
        }
        release(job);
        std::lock_guard<std::mutex> g(g_io_mu);
        if (r && !g_io_status) {
            g_io_status = r;
            g_io_message = msg;
        }
    });
    return SCLBM_OK;
}

extern "C" int sclbm_io_wait(void)
{
    std::vector<std::thread> ts;
    {
        std::lock_guard<std::mutex> lk(g_io_mu);
        ts.swap(g_io_threads);
    }
    for (auto &t : ts) t.join();
    std::lock_guard<std::mutex> lk(g_io_mu);
    const int rc = g_io_status;
    const std::string msg = g_io_message;
    g_io_status = SCLBM_OK;
    g_io_message.clear();
    return rc ? set_error(rc, msg) : SCLBM_OK;
}

extern "C" int sclbm_domain_read_text_f(sclbm_domain *d, int comp, const char *prefix)
{
    if (!d || !prefix) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    if (comp < 0 || comp >= d->ncomp) return set_error(SCLBM_E_INVALID_ARGUMENT, "bad component");
    std::vector<double> f(9 * d->N);
    for (int i = 0; i < 9; ++i) {
        const int rc = read_rows(dir_path(prefix, i), f.data() + i * d->N, d->nx, d->ny);
        if (rc) return rc;
    }
    return sclbm_domain_upload_f(d, comp, f.data(), f.size());
}

extern "C" int sclbm_domain_checkpoint_save(sclbm_domain *d, const char *path)
{
    if (!d || !path) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    const size_t es = elem_size(d->prec), bytes = 9 * d->N * es;
    std::vector<unsigned char> host(bytes), mask(d->N);
    cudaStream_t s = stream();
    SCLBM_CUDA(cudaMemcpyAsync(mask.data(), d->d_mask, d->N, cudaMemcpyDeviceToHost, s));
    std::FILE *fp = std::fopen(path, "wb");
    if (!fp) return set_error(SCLBM_E_RUNTIME, std::string("cannot open ") + path);
    CkHeader h{};
    std::memcpy(h.magic, "SCLBMCK1", 8);
    h.version = 1;
    h.precision = (uint32_t)d->prec;
    h.nx = d->nx;
    h.ny = d->ny;
    h.ncomp = (uint32_t)d->ncomp;
    h.elem = (uint32_t)es;
    bool ok = std::fwrite(&h, sizeof h, 1, fp) == 1;
    cudaError_t e = cudaStreamSynchronize(s);
    ok = ok && e == cudaSuccess && std::fwrite(mask.data(), 1, d->N, fp) == d->N;
    for (int k = 0; ok && k < d->ncomp; ++k) {
        e = cudaMemcpyAsync(host.data(), d->buf[d->parity][k], bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        ok = e == cudaSuccess && std::fwrite(host.data(), 1, bytes, fp) == bytes;
    }
    ok = (std::fclose(fp) == 0) && ok;
    if (e != cudaSuccess) return cuda_fail(e, "checkpoint copy");
    if (!ok) return set_error(SCLBM_E_RUNTIME, std::string("cannot write ") + path);
    return SCLBM_OK;
}

extern "C" int sclbm_domain_checkpoint_load(sclbm_domain *d, const char *path)
{
    if (!d || !path) return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    std::FILE *fp = std::fopen(path, "rb");
    if (!fp) return set_error(SCLBM_E_RUNTIME, std::string("cannot open ") + path);
    CkHeader h{};
    const size_t es = elem_size(d->prec), bytes = 9 * d->N * es;
    std::vector<unsigned char> mask(d->N), dmask(d->N), host(bytes);
    int rc = SCLBM_OK;
    if (std::fread(&h, sizeof h, 1, fp) != 1 || std::memcmp(h.magic, "SCLBMCK1", 8) != 0 ||
        h.version != 1)
        rc = set_error(SCLBM_E_INVALID_ARGUMENT, std::string(path) + " is not a checkpoint");
    else if (h.nx != d->nx || h.ny != d->ny || h.ncomp != (uint32_t)d->ncomp ||
             h.precision != (uint32_t)d->prec || h.elem != es)
        rc = set_error(SCLBM_E_INVALID_ARGUMENT,
                       "checkpoint was written by a domain of another size, component count or precision");
    else if (std::fread(mask.data(), 1, d->N, fp) != d->N)
        rc = set_error(SCLBM_E_RUNTIME, std::string(path) + " is truncated");
    cudaStream_t s = stream();
    if (!rc) {
        cudaError_t e = cudaMemcpyAsync(dmask.data(), d->d_mask, d->N, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(e, "mask copy");
        else if (mask != dmask)
            rc = set_error(SCLBM_E_INVALID_ARGUMENT, "checkpoint mask differs from the domain's");
    }
    for (int k = 0; !rc && k < d->ncomp; ++k) {
        if (std::fread(host.data(), 1, bytes, fp) != bytes) {
            rc = set_error(SCLBM_E_RUNTIME, std::string(path) + " is truncated");
            break;
        }
        cudaError_t e = cudaMemcpyAsync(d->buf[d->parity][k], host.data(), bytes,
                                        cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(e, "checkpoint upload");
    }
    std::fclose(fp);
    return rc;
}
