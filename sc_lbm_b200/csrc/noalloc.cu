// noalloc.cu -- mass/momentum monitor that allocates nothing.
//
// Some callers cannot allocate device memory: a host application that hands
// the library a fixed arena and forbids further cudaMalloc (hard memory
// budgets, custom allocators), or a region of a program in which the caller
// has promised its memory manager that no further device allocation happens.
// For them this variant of sclbm_domain_mass_momentum works directly on the
// caller's device buffers and keeps its per-chunk partial sums in a file-scope
// __device__ array instead of memory it allocates.
//
// It returns its result to the host, so it synchronises its stream: it must
// not be called while that stream is being captured into a CUDA graph, and it
// refuses a capturing stream (SCLBM_E_INVALID_ARGUMENT) before touching it, so
// the caller's capture stays intact.
//
// The array holds NOALLOC_MAX_PARTIALS partial sums of NOALLOC_CHUNK nodes
// each, which bounds the lattice to NOALLOC_MAX_PARTIALS * NOALLOC_CHUNK
// nodes (2^27, e.g. 16384 x 8192); larger lattices are rejected.  Every GPU
// that loads the library holds the array (about 128 KB) until the process
// exits.  Each chunk's slot is overwritten on every call, so nothing needs
// clearing between calls, but all calls share the one array: calls that
// overlap on the GPU (different streams, or host threads) race.
//
// The first call on a device looks the array's device address up and loads
// all of this file's kernels (every precision), so later calls on that device
// make the runtime neither allocate nor load a module.
#include <mutex>

#include "domain.h"
#include "lattice.cuh"

namespace sclbm {
namespace {

constexpr long long NOALLOC_CHUNK = 1 << 16;  // nodes per partial sum
constexpr int NOALLOC_MAX_PARTIALS = 2048;    // => at most 2^27 nodes
constexpr int NOALLOC_VALUES = 7;             // m, jx, jy per component + non-finite count
constexpr int NOALLOC_STRIDE = 8;

// partial sums of every chunk, then the final 7 values
static __device__ __align__(256) double g_noalloc_scratch[(NOALLOC_MAX_PARTIALS + 1) * NOALLOC_STRIDE];

template <typename S> __device__ __forceinline__ double to_f64(S v) { return (double)v; }
template <> __device__ __forceinline__ double to_f64<__half>(__half v) { return (double)__half2float(v); }

// block b reduces nodes [b*CHUNK, (b+1)*CHUNK) in a fixed order
template <typename S>
__global__ void __launch_bounds__(256)
    k_noalloc_partials(size_t N, int ncomp, const uint8_t *__restrict__ mask,
                       const S *__restrict__ f0, const S *__restrict__ f1, double rr0, double rr1,
                       int shifted, double *__restrict__ partials)
{
    double acc[NOALLOC_VALUES] = {0, 0, 0, 0, 0, 0, 0};
    const size_t n0 = (size_t)blockIdx.x * NOALLOC_CHUNK;
    const size_t n1 = min(N, n0 + (size_t)NOALLOC_CHUNK);
    for (size_t n = n0 + threadIdx.x; n < n1; n += blockDim.x) {
        if (!mask[n]) continue;
        for (int k = 0; k < ncomp; ++k) {
            const S *f = k ? f1 : f0;
            const double rr = k ? rr1 : rr0;
            double m = 0.0, jx = 0.0, jy = 0.0;
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const double d = to_f64(f[i * N + n]);
                if (!isfinite(d)) acc[6] += 1.0;
                m += d + (shifted ? w_eq(i) * rr : 0.0);
                jx += d * double(cx(i));
                jy += d * double(cy(i));
            }
            acc[3 * k + 0] += m;
            acc[3 * k + 1] += jx;
            acc[3 * k + 2] += jy;
        }
    }
    __shared__ double s[NOALLOC_VALUES][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < NOALLOC_VALUES; ++v) {
        double x = acc[v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) s[v][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x < NOALLOC_VALUES) {
        double x = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += s[threadIdx.x][w];
        partials[(size_t)blockIdx.x * NOALLOC_STRIDE + threadIdx.x] = x;
    }
}

// one block folds the partial sums of the chunks in a fixed order
__global__ void __launch_bounds__(256) k_noalloc_final(int nparts, double *__restrict__ scratch)
{
    __shared__ double s[NOALLOC_VALUES][256];
    for (int v = 0; v < NOALLOC_VALUES; ++v) {
        double x = 0.0;
        for (int b = threadIdx.x; b < nparts; b += blockDim.x) x += scratch[(size_t)b * NOALLOC_STRIDE + v];
        s[v][threadIdx.x] = x;
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int v = 0; v < NOALLOC_VALUES; ++v) s[v][threadIdx.x] += s[v][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < NOALLOC_VALUES)
        scratch[(size_t)NOALLOC_MAX_PARTIALS * NOALLOC_STRIDE + threadIdx.x] = s[threadIdx.x][0];
}

// device address of the scratch array, looked up once per device (host code
// may not use the symbol itself: it names the host-side shadow, not device memory)
std::mutex g_scratch_mu;
double *g_scratch_ptr[64] = {nullptr};

int scratch_for_current_device(double **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64) return set_error(SCLBM_E_NO_DEVICE, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(scratch)");
        // with lazy module loading each kernel would otherwise be loaded at its
        // own first launch, i.e. possibly inside the caller's no-allocation region
        cudaFuncAttributes fa;
        const void *kernels[] = {(const void *)k_noalloc_partials<double>,
                                 (const void *)k_noalloc_partials<float>,
                                 (const void *)k_noalloc_partials<__half>,
                                 (const void *)k_noalloc_final};
        for (const void *k : kernels) {
            e = cudaFuncGetAttributes(&fa, k);
            if (e != cudaSuccess) return cuda_fail(e, "cudaFuncGetAttributes(allocation-free monitor)");
        }
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_ptr[dev];
    return SCLBM_OK;
}

} // namespace
} // namespace sclbm

using namespace sclbm;

extern "C" int sclbm_mass_momentum_noalloc(const void *f0, const void *f1, const uint8_t *mask,
                                           size_t nx, size_t ny, int ncomp, int precision,
                                           const double *rho_ref, void *cuda_stream,
                                           double out[7])
{
    static_assert((long long)NOALLOC_MAX_PARTIALS * NOALLOC_CHUNK == (1LL << 27),
                  "lattice limit of the scratch array");
    if (!f0 || !mask || !out || (ncomp == 2 && !f1))
        return set_error(SCLBM_E_INVALID_ARGUMENT, "null argument");
    if (ncomp != 1 && ncomp != 2) return set_error(SCLBM_E_INVALID_ARGUMENT, "ncomp must be 1 or 2");
    if (precision < SCLBM_FP64 || precision > SCLBM_FP16_SHIFTED)
        return set_error(SCLBM_E_INVALID_ARGUMENT, "unknown precision");
    if (nx == 0 || ny == 0) return set_error(SCLBM_E_INVALID_ARGUMENT, "empty lattice");
    // compare before multiplying: nx * ny may wrap around
    if (ny > (size_t(1) << 27) / nx)
        return set_error(SCLBM_E_INVALID_ARGUMENT,
                         "lattice too large for the allocation-free monitor: at most 2^27 nodes "
                         "(its fixed scratch holds 2048 partial sums of 65536 nodes)");
    const size_t N = nx * ny;
    const long long nparts = ((long long)N + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK;
    if (nparts > NOALLOC_MAX_PARTIALS)
        return set_error(SCLBM_E_INVALID_ARGUMENT,
                         "lattice too large for the allocation-free monitor: at most 2^27 nodes "
                         "(its fixed scratch holds 2048 partial sums of 65536 nodes)");
    cudaStream_t s = (cudaStream_t)cuda_stream;
    // the result is read back with a stream synchronisation, which would
    // invalidate a capture in progress: refuse before enqueueing anything
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t ce = cudaStreamIsCapturing(s, &cap);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamIsCapturing");
    if (cap != cudaStreamCaptureStatusNone)
        return set_error(SCLBM_E_INVALID_ARGUMENT,
                         "the allocation-free monitor synchronises its stream and cannot run "
                         "while the stream is being captured");
    double *scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    const int shifted = precision != SCLBM_FP64;
    const double r0 = shifted && rho_ref ? rho_ref[0] : 0.0;
    const double r1 = shifted && rho_ref && ncomp > 1 ? rho_ref[1] : 0.0;
    const void *g1 = ncomp > 1 ? f1 : f0;
    const int g = (int)nparts;
    switch (precision) {
    case SCLBM_FP64:
        k_noalloc_partials<double><<<g, 256, 0, s>>>(N, ncomp, mask, (const double *)f0, (const double *)g1, r0, r1, 0, scratch);
        break;
    case SCLBM_FP32_SHIFTED:
        k_noalloc_partials<float><<<g, 256, 0, s>>>(N, ncomp, mask, (const float *)f0, (const float *)g1, r0, r1, 1, scratch);
        break;
    default:
        k_noalloc_partials<__half><<<g, 256, 0, s>>>(N, ncomp, mask, (const __half *)f0, (const __half *)g1, r0, r1, 1, scratch);
        break;
    }
    SCLBM_LAUNCHED("allocation-free monitor");
    k_noalloc_final<<<1, 256, 0, s>>>(g, scratch);
    SCLBM_LAUNCHED("allocation-free monitor (final)");
    SCLBM_CUDA(cudaMemcpyAsync(out, scratch + (size_t)NOALLOC_MAX_PARTIALS * NOALLOC_STRIDE,
                               NOALLOC_VALUES * sizeof(double), cudaMemcpyDeviceToHost, s));
    SCLBM_CUDA(cudaStreamSynchronize(s));
    if (out[6] != 0.0) return set_error(SCLBM_E_NONFINITE, "non-finite populations in the lattice");
    return SCLBM_OK;
}
