// tensor_map.cpp -- host encoding of TMA tensor maps (CUtensorMap) for the
// ring kernel.  cuTensorMapEncodeTiled is a driver API function; it is looked
// up once through the runtime's driver entry point, so the library needs no
// link against libcuda.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <mutex>

namespace sclbm {

int encode_tensor_map(CUtensorMap *m, CUtensorMapDataType dt, unsigned rank, void *base,
                      const cuuint64_t *dim, const cuuint64_t *stride_bytes, const cuuint32_t *box,
                      const cuuint32_t *elem_strides)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    if (!encode) return 1;
    const CUresult r = encode(m, dt, rank, base, dim, stride_bytes, box, elem_strides,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : 1;
}

} // namespace sclbm
