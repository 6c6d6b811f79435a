// Host-side tensor-map encoding for the TMA loads (driver entry point fetched through the runtime,
// so the library does not link libcuda directly).
#include <cudaTypedefs.h>

#include <mutex>

#include "wfd_tma.cuh"

namespace wfd {

namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_once;

void resolve() {
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
}
}  // namespace

bool make_tensor_map_3d(CUtensorMap *map, const float *base, long nx, long ny, long nz, unsigned box_z,
                        unsigned box_y, unsigned box_x) {
    std::call_once(g_once, resolve);
    if (!g_encode) return false;
    if ((nz * 4) % 16 != 0 || (reinterpret_cast<uintptr_t>(base) % 16) != 0) return false;
    cuuint64_t dims[3] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx};
    cuuint64_t strides[2] = {(cuuint64_t)nz * 4, (cuuint64_t)ny * (cuuint64_t)nz * 4};
    cuuint32_t box[3] = {box_z, box_y, box_x};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box,
                          estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace wfd
