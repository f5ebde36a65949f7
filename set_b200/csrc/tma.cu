// tma.cu -- tensor maps for the plane copies of the stage kernels.
//
// The stage kernels stage every plane of their column tile (cells + 2-cell halo, all 8 conserved
// variables) into shared memory with one 4-D tensor copy (cp.async.bulk.tensor) completed on an
// mbarrier.  The map is encoded on the host through the driver entry point
// cuTensorMapEncodeTiled, fetched with cudaGetDriverEntryPointByVersion so the library needs no
// link-time dependency on libcuda.
#include <cudaTypedefs.h>
#include "setb200.h"
#include "setb_internal.cuh"

namespace sb {

namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    }
    return fn;
}
}  // namespace

int encode_state_tmap(const GridGeom& g, const double* base, int ty, CUtensorMap* out) {
    // Tensor copies need 16-byte aligned bases and strides, and a 16-byte multiple inner box.
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (g.px & 1) || (g.ps & 1) || (g.vs & 1)) return SETB_EINVAL;
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn) return SETB_ECUDA;
    const cuuint64_t dims[4] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz, 8};
    const cuuint64_t strides[3] = {(cuuint64_t)g.px * 8, (cuuint64_t)g.ps * 8, (cuuint64_t)g.vs * 8};
    const cuuint32_t box[4] = {(cuuint32_t)(kTileX + 4), (cuuint32_t)(ty + 4), 1, 8};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? SETB_OK : SETB_ECUDA;
}

}  // namespace sb
