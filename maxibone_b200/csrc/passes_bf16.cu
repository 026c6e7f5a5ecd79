// Instantiation of the unrolled passes for the bf16 field storage type.
#include "unrolled_impl.cuh"

namespace maxi {

template cudaError_t dispatch_unrolled<__nv_bfloat16>(const Volume &, const void *, int, const float *, int, int64_t,
                                           __nv_bfloat16 *, __nv_bfloat16 *, uint16_t *, float *, int32_t,
                                           cudaStream_t, const RunOpts &);

template cudaError_t launch_init_field<__nv_bfloat16>(const void *, int, __nv_bfloat16 *, int64_t, cudaStream_t);

}  // namespace maxi
