// Instantiation of the unrolled passes for the f16 field storage type.
#include "unrolled_impl.cuh"

namespace maxi {

template cudaError_t dispatch_unrolled<__half>(const Volume &, const void *, int, const float *, int, int64_t,
                                           __half *, __half *, uint16_t *, float *, int32_t,
                                           cudaStream_t, const RunOpts &);

template cudaError_t launch_init_field<__half>(const void *, int, __half *, int64_t, cudaStream_t);

}  // namespace maxi
