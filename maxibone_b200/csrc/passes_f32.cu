// Instantiation of the unrolled passes for the f32 field storage type.
#include "unrolled_impl.cuh"

namespace maxi {

int radius_bucket(int r) { return radius_bucket_impl(r); }

template cudaError_t dispatch_unrolled<float>(const Volume &, const void *, int, const float *, int, int64_t,
                                           float *, float *, uint16_t *, float *, int32_t,
                                           cudaStream_t, const RunOpts &);

template cudaError_t launch_init_field<float>(const void *, int, float *, int64_t, cudaStream_t);

}  // namespace maxi
