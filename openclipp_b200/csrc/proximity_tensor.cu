// Tensor-core (tcgen05) ImageProximity path for sm_100a.
#include "tensor.h"

namespace ocipb {

bool tensor_supports(Measure, const DevImage&, const DevImage&, const DevImage&, bool) {
  return false;
}

cudaError_t launch_proximity_tensor(Context&, Measure, const DevImage&, const DevImage&,
                                    const DevImage&) {
  return cudaErrorNotSupported;
}

}  // namespace ocipb
