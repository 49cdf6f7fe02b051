// Tensor-core (tcgen05) ImageProximity path.
#pragma once

#include "host.h"
#include "internal.h"

namespace ocipb {

// Whether the tensor kernels cover this call. `forced` is true when the
// caller asked for the tensor path explicitly (OCIP_PATH_TENSOR); AUTO only
// takes it where results are exact.
bool tensor_supports(Measure m, const DevImage& src, const DevImage& tmpl,
                     const DevImage& dst, bool forced);

cudaError_t launch_proximity_tensor(Context& ctx, Measure m, const DevImage& src,
                                    const DevImage& tmpl, const DevImage& dst);

}  // namespace ocipb
