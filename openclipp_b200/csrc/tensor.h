// Tensor-core (tcgen05) ImageProximity path.
#pragma once

#include <vector>

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

// A prepared batch: every (image i, template j) pair into dsts[i * ntpl + j],
// one persistent launch over a work queue of (pair, channel, strip, band)
// items, captured in a CUDA graph. All images share one type; every pair must
// pass tensor_supports with forced = true.
struct TensorBatch;
TensorBatch* tensor_batch_create(Context& ctx, Measure m, const std::vector<DevImage>& imgs,
                                 const std::vector<DevImage>& tpls,
                                 const std::vector<DevImage>& dsts, cudaError_t* err);
cudaError_t tensor_batch_run(TensorBatch* b);
int tensor_batch_items(const TensorBatch* b);
// Band height the batch uses for templates of this size (0 if none).
int tensor_batch_band_height(const TensorBatch* b, int tw, int th);
void tensor_batch_destroy(TensorBatch* b);

}  // namespace ocipb
