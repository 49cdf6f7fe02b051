// Index reductions (ocipMinIndx family) on the device.
#pragma once

#include "host.h"
#include "internal.h"

namespace ocipb {

enum IndexOp { kIdxMin = 0, kIdxMax = 1, kIdxMinAbs = 2, kIdxMaxAbs = 3 };

// Device scratch for the per-group results of a W x H image.
size_t index_reduce_scratch_bytes(int W, int H);

// Minimum / maximum (of the value or of its absolute value) of a one-channel
// image and the (x, y) of the pixel that holds it, with the reference's
// comparison order. Synchronous (reads the group results back).
cudaError_t index_reduce(Context& ctx, int op, const DevImage& s, void* scratch, double* value,
                         int* x, int* y);

}  // namespace ocipb
