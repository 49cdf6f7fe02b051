// Row-energy maps for the tensor-core ImageProximity path.
#pragma once

#include <cuda_runtime.h>

#include "internal.h"

namespace ocipb {

// Row pitch (bytes) of a row-energy plane of the given width (4-byte entries).
size_t row_energy_pitch(int width);

// R(x, r, c) = sum_{w < tw} S(x + w - ax, r, c)^2 (zero outside the image) for
// every output column x and source row r, written to dst + c * dst_plane +
// r * dst_pitch (bytes): int32 for U8 sources (exact), FP32 for U16 and F32
// sources (FP64 sums rounded once). tw <= 1024.
cudaError_t launch_row_energy(const DevImage& src, int tw, int ax, void* dst, size_t dst_pitch,
                              size_t dst_plane, cudaStream_t stream);

}  // namespace ocipb
