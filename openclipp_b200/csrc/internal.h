// Internal interfaces between the C ABI layer (capi.cpp) and the CUDA
// launchers. Nothing here is exported from the shared library.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace ocipb {

// Pixel element types, same order as SImage::EDataType.
enum PixType : int { U8 = 0, S8, U16, S16, U32, S32, F32, F64, NbTypes };

// ImageProximity measures (reference cl-files/ImageProximity.cl:44-466).
enum Measure : int {
  kSqrDistance = 0,
  kSqrDistanceNorm = 1,
  kAbsDistance = 2,
  kCrossCorr = 3,
  kCrossCorrNorm = 4,
};

// Kernel launches issued by this library (reported by ocipGetLaunchCount).
extern unsigned long long g_launches;
inline void count_launches(int n) { g_launches += (unsigned long long)n; }

inline int type_bytes(int t) {
  static const int b[8] = {1, 1, 2, 2, 4, 4, 4, 8};
  return (t >= 0 && t < 8) ? b[t] : 0;
}
inline bool type_is_float(int t) { return t == F32 || t == F64; }
inline bool type_is_unsigned(int t) { return t == U8 || t == U16 || t == U32; }

// Device view of an image: `nch` interleaved channels of `type` per pixel,
// rows `pitch` bytes apart.
struct DevImage {
  void* ptr = nullptr;
  size_t pitch = 0;
  int width = 0;
  int height = 0;
  int nch = 1;
  int type = U8;
};

// Plain (CUDA-core) sliding-window kernels: every measure, type and channel
// count. Accumulation per output follows the reference's order (template
// row outer, column inner) with one fused multiply-add per product term.
// tt_scratch: 64 bytes of device memory for the per-channel template energy.
cudaError_t launch_proximity_plain(Measure m, const DevImage& src,
                                   const DevImage& tmpl, const DevImage& dst,
                                   void* tt_scratch, cudaStream_t stream);

// AbsDistance of a U8 or S8 source with packed-byte SAD (four taps per
// instruction, exact uint32 sums); launch_proximity_plain routes 8-bit
// AbsDistance here when proximity_sad_8bit_supported() holds.
size_t proximity_sad_8bit_smem(int tw, int th);
bool proximity_sad_8bit_supported(const DevImage& src, const DevImage& tmpl);
cudaError_t launch_proximity_sad_8bit(const DevImage& src, const DevImage& tmpl,
                                    const DevImage& dst, cudaStream_t stream);

// Scratch for the integral scan: per-row tile sums and per-band column
// prefixes (the counterpart of the reference's junction buffers,
// C++/programs/Integral.cpp:42-95).
struct IntegralScratch {
  void* buf = nullptr;
  size_t bytes = 0;
};
size_t integral_scratch_bytes(int width, int height, int nch);

// Inclusive integral of S (sqr = false) or S^2 (sqr = true) per channel into
// an F32 or F64 destination, accumulated exactly (int64 for integer sources,
// FP64 for float sources and for the squares of 32-bit integers).
cudaError_t launch_integral(bool sqr, const DevImage& src, const DevImage& dst,
                            void* scratch, size_t scratch_bytes,
                            cudaStream_t stream);

}  // namespace ocipb
