/* Extensions of the OpenCLIPP C interface specific to this implementation.
 *
 * Kept out of OpenCLIPP.h so that the drop-in header stays the reference's
 * interface. Nothing here has a counterpart in the reference unless stated.
 */
#ifndef OPENCLIPP_B200_EXT_H
#define OPENCLIPP_B200_EXT_H

#include "OpenCLIPP.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Which kernels serve the ImageProximity calls of the current context.
 *   OCIP_PATH_PLAIN : CUDA-core sliding window, the reference's arithmetic
 *                     (the drop-in default).
 *   OCIP_PATH_TENSOR: tcgen05 tensor cores for the product term of
 *                     SqrDistance[_Norm] and CrossCorr[_Norm] (i8 MMA with exact
 *                     s32 sums for 8-bit sources, split BF16 for F32) with
 *                     FP64/int64 window statistics; AbsDistance and shapes
 *                     the tensor kernels do not cover fall back to PLAIN.
 *   OCIP_PATH_AUTO  : TENSOR where it is exact (8-bit sources), PLAIN
 *                     otherwise. */
enum ocipProximityPath {
  OCIP_PATH_AUTO = 0,
  OCIP_PATH_PLAIN = 1,
  OCIP_PATH_TENSOR = 2,
};
ocipError ocip_API ocipSetProximityPath(int Path);
ocipError ocip_API ocipGetProximityPath(int* Path);

/* Path that served the last ImageProximity call of the current context
 * (an ocipProximityPath value other than AUTO). */
ocipError ocip_API ocipGetLastProximityPath(int* Path);

/* Human-readable detail of the last error returned on this thread. */
ocip_API const char* ocipGetLastErrorMessage(void);

/* The current context's CUDA stream (a cudaStream_t), for callers that time
 * or order work with CUDA events. */
ocipError ocip_API ocipGetStream(void** Stream);

/* Number of CUDA kernels this library has launched in this process. */
ocipError ocip_API ocipGetLaunchCount(uint64_t* Count);

/* Device address and row pitch (bytes) of an image's device buffer. */
ocipError ocip_API ocipGetImageDevicePtr(ocipImage Image, void** DevicePtr,
                                         size_t* Pitch);

#ifdef __cplusplus
}
#endif
#endif
