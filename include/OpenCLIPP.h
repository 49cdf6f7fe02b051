/* OpenCLIPP C interface: the template-matching subset, served on NVIDIA B200.
 *
 * Drop-in replacement for the reference's include/OpenCLIPP.h for the calls
 * that template matching needs: context and image management, the five
 * ImageProximity measures, the Integral scans and the FFT-named proximity
 * entry points. Every function keeps the reference's name, argument order,
 * argument meaning and error convention (0 on success, a negative OpenCL-style
 * code otherwise). Each declaration cites the reference line it replaces.
 *
 * OpenCL types are not needed: ocipError is a 32-bit signed integer carrying
 * the same numeric codes as cl_int, cl_device_type and cl_mem_flags are 64-bit
 * bitfields with the Khronos values. A caller that also includes the Khronos
 * headers gets compatible definitions (the ones below are skipped).
 *
 * Calls are asynchronous on the context's CUDA stream, like the reference's
 * in-order OpenCL queue: processing functions return once the work is
 * enqueued; ocipReadImage() and ocipFinish() wait for it.
 * The library keeps a process-wide current context and is not thread-safe,
 * as the reference (OpenCLIPP/OpenCLIPP.cpp:73-75).
 */
#ifndef OPENCLIPP_B200_OPENCLIPP_H
#define OPENCLIPP_B200_OPENCLIPP_H

#include <stdint.h>

#include "SImage.h"

#if defined(_WIN32)
#define ocip_API __declspec(dllexport)
#else
#define ocip_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

#ifndef __OPENCL_CL_H
typedef int32_t cl_int;
typedef uint64_t cl_bitfield;
typedef cl_bitfield cl_device_type;
typedef cl_bitfield cl_mem_flags;
#define CL_SUCCESS 0
#define CL_DEVICE_NOT_FOUND -1
#define CL_DEVICE_NOT_AVAILABLE -2
#define CL_MEM_OBJECT_ALLOCATION_FAILURE -4
#define CL_OUT_OF_RESOURCES -5
#define CL_OUT_OF_HOST_MEMORY -6
#define CL_IMAGE_FORMAT_MISMATCH -9
#define CL_IMAGE_FORMAT_NOT_SUPPORTED -10
#define CL_INVALID_VALUE -30
#define CL_INVALID_DEVICE_TYPE -31
#define CL_INVALID_DEVICE -33
#define CL_INVALID_CONTEXT -34
#define CL_INVALID_MEM_OBJECT -38
#define CL_INVALID_IMAGE_SIZE -40
#define CL_INVALID_PROGRAM -44
#define CL_INVALID_OPERATION -59
#define CL_INVALID_BUFFER_SIZE -61
#define CL_DEVICE_TYPE_DEFAULT (1 << 0)
#define CL_DEVICE_TYPE_CPU (1 << 1)
#define CL_DEVICE_TYPE_GPU (1 << 2)
#define CL_DEVICE_TYPE_ACCELERATOR (1 << 3)
#define CL_DEVICE_TYPE_ALL 0xFFFFFFFF
#define CL_MEM_READ_WRITE (1 << 0)
#define CL_MEM_WRITE_ONLY (1 << 1)
#define CL_MEM_READ_ONLY (1 << 2)
#endif

typedef char ocipBool; /* reference include/OpenCLIPP.h:48 */
#ifndef OPENCLIPP_B200_NO_UINT
typedef unsigned int uint; /* reference include/OpenCLIPP.h:49 */
#endif
typedef struct SImage SImage;

/* 0 on success, negative cl_int-compatible code otherwise
 * (reference include/OpenCLIPP.h:58-62). */
typedef cl_int ocipError;

/* Opaque handles (reference include/OpenCLIPP.h:64-66). */
typedef struct _cl_context* ocipContext;
typedef struct _cl_image* ocipImage;
typedef struct _cl_program* ocipProgram;

/* ---- Context ---------------------------------------------------------- */

/* Creates a context on a CUDA device and makes it current
 * (reference include/OpenCLIPP.h:99). PreferredPlatform may name a device
 * index ("0", "1", ...); NULL or any other string selects the calling
 * thread's current CUDA device.
 * deviceType must include CL_DEVICE_TYPE_GPU (DEFAULT and ALL do);
 * CL_DEVICE_TYPE_CPU alone gives CL_DEVICE_NOT_FOUND. */
ocipError ocip_API ocipInitialize(ocipContext* ContextPtr,
                                  const char* PreferredPlatform,
                                  cl_device_type deviceType);

/* Releases a context (reference include/OpenCLIPP.h:104). */
ocipError ocip_API ocipUninitialize(ocipContext Context);

/* Selects the context used by the next calls (reference :112). */
ocipError ocip_API ocipChangeContext(ocipContext Context);

/* Accepted and ignored: kernels are compiled into the library
 * (reference :118). */
void ocip_API ocipSetCLFilesPath(const char* Path);

/* Name of an error code, e.g. "CL_INVALID_VALUE" (reference :124). */
ocip_API const char* ocipGetErrorName(ocipError Error);

/* Name of the current context's device (reference :130). */
ocipError ocip_API ocipGetDeviceName(char* Name, uint BufferLength);

/* Waits for every operation queued on the current context (reference :135). */
ocipError ocip_API ocipFinish(void);

/* ---- Images ----------------------------------------------------------- */

/* Allocates device memory for an image described by Image; ImageData, when
 * not NULL, is the host buffer used by ocipSendImage/ocipReadImage and by the
 * automatic upload of a source image on its first use (reference :159).
 * 3-channel images keep 3 interleaved channels on the device; the reference
 * widens them to 4 (ColorImage, C++/Image.cpp:243-275) and drops the 4th on
 * read, which gives the same 3 channels of results. */
ocipError ocip_API ocipCreateImage(ocipImage* ImagePtr, SImage Image,
                                   void* ImageData, cl_mem_flags flags);

/* Queues a host-to-device copy of the image's host buffer (reference :170). */
ocipError ocip_API ocipSendImage(ocipImage Image);

/* Copies the device image into its host buffer and waits (reference :177). */
ocipError ocip_API ocipReadImage(ocipImage Image);

/* Releases an image (reference :182). */
ocipError ocip_API ocipReleaseImage(ocipImage Image);

/* Releases a program handle (reference :231). */
ocipError ocip_API ocipReleaseProgram(ocipProgram Program);

/* ---- Integral (reference include/OpenCLIPP.h:638-645) ------------------ */

/* Creates a program holding the scratch buffers sized for Image; Image may
 * be NULL (buffers are then sized on first use). */
ocipError ocip_API ocipPrepareIntegral(ocipProgram* ProgramPtr, ocipImage Image);

/* Inclusive integral: Dest(x, y) = sum of Source over [0..x] x [0..y].
 * Dest must be F32 or F64, same size and channel count as Source. */
ocipError ocip_API ocipIntegral(ocipProgram Program, ocipImage Source,
                                ocipImage Dest);

/* Same as ocipIntegral for the squares of the Source values. */
ocipError ocip_API ocipSqrIntegral(ocipProgram Program, ocipImage Source,
                                   ocipImage Dest);

/* ---- Statistics: arg-min / arg-max of a map (reference
 * include/OpenCLIPP.h:544-563; only the index reductions, the consumers of a
 * score map, are provided) ------------------------------------------------ */
/* Program for the statistics calls; Image may be NULL. */
ocipError ocip_API ocipPrepareStatistics(ocipProgram* ProgramPtr, ocipImage Image);

/* Minimum (maximum; of the absolute values for the Abs forms) of a one-channel
 * image and the coordinate of a pixel that holds it. Synchronous. Value,
 * position and tie-breaking are the reference's: the minimum as a float, the
 * first such pixel in the reference's reduction order. More than one channel
 * gives CL_INVALID_VALUE. */
ocipError ocip_API ocipMinIndx(ocipProgram Program, ocipImage Source, double* Result,
                               int* IndexX, int* IndexY);
ocipError ocip_API ocipMaxIndx(ocipProgram Program, ocipImage Source, double* Result,
                               int* IndexX, int* IndexY);
ocipError ocip_API ocipMinAbsIndx(ocipProgram Program, ocipImage Source, double* Result,
                                  int* IndexX, int* IndexY);
ocipError ocip_API ocipMaxAbsIndx(ocipProgram Program, ocipImage Source, double* Result,
                                  int* IndexX, int* IndexY);

/* ---- Image proximity (reference include/OpenCLIPP.h:649-669) ----------- */
/* Dest has the size and channel count of Source and a float type (F32; F64
 * sources compute in double). The window of Dest(x, y) covers Source
 * [x - tw/2, x - tw/2 + tw) x [y - th/2, y - th/2 + th) and pixels outside
 * Source read as 0. Template must not be larger than Source and must have
 * the type and channel count of Source. */

ocipError ocip_API ocipPrepareProximity(ocipImage Image);

/* sum (S - T)^2 / sqrt(sum S^2 * sum T^2) */
ocipError ocip_API ocipSqrDistance_Norm(ocipImage Source, ocipImage Template,
                                        ocipImage Dest);
/* sum (S - T)^2 */
ocipError ocip_API ocipSqrDistance(ocipImage Source, ocipImage Template,
                                   ocipImage Dest);
/* sum |S - T| */
ocipError ocip_API ocipAbsDistance(ocipImage Source, ocipImage Template,
                                   ocipImage Dest);
/* sum S * T */
ocipError ocip_API ocipCrossCorr(ocipImage Source, ocipImage Template,
                                 ocipImage Dest);
/* sum S * T / sqrt(sum S^2 * sum T^2) */
ocipError ocip_API ocipCrossCorr_Norm(ocipImage Source, ocipImage Template,
                                      ocipImage Dest);

/* ---- Proximity entry points named after the FFT path ------------------- */
/* (reference include/OpenCLIPP.h:673-688). The reference computes these with
 * clFFT on F32, 1-channel images, for large templates. Here they compute the
 * same measures on the tensor-core path (no FFT), templates beyond 64 x 64 as
 * tiles whose product sums add up in FP64; ocipIsFFTAvailable() returns 1. */
ocipBool ocip_API ocipIsFFTAvailable(void);
ocipError ocip_API ocipPrepareImageProximityFFT(ocipProgram* ProgramPtr,
                                                ocipImage Image,
                                                ocipImage Template);
ocipError ocip_API ocipSqrDistanceFFT(ocipProgram Program, ocipImage Source,
                                      ocipImage Template, ocipImage Dest);
ocipError ocip_API ocipSqrDistanceFFT_Norm(ocipProgram Program,
                                           ocipImage Source,
                                           ocipImage Template, ocipImage Dest);
ocipError ocip_API ocipCrossCorrFFT(ocipProgram Program, ocipImage Source,
                                    ocipImage Template, ocipImage Dest);
ocipError ocip_API ocipCrossCorrFFT_Norm(ocipProgram Program, ocipImage Source,
                                         ocipImage Template, ocipImage Dest);

#ifdef __cplusplus
}
#endif
#endif
