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
 *                     s32 sums for U8 sources, split BF16 for F32 and U16;
 *                     1-4 channels; templates up to 1024 columns: beyond
 *                     64 x 64 they run as tiles of at most 64 x 64 whose
 *                     product sums add up in FP64) with FP64/exact window
 *                     statistics; AbsDistance and shapes the tensor kernels
 *                     do not cover fall back to PLAIN.
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

/* Output rows per work item of the one-pair tensor-path launches of the
 * current context (each item also reads the template's height less one rows
 * above its band). 0, the default, picks the height per launch from the SM
 * count and the number of column strips; a positive value (clamped to the
 * image height) fixes it, for tuning and for tests. */
ocipError ocip_API ocipSetProximityBandHeight(int Rows);

/* Human-readable detail of the last error returned on this thread. */
ocip_API const char* ocipGetLastErrorMessage(void);

/* The current context's CUDA stream (a cudaStream_t), for callers that time
 * or order work with CUDA events. */
ocipError ocip_API ocipGetStream(void** Stream);

/* Number of CUDA kernels this library has launched in this process. */
ocipError ocip_API ocipGetLaunchCount(uint64_t* Count);

/* Integral (Square = 0) or SqrIntegral (Square != 0) that allocates no device
 * memory. It has no counterpart in the reference.
 * It is for callers that cannot let a library call cudaMalloc: their device
 * memory belongs to another allocator, or they must not allocate while running
 * because allocation can block and synchronise the device. The caller passes
 * device pointers and row pitches (bytes) for Source and Dest, their SImage
 * descriptions (Step is ignored; the pitches are used) and a cudaStream_t
 * (NULL for the default stream); the work is queued on that stream on the
 * calling thread's current CUDA device, and no context is needed.
 * The scan's scratch is a fixed 16 MiB array that every device which loads
 * the library holds until the process exits; images whose scratch would not
 * fit (about 7300 x 7300 pixels per channel) are refused with
 * CL_INVALID_IMAGE_SIZE. The first call in a CUDA context (on each device,
 * and again after the device is reset) looks up that array's device address
 * and may load the module; make that first call before capturing the stream
 * into a CUDA graph. All calls share the array: calls that overlap on the GPU
 * (on different streams, or on the same device from several threads) race,
 * so the caller must serialise them. */
ocipError ocip_API ocipIntegralNoAlloc(int Square, SImage SourceDesc, const void* Source,
                                       size_t SourcePitch, SImage DestDesc, void* Dest,
                                       size_t DestPitch, void* Stream);

/* Measures, for the batched calls below. */
enum ocipMeasure {
  OCIP_MEASURE_SQR_DISTANCE = 0,
  OCIP_MEASURE_SQR_DISTANCE_NORM = 1,
  OCIP_MEASURE_ABS_DISTANCE = 2,
  OCIP_MEASURE_CROSS_CORR = 3,
  OCIP_MEASURE_CROSS_CORR_NORM = 4,
};

/* Batched template matching. No reference counterpart: the reference matches
 * one (image, template) pair per call.
 * Prepares one persistent launch that computes Measure for every pair:
 *   Dests[i * NbTemplates + j] = Measure(Images[i], Templates[j])
 * with the same definition, zero padding and Dest types as the one-pair calls.
 * All images and templates share one type (U8, U16 or F32) and channel count
 * (1-4); templates are at most 64 x 64 and no larger than any image; each
 * Dest is F32 or F64 with its image's size and channels. AbsDistance has no
 * tensor-core form and is refused (CL_INVALID_VALUE). The work is a queue of
 * (pair, channel, column strip, band of rows) items, largest first,
 * taken by one persistent CTA per SM on the tensor path (U8 exact; F32 and
 * U16 within 1e-5 relative). Band heights are chosen per (template size
 * class, type, channels) by timing candidates on the device the first time a
 * class is seen in the process. The queue reset and the launch are captured
 * in a CUDA graph that ocipRunProximityBatch replays on the context's stream.
 * Images and templates with host data are uploaded here; the batch reads
 * their device buffers when it runs, so later changes must be sent with
 * ocipSendImage. Dests are marked as written. Release with ocipReleaseProgram;
 * the images must outlive the program. */
ocipError ocip_API ocipPrepareProximityBatch(ocipProgram* Program, int Measure,
                                             const ocipImage* Images, int NbImages,
                                             const ocipImage* Templates, int NbTemplates,
                                             const ocipImage* Dests);
ocipError ocip_API ocipRunProximityBatch(ocipProgram Program);
/* Work items of a prepared batch, and the band height (rows per item) it
 * uses for templates of the given size (0 if the batch has none). */
ocipError ocip_API ocipGetProximityBatchInfo(ocipProgram Program, int TemplateWidth,
                                             int TemplateHeight, int* NbItems,
                                             int* BandHeight);

/* Best match of a template in one call (no reference counterpart).
 * Computes the Measure (an ocipMeasure value) map of (Source, Template) and
 * its index reduction IndexOp (0: ocipMinIndx, 1: ocipMaxIndx,
 * 2: ocipMinAbsIndx, 3: ocipMaxAbsIndx), with the same answer as those calls
 * on the map, ties included: the smallest (or largest) value and its (X, Y).
 * One channel; Dest, when given, is F32 of the source's size and receives the
 * map; it may be NULL. On the tensor path (templates up to 64 x 64) the
 * reduction runs in the scoring kernel's epilogue, so without Dest no map is
 * written at all. A map that holds a NaN (a _Norm measure over a zero-energy
 * window) is reduced from the written map instead, because the reference's
 * answer then depends on where the NaNs lie; the plain path and other shapes
 * also compute the map (into Dest, or scratch) and reduce it. Synchronous. */
ocipError ocip_API ocipProximityIndx(int Measure, int IndexOp, ocipImage Source,
                                     ocipImage Template, ocipImage Dest, double* Value,
                                     int* X, int* Y);

/* Gradients of template matching (no reference counterpart).
 * For L = sum_{x,y} GradSqrDistance(x,y) * SqrDistance(Source, Template)(x,y)
 *       + sum_{x,y} GradCrossCorrNorm(x,y) * CrossCorr_Norm(Source, Template)(x,y)
 * writes dL/dSource into GradSource and dL/dTemplate into GradTemplate, with
 * the forward definitions of ocipSqrDistance and ocipCrossCorr_Norm (window
 * anchored at (tw/2, th/2), zero padding; padded pixels receive no gradient).
 * Source and Template are F32 with one channel, the template at most 64 x 64.
 * GradSqrDistance and GradCrossCorrNorm are F32 maps of the source's size;
 * either may be NULL (but not both). CrossCorrNorm is the forward
 * ocipCrossCorr_Norm map (F32), required with GradCrossCorrNorm; the window
 * energies are recomputed, not stored. GradSource (source size) and
 * GradTemplate (template size) are F32 or F64; either may be NULL. Positions
 * whose window energy is 0 (CrossCorr_Norm undefined) contribute nothing.
 * Both measures are served by one pass: a correlation of an adjoint map with
 * the flipped template and a template-gradient reduction, both on the tensor
 * cores (split BF16), with FP64 window sums. */
ocipError ocip_API ocipProximityBackward(ocipImage Source, ocipImage Template,
                                         ocipImage GradSqrDistance, ocipImage GradCrossCorrNorm,
                                         ocipImage CrossCorrNorm, ocipImage GradSource,
                                         ocipImage GradTemplate);

/* Every wait in the tensor-core kernels is bounded: when one expires (about 2 s
 * of SM clock), the kernel sets an error flag and returns instead of hanging,
 * and the next ocipFinish or ocipReadImage of the context returns
 * CL_OUT_OF_RESOURCES (the results since the previous such call are not
 * valid); the context stays usable.
 * This diagnostic runs that path on purpose: a kernel waits on a barrier that
 * nothing arrives on for LimitCycles SM clock cycles (at most 2^31 - 1). It
 * returns what ocipFinish returns afterwards: CL_OUT_OF_RESOURCES when the
 * bounded wait expired as designed. */
ocipError ocip_API ocipTestBoundedWait(int LimitCycles);

/* Device address and row pitch (bytes) of an image's device buffer. Writes
 * made through this address are not tracked by the library, so from then on
 * ocipReadImage of this image waits for all work queued on the context's
 * stream (otherwise a read waits only for the image's last writer). */
ocipError ocip_API ocipGetImageDevicePtr(ocipImage Image, void** DevicePtr,
                                         size_t* Pitch);

/* Row band of one image that part Part of Parts computes when the
 * ImageProximity calls of an image of Height rows and a template of
 * TemplateHeight rows are split across GPUs (one context per GPU; no
 * counterpart in the reference, whose contexts never share an image).
 * Rows[0] .. Rows[1] (exclusive) are the destination rows the part owns: the
 * image's rows split as evenly as possible, in order. Rows[2] .. Rows[3] are
 * the source rows it needs: its own rows shifted by the template anchor
 * (TemplateHeight / 2) plus a halo of TemplateHeight - 1 rows, clipped to the
 * image and, near its edges, widened to at least TemplateHeight rows (the
 * measures refuse a source shorter than the template). Running a measure on the image made of those source rows gives, at
 * its rows Rows[0] - Rows[2] .. Rows[1] - Rows[2], the same values as the
 * whole image gives at rows Rows[0] .. Rows[1]: the zero padding then falls
 * only outside the whole image. A part may own no rows (Parts > Height); its
 * source band is then empty too. Host arithmetic only: needs no context. */
ocipError ocip_API ocipGetProximityBand(unsigned int Height, unsigned int TemplateHeight,
                                        int Part, int Parts, unsigned int Rows[4]);

#ifdef __cplusplus
}
#endif
#endif
