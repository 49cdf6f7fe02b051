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

// Same with a general window anchor: output (x, y) reads
// S(x + w - ax, y + h - ay) (the one-pair calls use ax = tw/2, ay = th/2).
// 0 <= ax < tw, 0 <= ay < th.
cudaError_t launch_proximity_tensor_anchored(Context& ctx, Measure m, const DevImage& src,
                                             const DevImage& tmpl, const DevImage& dst, int ax,
                                             int ay);

// Product sums C(x, y) = sum_{w, h} S(x + w - ax, y + h - ay) T(w, h) of one
// template of at most 64 x 64 (a tile of a larger one) on the tensor cores,
// written into (accumulate = false) or added to (true) the F64 map c_map of
// the source's size and channels. Any anchor, including ones outside the
// template (a tile's offset within the whole template).
cudaError_t launch_tensor_product_sums(Context& ctx, const DevImage& src, const DevImage& tmpl,
                                       const DevImage& c_map, int ax, int ay, bool accumulate);

// A measure of a template larger than 64 x 64 (up to 1024 columns): the
// template is cut into tiles of at most 64 x 64 whose product sums accumulate
// in an F64 map, and a scoring pass adds the window energies (row energies
// plus running column sums) and the template energy.
cudaError_t launch_proximity_tensor_large(Context& ctx, Measure m, const DevImage& src,
                                          const DevImage& tmpl, const DevImage& dst);

// Best match of a one-channel F32 score map on the tensor path, fused into the
// scoring epilogue (ocipProximityIndx): the index reduction idx_op (0 min,
// 1 max, 2 min |v|, 3 max |v|) of the F32 scores, with the reference's tie
// order. dst may have a null pointer (no map written). records is device
// scratch of tensor_index_records_bytes() bytes. Synchronises the stream;
// *has_nan reports a NaN score (the caller then reduces a written map, whose
// answer depends on where the NaNs lie).
size_t tensor_index_records_bytes(const Context& ctx, const DevImage& src, const DevImage& tmpl);
cudaError_t launch_proximity_tensor_indexed(Context& ctx, Measure m, const DevImage& src,
                                            const DevImage& tmpl, const DevImage& dst, int idx_op,
                                            void* records, int* nrec, float* best, int* bx,
                                            int* by, bool* has_nan);

// Gradients of L = sum G1 * SqrDistance(S, T) + sum G2 * CrossCorr_Norm(S, T)
// (F32 sources, one channel, templates up to 64 x 64) into dS (S's size) and
// dT (T's size), F32 or F64; G1 or G2 may be null, N2 is CrossCorr_Norm(S, T)
// (needed with G2), dS or dT may be null.
cudaError_t proximity_backward(Context& ctx, const DevImage& S, const DevImage& T,
                               const DevImage* G1, const DevImage* G2, const DevImage* N2,
                               const DevImage* dS, const DevImage* dT);

// Launches a kernel whose one thread waits on an mbarrier that nothing arrives
// on, bounded to `limit_cycles` SM clock cycles (the failure path of every
// wait in the tensor kernels, exercised without a fault).
cudaError_t launch_bounded_wait_probe(Context& ctx, long long limit_cycles);

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
