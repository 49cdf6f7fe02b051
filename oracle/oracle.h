/* CPU oracle for the template-matching path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the tests,
 * smoke() and the bench's CPU baseline compare against; the shipped library
 * never links or calls it.
 *
 * Two restatements of the reference's arithmetic:
 *   orc_*_refexact : the reference's own arithmetic, operation by operation
 *                    (cl-files/ImageProximity.cl:44-466: REAL accumulators,
 *                    h-outer / w-inner loop, zero padding, same-size output,
 *                    centred anchor). Built with FP contraction off, it is bit
 *                    identical to the reference kernel source run through
 *                    ref_shim.h (checked by tests/test_oracle.py).
 *   orc_*_exact    : the mathematically exact (integer inputs: int64 /
 *                    __int128) or extended-precision (float inputs: long
 *                    double) value of the same quantity, returned as double.
 *
 * Pixel types follow SImage::EDataType (include/SImage.h:36-46 in the
 * reference): 0 U8, 1 S8, 2 U16, 3 S16, 4 U32, 5 S32, 6 F32, 7 F64.
 * Measures: 0 SqrDistance, 1 SqrDistance_Norm, 2 AbsDistance, 3 CrossCorr,
 * 4 CrossCorr_Norm. Steps are in bytes. Channels are interleaved.
 */
#ifndef OPENCLIPP_B200_ORACLE_H
#define OPENCLIPP_B200_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Reference arithmetic; dst holds REAL (float, or double for F64 sources).
 * fused = 0: every operation rounded separately; fused = 1: each
 * `acc += a * b` of the reference evaluated as fma(a, b, acc). */
int orc_proximity_refexact(int measure, int type, int nch, const void* src,
                           int src_step, const void* tmpl, int tmpl_step,
                           void* dst, int dst_step, int W, int H, int tw, int th,
                           int row_begin, int row_end, int fused);

/* Exact / extended precision; dst is double[H][W*nch] (dense). */
int orc_proximity_exact(int measure, int type, int nch, const void* src,
                        int src_step, const void* tmpl, int tmpl_step,
                        double* dst, int W, int H, int tw, int th);

/* The same for the listed output rows only: dst is double[nrows][W*nch],
 * row i holding output row rows[i]. */
int orc_proximity_exact_rows(int measure, int type, int nch, const void* src,
                             int src_step, const void* tmpl, int tmpl_step,
                             double* dst, int W, int H, int tw, int th,
                             const int* rows, int nrows);

/* Window statistics of the same windows, exact: energy of the source window
 * (sum of squares, zero padding), cross term (sum S*T) and template energy.
 * Each array is double[H][W*nch]; tt is double[nch]. Any pointer may be NULL. */
int orc_window_terms_exact(int type, int nch, const void* src, int src_step,
                           const void* tmpl, int tmpl_step, double* ss,
                           double* st, double* tt, int W, int H, int tw, int th);

/* Inclusive integral of S (sqr=0) or S^2 (sqr=1) per channel, exact
 * (integer sources: integer arithmetic; float sources: long double),
 * returned as double[H][W*nch]. */
int orc_integral_exact(int sqr, int type, int nch, const void* src,
                       int src_step, double* dst, int W, int H);

/* Gradients of the score map with respect to the template and the source,
 * in long double, for CrossCorr_Norm (measure 4) and SqrDistance (measure 0),
 * single channel float or double inputs given as double arrays (dense).
 * g is the upstream gradient (double[H][W]); dT is double[th][tw], dS is
 * double[H][W]. */
int orc_proximity_backward(int measure, const double* S, const double* T,
                           const double* g, double* dS, double* dT, int W,
                           int H, int tw, int th);

#ifdef __cplusplus
}
#endif

/* MinIndx (op 0), MaxIndx (1), MinAbsIndx (2), MaxAbsIndx (3) of a
 * one-channel image, in the reference's comparison order
 * (statistics_oracle.c). */
int orc_index_reduce(int op, int type, const void* src, int step, int W, int H, double* value,
                     int* x, int* y);

#endif
