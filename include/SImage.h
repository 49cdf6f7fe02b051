/* Image descriptor shared by every ocip* call.
 *
 * Replaces the reference's include/SImage.h:28-48 with the same field order,
 * widths and enum values, so that code written against the reference passes
 * the same struct by value. Width/Height are in pixels, Step is the number of
 * bytes between the starts of two rows in the caller's (host) buffer,
 * Channels is 1, 2, 3 or 4 and Type is the per-channel element type.
 */
#ifndef OPENCLIPP_B200_SIMAGE_H
#define OPENCLIPP_B200_SIMAGE_H

#ifdef __cplusplus
extern "C" {
#endif

struct SImage {
  unsigned int Width;    /* width of the image, in pixels */
  unsigned int Height;   /* height of the image, in pixels */
  unsigned int Step;     /* bytes between the starts of two rows */
  unsigned int Channels; /* 1, 2, 3 or 4 */

  /* Element type of each channel (same order and values as the reference). */
  enum EDataType {
    U8,  /* unsigned 8-bit integer */
    S8,  /* signed 8-bit integer */
    U16, /* unsigned 16-bit integer */
    S16, /* signed 16-bit integer */
    U32, /* unsigned 32-bit integer */
    S32, /* signed 32-bit integer */
    F32, /* 32-bit float */
    F64, /* 64-bit float */
    NbDataTypes
  } Type;
};

#ifdef __cplusplus
}
#endif
#endif
