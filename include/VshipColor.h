/*
 * VshipColor.h -- colourspace descriptor of the Vship C ABI, as implemented by the
 * B200 engine in vship_b200/csrc.
 *
 * Every enum value and struct layout below is ABI-identical to the reference header
 * src/VshipColor.h of Line-fr/Vship 4.1.0 (enums src/VshipColor.h:7-71, crop rectangle
 * :73-78, colourspace struct :81-96), so that a caller compiled against the reference
 * header links against this library unchanged.  The declarations are restated here, not
 * copied; the numeric values are the contract.
 */
#ifndef VSHIP_B200_COLOR_H
#define VSHIP_B200_COLOR_H

#include <stdint.h>
#include <stdbool.h>

/* Storage type of one sample.  Integer types are stored in 1 byte (UINT8) or in the low
 * bits of a little-endian 16-bit word (UINT9..UINT16); the unused high bits may hold
 * garbage and are masked off.  Reference: src/VshipColor.h:7-16. */
typedef enum Vship_Sample_t {
    Vship_SampleFLOAT  = 0,
    Vship_SampleHALF   = 1,
    Vship_SampleUINT8  = 2,
    Vship_SampleUINT9  = 3,
    Vship_SampleUINT10 = 5,
    Vship_SampleUINT12 = 7,
    Vship_SampleUINT14 = 9,
    Vship_SampleUINT16 = 11
} Vship_Sample_t;

/* Reference: src/VshipColor.h:18-21. */
typedef enum Vship_Range_t {
    Vship_RangeLimited = 0,
    Vship_RangeFull    = 1
} Vship_Range_t;

/* log2 of the chroma decimation factor per axis (0, 1 or 2 horizontally; 0 or 1
 * vertically).  Reference: src/VshipColor.h:23-26. */
typedef struct Vship_ChromaSubsample_t {
    int subw;
    int subh;
} Vship_ChromaSubsample_t;

/* Reference: src/VshipColor.h:28-33. */
typedef enum Vship_ChromaLocation_t {
    Vship_ChromaLoc_Left    = 0,
    Vship_ChromaLoc_Center  = 1,
    Vship_ChromaLoc_TopLeft = 2,
    Vship_ChromaLoc_Top     = 3
} Vship_ChromaLocation_t;

/* Reference: src/VshipColor.h:35-38 (implicit values 0 and 1). */
typedef enum Vship_ColorFamily_t {
    Vship_ColorYUV = 0,
    Vship_ColorRGB = 1
} Vship_ColorFamily_t;

/* Reference: src/VshipColor.h:40-48. */
typedef enum Vship_YUVMatrix_t {
    Vship_MATRIX_RGB          = 0,
    Vship_MATRIX_BT709        = 1,
    Vship_MATRIX_BT470_BG     = 5,
    Vship_MATRIX_ST170_M      = 6,
    Vship_MATRIX_BT2020_NCL   = 9,
    Vship_MATRIX_BT2020_CL    = 10,
    Vship_MATRIX_BT2100_ICTCP = 14
} Vship_YUVMatrix_t;

/* Reference: src/VshipColor.h:50-61. */
typedef enum Vship_TransferFunction_t {
    Vship_TRC_BT709    = 1,
    Vship_TRC_BT470_M  = 4,
    Vship_TRC_BT470_BG = 5,
    Vship_TRC_BT601    = 6,
    Vship_TRC_ST240_M  = 7,
    Vship_TRC_Linear   = 8,
    Vship_TRC_sRGB     = 13,
    Vship_TRC_PQ       = 16,
    Vship_TRC_ST428    = 17,
    Vship_TRC_HLG      = 18
} Vship_TransferFunction_t;

/* INTERNAL means CIE XYZ.  Reference: src/VshipColor.h:63-71. */
typedef enum Vship_Primaries_t {
    Vship_PRIMARIES_INTERNAL  = -1,
    Vship_PRIMARIES_BT709     = 1,
    Vship_PRIMARIES_BT470_M   = 4,
    Vship_PRIMARIES_BT470_BG  = 5,
    Vship_PRIMARIES_ST170_M   = 6,
    Vship_PRIMARIES_ST240_M   = 7,
    Vship_PRIMARIES_BT2020    = 9
} Vship_Primaries_t;

/* Pixels removed from each side after the optional resize.  Reference: src/VshipColor.h:73-78. */
typedef struct Vship_CropRectangle_t {
    int top;
    int bottom;
    int left;
    int right;
} Vship_CropRectangle_t;

/* Full description of one input clip.  target_width/target_height of -1 mean "no resize".
 * The metric runs at (target_width - left - right) x (target_height - top - bottom).
 * Reference: src/VshipColor.h:81-96. */
typedef struct Vship_Colorspace_t {
    int64_t width;
    int64_t height;
    int64_t target_width;
    int64_t target_height;
    Vship_Sample_t sample;
    Vship_Range_t range;
    Vship_ChromaSubsample_t subsampling;
    Vship_ChromaLocation_t chromaLocation;
    Vship_ColorFamily_t colorFamily;
    Vship_YUVMatrix_t YUVMatrix;
    Vship_TransferFunction_t transferFunction;
    Vship_Primaries_t primaries;
    Vship_CropRectangle_t crop;
} Vship_Colorspace_t;

#endif /* VSHIP_B200_COLOR_H */
