"""ctypes mirror of the Vship C ABI declared in include/VshipAPI.h and include/VshipColor.h.

Pure data definitions (no library is loaded here).  Enum values and struct layouts follow
the reference headers src/VshipColor.h:7-96 and src/VshipAPI.h:23-129 of Line-fr/Vship.
"""
import ctypes

# Vship_Sample_t (src/VshipColor.h:7-16)
SampleFLOAT, SampleHALF, SampleUINT8, SampleUINT9 = 0, 1, 2, 3
SampleUINT10, SampleUINT12, SampleUINT14, SampleUINT16 = 5, 7, 9, 11
# Vship_Range_t
RangeLimited, RangeFull = 0, 1
# Vship_ChromaLocation_t
ChromaLoc_Left, ChromaLoc_Center, ChromaLoc_TopLeft, ChromaLoc_Top = 0, 1, 2, 3
# Vship_ColorFamily_t
ColorYUV, ColorRGB = 0, 1
# Vship_YUVMatrix_t
MATRIX_RGB, MATRIX_BT709, MATRIX_BT470_BG, MATRIX_ST170_M = 0, 1, 5, 6
MATRIX_BT2020_NCL, MATRIX_BT2020_CL, MATRIX_BT2100_ICTCP = 9, 10, 14
# Vship_TransferFunction_t
TRC_BT709, TRC_BT470_M, TRC_BT470_BG, TRC_BT601, TRC_ST240_M = 1, 4, 5, 6, 7
TRC_Linear, TRC_sRGB, TRC_PQ, TRC_ST428, TRC_HLG = 8, 13, 16, 17, 18
# Vship_Primaries_t
PRIMARIES_INTERNAL, PRIMARIES_BT709, PRIMARIES_BT470_M, PRIMARIES_BT470_BG = -1, 1, 4, 5
PRIMARIES_ST170_M, PRIMARIES_ST240_M, PRIMARIES_BT2020 = 6, 7, 9

# Vship_Exception (src/VshipAPI.h:38-65)
EXCEPTIONS = {
    0: "NoError", 1: "OutOfVRAM", 2: "OutOfRAM", 12: "HIPError", 3: "BadDisplayModel",
    4: "DifferingInputType", 5: "NonRGBSInput", 13: "BadPath", 14: "BadJson",
    6: "DeviceCountError", 7: "NoDeviceDetected", 8: "BadDeviceArgument", 9: "BadDeviceCode",
    10: "BadHandler", 11: "BadPointer", 15: "BadErrorType",
}
NoError, OutOfVRAM, OutOfRAM, HIPError = 0, 1, 2, 12
DifferingInputType, DeviceCountError, NoDeviceDetected = 4, 6, 7
BadDeviceArgument, BadDeviceCode, BadHandler, BadPointer, BadErrorType = 8, 9, 10, 11, 15
BadDisplayModel, NonRGBSInput, BadPath, BadJson = 3, 5, 13, 14

SAMPLE_BYTES = {SampleFLOAT: 4, SampleHALF: 2, SampleUINT8: 1, SampleUINT9: 2, SampleUINT10: 2,
                SampleUINT12: 2, SampleUINT14: 2, SampleUINT16: 2}
SAMPLE_BITS = {SampleUINT8: 8, SampleUINT9: 9, SampleUINT10: 10, SampleUINT12: 12,
               SampleUINT14: 14, SampleUINT16: 16}


class ChromaSubsample(ctypes.Structure):
    _fields_ = [("subw", ctypes.c_int), ("subh", ctypes.c_int)]


class CropRectangle(ctypes.Structure):
    _fields_ = [("top", ctypes.c_int), ("bottom", ctypes.c_int),
                ("left", ctypes.c_int), ("right", ctypes.c_int)]


class Colorspace(ctypes.Structure):
    """Vship_Colorspace_t (src/VshipColor.h:81-96)."""
    _fields_ = [
        ("width", ctypes.c_int64), ("height", ctypes.c_int64),
        ("target_width", ctypes.c_int64), ("target_height", ctypes.c_int64),
        ("sample", ctypes.c_int), ("range", ctypes.c_int),
        ("subsampling", ChromaSubsample), ("chromaLocation", ctypes.c_int),
        ("colorFamily", ctypes.c_int), ("YUVMatrix", ctypes.c_int),
        ("transferFunction", ctypes.c_int), ("primaries", ctypes.c_int),
        ("crop", CropRectangle),
    ]

    def plane_dims(self):
        """(width, height) of each of the three input planes before chroma upsampling."""
        sw, sh = self.subsampling.subw, self.subsampling.subh
        cw, ch = ((self.width - 1) >> sw) + 1, ((self.height - 1) >> sh) + 1
        return [(self.width, self.height), (cw, ch), (cw, ch)]

    def out_dims(self):
        """(width, height) the metric runs at, after resize and crop."""
        tw = self.width if self.target_width == -1 else self.target_width
        th = self.height if self.target_height == -1 else self.target_height
        return (tw - self.crop.left - self.crop.right, th - self.crop.top - self.crop.bottom)


def colorspace(width, height, sample=SampleUINT8, range_=RangeFull, subw=0, subh=0,
               chroma_location=ChromaLoc_Left, family=ColorRGB, matrix=MATRIX_RGB,
               transfer=TRC_sRGB, primaries=PRIMARIES_BT709, target_width=-1, target_height=-1,
               crop=(0, 0, 0, 0)):
    cs = Colorspace()
    cs.width, cs.height = width, height
    cs.target_width, cs.target_height = target_width, target_height
    cs.sample, cs.range = sample, range_
    cs.subsampling = ChromaSubsample(subw, subh)
    cs.chromaLocation, cs.colorFamily = chroma_location, family
    cs.YUVMatrix, cs.transferFunction, cs.primaries = matrix, transfer, primaries
    cs.crop = CropRectangle(*crop)
    return cs


def srgb8(width, height):
    """8-bit full-range sRGB, BT.709 primaries (the 1-pair 1080p configuration)."""
    return colorspace(width, height)


def yuv420_10bit_bt709(width, height):
    """10-bit limited-range Y'CbCr 4:2:0, Left chroma siting, BT.709 matrix, transfer and primaries."""
    return colorspace(width, height, sample=SampleUINT10, range_=RangeLimited, subw=1, subh=1,
                      chroma_location=ChromaLoc_Left, family=ColorYUV, matrix=MATRIX_BT709,
                      transfer=TRC_BT709, primaries=PRIMARIES_BT709)


class Version(ctypes.Structure):
    _fields_ = [("major", ctypes.c_int), ("minor", ctypes.c_int),
                ("minorMinor", ctypes.c_int), ("backend", ctypes.c_int)]


class DeviceInfo(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 256), ("VRAMSize", ctypes.c_uint64),
                ("integrated", ctypes.c_int), ("MultiProcessorCount", ctypes.c_int),
                ("WarpSize", ctypes.c_int)]


class SSIMU2Handler(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint)]


class ButteraugliHandler(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint)]


class CVVDPHandler(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint)]


class CVVDPDisplay(ctypes.Structure):
    """VshipExt_CVVDPDisplay (include/VshipAPI_ext.h)."""
    _fields_ = [("width", ctypes.c_int64), ("height", ctypes.c_int64), ("hdr", ctypes.c_int),
                ("viewing_distance_meters", ctypes.c_float), ("diagonal_size_inches", ctypes.c_float),
                ("max_luminance", ctypes.c_float), ("contrast", ctypes.c_float), ("E_ambient", ctypes.c_float),
                ("k_refl", ctypes.c_float), ("exposure", ctypes.c_float), ("ppd", ctypes.c_float),
                ("black_level", ctypes.c_float), ("reflected_level", ctypes.c_float)]


class ButteraugliScore(ctypes.Structure):
    _fields_ = [("normQ", ctypes.c_double), ("norm3", ctypes.c_double), ("norminf", ctypes.c_double)]


PlanePtrs = ctypes.POINTER(ctypes.c_uint8) * 3
LineSizes = ctypes.c_int64 * 3


class SSIMU2BatchHandler(ctypes.Structure):
    """Extension (include/VshipAPI_ext.h): handler of uneven SSIMULACRA2 batches."""
    _fields_ = [("id", ctypes.c_uint)]


class SurrogateHandler(ctypes.Structure):
    """Extension (include/VshipAPI_ext.h): handler of the learned SSIMULACRA2 surrogate."""
    _fields_ = [("id", ctypes.c_uint)]


class FramePair(ctypes.Structure):
    """Extension (include/VshipAPI_ext.h): one pair of an uneven batch."""
    _fields_ = [("src_colorspace", Colorspace), ("dis_colorspace", Colorspace),
                ("srcp1", ctypes.c_void_p * 3), ("srcp2", ctypes.c_void_p * 3),
                ("lineSize", ctypes.c_int64 * 3), ("lineSize2", ctypes.c_int64 * 3)]
