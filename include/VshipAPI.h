/*
 * VshipAPI.h -- the Vship C ABI served by the B200 engine (libvship.so built from
 * vship_b200/csrc).
 *
 * Each declaration below replaces the reference declaration cited beside it
 * (Line-fr/Vship 4.1.0, src/VshipAPI.h).  Names, argument order, types and enum values are
 * ABI-identical so that FFVship, VapourSynth scripts and other callers of the reference
 * library link against this one unchanged.  Behaviour differences: a freed or never-
 * initialised handler id returns Vship_BadHandler (undefined behaviour in the reference), and
 * device memory is taken at Init rather than per frame.
 *
 * Threading contract (same as the reference): any number of handlers may be used from
 * different threads at the same time; one handler must not be used by two threads at once
 * (this build detects that case and returns Vship_BadHandler instead of racing).
 */
#ifndef VSHIP_B200_API_H
#define VSHIP_B200_API_H

#include <stdint.h>
#include <stdbool.h>

#include "VshipColor.h"

#if defined(_WIN32)
#  if defined(EXPORTVSHIPLIB)
#    define EXPORTPREPROCESS __declspec(dllexport)
#  else
#    define EXPORTPREPROCESS __declspec(dllimport)
#  endif
#else
#  define EXPORTPREPROCESS __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Reference: src/VshipAPI.h:23-26. */
typedef enum {
    Vship_HIP  = 0,
    Vship_Cuda = 1
} Vship_Backend;

/* Reference: src/VshipAPI.h:28-33. */
typedef struct {
    int major;
    int minor;
    int minorMinor;
    Vship_Backend backend;
} Vship_Version;

/* Library version: 4.1.0 on the CUDA backend.  Replaces src/VshipAPI.h:35. */
EXPORTPREPROCESS Vship_Version Vship_GetVersion(void);

/* Error codes.  Reference: src/VshipAPI.h:38-65. */
typedef enum {
    Vship_NoError = 0,
    Vship_OutOfVRAM = 1,
    Vship_OutOfRAM = 2,
    Vship_HIPError = 12,
    Vship_BadDisplayModel = 3,
    Vship_DifferingInputType = 4,
    Vship_NonRGBSInput = 5,
    Vship_BadPath = 13,
    Vship_BadJson = 14,
    Vship_DeviceCountError = 6,
    Vship_NoDeviceDetected = 7,
    Vship_BadDeviceArgument = 8,
    Vship_BadDeviceCode = 9,
    Vship_BadHandler = 10,
    Vship_BadPointer = 11,
    Vship_BadErrorType = 15
} Vship_Exception;

/* Number of visible CUDA devices.  Replaces src/VshipAPI.h:68. */
EXPORTPREPROCESS Vship_Exception Vship_GetDeviceCount(int* number);

/* Default device for the Init functions without a gpu_id.  Replaces src/VshipAPI.h:71. */
EXPORTPREPROCESS Vship_Exception Vship_SetDevice(int gpu_id);

/* Reference: src/VshipAPI.h:74-80. */
typedef struct Vship_DeviceInfo {
    char name[256];
    uint64_t VRAMSize;
    int integrated;
    int MultiProcessorCount;
    int WarpSize;
} Vship_DeviceInfo;

/* Replaces src/VshipAPI.h:82. */
EXPORTPREPROCESS Vship_Exception Vship_GetDeviceInfo(Vship_DeviceInfo* device_info, int gpu_id);

/* Runs a one-thread kernel on gpu_id and checks its result.  Replaces src/VshipAPI.h:85. */
EXPORTPREPROCESS Vship_Exception Vship_GPUFullCheck(int gpu_id);

/* Writes the generic message of an error code (truncated to len-1 bytes plus NUL) and
 * returns the buffer size the full message needs; len == 0 only returns that size.
 * Replaces src/VshipAPI.h:89. */
EXPORTPREPROCESS int Vship_GetErrorMessage(Vship_Exception exception, char* out_message, int len);

/* Same convention, for the detailed text of the last error raised by any call.
 * Replaces src/VshipAPI.h:93. */
EXPORTPREPROCESS int Vship_GetDetailedLastError(char* out_message, int len);

/* Opaque handle: an index into the library's handler table.  Reference: src/VshipAPI.h:98-100. */
typedef struct Vship_SSIMU2Handler {
    unsigned int id;
} Vship_SSIMU2Handler;

/* Page-locked host allocation (cudaMallocHost).  Replaces src/VshipAPI.h:102. */
EXPORTPREPROCESS Vship_Exception Vship_PinnedMalloc(void** ptr, uint64_t size);

/* Replaces src/VshipAPI.h:104. */
EXPORTPREPROCESS Vship_Exception Vship_PinnedFree(void* ptr);

/* Creates an SSIMULACRA2 handler on the default device.  Replaces src/VshipAPI.h:107. */
EXPORTPREPROCESS Vship_Exception Vship_SSIMU2Init(Vship_SSIMU2Handler* handler, Vship_Colorspace_t src_colorspace, Vship_Colorspace_t dis_colorspace);

/* Creates an SSIMULACRA2 handler on gpu_id; all device memory is allocated here, none per
 * frame.  Replaces src/VshipAPI.h:109. */
EXPORTPREPROCESS Vship_Exception Vship_SSIMU2Init2(Vship_SSIMU2Handler* handler, Vship_Colorspace_t src_colorspace, Vship_Colorspace_t dis_colorspace, int gpu_id);

/* Replaces src/VshipAPI.h:112. */
EXPORTPREPROCESS Vship_Exception Vship_SSIMU2Free(Vship_SSIMU2Handler handler);

/* Scores one frame pair.  srcp1/srcp2 are three host plane pointers (pageable or pinned)
 * with byte strides lineSize/lineSize2; the frames are not modified.  Blocks until *score
 * is written.  Replaces src/VshipAPI.h:115. */
EXPORTPREPROCESS Vship_Exception Vship_ComputeSSIMU2(Vship_SSIMU2Handler handler, double* score, const uint8_t* srcp1[3], const uint8_t* srcp2[3], const int64_t lineSize[3], const int64_t lineSize2[3]);

/* Detailed text of the handler's last error (same size convention as above); returns 0 for
 * an invalid handler.  Replaces src/VshipAPI.h:119. */
EXPORTPREPROCESS int Vship_SSIMU2GetDetailedLastError(Vship_SSIMU2Handler handler, char* out_message, int len);

/* Reference: src/VshipAPI.h:121-123. */
typedef struct Vship_ButteraugliHandler {
    unsigned int id;
} Vship_ButteraugliHandler;

/* Reference: src/VshipAPI.h:125-129. */
typedef struct Vship_ButteraugliScore {
    double normQ;
    double norm3;
    double norminf;
} Vship_ButteraugliScore;

/* Replaces src/VshipAPI.h:132. */
EXPORTPREPROCESS Vship_Exception Vship_ButteraugliInit(Vship_ButteraugliHandler* handler, Vship_Colorspace_t src_colorspace, Vship_Colorspace_t dis_colorspace, int Qnorm, float intensity_multiplier);

/* Replaces src/VshipAPI.h:134. */
EXPORTPREPROCESS Vship_Exception Vship_ButteraugliInit2(Vship_ButteraugliHandler* handler, Vship_Colorspace_t src_colorspace, Vship_Colorspace_t dis_colorspace, int Qnorm, float intensity_multiplier, int gpu_id);

/* Replaces src/VshipAPI.h:137. */
EXPORTPREPROCESS Vship_Exception Vship_ButteraugliFree(Vship_ButteraugliHandler handler);

/* Scores one frame pair.  dstp is NULL (no distortion map) or a host buffer of
 * dststride*height bytes that receives the FP32 distortion map row by row.
 * Replaces src/VshipAPI.h:143. */
EXPORTPREPROCESS Vship_Exception Vship_ComputeButteraugli(Vship_ButteraugliHandler handler, Vship_ButteraugliScore* score, const uint8_t* dstp, int64_t dststride, const uint8_t* srcp1[3], const uint8_t* srcp2[3], const int64_t lineSize[3], const int64_t lineSize2[3]);

/* Replaces src/VshipAPI.h:147. */
EXPORTPREPROCESS int Vship_ButteraugliGetDetailedLastError(Vship_ButteraugliHandler handler, char* out_message, int len);

/* Reference: src/VshipAPI.h:149-151. */
typedef struct Vship_CVVDPHandler {
    unsigned int id;
} Vship_CVVDPHandler;

/* CVVDP is outside this engine's scope.  The entry points exist so that the symbol table
 * matches the reference; they return Vship_BadErrorType with the detail
 * "CVVDP is not provided by this build" (or 0 for the *GetDetailedLastError getter).
 * Replace src/VshipAPI.h:154, :161, :163, :166, :169, :173, :176, :180, :186 and :190. */
EXPORTPREPROCESS Vship_Exception Vship_CVVDPInit(Vship_CVVDPHandler* handler, Vship_Colorspace_t src_colorspace, Vship_Colorspace_t dis_colorspace, float fps, bool resizeToDisplay, const char* model_key_cstr);
EXPORTPREPROCESS Vship_Exception Vship_CVVDPInit2(Vship_CVVDPHandler* handler, Vship_Colorspace_t src_colorspace, Vship_Colorspace_t dis_colorspace, float fps, bool resizeToDisplay, const char* model_key_cstr, const char* model_config_json_cstr);
EXPORTPREPROCESS Vship_Exception Vship_CVVDPInit3(Vship_CVVDPHandler* handler, Vship_Colorspace_t src_colorspace, Vship_Colorspace_t dis_colorspace, float fps, bool resizeToDisplay, const char* model_key_cstr, const char* model_config_json_cstr, int gpu_id);
EXPORTPREPROCESS Vship_Exception Vship_CVVDPFree(Vship_CVVDPHandler handler);
EXPORTPREPROCESS Vship_Exception Vship_CVVDPGetDistmapResolution(Vship_CVVDPHandler handler, int64_t* width, int64_t* height);
EXPORTPREPROCESS Vship_Exception Vship_ResetCVVDP(Vship_CVVDPHandler handler);
EXPORTPREPROCESS Vship_Exception Vship_ResetScoreCVVDP(Vship_CVVDPHandler handler);
EXPORTPREPROCESS Vship_Exception Vship_LoadTemporalCVVDP(Vship_CVVDPHandler handler, const uint8_t* srcp1[3], const uint8_t* srcp2[3], const int64_t lineSize[3], const int64_t lineSize2[3]);
EXPORTPREPROCESS Vship_Exception Vship_ComputeCVVDP(Vship_CVVDPHandler handler, double* score, const uint8_t* dstp, int64_t dststride, const uint8_t* srcp1[3], const uint8_t* srcp2[3], const int64_t lineSize[3], const int64_t lineSize2[3]);
EXPORTPREPROCESS int Vship_CVVDPGetDetailedLastError(Vship_CVVDPHandler handler, char* out_message, int len);

#ifdef __cplusplus
}
#endif

#endif /* VSHIP_B200_API_H */
