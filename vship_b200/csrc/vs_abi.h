/* The parts of the VapourSynth API 4 ABI that the library's plugin entry uses, declared here
 * (C and C++): opaque handles, the structures and enum values the filters read or pass, and
 * the two function tables up to the last slot the plugin calls.  Slots the plugin does not
 * call are untyped placeholders; only their count and position matter.  The layout follows
 * the public VapourSynth 4 API (VapourSynth4.h, API 4.0); tests/test_vs_plugin.py checks
 * every slot offset against that header where it is available. */
#ifndef VSHIP_B200_VS_ABI_H
#define VSHIP_B200_VS_ABI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct VSFrame VSFrame;
typedef struct VSNode VSNode;
typedef struct VSCore VSCore;
typedef struct VSPlugin VSPlugin;
typedef struct VSMap VSMap;
typedef struct VSFrameContext VSFrameContext;
typedef struct VsAbiApi VsAbiApi;

enum { vsCfGray = 1, vsCfRGB = 2, vsCfYUV = 3 };
enum { vsStInteger = 0, vsStFloat = 1 };
enum { vsArInitial = 0, vsArAllFramesReady = 1 };
enum { vsFmParallel = 0, vsFmParallelRequests = 1 };
enum { vsRpStrictSpatial = 2 };
enum { vsMaReplace = 0 };
enum { vsPeSuccess = 0 };
enum { vsDtUtf8 = 1 };

#define VS_ABI_MAKE_VERSION(major, minor) (((major) << 16) | (minor))
#define VS_ABI_API_VERSION VS_ABI_MAKE_VERSION(4, 0)
#define VS_ABI_MAKE_VIDEO_ID(cf, st, bits, sw, sh) (((cf) << 28) | ((st) << 24) | ((bits) << 16) | ((sw) << 8) | (sh))

typedef struct VsAbiVideoFormat {
    int colorFamily;
    int sampleType;
    int bitsPerSample;
    int bytesPerSample;
    int subSamplingW;
    int subSamplingH;
    int numPlanes;
} VsAbiVideoFormat;

typedef struct VsAbiVideoInfo {
    VsAbiVideoFormat format;
    int64_t fpsNum;
    int64_t fpsDen;
    int width;
    int height;
    int numFrames;
} VsAbiVideoInfo;

typedef struct VsAbiCoreInfo {
    const char* versionString;
    int core;
    int api;
    int numThreads;
    int64_t maxFramebufferSize;
    int64_t usedFramebufferSize;
} VsAbiCoreInfo;

typedef struct VsAbiFilterDependency {
    VSNode* source;
    int requestPattern;
} VsAbiFilterDependency;

typedef const VSFrame* (*VsAbiGetFrame)(int n, int activationReason, void* instanceData, void** frameData,
                                        VSFrameContext* frameCtx, VSCore* core, const VsAbiApi* vsapi);
typedef void (*VsAbiFilterFree)(void* instanceData, VSCore* core, const VsAbiApi* vsapi);
typedef void (*VsAbiPublicFunction)(const VSMap* in, VSMap* out, void* userData, VSCore* core, const VsAbiApi* vsapi);
typedef void (*VsAbiSlot)(void);

/* VSPLUGINAPI */
typedef struct VsAbiPluginApi {
    int (*getAPIVersion)(void);
    int (*configPlugin)(const char* identifier, const char* pluginNamespace, const char* name, int pluginVersion,
                        int apiVersion, int flags, VSPlugin* plugin);
    int (*registerFunction)(const char* name, const char* args, const char* returnType, VsAbiPublicFunction argsFunc,
                            void* functionData, VSPlugin* plugin);
} VsAbiPluginApi;

/* VSAPI, slots 1..102 (numbered from 1 as the comments below). */
struct VsAbiApi {
    void (*createVideoFilter)(VSMap* out, const char* name, const VsAbiVideoInfo* vi, VsAbiGetFrame getFrame,
                              VsAbiFilterFree free, int filterMode, const VsAbiFilterDependency* dependencies,
                              int numDeps, void* instanceData, VSCore* core);       /* 1 */
    VsAbiSlot slots_2_7[6];
    void (*freeNode)(VSNode* node);                                                  /* 8 */
    VsAbiSlot slots_9_10[2];
    const VsAbiVideoInfo* (*getVideoInfo)(VSNode* node);                             /* 11 */
    VsAbiSlot slot_12;
    VSFrame* (*newVideoFrame)(const VsAbiVideoFormat* format, int width, int height, const VSFrame* propSrc,
                              VSCore* core);                                         /* 13 */
    VsAbiSlot slots_14_16[3];
    void (*freeFrame)(const VSFrame* f);                                             /* 17 */
    VsAbiSlot slot_18;
    VSFrame* (*copyFrame)(const VSFrame* f, VSCore* core);                           /* 19 */
    VsAbiSlot slot_20;
    VSMap* (*getFramePropertiesRW)(VSFrame* f);                                      /* 21 */
    ptrdiff_t (*getStride)(const VSFrame* f, int plane);                             /* 22 */
    const uint8_t* (*getReadPtr)(const VSFrame* f, int plane);                       /* 23 */
    uint8_t* (*getWritePtr)(VSFrame* f, int plane);                                  /* 24 */
    VsAbiSlot slots_25_27[3];
    int (*getFrameWidth)(const VSFrame* f, int plane);                               /* 28 */
    int (*getFrameHeight)(const VSFrame* f, int plane);                              /* 29 */
    VsAbiSlot slots_30_32[3];
    int (*queryVideoFormat)(VsAbiVideoFormat* format, int colorFamily, int sampleType, int bitsPerSample,
                            int subSamplingW, int subSamplingH, VSCore* core);       /* 33 */
    VsAbiSlot slots_34_38[5];
    const VSFrame* (*getFrameFilter)(int n, VSNode* node, VSFrameContext* frameCtx); /* 39 */
    void (*requestFrameFilter)(int n, VSNode* node, VSFrameContext* frameCtx);       /* 40 */
    VsAbiSlot slots_41_42[2];
    void (*setFilterError)(const char* errorMessage, VSFrameContext* frameCtx);      /* 43 */
    VsAbiSlot slots_44_47[4];
    VSMap* (*createMap)(void);                                                       /* 48 */
    void (*freeMap)(VSMap* map);                                                     /* 49 */
    VsAbiSlot slots_50_51[2];
    void (*mapSetError)(VSMap* map, const char* errorMessage);                       /* 52 */
    const char* (*mapGetError)(const VSMap* map);                                    /* 53 */
    VsAbiSlot slots_54_59[6];
    int64_t (*mapGetInt)(const VSMap* map, const char* key, int index, int* error);  /* 60 */
    VsAbiSlot slots_61_62[2];
    int (*mapSetInt)(VSMap* map, const char* key, int64_t i, int append);            /* 63 */
    VsAbiSlot slot_64;
    double (*mapGetFloat)(const VSMap* map, const char* key, int index, int* error); /* 65 */
    VsAbiSlot slots_66_67[2];
    int (*mapSetFloat)(VSMap* map, const char* key, double d, int append);           /* 68 */
    VsAbiSlot slot_69;
    const char* (*mapGetData)(const VSMap* map, const char* key, int index, int* error); /* 70 */
    VsAbiSlot slots_71_72[2];
    int (*mapSetData)(VSMap* map, const char* key, const char* data, int size, int type, int append); /* 73 */
    VSNode* (*mapGetNode)(const VSMap* map, const char* key, int index, int* error); /* 74 */
    VsAbiSlot slot_75;
    int (*mapConsumeNode)(VSMap* map, const char* key, VSNode* node, int append);    /* 76 */
    VsAbiSlot slots_77_83[7];
    VSPlugin* (*getPluginByID)(const char* identifier, VSCore* core);                /* 84 */
    VsAbiSlot slots_85_96[12];
    VSMap* (*invoke)(VSPlugin* plugin, const char* name, const VSMap* args);         /* 97 */
    VsAbiSlot slots_98_101[4];
    void (*getCoreInfo)(VSCore* core, VsAbiCoreInfo* info);                          /* 102 */
};

#ifdef __cplusplus
}
#endif

#endif /* VSHIP_B200_VS_ABI_H */
