/* A minimal stand-in for a VapourSynth core, for testing the library's plugin entry without a
 * VapourSynth installation.  It implements the API slots the plugin calls (vship_b200/csrc/
 * vs_abi.h), keeps clips as in-memory frames, and drives a filter's frame requests the way the
 * VapourSynth scheduler does (arInitial, then arAllFramesReady).  Driven from Python through
 * ctypes by tests/test_vs_plugin.py.  Test infrastructure only. */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../vship_b200/csrc/vs_abi.h"

/* ---- maps ---------------------------------------------------------------------------- */
enum { tInt = 1, tFloat, tNode, tData };
typedef struct Entry {
    char key[64];
    int type;
    int64_t i;
    double f;
    VSNode* node;
    char* data;
} Entry;
struct VSMap {
    Entry e[32];
    int n;
    char error[4096];
    int has_error;
};

static Entry* find(const VSMap* m, const char* key) {
    for (int k = 0; k < m->n; k++)
        if (!strcmp(m->e[k].key, key)) return (Entry*)&m->e[k];
    return NULL;
}
static Entry* put(VSMap* m, const char* key) {
    Entry* x = find(m, key);
    if (x) return x;
    x = &m->e[m->n++];
    memset(x, 0, sizeof(*x));
    snprintf(x->key, sizeof(x->key), "%s", key);
    return x;
}

/* ---- frames and nodes ---------------------------------------------------------------- */
struct VSFrame {
    VsAbiVideoFormat fmt;
    int w, h;
    uint8_t* plane[3];
    ptrdiff_t stride[3];
    VSMap props;
};
struct VSNode {
    VsAbiVideoInfo vi;
    VSFrame** frames;  /* source clips */
    VsAbiGetFrame get;  /* filters */
    VsAbiFilterFree free_fn;
    void* instance;
};
struct VSCore {
    int threads;
};
struct VSFrameContext {
    char error[4096];
    int has_error;
};
struct VSPlugin {
    int dummy;
};

static VSFrame* new_frame(const VsAbiVideoFormat* f, int w, int h) {
    VSFrame* fr = (VSFrame*)calloc(1, sizeof(VSFrame));
    fr->fmt = *f;
    fr->w = w;
    fr->h = h;
    for (int p = 0; p < f->numPlanes; p++) {
        fr->stride[p] = ((ptrdiff_t)w * f->bytesPerSample + 63) / 64 * 64; /* padded rows, as VapourSynth */
        fr->plane[p] = (uint8_t*)calloc((size_t)fr->stride[p] * h, 1);
    }
    return fr;
}
static void free_frame(const VSFrame* f) {
    if (!f) return;
    for (int p = 0; p < 3; p++) free(f->plane[p]);
    free((void*)f);
}
static VSFrame* copy_frame(const VSFrame* f, VSCore* core) {
    (void)core;
    VSFrame* c = new_frame(&f->fmt, f->w, f->h);
    for (int p = 0; p < f->fmt.numPlanes; p++) memcpy(c->plane[p], f->plane[p], (size_t)f->stride[p] * f->h);
    c->props = f->props;
    return c;
}

/* ---- API slots ------------------------------------------------------------------------ */
static void api_create_video_filter(VSMap* out, const char* name, const VsAbiVideoInfo* vi, VsAbiGetFrame get,
                                    VsAbiFilterFree fr, int mode, const VsAbiFilterDependency* deps, int ndeps,
                                    void* instance, VSCore* core) {
    (void)name; (void)mode; (void)deps; (void)ndeps; (void)core;
    VSNode* n = (VSNode*)calloc(1, sizeof(VSNode));
    n->vi = *vi;
    n->get = get;
    n->free_fn = fr;
    n->instance = instance;
    Entry* e = put(out, "clip");
    e->type = tNode;
    e->node = n;
}
static void api_free_node(VSNode* n) { (void)n; /* nodes are released by vsfake_free_node */ }
static const VsAbiVideoInfo* api_get_video_info(VSNode* n) { return &n->vi; }
static VSFrame* api_new_video_frame(const VsAbiVideoFormat* f, int w, int h, const VSFrame* src, VSCore* core) {
    (void)src; (void)core;
    return new_frame(f, w, h);
}
static void api_free_frame(const VSFrame* f) {
    /* source frames stay owned by their node; only frames made for a request are freed */
    (void)f;
}
static VSMap* api_props_rw(VSFrame* f) { return &f->props; }
static ptrdiff_t api_get_stride(const VSFrame* f, int p) { return f->stride[p]; }
static const uint8_t* api_get_read_ptr(const VSFrame* f, int p) { return f->plane[p]; }
static uint8_t* api_get_write_ptr(VSFrame* f, int p) { return f->plane[p]; }
static int api_get_frame_width(const VSFrame* f, int p) { (void)p; return f->w; }
static int api_get_frame_height(const VSFrame* f, int p) { (void)p; return f->h; }
static int api_query_video_format(VsAbiVideoFormat* f, int cf, int st, int bits, int sw, int sh, VSCore* core) {
    (void)core;
    f->colorFamily = cf;
    f->sampleType = st;
    f->bitsPerSample = bits;
    f->bytesPerSample = bits <= 8 ? 1 : bits <= 16 ? 2 : 4;
    f->subSamplingW = sw;
    f->subSamplingH = sh;
    f->numPlanes = cf == vsCfGray ? 1 : 3;
    return 1;
}
static const VSFrame* api_get_frame_filter(int n, VSNode* node, VSFrameContext* ctx) {
    (void)ctx;
    return node->frames ? node->frames[n] : NULL;
}
static void api_request_frame_filter(int n, VSNode* node, VSFrameContext* ctx) { (void)n; (void)node; (void)ctx; }
static void api_set_filter_error(const char* msg, VSFrameContext* ctx) {
    snprintf(ctx->error, sizeof(ctx->error), "%s", msg);
    ctx->has_error = 1;
}
static VSMap* api_create_map(void) { return (VSMap*)calloc(1, sizeof(VSMap)); }
static void api_free_map(VSMap* m) { free(m); }
static void api_map_set_error(VSMap* m, const char* msg) {
    snprintf(m->error, sizeof(m->error), "%s", msg);
    m->has_error = 1;
}
static const char* api_map_get_error(const VSMap* m) { return m->has_error ? m->error : NULL; }
static int64_t api_map_get_int(const VSMap* m, const char* key, int idx, int* err) {
    (void)idx;
    Entry* e = find(m, key);
    if (!e || e->type != tInt) { if (err) *err = 1; return 0; }
    if (err) *err = 0;
    return e->i;
}
static int api_map_set_int(VSMap* m, const char* key, int64_t v, int append) {
    (void)append;
    Entry* e = put(m, key);
    e->type = tInt;
    e->i = v;
    return 0;
}
static double api_map_get_float(const VSMap* m, const char* key, int idx, int* err) {
    (void)idx;
    Entry* e = find(m, key);
    if (!e || e->type != tFloat) { if (err) *err = 1; return 0; }
    if (err) *err = 0;
    return e->f;
}
static int api_map_set_float(VSMap* m, const char* key, double v, int append) {
    (void)append;
    Entry* e = put(m, key);
    e->type = tFloat;
    e->f = v;
    return 0;
}
static int api_map_set_data(VSMap* m, const char* key, const char* d, int size, int type, int append) {
    (void)type; (void)append;
    Entry* e = put(m, key);
    e->type = tData;
    e->data = (char*)calloc((size_t)size + 1, 1);
    memcpy(e->data, d, (size_t)size);
    return 0;
}
static const char* api_map_get_data(const VSMap* m, const char* key, int idx, int* err) {
    (void)idx;
    Entry* e = find(m, key);
    if (!e || e->type != tData) { if (err) *err = 1; return NULL; }
    if (err) *err = 0;
    return e->data;
}
static VSNode* api_map_get_node(const VSMap* m, const char* key, int idx, int* err) {
    (void)idx;
    Entry* e = find(m, key);
    if (!e || e->type != tNode) { if (err) *err = 1; return NULL; }
    if (err) *err = 0;
    return e->node;
}
static int api_map_consume_node(VSMap* m, const char* key, VSNode* n, int append) {
    (void)append;
    Entry* e = put(m, key);
    e->type = tNode;
    e->node = n;
    return 0;
}
static VSPlugin* api_get_plugin_by_id(const char* id, VSCore* core) { (void)id; (void)core; return NULL; }
static VSMap* api_invoke(VSPlugin* p, const char* name, const VSMap* args) { (void)p; (void)name; (void)args; return NULL; }
static void api_get_core_info(VSCore* core, VsAbiCoreInfo* info) {
    memset(info, 0, sizeof(*info));
    info->versionString = "fake";
    info->core = 70;
    info->api = VS_ABI_API_VERSION;
    info->numThreads = core->threads;
}

static VsAbiApi g_api;
static VSCore g_core = {4};

/* ---- plugin registration ---------------------------------------------------------------- */
typedef struct Fn {
    char name[64];
    char args[512];
    char ret[64];
    VsAbiPublicFunction fn;
} Fn;
static Fn g_fns[16];
static int g_nfns;
static char g_plugin_id[128], g_plugin_ns[64];
static int g_plugin_version, g_plugin_api;

static int papi_api_version(void) { return VS_ABI_API_VERSION; }
static int papi_config(const char* id, const char* ns, const char* name, int version, int api, int flags, VSPlugin* p) {
    (void)name; (void)flags; (void)p;
    snprintf(g_plugin_id, sizeof(g_plugin_id), "%s", id);
    snprintf(g_plugin_ns, sizeof(g_plugin_ns), "%s", ns);
    g_plugin_version = version;
    g_plugin_api = api;
    return 1;
}
static int papi_register(const char* name, const char* args, const char* ret, VsAbiPublicFunction fn, void* data,
                         VSPlugin* p) {
    (void)data; (void)p;
    Fn* f = &g_fns[g_nfns++];
    snprintf(f->name, sizeof(f->name), "%s", name);
    snprintf(f->args, sizeof(f->args), "%s", args);
    snprintf(f->ret, sizeof(f->ret), "%s", ret);
    f->fn = fn;
    return 1;
}

/* Loads the library and runs its plugin entry; returns the number of registered functions. */
int vsfake_load(const char* libpath) {
    g_api.createVideoFilter = api_create_video_filter;
    g_api.freeNode = api_free_node;
    g_api.getVideoInfo = api_get_video_info;
    g_api.newVideoFrame = api_new_video_frame;
    g_api.freeFrame = api_free_frame;
    g_api.copyFrame = copy_frame;
    g_api.getFramePropertiesRW = api_props_rw;
    g_api.getStride = api_get_stride;
    g_api.getReadPtr = api_get_read_ptr;
    g_api.getWritePtr = api_get_write_ptr;
    g_api.getFrameWidth = api_get_frame_width;
    g_api.getFrameHeight = api_get_frame_height;
    g_api.queryVideoFormat = api_query_video_format;
    g_api.getFrameFilter = api_get_frame_filter;
    g_api.requestFrameFilter = api_request_frame_filter;
    g_api.setFilterError = api_set_filter_error;
    g_api.createMap = api_create_map;
    g_api.freeMap = api_free_map;
    g_api.mapSetError = api_map_set_error;
    g_api.mapGetError = api_map_get_error;
    g_api.mapGetInt = api_map_get_int;
    g_api.mapSetInt = api_map_set_int;
    g_api.mapGetFloat = api_map_get_float;
    g_api.mapSetFloat = api_map_set_float;
    g_api.mapSetData = api_map_set_data;
    g_api.mapGetData = api_map_get_data;
    g_api.mapGetNode = api_map_get_node;
    g_api.mapConsumeNode = api_map_consume_node;
    g_api.getPluginByID = api_get_plugin_by_id;
    g_api.invoke = api_invoke;
    g_api.getCoreInfo = api_get_core_info;
    void* lib = dlopen(libpath, RTLD_NOW | RTLD_LOCAL);
    if (!lib) return -1;
    void (*init)(VSPlugin*, const VsAbiPluginApi*) = (void (*)(VSPlugin*, const VsAbiPluginApi*))dlsym(lib, "VapourSynthPluginInit2");
    if (!init) return -2;
    static VsAbiPluginApi papi = {papi_api_version, papi_config, papi_register};
    static VSPlugin plugin;
    g_nfns = 0;
    init(&plugin, &papi);
    return g_nfns;
}

int vsfake_registered(int i, char* name, char* args, char* ret) {
    if (i < 0 || i >= g_nfns) return -1;
    strcpy(name, g_fns[i].name);
    strcpy(args, g_fns[i].args);
    strcpy(ret, g_fns[i].ret);
    return 0;
}

int vsfake_plugin(char* id, char* ns, int* version, int* api) {
    strcpy(id, g_plugin_id);
    strcpy(ns, g_plugin_ns);
    *version = g_plugin_version;
    *api = g_plugin_api;
    return 0;
}

/* A source clip of nframes planar frames (cf/st/bits), copied from `data` laid out
 * [frame][plane][h][w] in bytesPerSample units. */
VSNode* vsfake_source(int w, int h, int nframes, int cf, int st, int bits, const uint8_t* data) {
    VSNode* n = (VSNode*)calloc(1, sizeof(VSNode));
    api_query_video_format(&n->vi.format, cf, st, bits, 0, 0, &g_core);
    n->vi.width = w;
    n->vi.height = h;
    n->vi.numFrames = nframes;
    n->vi.fpsNum = 24;
    n->vi.fpsDen = 1;
    n->frames = (VSFrame**)calloc((size_t)nframes, sizeof(VSFrame*));
    const int bps = n->vi.format.bytesPerSample, np = n->vi.format.numPlanes;
    for (int k = 0; k < nframes; k++) {
        VSFrame* f = new_frame(&n->vi.format, w, h);
        for (int p = 0; p < np; p++)
            for (int y = 0; y < h; y++)
                memcpy(f->plane[p] + (size_t)y * f->stride[p], data + (((size_t)k * np + p) * h + y) * (size_t)w * bps,
                       (size_t)w * bps);
        n->frames[k] = f;
    }
    return n;
}

/* Calls registered function `fname` with reference/distorted clips and optional integer,
 * float and string arguments ("key=value" lists, separated by ';'); returns the output clip
 * or NULL with the error copied to `err`. */
VSNode* vsfake_call(const char* fname, VSNode* ref, VSNode* dis, const char* ints, const char* floats, const char* datas,
                    char* err) {
    VSMap* in = api_create_map();
    VSMap* out = api_create_map();
    if (ref) api_map_consume_node(in, "reference", ref, 0);
    if (dis) api_map_consume_node(in, "distorted", dis, 0);
    char buf[1024];
    for (int pass = 0; pass < 3; pass++) {
        const char* list = pass == 0 ? ints : pass == 1 ? floats : datas;
        if (!list || !*list) continue;
        snprintf(buf, sizeof(buf), "%s", list);
        for (char* tok = strtok(buf, ";"); tok; tok = strtok(NULL, ";")) {
            char* eq = strchr(tok, '=');
            if (!eq) continue;
            *eq = 0;
            if (pass == 1) api_map_set_float(in, tok, atof(eq + 1), 0);
            else if (pass == 0) api_map_set_int(in, tok, atoll(eq + 1), 0);
            else api_map_set_data(in, tok, eq + 1, (int)strlen(eq + 1), vsDtUtf8, 0);
        }
    }
    VsAbiPublicFunction fn = NULL;
    for (int k = 0; k < g_nfns; k++)
        if (!strcmp(g_fns[k].name, fname)) fn = g_fns[k].fn;
    VSNode* node = NULL;
    if (!fn) {
        strcpy(err, "no such function");
    } else {
        fn(in, out, NULL, &g_core, &g_api);
        if (out->has_error) strcpy(err, out->error);
        else node = api_map_get_node(out, "clip", 0, NULL);
        Entry* d = find(out, "gpu_human_data");
        if (d && d->type == tData) { strncpy(err, d->data, 4095); err[4095] = 0; }
    }
    api_free_map(in);
    api_free_map(out);
    return node;
}

/* Produces frame n of a filter clip: float property `prop` into *value and, when `plane0` is
 * not NULL, the first plane (w*h floats); returns 0, or -1 with the filter's error in `err`. */
int vsfake_frame(VSNode* node, int n, const char* prop, double* value, float* plane0, char* err) {
    VSFrameContext ctx;
    memset(&ctx, 0, sizeof(ctx));
    void* fd = NULL;
    node->get(n, vsArInitial, node->instance, &fd, &ctx, &g_core, &g_api);
    const VSFrame* f = node->get(n, vsArAllFramesReady, node->instance, &fd, &ctx, &g_core, &g_api);
    if (!f) {
        strcpy(err, ctx.has_error ? ctx.error : "no frame");
        return -1;
    }
    Entry* e = find(&f->props, prop);
    *value = e && e->type == tFloat ? e->f : -1e300;
    if (plane0)
        for (int y = 0; y < f->h; y++) memcpy(plane0 + (size_t)y * f->w, f->plane[0] + (size_t)y * f->stride[0], (size_t)f->w * 4);
    free_frame(f);
    return 0;
}

void vsfake_free_node(VSNode* node) {
    if (node->free_fn) node->free_fn(node->instance, &g_core, &g_api);
    free(node);
}
