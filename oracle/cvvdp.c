/*
 * cvvdp.c -- FP64 CPU restatement of Vship's CVVDP (src/cvvdp/*.hpp).
 *
 * TEST INFRASTRUCTURE ONLY: the checker the CUDA CVVDP engine is compared against; the
 * product never links, loads or calls it.  Stateful like the reference's
 * CVVDPComputingImplementation (src/cvvdp/main.hpp:161-398): a ring of past frames per
 * clip, the temporal score accumulator, and the same reset semantics.
 *
 * Input frames are planar linear RGB in the clip's own primaries at the metric size (what
 * the reference's Converter delivers with destination linRGB; oracle_convert_native makes
 * them from raw planes).  Pixel arithmetic is in double.  The small host-side quantities the
 * reference forms in float before any pixel is touched (pixels per degree, pyramid depth,
 * band frequencies, temporal filter taps, per-band CSF tables, the pyramid kernel) are formed
 * in float here too, so that integer decisions (number of bands) and table interpolation
 * follow the reference exactly.  Reference quirks kept: the swapped interpolation weights of
 * the CSF lookup (csf.hpp:73), the frame count used before it is incremented in the temporal
 * pooling (main.hpp:379-385), the mixed mirror padding of the pyramid kernels
 * (lpyr.hpp:21-25, 66-71), the halved last coefficient of the inverse real DFT
 * (temporalFilter.hpp:8-12).  One deliberate difference: a background luminance above the
 * table's range clamps to the last table entry (the reference reads past the table).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/VshipColor.h"
#include "../vship_b200/csrc/cvvdp_csf_table.h"

#define ORACLE_API __attribute__((visibility("default")))
#define CV_PI 3.14159265359 /* the reference's PI (src/util/preprocessor.hpp:83) */

void oracle_resize_transpose(const double* src, int64_t sw, int64_t sh, int64_t rw, double* dst);

/* Model constants (src/cvvdp/parameters.hpp:5-68). */
static const double mask_p = 2.264355182647705, mask_c = -0.7954971194267273;
static const double sensitivity_correction = -0.2797423303127289;
static const double jod_a = 0.0439569391310215, jod_exp = 0.9302042722702026;
static const double mask_q[4] = {1.302622675895691, 2.8885908126831055, 3.6807713508605957, 3.588787317276001};
static const double ch_chrom_w = 1.0, ch_trans_w = 0.8081134557723999;
static const float sigma_tf[4] = {5.79336f, 14.1255f, 6.63661f, 0.12314f};
static const float beta_tf[4] = {1.3314f, 1.1196f, 0.947901f, 0.1898f};
static const double xcm_weights[16] = {
    -0.18950104713439941, -5.962151050567627, -4.31834602355957, -1.9321587085723877,
    2.5655593872070312,   0.34406712651252747, -2.719646453857422, -0.4970424771308899,
    3.8118371963500977,   -1.0051705837249756, -0.5193376541137695, -0.5653647780418396,
    -7.054771423339844,   -5.527150630950928, -3.5106418132781982, -2.08804988861084};
static const double baseband_weight[4] = {0.0036334486212581396, 1.6627724170684814, 4.11874532699585, 25.25969886779785};
static const double d_max = 2.5642454624176025, image_int = 0.577918291091919;

#define CV_MAX_LEVELS 14

typedef struct oracle_cvvdp {
    int64_t sw, sh, rw, rh, mw, mh;
    int taps;
    double filt[4][64];
    double* ring[2];            /* [taps][3][mw*mh] per clip */
    int ind0, tsize;
    int levels;
    int64_t lw[CV_MAX_LEVELS], lh[CV_MAX_LEVELS];
    float band_freq[CV_MAX_LEVELS];
    float csf[CV_MAX_LEVELS][4][32]; /* log10 S over the luminance axis, per band and channel */
    float lum_log[32];
    int hdr;
    double y_peak, y_black, y_refl, exposure;
    int trc[2], prim[2];
    int num_frame;
    double sq_sum;
    double vals[CV_MAX_LEVELS * 4];
    double q;
} oracle_cvvdp;

/* ---- display model (display_models.hpp:153-170) ---------------------------------------- */
static float screen_ppd(const double m[10]) {
    const float res0 = (float)m[0], res1 = (float)m[1];
    const float diag = (float)m[4], dist = (float)m[3];
    const float ar = res0 / res1;
    const float height_meter = (float)(sqrt(((double)diag * 25.4) * ((double)diag * 25.4) / (double)(1 + ar * ar)) / 1000);
    const float width_meter = ar * height_meter;
    const float pix_deg = (float)(2 * 180 * atan(0.5 * width_meter / (double)res0 / (double)dist) / CV_PI);
    return 1 / pix_deg;
}

/* get_frequencies (lpyr.hpp:148-161). */
static int band_frequencies(int64_t w, int64_t h, float ppd, float* bf) {
    const float min_freq = 0.2f;
    const int for_res = (int)(log2((double)(w < h ? w : h)) - 1);
    const int for_ppd = (int)(ceil(-log2(2 * min_freq / 0.3228 / (double)ppd)) + 1);
    int levels = for_res < 14 ? for_res : 14;
    if (for_ppd < levels) levels = for_ppd;
    if (levels < 1 || levels > CV_MAX_LEVELS) return levels;
    bf[0] = (float)(0.5 * ppd);
    for (int i = 0; i < levels - 1; i++) bf[i + 1] = (float)(0.3228 * 0.5 * ppd / (double)(float)(1 << i));
    return levels;
}

/* CSF_Handler::init (csf.hpp:23-54): per band and channel, the 32-entry log-sensitivity
 * column at the band's frequency, interpolated linearly in log frequency. */
static void csf_tables(oracle_cvvdp* o) {
    float lut_logrho[32];
    for (int i = 0; i < 32; i++) {
        lut_logrho[i] = log10f(kCsfRho[i]);
        o->lum_log[i] = log10f(kCsfLum[i]);
    }
    for (int b = 0; b < o->levels; b++) {
        const float logrho = log10f(o->band_freq[b]);
        int x0 = 31;
        for (int i = 1; i < 32; i++)
            if (lut_logrho[i] > logrho) { x0 = i - 1; break; }   /* indexSearch, csf.hpp:9-16 */
        if (x0 > 30) x0 = 30;
        const float slope = (logrho - lut_logrho[x0]) / (lut_logrho[x0 + 1] - lut_logrho[x0]);
        for (int c = 0; c < 4; c++)
            for (int i = 0; i < 32; i++) {
                const float y0 = kCsfLogS[c][i][x0], y1 = kCsfLogS[c][i][x0 + 1];
                o->csf[b][c][i] = y0 + (y1 - y0) * slope;
            }
    }
}

/* computeSensitivityGPU (csf.hpp:60-82), with the reference's swapped weights. */
static double sensitivity(const oracle_cvvdp* o, double lbkg, int band, int ch) {
    const double x = log10(lbkg);
    double frac = 31 * (x - o->lum_log[0]) / ((double)o->lum_log[31] - o->lum_log[0]);
    int imin = (int)frac;
    if (imin > 31) imin = 31;
    if (imin < 0) imin = 0;
    const int imax = imin + 1 < 31 ? imin + 1 : 31;
    frac -= imin;
    const float* y = o->csf[band][ch];
    const double logs = y[imin] * frac + y[imax] * (1.0 - frac) + sensitivity_correction / 20.0;
    return pow(10.0, logs);
}

/* TemporalFilter::init and inverseRealFourrierTransform (temporalFilter.hpp:5-73). */
static void temporal_filters(oracle_cvvdp* o, float fps) {
    int size = (int)(ceil(0.25 * fps / 2) * 2) + 1;
    if (size < 1) size = 1;
    o->taps = size;
    const int nf = size / 2 + 1;
    float freq[64], spec[4][64];
    for (int i = 0; i < nf; i++) freq[i] = fps * i / 2;
    for (int j = 0; j < 3; j++)
        for (int i = 0; i < nf; i++) spec[j][i] = expf(-powf(freq[i], beta_tf[j]) / sigma_tf[j]);
    for (int i = 0; i < nf; i++) {
        float t = (float)((double)powf(freq[i], beta_tf[3]) - pow(5, beta_tf[3]));
        t *= t;
        spec[3][i] = expf(-t / sigma_tf[3]);
    }
    for (int j = 0; j < 4; j++) {
        float inp[64], res[64];
        memcpy(inp, spec[j], sizeof(float) * nf);
        if (nf > size / 2) inp[size / 2] /= 2;
        inp[0] /= 2;
        for (int i = 0; i < size; i++) res[i] = 0;
        for (int i = 0; i < size; i++)
            for (int k = 0; k < nf; k++)
            {
                float* r = &res[(i + nf - 1) % size];
                *r = (float)((double)*r + 2 * inp[k] * cos(2 * CV_PI * k * i / size) / size);
            }
        for (int i = 0; i < size; i++) o->filt[j][i] = res[i];
    }
}

/* ---- pyramid (lpyr.hpp:3-95) ------------------------------------------------------------ */
static double pyr_k[5];

static void pyr_kernel_init(void) {
    const float a = 0.4f;
    const float k[5] = {(float)(0.25 - a / 2.), 0.25f, a, 0.25f, (float)(0.25 - a / 2.)};
    for (int i = 0; i < 5; i++) pyr_k[i] = k[i];
}

static void pyr_reduce(const double* src, int64_t w, int64_t h, double* dst) {
    const int64_t nw = (w + 1) / 2, nh = (h + 1) / 2;
    for (int64_t y = 0; y < nh; y++)
        for (int64_t x = 0; x < nw; x++) {
            double v = 0;
            for (int dx = -2; dx <= 2; dx++) {
                int64_t rx = 2 * x + dx;
                if (rx < 0) rx = -rx - 1;
                if (rx >= w) rx = 2 * w - rx - 2;
                for (int dy = -2; dy <= 2; dy++) {
                    int64_t ry = 2 * y + dy;
                    if (ry < 0) ry = -ry - 1;
                    if (ry >= h) ry = 2 * h - ry - 2;
                    v += pyr_k[dx + 2] * pyr_k[dy + 2] * src[ry * w + rx];
                }
            }
            dst[y * nw + x] = v;
        }
}

/* Expansion of a coarse plane to w x h (gaussPyrExpand_Kernel, lpyr.hpp:48-90). */
static double pyr_expand_at(const double* src, int64_t w, int64_t h, int64_t x, int64_t y) {
    const int64_t ow = (w + 1) / 2, oh = (h + 1) / 2;
    double v = 0;
    for (int dx = -2 + (int)(x & 1); dx <= 2; dx += 2) {
        int64_t rx = (x + dx) / 2;
        if (rx < 0) rx = -rx - 1;
        if (rx >= ow) rx = 2 * ow - rx - 2;
        for (int dy = -2 + (int)(y & 1); dy <= 2; dy += 2) {
            int64_t ry = (y + dy) / 2;
            if (ry < 0) ry = -ry - 1;
            if (ry >= oh) ry = 2 * oh - ry - 2;
            v += 2 * pyr_k[dx + 2] * 2 * pyr_k[dy + 2] * src[ry * ow + rx];
        }
    }
    return v;
}

/* ---- per-pixel colour (colors.hpp, main.hpp:327-346) ------------------------------------- */
static double display_encode(const oracle_cvvdp* o, double a, int trc) {
    if (o->hdr && trc == Vship_TRC_PQ) {
        a *= 100.0;
        double lo = o->y_black > 0.005 ? o->y_black : 0.005;
        double v = a * o->exposure < o->y_peak ? a * o->exposure : o->y_peak;
        return (v > lo ? v : lo) + o->y_black + o->y_refl;
    }
    if (o->hdr && trc == Vship_TRC_Linear) {
        double lo = o->y_black > 0.005 ? o->y_black : 0.005;
        double v = a * o->exposure < o->y_peak ? a * o->exposure : o->y_peak;
        return (v > lo ? v : lo) + o->y_refl;
    }
    double c = a * o->exposure;
    c = c < 0 ? 0 : (c > 1 ? 1 : c);
    return (o->y_peak - o->y_black) * c + o->y_black + o->y_refl;
}

static const double* rgb_to_xyz(int prim) { /* primaries.hpp: <P, INTERNAL> matrices */
    static const double st170[9] = {0.39349893, 0.3652766, 0.19162447, 0.2123645, 0.70109542, 0.08654008, 0.01873804, 0.1119396, 0.95812235};
    static const double bg[9] = {0.4305, 0.3416, 0.1783, 0.2220, 0.7067, 0.07132, 0.0202, 0.1296, 0.9391};
    static const double m470[9] = {0.6068, 0.1735, 0.2003, 0.2989, 0.5866, 0.1145, 0.0, 0.06609, 1.116};
    static const double bt709[9] = {0.4124, 0.3576, 0.1805, 0.2126, 0.7152, 0.0722, 0.0193, 0.1192, 0.9505};
    static const double bt2020[9] = {0.6370, 0.1446, 0.1689, 0.2627, 0.6780, 0.0593, 0.0, 0.0281, 1.0610};
    switch (prim) {
    case Vship_PRIMARIES_ST170_M: case Vship_PRIMARIES_ST240_M: return st170;
    case Vship_PRIMARIES_BT470_BG: return bg;
    case Vship_PRIMARIES_BT470_M: return m470;
    case Vship_PRIMARIES_BT709: return bt709;
    case Vship_PRIMARIES_BT2020: return bt2020;
    default: return NULL;
    }
}

static void to_dkl(double v[3], int prim) {
    const double* m = rgb_to_xyz(prim);
    if (m) {
        const double x = m[0] * v[0] + m[1] * v[1] + m[2] * v[2];
        const double y = m[3] * v[0] + m[4] * v[1] + m[5] * v[2];
        const double z = m[6] * v[0] + m[7] * v[1] + m[8] * v[2];
        v[0] = x; v[1] = y; v[2] = z;
    }
    /* xyz_to_LMS2006 and LMS2006_to_DKLd65 (colors.hpp:30-49) */
    const double l = 0.187596268556126 * v[0] + 0.585168649077728 * v[1] - 0.026384263306304 * v[2];
    const double mm = -0.133397430663221 * v[0] + 0.405505777260049 * v[1] + 0.034502127690364 * v[2];
    const double s = 0.000244379021663 * v[0] - 0.000542995890619 * v[1] + 0.019406849066323 * v[2];
    const double a = l + mm;
    v[0] = a;
    v[1] = a - 3.311130179947035 * mm;
    v[2] = 50.977571328718781 * s - a;
}

static double to_jod(double a) { /* distmap_specifics.hpp:5-12 */
    if (a > 0.1) return 10.0 - jod_a * pow(a, jod_exp);
    return 10.0 - jod_a * pow(0.1, jod_exp - 1.0) * a;
}

/* ---- lifecycle --------------------------------------------------------------------------- */
/* model = {res_x, res_y, hdr, viewing_distance_m, diagonal_in, max_luminance, contrast,
 *          E_ambient, k_refl, exposure}; (sw, sh) = metric input size.  Returns NULL when the
 * size gives no pyramid band. */
ORACLE_API oracle_cvvdp* oracle_cvvdp_new(int64_t sw, int64_t sh, double fps, int resize_to_display,
                                          const double model[10], int trc1, int prim1, int trc2, int prim2) {
    pyr_kernel_init();
    oracle_cvvdp* o = (oracle_cvvdp*)calloc(1, sizeof(oracle_cvvdp));
    o->sw = sw; o->sh = sh;
    const int64_t rx = (int64_t)model[0], ry = (int64_t)model[1];
    if (resize_to_display) { /* main.hpp:201-214 */
        if (sw * ry >= sh * rx) { o->rw = rx; o->rh = sh * rx / sw; }
        else { o->rh = ry; o->rw = sw * ry / sh; }
    } else { o->rw = sw; o->rh = sh; }
    o->mw = o->rw < sw ? o->rw : sw;
    o->mh = o->rh < sh ? o->rh : sh;
    o->hdr = model[2] != 0;
    const float max_lum = (float)model[5], contrast = (float)model[6], e_amb = (float)model[7], k_refl = (float)model[8];
    o->y_peak = max_lum;
    o->y_black = (float)(max_lum / contrast);
    o->y_refl = (float)(e_amb * k_refl / CV_PI);
    o->exposure = (float)model[9];
    o->trc[0] = trc1; o->trc[1] = trc2; o->prim[0] = prim1; o->prim[1] = prim2;
    const float ppd = screen_ppd(model);
    o->levels = band_frequencies(o->rw, o->rh, ppd, o->band_freq);
    if (o->levels < 1 || o->levels > CV_MAX_LEVELS) { free(o); return NULL; }
    int64_t w = o->rw, h = o->rh;
    for (int i = 0; i < o->levels; i++) { o->lw[i] = w; o->lh[i] = h; w = (w + 1) / 2; h = (h + 1) / 2; }
    csf_tables(o);
    temporal_filters(o, (float)fps);
    const int64_t n = o->mw * o->mh;
    for (int k = 0; k < 2; k++) o->ring[k] = (double*)calloc((size_t)(o->taps * 3 * n), sizeof(double));
    return o;
}

ORACLE_API void oracle_cvvdp_free(oracle_cvvdp* o) {
    if (!o) return;
    free(o->ring[0]);
    free(o->ring[1]);
    free(o);
}

ORACLE_API void oracle_cvvdp_info(const oracle_cvvdp* o, int64_t* out) {
    out[0] = o->rw; out[1] = o->rh; out[2] = o->levels; out[3] = o->taps; out[4] = o->mw; out[5] = o->mh;
}

ORACLE_API void oracle_cvvdp_filters(const oracle_cvvdp* o, double* out) {
    for (int j = 0; j < 4; j++)
        for (int i = 0; i < o->taps; i++) out[j * o->taps + i] = o->filt[j][i];
}

/* flushTemporalRing (only_score = 0) and flushOnlyScore (main.hpp:389-397). */
ORACLE_API void oracle_cvvdp_reset(oracle_cvvdp* o, int only_score) {
    o->num_frame = 0;
    o->sq_sum = 0;
    if (!only_score) o->tsize = 0;
}

static double* slot(oracle_cvvdp* o, int img, int age) {
    if (age >= o->tsize) age = o->tsize - 1;
    return o->ring[img] + (int64_t)((o->ind0 + age) % o->taps) * 3 * o->mw * o->mh;
}

/* loadImageToRing (main.hpp:234-347) for both clips; lin1/lin2 are 3 x sh x sw. */
static void load_frame(oracle_cvvdp* o, const double* lin1, const double* lin2) {
    o->tsize = o->tsize + 1 < o->taps ? o->tsize + 1 : o->taps;
    o->ind0 = (o->ind0 + o->taps - 1) % o->taps;
    const int64_t sw = o->sw, sh = o->sh, n = o->mw * o->mh;
    const int down = (o->sw != o->rw || o->sh != o->rh) && sw > o->rw;
    for (int k = 0; k < 2; k++) {
        const double* lin = k ? lin2 : lin1;
        double* dst = slot(o, k, 0);
        if (down) {
            double* tmp = (double*)malloc(sizeof(double) * o->rw * sh);
            for (int c = 0; c < 3; c++) {
                oracle_resize_transpose(lin + c * sw * sh, sw, sh, o->rw, tmp);
                oracle_resize_transpose(tmp, sh, o->rw, o->rh, dst + c * n);
            }
            free(tmp);
        } else {
            memcpy(dst, lin, sizeof(double) * 3 * n);
        }
        for (int64_t i = 0; i < n; i++) {
            double v[3];
            for (int c = 0; c < 3; c++) v[c] = display_encode(o, dst[c * n + i], o->trc[k]);
            to_dkl(v, o->prim[k]);
            for (int c = 0; c < 3; c++) dst[c * n + i] = v[c];
        }
    }
}

/* One clip's Laplacian contrast pyramid (LpyrManager, lpyr.hpp:177-244) from its four
 * temporal channels at level 0.  con[c][level] receives the contrast planes; lbkg[level]
 * the background luminance (levels < L-1), lbkg_mean the baseband mean. */
typedef struct {
    double* con[4][CV_MAX_LEVELS];
    double* lbkg[CV_MAX_LEVELS];
    double mean;
} pyramid;

static void build_pyramid(const oracle_cvvdp* o, double* g0[4], pyramid* p) {
    double* g[4];
    for (int c = 0; c < 4; c++) g[c] = g0[c];
    for (int i = 0; i < o->levels; i++) {
        const int64_t w = o->lw[i], h = o->lh[i], n = w * h;
        if (i < o->levels - 1) {
            double* next[4];
            for (int c = 0; c < 4; c++) {
                next[c] = (double*)malloc(sizeof(double) * ((w + 1) / 2) * ((h + 1) / 2));
                pyr_reduce(g[c], w, h, next[c]);
            }
            double* lb = (double*)malloc(sizeof(double) * n);
            for (int64_t y = 0; y < h; y++)
                for (int64_t x = 0; x < w; x++) {
                    const double e = pyr_expand_at(next[0], w, h, x, y);
                    lb[y * w + x] = e > 0.01 ? e : 0.01;
                }
            const double mult = i == 0 ? 1.0 : 2.0;
            for (int c = 0; c < 4; c++) {
                double* out = (double*)malloc(sizeof(double) * n);
                for (int64_t y = 0; y < h; y++)
                    for (int64_t x = 0; x < w; x++) {
                        const int64_t j = y * w + x;
                        const double layer = c == 0 ? g[0][j] - lb[j] : g[c][j] - pyr_expand_at(next[c], w, h, x, y);
                        const double den = lb[j] > 0.01 ? lb[j] : 0.01;
                        const double con = layer / den;
                        out[j] = (con < 1000.0 ? con : 1000.0) * mult;
                    }
                p->con[c][i] = out;
            }
            p->lbkg[i] = lb;
            for (int c = 0; c < 4; c++) {
                if (g[c] != g0[c]) free(g[c]);
                g[c] = next[c];
            }
        } else {
            double s = 0;
            for (int64_t j = 0; j < n; j++) s += g[0][j];
            p->mean = s / (double)n;
            const double den = p->mean > 0.01 ? p->mean : 0.01;
            for (int c = 0; c < 4; c++) {
                double* out = (double*)malloc(sizeof(double) * n);
                for (int64_t j = 0; j < n; j++) {
                    const double con = g[c][j] / den;
                    out[j] = con < 1000.0 ? con : 1000.0;
                }
                p->con[c][i] = out;
            }
            p->lbkg[i] = NULL;
            for (int c = 0; c < 4; c++)
                if (g[c] != g0[c]) free(g[c]);
        }
    }
}

static void free_pyramid(const oracle_cvvdp* o, pyramid* p) {
    for (int i = 0; i < o->levels; i++) {
        for (int c = 0; c < 4; c++) free(p->con[c][i]);
        free(p->lbkg[i]);
    }
}

/* Renormalised 17-tap Gaussian of sigma 3 with zero padding (gaussianBlur.hpp:5-119). */
static void mask_blur(const double* src, double* dst, int64_t w, int64_t h) {
    double g[17];
    for (int i = 0; i < 17; i++) g[i] = exp(-(double)((8 - i) * (8 - i)) / (2.0 * 3.0 * 3.0));
    double* tmp = (double*)malloc(sizeof(double) * w * h);
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x < w; x++) {
            double s = 0, t = 0;
            for (int i = 0; i < 17; i++) {
                const int64_t xx = x - 8 + i;
                if (xx < 0 || xx >= w) continue;
                s += g[i] * src[y * w + xx];
                t += g[i];
            }
            tmp[y * w + x] = s / t;
        }
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x < w; x++) {
            double s = 0, t = 0;
            for (int i = 0; i < 17; i++) {
                const int64_t yy = y - 8 + i;
                if (yy < 0 || yy >= h) continue;
                s += g[i] * tmp[yy * w + x];
                t += g[i];
            }
            dst[y * w + x] = s / t;
        }
    free(tmp);
}

/* CVVDPprocess (main.hpp:24-158) on the ring's current content; fills o->vals / o->q and,
 * when `dmap` is not NULL, the rw x rh distortion map (distmap_specifics.hpp:47-71). */
static void process(oracle_cvvdp* o, double* dmap) {
    const int64_t mw = o->mw, mh = o->mh, mn = mw * mh, rw = o->rw, rh = o->rh, rn = rw * rh;
    const int L = o->levels;
    pyramid pyr[2];
    for (int k = 0; k < 2; k++) {
        double* ch[4];
        for (int c = 0; c < 4; c++) ch[c] = (double*)calloc((size_t)(mn > rn ? mn : rn), sizeof(double));
        /* temporalConvolutionKernel_d (temporalFilter.hpp:150-193) */
        for (int64_t i = 0; i < mn; i++) {
            if (o->tsize == 1) {
                const double* f = slot(o, k, 0);
                ch[0][i] = f[i]; ch[1][i] = f[mn + i]; ch[2][i] = f[2 * mn + i]; ch[3][i] = 0.0;
                continue;
            }
            double ys = 0, yt = 0, rg = 0, yv = 0;
            for (int t = 0; t < o->taps; t++) {
                const double* f = slot(o, k, t);
                ys += o->filt[0][t] * f[i];
                yt += o->filt[3][t] * f[i];
                rg += o->filt[1][t] * f[mn + i];
                yv += o->filt[2][t] * f[2 * mn + i];
            }
            ch[0][i] = ys; ch[1][i] = rg; ch[2][i] = yv; ch[3][i] = yt;
        }
        if (mw < rw) { /* main.hpp:71-82 */
            double* tmp = (double*)malloc(sizeof(double) * rw * mh);
            double* big = (double*)malloc(sizeof(double) * rn);
            for (int c = 0; c < 4; c++) {
                oracle_resize_transpose(ch[c], mw, mh, rw, tmp);
                oracle_resize_transpose(tmp, mh, rw, rh, big);
                memcpy(ch[c], big, sizeof(double) * rn);
            }
            free(tmp);
            free(big);
        }
        build_pyramid(o, ch, &pyr[k]);
        for (int c = 0; c < 4; c++) free(ch[c]);
    }
    const double powmaskc = pow(10.0, mask_c), max_v = pow(10.0, d_max);
    const double ch_w[4] = {1.0, ch_chrom_w, ch_chrom_w, ch_trans_w};
    double* dplanes[CV_MAX_LEVELS][4];
    for (int b = 0; b < L; b++) {
        const int64_t w = o->lw[b], h = o->lh[b], n = w * h;
        for (int c = 0; c < 4; c++) dplanes[b][c] = (double*)malloc(sizeof(double) * n);
        if (b < L - 1) {
            double* R[4];
            double* T[4];
            double* M[4];
            for (int c = 0; c < 4; c++) {
                R[c] = (double*)malloc(sizeof(double) * n);
                T[c] = (double*)malloc(sizeof(double) * n);
                M[c] = (double*)malloc(sizeof(double) * n);
                const double gain = c == 1 ? 1.45 : 1.0;
                for (int64_t j = 0; j < n; j++) { /* preGaussianPreCompute_kernel (maskingModel.hpp:5-15) */
                    const double s = sensitivity(o, pyr[0].lbkg[b][j], b, c) * gain;
                    R[c][j] = pyr[0].con[c][b][j] * s;
                    T[c][j] = pyr[1].con[c][b][j] * s;
                }
                double* mn_in = (double*)malloc(sizeof(double) * n);
                for (int64_t j = 0; j < n; j++) mn_in[j] = fmin(fabs(R[c][j]), fabs(T[c][j]));
                mask_blur(mn_in, M[c], w, h);
                free(mn_in);
            }
            for (int64_t j = 0; j < n; j++) { /* computeD_Kernel (maskingModel.hpp:28-96) */
                double cm[4];
                for (int c = 0; c < 4; c++) cm[c] = pow(powmaskc * fabs(M[c][j]), mask_q[c]);
                for (int c = 0; c < 4; c++) {
                    double cmask = 0;
                    for (int k = 0; k < 4; k++) cmask += cm[k] * pow(2.0, xcm_weights[k * 4 + c]);
                    const double du = pow(fabs(R[c][j] - T[c][j]), mask_p) / (1 + cmask);
                    dplanes[b][c][j] = max_v * du / (max_v + du) * ch_w[c];
                }
            }
            for (int c = 0; c < 4; c++) { free(R[c]); free(T[c]); free(M[c]); }
        } else {
            for (int c = 0; c < 4; c++) { /* computeD_baseband_kernel (maskingModel.hpp:106-114) */
                const double s = sensitivity(o, pyr[0].mean, b, c);
                for (int64_t j = 0; j < n; j++)
                    dplanes[b][c][j] = fabs(pyr[0].con[c][b][j] - pyr[1].con[c][b][j]) * s * baseband_weight[c];
            }
        }
        for (int c = 0; c < 4; c++) { /* computeMean<2> (pooling.hpp:54-85) */
            double s = 0;
            for (int64_t j = 0; j < n; j++) s += dplanes[b][c][j] * dplanes[b][c][j];
            o->vals[b * 4 + c] = sqrt(s / (double)n);
        }
    }
    double q = 0;
    for (int i = 0; i < 4 * L; i++) q += pow(o->vals[i], 4);
    o->q = pow(q, 0.25);
    if (dmap) {
        double* m[CV_MAX_LEVELS];
        for (int b = 0; b < L; b++) { /* mergeChromaNorm_Kernel */
            const int64_t n = o->lw[b] * o->lh[b];
            const double div = (b == 0 || b == L - 1) ? 1.0 : 2.0;
            m[b] = (double*)malloc(sizeof(double) * n);
            for (int64_t j = 0; j < n; j++) {
                double s = 0;
                for (int c = 0; c < 4; c++) s += pow(dplanes[b][c][j], 4);
                m[b][j] = pow(s * 0.25, 0.25) / div;
            }
        }
        for (int b = L - 2; b >= 0; b--) /* reconstruction, getDistMap */
            for (int64_t y = 0; y < o->lh[b]; y++)
                for (int64_t x = 0; x < o->lw[b]; x++)
                    m[b][y * o->lw[b] + x] += pyr_expand_at(m[b + 1], o->lw[b], o->lh[b], x, y);
        for (int64_t j = 0; j < rn; j++) dmap[j] = 1.0 - to_jod(m[0][j]) * 0.1;
        for (int b = 0; b < L; b++) free(m[b]);
    }
    for (int b = 0; b < L; b++)
        for (int c = 0; c < 4; c++) free(dplanes[b][c]);
    free_pyramid(o, &pyr[0]);
    free_pyramid(o, &pyr[1]);
}

/* Vship_LoadTemporalCVVDP (compute = 0) or Vship_ComputeCVVDP (compute = 1, run(),
 * main.hpp:376-388).  Returns the JOD score through *score when computing. */
ORACLE_API void oracle_cvvdp_frame(oracle_cvvdp* o, const double* lin1, const double* lin2, int compute,
                                   double* score, double* dmap) {
    load_frame(o, lin1, lin2);
    if (!compute) return;
    process(o, dmap);
    o->sq_sum += o->q * o->q;
    const double resq = o->num_frame == 0 ? o->q * image_int : sqrt(o->sq_sum / (double)o->num_frame);
    o->num_frame++;
    *score = to_jod(resq);
}

/* Per-band, per-channel pooled distortions of the last computed frame and their 4-norm. */
ORACLE_API double oracle_cvvdp_bands(const oracle_cvvdp* o, double* vals) {
    for (int i = 0; i < 4 * o->levels; i++) vals[i] = o->vals[i];
    return o->q;
}
