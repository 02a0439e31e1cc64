/*
 * tm_oracle.c -- CPU oracle for imageproc's template matching.
 *
 * TEST INFRASTRUCTURE ONLY (see tm_oracle.h). Every function names the lines
 * of imageproc 0.27.0 src/template_matching.rs it restates.
 *
 * Build with -ffp-contract=off: the reference's Rust code never fuses a
 * multiply and an add, so neither may this restatement.
 */
#include "tm_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Argument checks: the reference's assertions, in the reference's order.   */
/* ImageTemplate::new (:394-404) and ImageTemplateMask::new (:432-440).     */
/* ------------------------------------------------------------------------ */
static int check_dims(uint32_t W, uint32_t H, uint32_t w, uint32_t h,
                      const uint8_t *mask, uint32_t mw, uint32_t mh) {
    if (mask && (mw != w || mh != h)) return TMO_ERR_MASK_SIZE;
    if (W < w) return TMO_ERR_TEMPLATE_WIDTH;
    if (H < h) return TMO_ERR_TEMPLATE_HEIGHT;
    return TMO_OK;
}

/* ------------------------------------------------------------------------ */
/* Row-parallel driver: rayon's into_par_iter over output rows (:184-203).  */
/* ------------------------------------------------------------------------ */
typedef void (*row_fn)(void *ctx, uint32_t row);

typedef struct {
    row_fn fn;
    void *ctx;
    uint32_t begin, end;
    int tid, nthreads;
} row_job;

static void *row_worker(void *arg) {
    row_job *j = (row_job *)arg;
    for (uint32_t r = j->begin + (uint32_t)j->tid; r < j->end;
         r += (uint32_t)j->nthreads)
        j->fn(j->ctx, r);
    return NULL;
}

static void run_rows(row_fn fn, void *ctx, uint32_t begin, uint32_t end,
                     int nthreads) {
    if (nthreads <= 1 || end - begin < 2) {
        for (uint32_t r = begin; r < end; ++r) fn(ctx, r);
        return;
    }
    if ((uint32_t)nthreads > end - begin) nthreads = (int)(end - begin);
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    row_job *jobs = (row_job *)malloc(sizeof(row_job) * (size_t)nthreads);
    for (int t = 0; t < nthreads; ++t) {
        jobs[t] = (row_job){fn, ctx, begin, end, t, nthreads};
        pthread_create(&th[t], NULL, row_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(th);
    free(jobs);
}

/* ------------------------------------------------------------------------ */
/* Reference f32 arithmetic.                                                 */
/* ------------------------------------------------------------------------ */
typedef struct {
    const uint8_t *image, *templ, *mask;
    uint32_t W, w, h, Wo, row_begin;
    int method;
    float tss; /* square_sum / mult_square_sum, f32 (:378-386) */
    float *out;
} ref_ctx;

/* methods::*::score_at for one output pixel. The closure bodies are
 * :223 (SSE), :245-246 (SSE-norm), :264 (CCORR), :286-287 (CCORR-norm),
 * :305 (masked SSE), :328-329, :346, :369-370 (masked), and the final
 * normalisation :249-250 / :290-291 / :332-333 / :373-374. The walk is
 * dy-outer, dx-inner (:410-416 / :447-454). */
static float ref_score_at(const ref_ctx *c, uint32_t x, uint32_t y) {
    const uint32_t W = c->W, w = c->w, h = c->h;
    float score = 0.0f, ii = 0.0f;
    if (!c->mask) {
        for (uint32_t dy = 0; dy < h; ++dy) {
            const uint8_t *irow = c->image + (size_t)(y + dy) * W + x;
            const uint8_t *trow = c->templ + (size_t)dy * w;
            for (uint32_t dx = 0; dx < w; ++dx) {
                const float i = (float)irow[dx];
                const float t = (float)trow[dx];
                switch (c->method) {
                case TMO_SSE: {
                    const float d = t - i;
                    score = score + d * d;
                } break;
                case TMO_SSE_NORMALIZED: {
                    const float d = t - i;
                    score = score + d * d;
                    ii = ii + i * i;
                } break;
                case TMO_CCORR:
                    score = score + i * t;
                    break;
                default:
                    score = score + i * t;
                    ii = ii + i * i;
                    break;
                }
            }
        }
        if (c->method == TMO_SSE_NORMALIZED ||
            c->method == TMO_CCORR_NORMALIZED) {
            const float norm = sqrtf(ii * c->tss);
            return norm > 0.0f ? score / norm : score;
        }
        return score;
    }
    for (uint32_t dy = 0; dy < h; ++dy) {
        const uint8_t *irow = c->image + (size_t)(y + dy) * W + x;
        const uint8_t *trow = c->templ + (size_t)dy * w;
        const uint8_t *mrow = c->mask + (size_t)dy * w;
        for (uint32_t dx = 0; dx < w; ++dx) {
            const float i = (float)irow[dx];
            const float t = (float)trow[dx];
            const float m = (float)mrow[dx];
            switch (c->method) {
            case TMO_SSE: {
                const float e = (t - i) * m;
                score = score + e * e;
            } break;
            case TMO_SSE_NORMALIZED: {
                const float e = (t - i) * m;
                score = score + e * e;
                const float q = i * m;
                ii = ii + q * q;
            } break;
            case TMO_CCORR:
                score = score + ((t * i) * m) * m;
                break;
            default: {
                score = score + ((t * i) * m) * m;
                const float q = i * m;
                ii = ii + q * q;
            } break;
            }
        }
    }
    if (c->method == TMO_SSE_NORMALIZED || c->method == TMO_CCORR_NORMALIZED) {
        /* (template_mask_squared_sum * im_im).sqrt() */
        const float norm = sqrtf(c->tss * ii);
        return norm > 0.0f ? score / norm : score;
    }
    return score;
}

static void ref_row(void *ctx, uint32_t y) {
    const ref_ctx *c = (const ref_ctx *)ctx;
    float *o = c->out + (size_t)(y - c->row_begin) * c->Wo;
    for (uint32_t x = 0; x < c->Wo; ++x) o[x] = ref_score_at(c, x, y);
}

int tmo_match_reference(const uint8_t *image, uint32_t W, uint32_t H,
                        const uint8_t *templ, uint32_t w, uint32_t h,
                        const uint8_t *mask, uint32_t mw, uint32_t mh,
                        int method, float *out, uint32_t row_begin,
                        uint32_t row_end, int nthreads) {
    int st = check_dims(W, H, w, h, mask, mw, mh);
    if (st) return st;
    if (method < 0 || method > 3) return TMO_ERR_INVALID_ARGUMENT;
    const uint32_t Wo = W - w + 1, Ho = H - h + 1;
    if (row_end > Ho) row_end = Ho;
    if (row_begin > row_end) return TMO_ERR_INVALID_ARGUMENT;
    ref_ctx c = {image, templ, mask, W, w, h, Wo, row_begin, method, 0.0f,
                 out};
    /* square_sum (:378-380) / mult_square_sum (:381-386): sequential f32
     * sums in raw-buffer order. */
    float acc = 0.0f;
    for (size_t k = 0; k < (size_t)w * h; ++k) {
        const float t = (float)templ[k];
        if (mask) {
            const float p = t * (float)mask[k];
            acc = acc + p * p;
        } else {
            acc = acc + t * t;
        }
    }
    c.tss = acc;
    run_rows(ref_row, &c, row_begin, row_end, nthreads);
    return TMO_OK;
}

/* ------------------------------------------------------------------------ */
/* Exact integer sums.                                                       */
/*   unmasked: X = sum I*T,      Y = sum I^2,        TSS = sum T^2           */
/*   masked:   X = sum I*T*m^2,  Y = sum I^2*m^2,    TSS = sum (T*m)^2       */
/* so that CCORR = X, SSE = Y - 2X + TSS and norm = sqrt(Y * TSS) for every  */
/* method of MatchTemplateMethod (:8-64) with and without a mask.           */
/* ------------------------------------------------------------------------ */
typedef struct {
    const uint8_t *image;
    uint32_t W, w, h, Wo;
    const uint32_t *U, *V; /* per template pixel: T*m^2 and m^2 (or T, 1) */
    uint64_t *X, *Y;
} sums_ctx;

static void sums_row(void *ctx, uint32_t y) {
    const sums_ctx *c = (const sums_ctx *)ctx;
    uint64_t *ax = (uint64_t *)calloc(c->Wo ? c->Wo : 1, sizeof(uint64_t));
    uint64_t *ay = (uint64_t *)calloc(c->Wo ? c->Wo : 1, sizeof(uint64_t));
    for (uint32_t dy = 0; dy < c->h; ++dy) {
        for (uint32_t dx = 0; dx < c->w; ++dx) {
            const uint64_t u = c->U[(size_t)dy * c->w + dx];
            const uint64_t v = c->V[(size_t)dy * c->w + dx];
            const uint8_t *row = c->image + (size_t)(y + dy) * c->W + dx;
            for (uint32_t x = 0; x < c->Wo; ++x) {
                const uint64_t i = row[x];
                ax[x] += i * u;
                ay[x] += i * i * v;
            }
        }
    }
    if (c->X) memcpy(c->X + (size_t)y * c->Wo, ax, sizeof(uint64_t) * c->Wo);
    if (c->Y) memcpy(c->Y + (size_t)y * c->Wo, ay, sizeof(uint64_t) * c->Wo);
    free(ax);
    free(ay);
}

int tmo_sums(const uint8_t *image, uint32_t W, uint32_t H,
             const uint8_t *templ, uint32_t w, uint32_t h,
             const uint8_t *mask, uint64_t *X, uint64_t *Y, uint64_t *tss,
             int nthreads) {
    int st = check_dims(W, H, w, h, NULL, 0, 0);
    if (st) return st;
    const size_t n = (size_t)w * h;
    uint32_t *U = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *V = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint64_t t2 = 0;
    for (size_t k = 0; k < n; ++k) {
        const uint32_t t = templ[k];
        const uint32_t m = mask ? mask[k] : 1u;
        U[k] = t * m * m;
        V[k] = m * m;
        t2 += (uint64_t)(t * m) * (t * m);
    }
    if (tss) *tss = t2;
    sums_ctx c = {image, W, w, h, W - w + 1, U, V, X, Y};
    run_rows(sums_row, &c, 0, H - h + 1, nthreads);
    free(U);
    free(V);
    return TMO_OK;
}

/* The per-pixel epilogue. FP64: the sqrt of Y*TSS and the divide in double,
 * rounded once to f32. F32: the reference's own normalisation sequence
 * (`(ii * tss).sqrt()` then `score / norm`, :249-250) applied to the exact
 * sums converted to f32. Zero norm returns the raw score (:250). */
float tmo_finish(int method, int precision, uint64_t X, uint64_t Y,
                 uint64_t tss) {
    const int sse = (method == TMO_SSE || method == TMO_SSE_NORMALIZED);
    const int norm = (method == TMO_SSE_NORMALIZED ||
                      method == TMO_CCORR_NORMALIZED);
    const uint64_t score = sse ? (Y + tss - 2u * X) : X;
    if (!norm) return (float)score;
    if (precision == TMO_PRECISION_EXACT_FP64) {
        const double n = sqrt((double)Y * (double)tss);
        return n > 0.0 ? (float)((double)score / n) : (float)score;
    }
    const float s = (float)score;
    const float n = sqrtf((float)Y * (float)tss);
    return n > 0.0f ? s / n : s;
}

int tmo_match_exact(const uint8_t *image, uint32_t W, uint32_t H,
                    const uint8_t *templ, uint32_t w, uint32_t h,
                    const uint8_t *mask, uint32_t mw, uint32_t mh,
                    int method, int precision, float *out, int nthreads) {
    int st = check_dims(W, H, w, h, mask, mw, mh);
    if (st) return st;
    if (method < 0 || method > 3) return TMO_ERR_INVALID_ARGUMENT;
    const size_t n = (size_t)(W - w + 1) * (H - h + 1);
    uint64_t *X = (uint64_t *)malloc(sizeof(uint64_t) * n);
    uint64_t *Y = (uint64_t *)malloc(sizeof(uint64_t) * n);
    uint64_t tss = 0;
    tmo_sums(image, W, H, templ, w, h, mask, X, Y, &tss, nthreads);
    for (size_t k = 0; k < n; ++k)
        out[k] = tmo_finish(method, precision, X[k], Y[k], tss);
    free(X);
    free(Y);
    return TMO_OK;
}

/* ------------------------------------------------------------------------ */
/* find_extremes (:479-511): seed from (0,0), strict < and > in row-major    */
/* order, so the first occurrence wins and a NaN seed is never replaced.     */
/* ------------------------------------------------------------------------ */
#define SCAN(T)                                                              \
    do {                                                                     \
        const T *p = (const T *)image;                                       \
        T mn = p[0], mx = p[0];                                              \
        for (uint64_t k = 0; k < n; ++k) {                                   \
            if (p[k] < mn) { mn = p[k]; *min_index = k; }                    \
            if (p[k] > mx) { mx = p[k]; *max_index = k; }                    \
        }                                                                    \
    } while (0)

int tmo_find_extremes_index(const void *image, uint32_t W, uint32_t H,
                            int type, uint64_t *max_index,
                            uint64_t *min_index) {
    if (W == 0 || H == 0) return TMO_ERR_EMPTY_IMAGE;
    const uint64_t n = (uint64_t)W * H;
    *max_index = 0;
    *min_index = 0;
    switch (type) {
    case 0: SCAN(uint8_t); break;
    case 1: SCAN(uint16_t); break;
    case 2: SCAN(uint32_t); break;
    case 3: SCAN(uint64_t); break;
    case 4: SCAN(int8_t); break;
    case 5: SCAN(int16_t); break;
    case 6: SCAN(int32_t); break;
    case 7: SCAN(int64_t); break;
    case 8: SCAN(float); break;
    case 9: SCAN(double); break;
    default: return TMO_ERR_INVALID_ARGUMENT;
    }
    return TMO_OK;
}

static double load_as_double(const void *image, int type, uint64_t k) {
    switch (type) {
    case 0: return ((const uint8_t *)image)[k];
    case 1: return ((const uint16_t *)image)[k];
    case 2: return ((const uint32_t *)image)[k];
    case 3: return (double)((const uint64_t *)image)[k];
    case 4: return ((const int8_t *)image)[k];
    case 5: return ((const int16_t *)image)[k];
    case 6: return ((const int32_t *)image)[k];
    case 7: return (double)((const int64_t *)image)[k];
    case 8: return ((const float *)image)[k];
    default: return ((const double *)image)[k];
    }
}

int tmo_find_extremes(const void *image, uint32_t W, uint32_t H, int type,
                      tmo_extremes *out) {
    uint64_t imax = 0, imin = 0;
    int st = tmo_find_extremes_index(image, W, H, type, &imax, &imin);
    if (st) return st;
    out->max_value = load_as_double(image, type, imax);
    out->min_value = load_as_double(image, type, imin);
    out->max_x = (uint32_t)(imax % W);
    out->max_y = (uint32_t)(imax / W);
    out->min_x = (uint32_t)(imin % W);
    out->min_y = (uint32_t)(imin / W);
    return TMO_OK;
}
