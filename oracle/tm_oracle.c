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

/* ------------------------------------------------------------------------ */
/* Fast exact form for unmasked templates (full-size parity checks).         */
/* The same sums as tmo_sums: X = sum I*T over the window (:260-268 with     */
/* exact integers), Y = sum I^2 over the window, read from the exclusive     */
/* u64 integral image of I^2 (src/integral_image.rs:11-22), TSS = sum T^2.   */
/* Only the loop order differs: per output row and template row, X gains    */
/* the row correlation, 32 outputs at a time with AVX2 where the CPU has it. */
/* ------------------------------------------------------------------------ */
/* acc[x] += sum over dx < w of irow[x + dx] * trow[dx], x < n. */
static void row_corr_scalar(uint32_t *acc, const uint8_t *irow, const uint8_t *trow, uint32_t w,
                            uint32_t x0, uint32_t n) {
    for (uint32_t dx = 0; dx < w; ++dx) {
        const uint32_t t = trow[dx];
        if (!t) continue;
        for (uint32_t x = x0; x < n; ++x) acc[x] += irow[x + dx] * t;
    }
}

#if defined(__x86_64__)
#include <immintrin.h>
/* The same sums from a pair row: prow[x] holds the 16-bit pair
 * (I[x], I[x+1]) (I[W] read as 0), so one multiply-add of 16-bit pairs into
 * 32-bit lanes adds I[x+dx]*T[dx] + I[x+dx+1]*T[dx+1] for eight outputs at
 * once (every product and pair sum is exact: 2 * 255 * 255 < 2^31). 32
 * outputs per block keep their sums in registers across the template row;
 * tpair[k] holds (T[2k], T[2k+1]) with T[w] = 0. */
__attribute__((target("avx2")))
static void row_corr_avx2(uint32_t *acc, const uint32_t *prow, const uint32_t *tpair, uint32_t w,
                          uint32_t n) {
    const uint32_t npairs = (w + 1) / 2;
    const uint32_t n32 = n & ~31u;
    for (uint32_t x0 = 0; x0 < n32; x0 += 32) {
        __m256i a0 = _mm256_setzero_si256(), a1 = a0, a2 = a0, a3 = a0;
        for (uint32_t k = 0; k < npairs; ++k) {
            if (!tpair[k]) continue;
            const __m256i t = _mm256_set1_epi32((int32_t)tpair[k]);
            const uint32_t *q = prow + x0 + 2 * k;
            a0 = _mm256_add_epi32(a0, _mm256_madd_epi16(_mm256_loadu_si256((const __m256i *)q), t));
            a1 = _mm256_add_epi32(a1, _mm256_madd_epi16(_mm256_loadu_si256((const __m256i *)(q + 8)), t));
            a2 = _mm256_add_epi32(a2, _mm256_madd_epi16(_mm256_loadu_si256((const __m256i *)(q + 16)), t));
            a3 = _mm256_add_epi32(a3, _mm256_madd_epi16(_mm256_loadu_si256((const __m256i *)(q + 24)), t));
        }
        __m256i *d = (__m256i *)(acc + x0);
        _mm256_storeu_si256(d, _mm256_add_epi32(_mm256_loadu_si256(d), a0));
        _mm256_storeu_si256(d + 1, _mm256_add_epi32(_mm256_loadu_si256(d + 1), a1));
        _mm256_storeu_si256(d + 2, _mm256_add_epi32(_mm256_loadu_si256(d + 2), a2));
        _mm256_storeu_si256(d + 3, _mm256_add_epi32(_mm256_loadu_si256(d + 3), a3));
    }
    for (uint32_t x = n32; x < n; ++x) {
        uint32_t v = 0;
        for (uint32_t k = 0; k < npairs; ++k) {
            const uint32_t pr = prow[x + 2 * k], tp = tpair[k];
            v += (pr & 0xFFFFu) * (tp & 0xFFFFu) + (pr >> 16) * (tp >> 16);
        }
        acc[x] += v;
    }
}
#endif

static int have_avx2(void) {
#if defined(__x86_64__)
    static int v = -1;
    if (v < 0) v = __builtin_cpu_supports("avx2") ? 1 : 0;
    return v;
#else
    return 0;
#endif
}

typedef struct {
    const uint8_t *image;
    const uint8_t *templ;   /* n templates of w x h, back to back */
    const uint64_t *sat;    /* (W+1) x (H+1) exclusive sums of I^2 */
    const uint32_t *prows;  /* per image row: the pair row (AVX2 form), or NULL */
    const uint32_t *tpairs; /* per template and row: (w+1)/2 column pairs */
    const uint64_t *tss;    /* per template: sum of T^2 */
    uint32_t W, w, h, Wo, n, row_begin, row_end;
    int method, precision, nthreads;
    float *out;             /* n maps of (row_end - row_begin) x Wo, or NULL */
    /* per thread and template: best (value, index) of min and max */
    float *tmin, *tmax;
    uint64_t *imin, *imax;
} fast_ctx;

typedef struct {
    fast_ctx *c;
    int tid;
} fast_job;

static void *fast_worker(void *arg) {
    const fast_job *j = (const fast_job *)arg;
    fast_ctx *c = j->c;
    uint32_t *acc = (uint32_t *)malloc(sizeof(uint32_t) * (c->Wo ? c->Wo : 1));
    float *row_out = (float *)malloc(sizeof(float) * (c->Wo ? c->Wo : 1));
    float *vmin = c->tmin + (size_t)j->tid * c->n, *vmax = c->tmax + (size_t)j->tid * c->n;
    uint64_t *imin = c->imin + (size_t)j->tid * c->n, *imax = c->imax + (size_t)j->tid * c->n;
    const uint32_t sp = c->W + 1, np = (c->w + 1) / 2;
    const size_t tsize = (size_t)c->w * c->h, band = (size_t)(c->row_end - c->row_begin) * c->Wo;
    for (uint32_t k = 0; k < c->n; ++k) imin[k] = imax[k] = UINT64_MAX;
    for (uint32_t y = c->row_begin + (uint32_t)j->tid; y < c->row_end; y += (uint32_t)c->nthreads) {
        const uint64_t *s0 = c->sat + (size_t)y * sp, *s1 = c->sat + (size_t)(y + c->h) * sp;
        for (uint32_t k = 0; k < c->n; ++k) {
            const uint8_t *templ = c->templ + k * tsize;
            memset(acc, 0, sizeof(uint32_t) * c->Wo);
            for (uint32_t dy = 0; dy < c->h; ++dy) {
#if defined(__x86_64__)
                if (c->prows) {
                    row_corr_avx2(acc, c->prows + (size_t)(y + dy) * c->W,
                                  c->tpairs + ((size_t)k * c->h + dy) * np, c->w, c->Wo);
                    continue;
                }
#endif
                row_corr_scalar(acc, c->image + (size_t)(y + dy) * c->W, templ + (size_t)dy * c->w,
                                c->w, 0, c->Wo);
            }
            for (uint32_t x = 0; x < c->Wo; ++x) {
                const uint64_t Y = s1[x + c->w] - s0[x + c->w] - s1[x] + s0[x];
                row_out[x] = tmo_finish(c->method, c->precision, acc[x], Y, c->tss[k]);
            }
            if (c->out)
                memcpy(c->out + k * band + (size_t)(y - c->row_begin) * c->Wo, row_out,
                       sizeof(float) * c->Wo);
            const uint64_t base = (uint64_t)y * c->Wo;
            for (uint32_t x = 0; x < c->Wo; ++x) {
                const float v = row_out[x];
                /* a thread's rows come in increasing order: strict compares
                 * keep the first occurrence */
                if (imin[k] == UINT64_MAX || v < vmin[k]) { vmin[k] = v; imin[k] = base + x; }
                if (imax[k] == UINT64_MAX || v > vmax[k]) { vmax[k] = v; imax[k] = base + x; }
            }
        }
    }
    free(acc);
    free(row_out);
    return NULL;
}

int tmo_many_exact_fast(const uint8_t *image, uint32_t W, uint32_t H,
                        const uint8_t *templates, uint32_t w, uint32_t h,
                        uint32_t n, int method, int precision,
                        uint32_t row_begin, uint32_t row_end, float *out,
                        struct tmo_extremes_s *ext, int nthreads) {
    int st = check_dims(W, H, w, h, NULL, 0, 0);
    if (st) return st;
    if (method < 0 || method > 3 || n == 0) return TMO_ERR_INVALID_ARGUMENT;
    if ((uint64_t)w * h > 66051u || w == 0 || h == 0) return TMO_ERR_INVALID_ARGUMENT;
    const uint32_t Wo = W - w + 1, Ho = H - h + 1;
    if (row_begin >= row_end || row_end > Ho) return TMO_ERR_INVALID_ARGUMENT;
    const uint32_t sp = W + 1;
    uint64_t *sat = (uint64_t *)calloc((size_t)sp * (H + 1), sizeof(uint64_t));
    uint64_t *tss = (uint64_t *)calloc(n, sizeof(uint64_t));
    if (!sat || !tss) {
        free(sat);
        free(tss);
        return TMO_ERR_INVALID_ARGUMENT;
    }
    for (uint32_t y = 0; y < H; ++y) {
        uint64_t run = 0;
        const uint8_t *r = image + (size_t)y * W;
        uint64_t *prev = sat + (size_t)y * sp, *cur = sat + (size_t)(y + 1) * sp;
        for (uint32_t x = 0; x < W; ++x) {
            run += (uint64_t)r[x] * r[x];
            cur[x + 1] = prev[x + 1] + run;
        }
    }
    const size_t tsize = (size_t)w * h;
    for (uint32_t k = 0; k < n; ++k)
        for (size_t i = 0; i < tsize; ++i)
            tss[k] += (uint64_t)templates[k * tsize + i] * templates[k * tsize + i];
    if (nthreads < 1) nthreads = 1;
    if ((uint32_t)nthreads > row_end - row_begin) nthreads = (int)(row_end - row_begin);
    if (nthreads > 256) nthreads = 256;
    uint32_t *prows = NULL, *tpairs = NULL;
    if (have_avx2()) {
        const uint32_t np = (w + 1) / 2;
        prows = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)W * H);
        tpairs = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)np * h * n);
        if (!prows || !tpairs) {
            free(prows);
            free(tpairs);
            prows = tpairs = NULL;
        } else {
            for (uint32_t y = 0; y < H; ++y) {
                const uint8_t *r = image + (size_t)y * W;
                uint32_t *pr = prows + (size_t)y * W;
                for (uint32_t x = 0; x < W; ++x)
                    pr[x] = (uint32_t)r[x] | ((x + 1 < W ? (uint32_t)r[x + 1] : 0u) << 16);
            }
            for (size_t row = 0; row < (size_t)n * h; ++row) {
                const uint8_t *t = templates + row * w;
                for (uint32_t k = 0; k < np; ++k)
                    tpairs[row * np + k] =
                        (uint32_t)t[2 * k] | ((2 * k + 1 < w ? (uint32_t)t[2 * k + 1] : 0u) << 16);
            }
        }
    }
    const size_t per = (size_t)nthreads * n;
    float *tmin = (float *)malloc(sizeof(float) * per), *tmax = (float *)malloc(sizeof(float) * per);
    uint64_t *imin = (uint64_t *)malloc(sizeof(uint64_t) * per);
    uint64_t *imax = (uint64_t *)malloc(sizeof(uint64_t) * per);
    fast_ctx c = {image, templates, sat, prows, tpairs, tss, W, w, h, Wo, n, row_begin, row_end,
                  method, precision, nthreads, out, tmin, tmax, imin, imax};
    pthread_t th[256];
    fast_job jobs[256];
    for (int t = 0; t < nthreads; ++t) {
        jobs[t] = (fast_job){&c, t};
        pthread_create(&th[t], NULL, fast_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    if (ext) {
        for (uint32_t k = 0; k < n; ++k) {
            size_t bmin = k, bmax = k;
            for (int t = 1; t < nthreads; ++t) {
                const size_t i = (size_t)t * n + k;
                if (tmin[i] < tmin[bmin] || (tmin[i] == tmin[bmin] && imin[i] < imin[bmin])) bmin = i;
                if (tmax[i] > tmax[bmax] || (tmax[i] == tmax[bmax] && imax[i] < imax[bmax])) bmax = i;
            }
            ext[k].min_value = tmin[bmin];
            ext[k].max_value = tmax[bmax];
            ext[k].min_x = (uint32_t)(imin[bmin] % Wo);
            ext[k].min_y = (uint32_t)(imin[bmin] / Wo);
            ext[k].max_x = (uint32_t)(imax[bmax] % Wo);
            ext[k].max_y = (uint32_t)(imax[bmax] / Wo);
        }
    }
    free(sat);
    free(tss);
    free(prows);
    free(tpairs);
    free(tmin);
    free(tmax);
    free(imin);
    free(imax);
    return TMO_OK;
}

int tmo_match_exact_fast(const uint8_t *image, uint32_t W, uint32_t H,
                         const uint8_t *templ, uint32_t w, uint32_t h,
                         int method, int precision, float *out,
                         struct tmo_extremes_s *ext, int nthreads) {
    if (W < w || H < h) return check_dims(W, H, w, h, NULL, 0, 0);
    return tmo_many_exact_fast(image, W, H, templ, w, h, 1, method, precision, 0, H - h + 1, out,
                               ext, nthreads);
}
