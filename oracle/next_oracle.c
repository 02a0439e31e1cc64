/*
 * next_oracle.c -- CPU restatement of imageproc's integral images
 * (src/integral_image.rs) and non-maximum suppression (src/suppress.rs).
 * TEST INFRASTRUCTURE ONLY; see next_oracle.h.
 */
#include "next_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ---- integral images: src/integral_image.rs:98-153 ---------------------- */

#define NXO_INTEGRAL(T, NAME)                                                         \
    void NAME(const uint8_t *img, uint32_t W, uint32_t H, uint32_t C, int square, T *out) { \
        const size_t pitch = (size_t)(W + 1) * C;                                     \
        memset(out, 0, sizeof(T) * pitch * (H + 1));                                  \
        if (W == 0 || H == 0) return;                                                 \
        T sum[4];                                                                     \
        for (uint32_t y = 0; y < H; ++y) {                                            \
            for (uint32_t c = 0; c < C; ++c) sum[c] = 0;                              \
            for (uint32_t x = 0; x < W; ++x) {                                        \
                for (uint32_t c = 0; c < C; ++c) {                                    \
                    const T pix = img[((size_t)y * W + x) * C + c];                   \
                    sum[c] += square ? pix * pix : pix;                               \
                }                                                                     \
                for (uint32_t c = 0; c < C; ++c)                                      \
                    out[(size_t)(y + 1) * pitch + (size_t)(x + 1) * C + c] =          \
                        out[(size_t)y * pitch + (size_t)(x + 1) * C + c] + sum[c];    \
            }                                                                         \
        }                                                                             \
    }

NXO_INTEGRAL(uint32_t, nxo_integral_u32)
NXO_INTEGRAL(uint64_t, nxo_integral_u64)

/* ---- suppress_non_maximum: src/suppress.rs:10-107 ------------------------ */

static uint32_t sat_sub(uint32_t a, uint32_t b) { return a > b ? a - b : 0; }
static uint32_t min_u64(uint64_t a, uint64_t b) { return (uint32_t)(a < b ? a : b); }

/* (ax, ay) < (bx, by) as Rust tuples: x first, then y */
static int lex_xy_less(uint32_t ax, uint32_t ay, uint32_t bx, uint32_t by) {
    return ax < bx || (ax == bx && ay < by);
}

/* contains_greater_value (:82-107) */
static int contains_greater(const uint64_t *k, uint32_t W, uint32_t x, uint32_t y, uint64_t v, uint32_t ylo,
                            uint32_t yhi, uint32_t xlo, uint32_t xhi) {
    for (uint32_t cy = ylo; cy < yhi; ++cy)
        for (uint32_t cx = xlo; cx < xhi; ++cx) {
            const uint64_t ci = k[(size_t)cy * W + cx];
            if (ci < v) continue;
            if (ci > v || lex_xy_less(cx, cy, x, y)) return 1;
        }
    return 0;
}

void nxo_suppress_non_maximum(const uint64_t *k, uint32_t W, uint32_t H, uint32_t r, uint8_t *keep) {
    memset(keep, 0, (size_t)W * H);
    if (W == 0 || H == 0) return;
    const uint64_t step = (uint64_t)r + 1;
    for (uint64_t yy = 0; yy < H; yy += step)
        for (uint64_t xx = 0; xx < W; xx += step) {
            const uint32_t x = (uint32_t)xx, y = (uint32_t)yy;
            uint32_t bx = x, by = y;
            uint64_t mi = k[(size_t)y * W + x];
            /* the grid cell's maximum, lexicographically first among equals */
            for (uint32_t cy = y; cy < min_u64(H, (uint64_t)y + r + 1); ++cy)
                for (uint32_t cx = x; cx < min_u64(W, (uint64_t)x + r + 1); ++cx) {
                    const uint64_t ci = k[(size_t)cy * W + cx];
                    if (ci < mi) continue;
                    if (ci > mi || lex_xy_less(cx, cy, bx, by)) {
                        bx = cx;
                        by = cy;
                        mi = ci;
                    }
                }
            const uint32_t x0 = sat_sub(bx, r), x1 = x, x2 = min_u64(W, (uint64_t)x + r + 1),
                           x3 = min_u64(W, (uint64_t)bx + r + 1);
            const uint32_t y0 = sat_sub(by, r), y1 = y, y2 = min_u64(H, (uint64_t)y + r + 1),
                           y3 = min_u64(H, (uint64_t)by + r + 1);
            int failed = contains_greater(k, W, bx, by, mi, y0, y1, x0, x3);  /* above */
            failed |= contains_greater(k, W, bx, by, mi, y1, y2, x0, x1);     /* left */
            failed |= contains_greater(k, W, bx, by, mi, y1, y2, x2, x3);     /* right */
            failed |= contains_greater(k, W, bx, by, mi, y2, y3, x0, x3);     /* below */
            if (!failed) keep[(size_t)by * W + bx] = 1;
        }
}

/* suppress_non_maximum_reference (:274-318) */
void nxo_suppress_non_maximum_naive(const uint64_t *k, uint32_t W, uint32_t H, uint32_t r, uint8_t *keep) {
    for (uint32_t y = 0; y < H; ++y)
        for (uint32_t x = 0; x < W; ++x) {
            const uint64_t v0 = k[(size_t)y * W + x];
            int is_max = 1;
            const int64_t ylo = (int64_t)y - r < 0 ? 0 : (int64_t)y - r;
            const int64_t yhi = (int64_t)y + r + 1 > H ? H : (int64_t)y + r + 1;
            const int64_t xlo = (int64_t)x - r < 0 ? 0 : (int64_t)x - r;
            const int64_t xhi = (int64_t)x + r + 1 > W ? W : (int64_t)x + r + 1;
            for (int64_t py = ylo; py < yhi && is_max; ++py)
                for (int64_t px = xlo; px < xhi; ++px) {
                    const uint64_t v = k[(size_t)py * W + px];
                    if (v > v0 || (v == v0 && lex_xy_less((uint32_t)px, (uint32_t)py, x, y))) {
                        is_max = 0;
                        break;
                    }
                }
            keep[(size_t)y * W + x] = (uint8_t)is_max;
        }
}

/* ---- local_maxima: src/suppress.rs:111-173 ------------------------------- */

static const uint32_t *g_xs, *g_ys;

/* sort_by_key((y, x)) is stable: the input index breaks ties */
static int by_yx_index(const void *a, const void *b) {
    const uint32_t i = *(const uint32_t *)a, j = *(const uint32_t *)b;
    if (g_ys[i] != g_ys[j]) return g_ys[i] < g_ys[j] ? -1 : 1;
    if (g_xs[i] != g_xs[j]) return g_xs[i] < g_xs[j] ? -1 : 1;
    return i < j ? -1 : (i > j);
}

uint32_t nxo_local_maxima(const uint32_t *xs, const uint32_t *ys, const float *scores, uint32_t n, uint32_t radius,
                          uint32_t *out_idx) {
    if (n == 0) return 0;
    uint32_t *ord = malloc(sizeof(uint32_t) * n);
    for (uint32_t i = 0; i < n; ++i) ord[i] = i;
    g_xs = xs;
    g_ys = ys;
    qsort(ord, n, sizeof(uint32_t), by_yx_index);
    const uint32_t height = ys[ord[n - 1]];
    /* ts_by_row: the sorted points of row y are ord[row_start[y] .. row_start[y + 1]) */
    uint32_t *row_start = calloc((size_t)height + 2, sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i) row_start[ys[ord[i]] + 1] += 1;
    for (uint32_t y = 0; y <= height; ++y) row_start[y + 1] += row_start[y];
    uint32_t count = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t t = ord[i], cx = xs[t], cy = ys[t];
        const float cs = scores[t];
        int is_max = 1;
        /* u32 arithmetic as in the reference (release builds wrap) */
        const uint32_t row_lower = cy > radius ? cy - radius : 0;
        const uint32_t row_upper = (uint32_t)(cy + radius + 1u) > height ? height : (uint32_t)(cy + radius + 1u);
        for (uint32_t y = row_lower; y < row_upper && is_max; ++y)
            for (uint32_t k = row_start[y]; k < row_start[y + 1]; ++k) {
                const uint32_t c = ord[k];
                if ((uint32_t)(xs[c] + radius) < cx) continue;
                if (xs[c] > (uint32_t)(cx + radius)) break;
                if (scores[c] > cs) {
                    is_max = 0;
                    break;
                }
                if (scores[c] < cs) continue;
                /* tie-break lexicographically on (y, x) */
                if (ys[c] < cy || (ys[c] == cy && xs[c] < cx)) {
                    is_max = 0;
                    break;
                }
            }
        if (is_max) out_idx[count++] = t;
    }
    free(row_start);
    free(ord);
    return count;
}

/* ---- filter_clamped: src/filter/mod.rs:29-70, :407-416 -------------------- */

/* Clamp<K> for S (src/definitions.rs:119-131): `if x < max { if x > min { x as S }
 * else { min } } else { max }` -- NaN fails both tests and gives max. */
static double clamp_d(double x, double lo, double hi) {
    if (x < hi) return x > lo ? x : lo;
    return hi;
}

void nxo_filter_clamped(const uint8_t *img, uint32_t W, uint32_t H, uint32_t C, const void *kernel,
                        int kernel_type, uint32_t kw, uint32_t kh, int out_type, void *out) {
    const int64_t kwi = kw, khi = kh, Wi = W, Hi = H;
    for (int64_t y = 0; y < Hi; ++y)
        for (int64_t x = 0; x < Wi; ++x) {
            float accf[4] = {0, 0, 0, 0};
            uint32_t acci[4] = {0, 0, 0, 0}; /* i32 arithmetic, wrapping */
            for (int64_t ky = 0; ky < khi; ++ky) {
                int64_t yp = y + ky - khi / 2;
                yp = yp < 0 ? 0 : (yp > Hi - 1 ? Hi - 1 : yp);
                for (int64_t kx = 0; kx < kwi; ++kx) {
                    int64_t xp = x + kx - kwi / 2;
                    xp = xp < 0 ? 0 : (xp > Wi - 1 ? Wi - 1 : xp);
                    const uint8_t *p = img + ((size_t)yp * W + (size_t)xp) * C;
                    for (uint32_t c = 0; c < C; ++c) {
                        if (kernel_type == 0) {
                            const float w = ((const float *)kernel)[ky * kwi + kx];
                            const float prod = (float)p[c] * w;
                            accf[c] = accf[c] + prod;
                        } else {
                            const int32_t w = ((const int32_t *)kernel)[ky * kwi + kx];
                            acci[c] = acci[c] + (uint32_t)p[c] * (uint32_t)w;
                        }
                    }
                }
            }
            for (uint32_t c = 0; c < C; ++c) {
                const size_t o = ((size_t)y * W + (size_t)x) * C + c;
                if (kernel_type == 0) {
                    const float a = accf[c];
                    if (out_type == 8) ((float *)out)[o] = a;
                    else if (out_type == 0) ((uint8_t *)out)[o] = (uint8_t)clamp_d(a, 0.0, 255.0);
                    else ((uint16_t *)out)[o] = (uint16_t)clamp_d(a, 0.0, 65535.0);
                } else {
                    const int32_t a = (int32_t)acci[c];
                    if (out_type == 6) ((int32_t *)out)[o] = a;
                    else if (out_type == 0) ((uint8_t *)out)[o] = (uint8_t)clamp_d(a, 0.0, 255.0);
                    else if (out_type == 1) ((uint16_t *)out)[o] = (uint16_t)clamp_d(a, 0.0, 65535.0);
                    else ((int16_t *)out)[o] = (int16_t)clamp_d(a, -32768.0, 32767.0);
                }
            }
        }
}
