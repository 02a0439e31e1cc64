/*
 * learned_oracle.c -- FP64 CPU restatement of the proposal network's forward
 * and backward passes. TEST INFRASTRUCTURE ONLY (see learned_oracle.h).
 */
#include "learned_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

double lo_bf16(double v) {
    float f = (float)v;
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) return v; /* inf / nan unchanged */
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7FFFu + lsb;
    u &= 0xFFFF0000u;
    memcpy(&f, &u, 4);
    return (double)f;
}

static double rnd(double v, int bf16) { return bf16 ? lo_bf16(v) : v; }

/* 4x4 block sums of n h x w u8 images -> (sum - 2048) / 1024, n x (h/4) x (w/4) */
static void downsample(const uint8_t *img, int n, int h, int w, double *D) {
    const int hs = h / 4, ws = w / 4;
    for (int k = 0; k < n; ++k)
        for (int y = 0; y < hs; ++y)
            for (int x = 0; x < ws; ++x) {
                int s = 0;
                for (int dy = 0; dy < 4; ++dy)
                    for (int dx = 0; dx < 4; ++dx)
                        s += img[((size_t)k * h + 4 * y + dy) * w + 4 * x + dx];
                D[((size_t)k * hs + y) * ws + x] = (double)(s - 2048) / 1024.0;
            }
}

/* Z = b + conv3x3(W, A), zero padding. A: n x cin x h x w; Z: n x cout x h x w. */
static void conv_fwd(const double *W, const double *b, const double *A, int n, int cin, int cout,
                     int h, int w, double *Z) {
    for (int k = 0; k < n; ++k)
        for (int co = 0; co < cout; ++co)
            for (int y = 0; y < h; ++y)
                for (int x = 0; x < w; ++x) {
                    double s = b[co];
                    for (int ci = 0; ci < cin; ++ci)
                        for (int ky = 0; ky < 3; ++ky) {
                            const int yy = y + ky - 1;
                            if (yy < 0 || yy >= h) continue;
                            for (int kx = 0; kx < 3; ++kx) {
                                const int xx = x + kx - 1;
                                if (xx < 0 || xx >= w) continue;
                                s += W[((co * cin + ci) * 3 + ky) * 3 + kx] *
                                     A[(((size_t)k * cin + ci) * h + yy) * w + xx];
                            }
                        }
                    Z[(((size_t)k * cout + co) * h + y) * w + x] = s;
                }
}

/* Gradients of conv_fwd: accumulates dW, db and (when dA != NULL) writes dA. */
static void conv_bwd(const double *W, const double *A, const double *dZ, int n, int cin, int cout, int h,
                     int w, double *dW, double *db, double *dA) {
    const size_t hw = (size_t)h * w;
    for (int k = 0; k < n; ++k)
        for (int co = 0; co < cout; ++co) {
            const double *dz = dZ + ((size_t)k * cout + co) * hw;
            for (size_t i = 0; i < hw; ++i) db[co] += dz[i];
            for (int ci = 0; ci < cin; ++ci) {
                const double *a = A + ((size_t)k * cin + ci) * hw;
                for (int ky = 0; ky < 3; ++ky)
                    for (int kx = 0; kx < 3; ++kx) {
                        double s = 0.0;
                        for (int y = 0; y < h; ++y) {
                            const int yy = y + ky - 1;
                            if (yy < 0 || yy >= h) continue;
                            for (int x = 0; x < w; ++x) {
                                const int xx = x + kx - 1;
                                if (xx < 0 || xx >= w) continue;
                                s += dz[(size_t)y * w + x] * a[(size_t)yy * w + xx];
                            }
                        }
                        dW[((co * cin + ci) * 3 + ky) * 3 + kx] += s;
                    }
            }
        }
    if (!dA) return;
    memset(dA, 0, sizeof(double) * (size_t)n * cin * hw);
    for (int k = 0; k < n; ++k)
        for (int co = 0; co < cout; ++co) {
            const double *dz = dZ + ((size_t)k * cout + co) * hw;
            for (int ci = 0; ci < cin; ++ci) {
                double *da = dA + ((size_t)k * cin + ci) * hw;
                for (int ky = 0; ky < 3; ++ky)
                    for (int kx = 0; kx < 3; ++kx) {
                        const double wv = W[((co * cin + ci) * 3 + ky) * 3 + kx];
                        for (int y = 0; y < h; ++y) {
                            const int yy = y + ky - 1;
                            if (yy < 0 || yy >= h) continue;
                            for (int x = 0; x < w; ++x) {
                                const int xx = x + kx - 1;
                                if (xx < 0 || xx >= w) continue;
                                da[(size_t)yy * w + xx] += wv * dz[(size_t)y * w + x];
                            }
                        }
                    }
            }
        }
}

void lo_trunk_forward(const lo_params *P, const uint8_t *img, int n, int h, int w, int bf16, double *F,
                      double **acts) {
    const int hs = h / 4, ws = w / 4;
    const size_t plane = (size_t)hs * ws;
    double *D = (double *)malloc(sizeof(double) * n * plane);
    downsample(img, n, h, w, D);
    double *cur = D;
    int cin = 1;
    for (int l = 0; l < LO_LAYERS; ++l) {
        double *Z = acts ? acts[2 * l] : (double *)malloc(sizeof(double) * n * LO_CH * plane);
        conv_fwd(P->W[l], P->b[l], cur, n, cin, LO_CH, hs, ws, Z);
        const size_t m = (size_t)n * LO_CH * plane;
        double *A;
        if (l + 1 < LO_LAYERS) {
            A = acts ? acts[2 * l + 1] : (double *)malloc(sizeof(double) * m);
            for (size_t i = 0; i < m; ++i) A[i] = rnd(Z[i] > 0.0 ? Z[i] : 0.0, bf16);
        } else {
            A = F;
            for (size_t i = 0; i < m; ++i) A[i] = rnd(Z[i], bf16);
        }
        if (!acts) free(Z);
        if (cur != D && !acts) free(cur);
        cur = A;
        cin = LO_CH;
    }
    free(D);
}

double lo_loss_grad(const lo_params *P, const uint8_t *scenes, int N, int sh, int sw,
                    const uint8_t *templates, int T, const int64_t *pos, int bf16, lo_grads *G,
                    double *zout) {
    const int hs = sh / 4, ws = sw / 4;
    const size_t plane = (size_t)hs * ws, tplane = 144;
    const size_t P_all = (size_t)N * plane;
    double *acts_s[2 * LO_LAYERS], *acts_t[2 * LO_LAYERS];
    for (int i = 0; i < 2 * LO_LAYERS; ++i) {
        acts_s[i] = (double *)malloc(sizeof(double) * N * LO_CH * plane);
        acts_t[i] = (double *)malloc(sizeof(double) * T * LO_CH * tplane);
    }
    double *F = (double *)malloc(sizeof(double) * N * LO_CH * plane);
    double *Ft = (double *)malloc(sizeof(double) * T * LO_CH * tplane);
    lo_trunk_forward(P, scenes, N, sh, sw, bf16, F, acts_s);
    lo_trunk_forward(P, templates, T, 48, 48, bf16, Ft, acts_t);
    /* G_t[c][o] = Ft[t][c][5 + oy][5 + ox] */
    double *Gt = (double *)malloc(sizeof(double) * T * LO_CH * 4);
    for (int t = 0; t < T; ++t)
        for (int c = 0; c < LO_CH; ++c)
            for (int o = 0; o < 4; ++o)
                Gt[(t * LO_CH + c) * 4 + o] = Ft[((size_t)t * LO_CH + c) * tplane + (5 + o / 2) * 12 + 5 + o % 2];
    /* logits */
    double *z = (double *)malloc(sizeof(double) * T * P_all);
    for (int t = 0; t < T; ++t)
        for (int n = 0; n < N; ++n)
            for (int y = 0; y < hs; ++y)
                for (int x = 0; x < ws; ++x) {
                    double s = 0.0;
                    for (int o = 0; o < 4; ++o) {
                        const int yy = y + o / 2, xx = x + o % 2;
                        if (yy >= hs || xx >= ws) continue;
                        for (int c = 0; c < LO_CH; ++c)
                            s += F[(((size_t)n * LO_CH + c) * hs + yy) * ws + xx] * Gt[(t * LO_CH + c) * 4 + o];
                    }
                    z[(size_t)t * P_all + ((size_t)n * hs + y) * ws + x] = P->alpha * s;
                }
    if (zout) memcpy(zout, z, sizeof(double) * T * P_all);
    /* loss and dz */
    double loss = 0.0;
    for (int t = 0; t < T; ++t) {
        double *zt = z + (size_t)t * P_all;
        double mx = zt[0];
        for (size_t i = 1; i < P_all; ++i) mx = zt[i] > mx ? zt[i] : mx;
        double se = 0.0;
        for (size_t i = 0; i < P_all; ++i) se += exp(zt[i] - mx);
        const double lse = mx + log(se);
        /* the positive set: the 3 x 3 neighbourhood of pos[t] inside its crop */
        const size_t pt = (size_t)pos[t], base = pt - pt % plane;
        const int py = (int)((pt % plane) / ws), px = (int)(pt % ws);
        double mn = -INFINITY, sn = 0.0;
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
                if (py + dy >= 0 && py + dy < hs && px + dx >= 0 && px + dx < ws) {
                    const double v = zt[base + (size_t)(py + dy) * ws + px + dx];
                    mn = v > mn ? v : mn;
                }
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
                if (py + dy >= 0 && py + dy < hs && px + dx >= 0 && px + dx < ws)
                    sn += exp(zt[base + (size_t)(py + dy) * ws + px + dx] - mn);
        const double lsen = mn + log(sn);
        loss += lse - lsen;
        /* reuse z as dz */
        for (size_t i = 0; i < P_all; ++i) {
            double d = exp(zt[i] - lse);
            const size_t k = i / plane;
            const int y = (int)((i % plane) / ws), x = (int)(i % ws);
            if (k == pt / plane && y - py <= 1 && py - y <= 1 && x - px <= 1 && px - x <= 1)
                d -= exp(zt[i] - lsen);
            zt[i] = d / T;
        }
    }
    loss /= T;
    if (G) {
        /* dF (scenes) and dG */
        double *dF = (double *)calloc((size_t)N * LO_CH * plane, sizeof(double));
        double *dG = (double *)calloc((size_t)T * LO_CH * 4, sizeof(double));
        for (int t = 0; t < T; ++t)
            for (int n = 0; n < N; ++n)
                for (int y = 0; y < hs; ++y)
                    for (int x = 0; x < ws; ++x) {
                        const double dz = P->alpha * z[(size_t)t * P_all + ((size_t)n * hs + y) * ws + x];
                        if (dz == 0.0) continue;
                        for (int o = 0; o < 4; ++o) {
                            const int yy = y + o / 2, xx = x + o % 2;
                            if (yy >= hs || xx >= ws) continue;
                            for (int c = 0; c < LO_CH; ++c) {
                                const size_t fi = (((size_t)n * LO_CH + c) * hs + yy) * ws + xx;
                                dF[fi] += dz * Gt[(t * LO_CH + c) * 4 + o];
                                dG[(t * LO_CH + c) * 4 + o] += dz * F[fi];
                            }
                        }
                    }
        double *dFt = (double *)calloc((size_t)T * LO_CH * tplane, sizeof(double));
        for (int t = 0; t < T; ++t)
            for (int c = 0; c < LO_CH; ++c)
                for (int o = 0; o < 4; ++o)
                    dFt[((size_t)t * LO_CH + c) * tplane + (5 + o / 2) * 12 + 5 + o % 2] = dG[(t * LO_CH + c) * 4 + o];
        /* trunk backward for scenes and templates */
        for (int side = 0; side < 2; ++side) {
            const int n = side ? T : N, h = side ? 12 : hs, w = side ? 12 : ws;
            const size_t pl = (size_t)h * w;
            double **acts = side ? acts_t : acts_s;
            const uint8_t *img = side ? templates : scenes;
            double *D = (double *)malloc(sizeof(double) * n * pl);
            downsample(img, n, side ? 48 : sh, side ? 48 : sw, D);
            double *dZ = (double *)malloc(sizeof(double) * n * LO_CH * pl);
            memcpy(dZ, side ? dFt : dF, sizeof(double) * n * LO_CH * pl); /* layer 5: no relu */
            double *dA = (double *)malloc(sizeof(double) * n * LO_CH * pl);
            for (int l = LO_LAYERS - 1; l >= 0; --l) {
                const double *A_in = l ? acts[2 * (l - 1) + 1] : D;
                const int cin = l ? LO_CH : 1;
                conv_bwd(P->W[l], A_in, dZ, n, cin, LO_CH, h, w, G->dW[l], G->db[l], l ? dA : NULL);
                if (l) {
                    const double *Zp = acts[2 * (l - 1)];
                    for (size_t i = 0; i < (size_t)n * LO_CH * pl; ++i) dZ[i] = Zp[i] > 0.0 ? dA[i] : 0.0;
                }
            }
            free(D);
            free(dZ);
            free(dA);
        }
        free(dF);
        free(dG);
        free(dFt);
    }
    for (int i = 0; i < 2 * LO_LAYERS; ++i) {
        free(acts_s[i]);
        free(acts_t[i]);
    }
    free(F);
    free(Ft);
    free(Gt);
    free(z);
    return loss;
}
