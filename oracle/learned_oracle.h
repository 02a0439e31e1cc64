/*
 * learned_oracle.h -- CPU oracle of the learned proposal network.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the GPU forward and backward
 * kernels of imageproc_b200's proposal network (csrc/tm_learned.cu). No
 * product code path links against it. The reference (imageproc) has no
 * learned component; this oracle restates the network this library defines,
 * in FP64, and is itself pinned by finite differences (tests/
 * test_oracle_learned.py).
 *
 * The network (all images row-major, zero padding):
 *   D      = (sum of each 4x4 block of the u8 image - 2048) / 1024
 *   A1     = R(relu(b1 + conv3x3(W1, D)))                1 -> 32 channels
 *   Al     = R(relu(bl + conv3x3(Wl, A(l-1))))  l = 2..4  32 -> 32
 *   F      = R(b5 + conv3x3(W5, A4))                     32 -> 32, no relu
 *   G_t(o) = F_template_t(5 + oy, 5 + ox), o in {0,1}^2   (the 2x2 centre of a
 *            12x12 downsampled 48x48 template's features)
 *   z_t(p) = alpha * sum_o F(p + o) . G_t(o)             (F outside the map = 0)
 * R() rounds to bfloat16 (round to nearest even) when `bf16` is set, and is
 * the identity otherwise. Weights are taken as given (already bf16 values on
 * the GPU side). Layout: activations [n][c][y][x]; conv weights
 * [co][ci][ky][kx]; biases [co].
 *
 * Loss of a batch of T templates against N scene crops (in-batch softmax):
 *   L = (1/T) sum_t ( logsumexp_{n,p} z_t(n, p) - logsumexp_{p in N_t} z_t(p) )
 * with pos_t a flat index into the N crops' heatmap positions and N_t its
 * 3 x 3 neighbourhood inside its crop (a multiple-instance positive). Backward
 * treats R() as the identity (straight-through).
 */
#ifndef LEARNED_ORACLE_H
#define LEARNED_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LO_CH 32
#define LO_LAYERS 5

typedef struct {
    /* W[0]: 32 x 1 x 3 x 3; W[1..4]: 32 x 32 x 3 x 3 */
    const double *W[LO_LAYERS];
    const double *b[LO_LAYERS];
    double alpha;
} lo_params;

typedef struct {
    double *dW[LO_LAYERS];
    double *db[LO_LAYERS];
} lo_grads;

/* Forward of the trunk on n images of h x w u8 pixels (h, w multiples of 4):
 * writes F (n x 32 x h/4 x w/4) and, when acts != NULL, the post-activation
 * maps A1..A4 and pre-activations Z1..Z5 for the backward pass
 * (acts[2*l] = Z(l+1), acts[2*l+1] = A(l+1); each n x 32 x h/4 x w/4). */
void lo_trunk_forward(const lo_params *P, const uint8_t *img, int n, int h, int w,
                      int bf16, double *F, double **acts);

/* Loss and gradients for N scene crops (sh x sw u8) and T templates
 * (48 x 48 u8) with positives pos[T]. Returns the loss; writes the
 * gradients when G != NULL, and the logits (T x N x sh/4 x sw/4) when z != NULL. */
double lo_loss_grad(const lo_params *P, const uint8_t *scenes, int N, int sh, int sw,
                    const uint8_t *templates, int T, const int64_t *pos, int bf16,
                    lo_grads *G, double *z);

/* Round to bfloat16, nearest even (the value as a double). */
double lo_bf16(double v);

#ifdef __cplusplus
}
#endif
#endif
