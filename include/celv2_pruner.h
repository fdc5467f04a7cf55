/* celv2_pruner.h: the learned partition / mode pruner of the B200 decision engine.
 *
 * No counterpart in the reference, which always searches exhaustively. A small convolutional
 * network reads, per 64x64 superblock, its luma at quarter resolution and the coarse motion
 * search's cost map against every reference, and proposes which references, whether intra, which
 * block levels of the partition tree and which intra modes the exact integer scorer evaluates (a
 * keep word per superblock, include/celv2_decision.h); the kept options are scored exactly as the
 * exhaustive engine scores them. Its weights are BF16 on
 * the tensor cores with FP32 accumulation (every GEMM operand is rounded to BF16, the products
 * accumulate in FP32); the master parameters are FP32. The forward, backward, loss and optimiser
 * kernels below train it on decision records the exhaustive engine wrote; celv2_set_pruner makes an
 * engine run it on every inter frame.
 *
 * Features per superblock (CELV2_PRUNER_FEATURES floats):
 *   [0, 256)    the superblock at pyramid level 2 (16 x 16 means of 4 x 4 samples), minus its mean,
 *               divided by 64, row-major;
 *   [256, 368)  per reference slot r (7), per level-1 cell of the superblock (4 x 4, row-major):
 *               log2(1 + SAD) / 14 of the 8x8 level-1 block at the level-1 motion vector; 0 for
 *               absent references;
 *   [368, 375)  1 where reference slot r is present, else 0;
 *   375         log2(lambda_q8) / 20.
 * Network: conv 3x3 1->16, ReLU; conv 3x3 stride 2 16->32, ReLU; conv 3x3 stride 2 32->32, ReLU;
 * flatten (y, x, channel) with the 120 non-image features; dense 632->64, ReLU; dense 64->24.
 * Outputs (logits of "the chosen partition uses this option"): 0-6 reference r, 7 intra, 8-11
 * block level l (64, 32, 16, 8-sample squares and their halves), 12-21 intra modes 3-12 (Smooth ..
 * D203), 22-23 unused.
 * Parameters (FP32, in this order): W1 [16][9], b1 [16], W2 [32][144], b2 [32], W3 [32][288],
 * b3 [32], W4 [64][632], b4 [64], W5 [24][64], b5 [24]; a convolution's column index is
 * (ky * 3 + kx) * Cin + ci.
 *
 * Buffers are device memory; `stream` is a cudaStream_t (NULL: the default stream). Every function
 * returns 0 or a negative CELV2_E* code (celv2_last_error() has the message). */
#ifndef CELV2_PRUNER_H
#define CELV2_PRUNER_H

#include <stdint.h>

#include "celv2_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

#define CELV2_PRUNER_FEATURES 376
#define CELV2_PRUNER_OUTPUTS 24
#define CELV2_PRUNER_PARAMS 56120
/* Forward activation cache, floats per sample; the logits are its last batch * 24 floats. */
#define CELV2_PRUNER_ACTS 23504
/* Backward workspace, floats per sample. */
#define CELV2_PRUNER_WORK 20544

/* Forward pass of `batch` samples (x: batch x FEATURES) into `acts` (batch x ACTS floats, the
 * logits at acts + batch * (ACTS - OUTPUTS), batch x OUTPUTS). */
int celv2_pruner_forward(const float* params, const float* x, int batch, float* acts, void* stream);

/* Gradients of the loss w.r.t. every parameter (`grads`, PARAMS floats, overwritten) from the
 * forward cache and dlogits (batch x OUTPUTS); `work`: batch x WORK floats. */
int celv2_pruner_backward(const float* params, int batch, const float* acts, const float* dlogits, float* work,
                          float* grads, void* stream);

/* Weighted binary cross-entropy of the logits against 0/1 labels (batch x OUTPUTS; weights 0 drop
 * an output): adds sum(w * bce) / batch to *loss and writes dlogits = w * (sigmoid - label) / batch. */
int celv2_pruner_bce(const float* logits, const float* labels, const float* weights, int batch, float* dlogits,
                     float* loss, void* stream);

/* One Adam step (bias-corrected, decoupled weight decay) on n parameters; step counts from 1. */
int celv2_pruner_adam(float* params, const float* grads, float* m, float* v, int n, float lr, float beta1,
                      float beta2, float eps, float weight_decay, int step, void* stream);

/* The engine side. celv2_set_pruner: from the next launch on, every inter frame of this engine
 * (that has no celv2_set_keep masks) is scored on the keep words the network proposes: reference r
 * where sigmoid(logit r) >= ref_threshold (the likeliest reference always), intra where
 * sigmoid(logit 7) >= intra_threshold, block level l where sigmoid(logit 8 + l) >= level_threshold
 * (the likeliest level always), and with intra the modes DC, V, H and each mode m of 3-12 where
 * sigmoid(logit 9 + m) >= mode_threshold; a superblock one of whose reference, intra or level
 * outputs lies within `band` of its threshold keeps everything (the fallback to the full search).
 * params: host, PARAMS floats; NULL turns the pruner off. */
int celv2_set_pruner(celv2_engine* e, const float* params, float ref_threshold, float intra_threshold,
                     float level_threshold, float mode_threshold, float band);
/* The features of the last launch's job (sb_cols * sb_rows x FEATURES floats, host), when
 * celv2_set_config(e, CELV2_CFG_FEATURES, 1) was on for it (an inter frame). Waits for the work. */
int celv2_features(celv2_engine* e, int job, float* out);
/* The keep words the pruner chose for the last launch's job (sb_cols * sb_rows words). Waits. */
int celv2_pruner_masks(celv2_engine* e, int job, uint32_t* out);

#ifdef __cplusplus
}
#endif

#endif /* CELV2_PRUNER_H */
