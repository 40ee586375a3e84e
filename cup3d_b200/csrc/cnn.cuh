// Learned per-block preconditioner: a 3-D CNN applied to each block's
// residual (block + one-cell halo) standing in for the block inverse inside
// BiCGSTAB.  No counterpart in the reference (it is the new slot at the
// preconditioner call sites PoissonSolverAMR.h:183-222 / BiCGSTAB.cu:526-527).
//
// Network: x (10^3, 1 channel) -> conv3^3 valid 1->C -> conv3^3 same C->C ->
// conv3^3 same C->C -> conv3^3 same C->1 -> z (8^3), C = 16.  The layers are
// linear (identity activations, no biases): a preconditioner inside BiCGSTAB
// must be a fixed linear map of the residual, or the short recurrences lose
// their meaning (a ReLU network, even one with a small output, doubled the
// iteration count of the two-level method it was added to).  The bias slots
// of the parameter vector are kept for its layout and are not used.  Being
// linear, the network equals one 512 x 896 matrix on the block's star lab,
// which the solver applies (lmap.cuh).  The input is normalised by its RMS s
// and the output scaled by s/h, so z has the units of A^-1 r (A = h *
// Laplacian).
#pragma once
#include "common.cuh"

namespace cup3d {

constexpr int CNN_C = 16;
// parameter counts (FP32 master copy, contiguous in this order)
constexpr int CNN_W0 = CNN_C * 27;            // [co][tap]
constexpr int CNN_B0 = CNN_C;
constexpr int CNN_W1 = CNN_C * CNN_C * 27;    // [co][ci][tap]
constexpr int CNN_B1 = CNN_C;
constexpr int CNN_W2 = CNN_C * CNN_C * 27;
constexpr int CNN_B2 = CNN_C;
constexpr int CNN_W3 = CNN_C * 27;            // [ci][tap]
constexpr int CNN_B3 = 1;
constexpr int CNN_NPARAM = CNN_W0 + CNN_B0 + CNN_W1 + CNN_B1 + CNN_W2 + CNN_B2 + CNN_W3 + CNN_B3;
// offsets
constexpr int OFF_W0 = 0;
constexpr int OFF_B0 = OFF_W0 + CNN_W0;
constexpr int OFF_W1 = OFF_B0 + CNN_B0;
constexpr int OFF_B1 = OFF_W1 + CNN_W1;
constexpr int OFF_W2 = OFF_B1 + CNN_B1;
constexpr int OFF_B2 = OFF_W2 + CNN_W2;
constexpr int OFF_W3 = OFF_B2 + CNN_B2;
constexpr int OFF_B3 = OFF_W3 + CNN_W3;

struct CnnWeights {
  float* master;      // CNN_NPARAM FP32 (training copy)
  uint16_t* w1_bf16;  // [tap][co][ci] bf16 packed for the tensor cores
  uint16_t* w2_bf16;
  uint16_t* w1t_bf16; // [tap][ci][co] flipped-tap transposes for backward-data
  uint16_t* w2t_bf16;
};

// Packs the BF16 tensor-core copies from the FP32 master weights.
int cnn_pack(const CnnWeights& W, cudaStream_t s);

// Folds the network into the solver's matrix (lmap.cuh): forward passes on
// the 896 unit inputs of the star lab (in: 896 * 1000 floats, out: 896 * 512
// floats of scratch), then the fragment-ordered BF16 copy into wfrag
// (LMAP_W_WORDS 16-byte words).  gpart: as cnn_forward_batch.
int cnn_fold(const CnnWeights& W, float* in, float* out, uint4* wfrag, float* gpart, int grid, cudaStream_t s);
// The fragment-ordered BF16 copy alone: W[c][j] = out[j * 512 + c].
int lmap_pack(const float* out, uint4* wfrag, cudaStream_t s);

// z = BJ(r) + (s/h) CNN(r_lab / s) per block (BJ: the exact block inverse;
// r_lab: the residual lab of lmap.cuh, s: its RMS); sum(z h^3) into
// *mean_sum when given.  mean_blk: the block of a mean-constraint row, -1 none.
template <class T>
int cnn_apply(const DevMesh& M, const T* r, T* z, const CnnWeights& W, int grid, cudaStream_t s, GridReduce G,
              double* mean_sum, int mean_blk);

// Appends one training sample per block from a residual r and a correction
// field corr (units of A^-1 r): input gather(r)/s (10^3), target corr h / s
// (8^3), at rows base.. of in/target (capacity cap); the new count into
// *count_dev.
int cnn_dataset_add(const DevMesh& M, const double* r, const double* corr, float* in, float* target, int base,
                    int cap, int* count_dev, int grid, cudaStream_t s, int mean_blk);

// Training on a device dataset of n samples: in[n*1000], target[n*512]
// (targets already divided by the sample's scale/h).  One Adam step over a
// minibatch of `batch` sample indices idx[batch]; the targets are read
// multiplied by target_scale; loss (the residual norm of cnn_residual_loss)
// into *loss_dev.
// grad_partial: grid*(CNN_NPARAM+1) floats of scratch.
int cnn_train_step(const CnnWeights& W, float* adam_m, float* adam_v, int t, float lr, const float* in,
                   const float* target, float target_scale, const int* idx, int batch, float* grad_partial,
                   float* grad, float* loss_dev, int grid, cudaStream_t s);

// Forward and gradient (no update) on a batch, for checks against the oracle.
// gpart: >= grid*(CNN_NPARAM+1) floats of scratch.
int cnn_forward_batch(const CnnWeights& W, const float* in, float* out, int n, float* gpart, int grid,
                      cudaStream_t s);
int cnn_grad_batch(const CnnWeights& W, const float* in, const float* target, int n, float* grad_partial,
                   float* grad, float* loss_dev, int grid, cudaStream_t s);
// Residual-norm loss |L (z - t)|^2 (mean over samples and cells; L the 7-point
// block Laplacian, zero outside the block) of the network (zero_pred = 0) or
// of the zero prediction (zero_pred = 1) on n samples; the training steps
// (cnn_train_step) minimise this loss.
int cnn_residual_loss(const CnnWeights& W, const float* in, const float* target, int n, int zero_pred,
                      float* grad_partial, float* loss_dev, int grid, cudaStream_t s);

}  // namespace cup3d
