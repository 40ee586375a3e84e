// C-ABI of the learned preconditioner: weights, dataset, training, checks.
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "context.h"
#include "lmap.cuh"
#include "profiler.h"

namespace cup3d {

static int ensure_cnn(cup_ctx* c) {
  CnnState& S = c->cnn;
  if (S.W.master) return 0;
  DevArena& A = S.arena;
  if (int rc = A.alloc(&S.W.master, CNN_NPARAM)) return rc;
  if (int rc = A.alloc(&S.W.w1_bf16, 27 * 256)) return rc;
  if (int rc = A.alloc(&S.W.w2_bf16, 27 * 256)) return rc;
  if (int rc = A.alloc(&S.W.w1t_bf16, 27 * 256)) return rc;
  if (int rc = A.alloc(&S.W.w2t_bf16, 27 * 256)) return rc;
  if (int rc = A.alloc(&S.adam_m, CNN_NPARAM)) return rc;
  if (int rc = A.alloc(&S.adam_v, CNN_NPARAM)) return rc;
  if (int rc = A.alloc(&S.grad, CNN_NPARAM)) return rc;
  if (int rc = A.alloc(&S.loss, 1)) return rc;
  S.train_grid = std::max(1, c->num_sms);
  if (int rc = A.alloc(&S.gpart, size_t(S.train_grid) * (CNN_NPARAM + 1))) return rc;
  CUP_CUDA_TRY(stream_zero(c->stream, S.adam_m, CNN_NPARAM * sizeof(float)));
  CUP_CUDA_TRY(stream_zero(c->stream, S.adam_v, CNN_NPARAM * sizeof(float)));
  return 0;
}

// sum of squares of v[0..n) into *out (deterministic grid reduction)
__global__ void __launch_bounds__(NT) k_sumsq(const float* __restrict__ v, size_t n, GridReduce g, double* out) {
  __shared__ double red[64];
  double acc[1] = {0.0};
  for (size_t i = size_t(blockIdx.x) * NT + threadIdx.x; i < n; i += size_t(gridDim.x) * NT) {
    const double x = v[i];
    acc[0] += x * x;
  }
  if (grid_reduce<1>(acc, g, red) && threadIdx.x == 0) *out = acc[0];
}

__global__ void k_scale(float* v, size_t n, float s) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) v[i] *= s;
}

// RMS of the stored training targets.
static int target_rms(cup_ctx* c, double* rms) {
  CnnState& S = c->cnn;
  const size_t n = size_t(S.count) * BN;
  GridReduce g{c->W.partial, c->W.counters + 16};
  double* d = c->d_scalars + SC_TARGET_SUMSQ;
  k_sumsq<<<c->W.grid, NT, 0, c->stream>>>(S.ds_target, n, g, d);
  CUP_CUDA_TRY(cudaGetLastError());
  double ss = 0.0;
  CUP_CUDA_TRY(stream_d2h(c->stream, &ss, d, sizeof(double)));
  *rms = std::sqrt(ss / double(std::max<size_t>(n, 1)));
  return 0;
}

// Scales the output layer (W3, b3) by s.  The output layer is linear, so the
// network's outputs scale by s as well.
static int scale_output_layer(cup_ctx* c, float s) {
  k_scale<<<2, NT, 0, c->stream>>>(c->cnn.W.master + OFF_W3, size_t(CNN_W3 + CNN_B3), s);
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

static int set_params(cup_ctx* c, const float* p) {
  if (int rc = ensure_cnn(c)) return rc;
  CUP_CUDA_TRY(stream_h2d(c->stream, c->cnn.W.master, p, CNN_NPARAM * sizeof(float)));
  c->cnn.folded = false;
  if (int rc = cnn_pack(c->cnn.W, c->stream)) return rc;
  CUP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->cnn.ready = true;
  c->cnn.adam_t = 0;
  CUP_CUDA_TRY(stream_zero(c->stream, c->cnn.adam_m, CNN_NPARAM * sizeof(float)));
  CUP_CUDA_TRY(stream_zero(c->stream, c->cnn.adam_v, CNN_NPARAM * sizeof(float)));
  return 0;
}

static bool dev_ok(cup_ctx* c) { return c && !c->host_only && c->mesh.nb > 0; }

// The learned map's two phases as kernels of their own (the solver runs
// them inside its persistent launch).
__global__ void __launch_bounds__(256) k_lmap_gather(DevMesh M, const double* v, uint16_t* lab, int mean_blk) {
  __shared__ LabMeta meta[LMAP_GATHER];
  lmap_gather<double>(M, v, lab, meta, mean_blk);
}

__global__ void __launch_bounds__(256) k_lmap_gemm(DevMesh M, const uint4* W, const uint16_t* lab, double* z) {
  extern __shared__ __align__(16) unsigned char lmap_smem[];
  (void)lmap_gemm<double>(M, W, lab, z, reinterpret_cast<uint16_t*>(lmap_smem));
}

// The mean-constraint row's block (cell 0) when the configured mean mode
// replaces a row (1 and 3), else -1.
int mean_block_of(const cup_ctx* c) {
  const int m = c->cfg.mean_constraint;
  return (m == 1 || m == 3) ? c->dm.mean_block : -1;
}

// The solver's lab buffer for the current mesh.
static int ensure_lab(cup_ctx* c) {
  CnnState& S = c->cnn;
  const size_t need = size_t(c->mesh.nb) * LMAP_K;
  if (S.lab_cap >= need) return 0;
  S.lab_arena.release();
  S.lab_cap = 0;
  if (int rc = S.lab_arena.alloc(&S.lmap_lab, need)) return rc;
  S.lab_cap = need;
  return 0;
}

int lmap_prepare(cup_ctx* c, LocalMap* out) {
  CnnState& S = c->cnn;
  if (!S.ready) return set_error(CUP_ERR_STATE, "learned preconditioner has no weights (cup_cnn_init / cup_cnn_set_params)");
  if (!S.lmap_w) {
    if (int rc = S.arena.alloc(&S.lmap_w, LMAP_W_WORDS)) return rc;
    if (int rc = S.arena.alloc(&S.fold_in, size_t(LMAP_K) * 1000)) return rc;
    if (int rc = S.arena.alloc(&S.fold_out, size_t(LMAP_K) * BN)) return rc;
    S.folded = false;
  }
  if (int rc = ensure_lab(c)) return rc;
  if (!S.folded) {
    if (int rc = cnn_fold(S.W, S.fold_in, S.fold_out, S.lmap_w, S.gpart, S.train_grid, c->stream)) return rc;
    S.folded = true;
  }
  *out = LocalMap{S.lmap_w, S.lmap_lab};
  return 0;
}

// Star-lab index of cube position q (x, y, z in -1..8): the block's cells,
// then the six one-cell face layers (LabGeom<1>); -1 for edges, corners and
// positions beyond the layers.
static int star_index(const int q[3]) {
  int out = -1, n = 0;
  for (int d = 0; d < 3; ++d) {
    if (q[d] < -1 || q[d] > BS) return -1;
    if (q[d] == -1 || q[d] == BS) {
      out = d;
      ++n;
    }
  }
  if (n == 0) return q[0] + BS * q[1] + BS * BS * q[2];
  if (n > 1) return -1;
  const int d = out, s = q[d] == BS ? 1 : 0;
  return BN + (2 * d + s) * 64 + q[tan1(d)] + 8 * q[tan2(d)];
}

// The one-cell-overlap local solve (restricted additive Schwarz with a
// one-cell overlap) as a local map: z_b = [L_s^-1 lab_b]_interior / h_b, with
// L_s the 7-point Laplacian of unit spacing on the 896 star cells (the block
// and its six face layers; zero beyond them: edges, corners and the next
// layer).  The solver's phases already apply the block inverse
// [L_b^-1 | 0] (L_b: the same operator on the block alone), so the map holds
// the difference [L_s^-1]_interior - [L_b^-1 | 0].  A = h L on a uniform
// neighbourhood (the AMR operator's same-level rows), hence the 1/h.
int schwarz_prepare(cup_ctx* c, LocalMap* out) {
  CnnState& S = c->cnn;
  if (!S.schwarz_w) {
    std::vector<double> Ls(size_t(LMAP_K) * LMAP_K, 0.0), Lb(size_t(BN) * BN, 0.0);
    for (int j = 0; j < LMAP_K; ++j) {
      int q[3];
      lmap_lab_pos(j, q);
      Ls[size_t(j) * LMAP_K + j] = -6.0;
      if (j < BN) Lb[size_t(j) * BN + j] = -6.0;
      for (int d = 0; d < 3; ++d)
        for (int e = -1; e <= 1; e += 2) {
          int r[3] = {q[0], q[1], q[2]};
          r[d] += e;
          const int k = star_index(r);
          if (k < 0) continue;
          Ls[size_t(j) * LMAP_K + k] = 1.0;
          if (j < BN && k < BN) Lb[size_t(j) * BN + k] = 1.0;
        }
    }
    DevArena tmp;
    double *dLs = nullptr, *dLb = nullptr;
    if (int rc = tmp.alloc(&dLs, Ls.size())) return rc;
    if (int rc = tmp.alloc(&dLb, Lb.size())) return rc;
    if (int rc = device_inverse(Ls.data(), LMAP_K, dLs, c->num_sms, c->stream)) return rc;
    if (int rc = device_inverse(Lb.data(), BN, dLb, c->num_sms, c->stream)) return rc;
    CUP_CUDA_TRY(stream_d2h(c->stream, Ls.data(), dLs, Ls.size() * sizeof(double)));
    CUP_CUDA_TRY(stream_d2h(c->stream, Lb.data(), dLb, Lb.size() * sizeof(double)));
    // W[r][j] in the fold's layout out[j * 512 + r]
    std::vector<float> w(size_t(LMAP_K) * BN);
    for (int r = 0; r < BN; ++r)
      for (int j = 0; j < LMAP_K; ++j)
        w[size_t(j) * BN + r] = float(Ls[size_t(r) * LMAP_K + j] - (j < BN ? Lb[size_t(r) * BN + j] : 0.0));
    float* dw = nullptr;
    if (int rc = tmp.alloc(&dw, w.size())) return rc;
    CUP_CUDA_TRY(stream_h2d(c->stream, dw, w.data(), w.size() * sizeof(float)));
    uint4* wf = nullptr;
    if (int rc = S.arena.alloc(&wf, LMAP_W_WORDS)) return rc;
    if (int rc = lmap_pack(dw, wf, c->stream)) return rc;
    CUP_CUDA_TRY(cudaStreamSynchronize(c->stream));
    S.schwarz_w = wf;
  }
  if (int rc = ensure_lab(c)) return rc;
  *out = LocalMap{S.schwarz_w, S.lmap_lab};
  return 0;
}

// z += the local map on r's labs (its two phases as kernels of their own).
static int map_correction(cup_ctx* c, const LocalMap& lm, const double* d_r, double* d_z) {
  const int grid = std::max(1, std::min(c->num_sms * 2, (c->mesh.nb + LMAP_GATHER - 1) / LMAP_GATHER));
  {
    ProfScope ps("lmap_gather", c->stream);
    k_lmap_gather<<<grid, 256, 0, c->stream>>>(c->dm, d_r, lm.lab, mean_block_of(c));
  }
  CUP_CUDA_TRY(cudaGetLastError());
  static unsigned long long attr = 0;
  if (first_on_device(attr))
    CUP_CUDA_TRY(cudaFuncSetAttribute(k_lmap_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, int(LMAP_TILE_BYTES)));
  {
    ProfScope ps("lmap_gemm", c->stream);
    k_lmap_gemm<<<std::max(1, c->num_sms * 2), 256, LMAP_TILE_BYTES, c->stream>>>(c->dm, lm.w, lm.lab, d_z);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

// z = block inverse of r + the local map on r's labs.
static int map_apply(cup_ctx* c, const LocalMap& lm, const double* d_r, double* d_z) {
  if (int rc = launch_block_inverse(c->dm, d_r, d_z, c->W, c->stream)) return rc;
  if (int rc = map_correction(c, lm, d_r, d_z)) return rc;
  CUP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return 0;
}

}  // namespace cup3d

using namespace cup3d;

extern "C" {

int32_t cup_cnn_num_params(void) { return CNN_NPARAM; }

int cup_cnn_init(cup_ctx* c, uint64_t seed) {
  if (!c || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_cnn_init: no device context");
  // Variance-preserving normal weights for linear layers (1 / fan-in, fan-in
  // 27 C_in); the last layer starts small, so the preconditioner starts close
  // to the two-level one without the network.
  std::mt19937_64 g(seed);
  std::normal_distribution<float> n01(0.f, 1.f);
  std::vector<float> p(CNN_NPARAM, 0.f);
  auto fill = [&](int off, int cnt, float stdv) {
    for (int i = 0; i < cnt; ++i) p[off + i] = stdv * n01(g);
  };
  fill(OFF_W0, CNN_W0, std::sqrt(1.f / 27.f));
  fill(OFF_W1, CNN_W1, std::sqrt(1.f / (27.f * CNN_C)));
  fill(OFF_W2, CNN_W2, std::sqrt(1.f / (27.f * CNN_C)));
  fill(OFF_W3, CNN_W3, 0.01f * std::sqrt(1.f / (27.f * CNN_C)));
  if (int rc = set_params(c, p.data())) return ctx_fail(c, rc, cup_last_error(nullptr));
  return 0;
}

int cup_cnn_set_params(cup_ctx* c, const float* params) {
  if (!c || c->host_only || !params) return ctx_fail(c, CUP_ERR_ARG, "cup_cnn_set_params: bad arguments");
  if (int rc = set_params(c, params)) return ctx_fail(c, rc, cup_last_error(nullptr));
  return 0;
}

int cup_cnn_get_params(cup_ctx* c, float* params) {
  if (!c || !params || !c->cnn.W.master) return ctx_fail(c, CUP_ERR_STATE, "cup_cnn_get_params: no weights");
  cudaError_t e = stream_d2h(c->stream, params, c->cnn.W.master, CNN_NPARAM * sizeof(float));
  if (e != cudaSuccess) return ctx_fail(c, set_cuda_error(e, "cnn_get", __FILE__, __LINE__), cup_last_error(nullptr));
  return 0;
}

int cup_cnn_dataset_reserve(cup_ctx* c, int32_t capacity) {
  if (!c || c->host_only || capacity <= 0) return ctx_fail(c, CUP_ERR_ARG, "cup_cnn_dataset_reserve: bad arguments");
  CnnState& S = c->cnn;
  S.data_arena.release();
  S.cap = S.count = 0;
  int rc = S.data_arena.alloc(&S.ds_in, size_t(capacity) * 1000);
  if (!rc) rc = S.data_arena.alloc(&S.ds_target, size_t(capacity) * BN);
  if (!rc) rc = S.data_arena.alloc(&S.ds_count, 1);
  if (rc) return ctx_fail(c, rc, cup_last_error(nullptr));
  S.cap = capacity;
  return 0;
}

int cup_cnn_dataset_add(cup_ctx* c, const double* d_r, const double* /*d_e*/) {
  ProfBind pb_(c);
  if (!dev_ok(c) || !d_r) return ctx_fail(c, CUP_ERR_ARG, "cup_cnn_dataset_add: bad arguments");
  CnnState& S = c->cnn;
  if (S.cap == 0) return ctx_fail(c, CUP_ERR_STATE, "cup_cnn_dataset_add: no dataset (cup_cnn_dataset_reserve)");
  if (S.count >= S.cap) return 0;
  // the target: the overlap solve's correction of r (its local map alone)
  LocalMap lm{};
  if (int rc = schwarz_prepare(c, &lm)) return ctx_fail(c, rc, cup_last_error(nullptr));
  double* corr = c->W.t;
  CUP_CUDA_TRY(cudaMemsetAsync(corr, 0, nbn(c) * sizeof(double), c->stream));
  if (int rc = map_correction(c, lm, d_r, corr)) return ctx_fail(c, rc, cup_last_error(nullptr));
  if (int rc = cnn_dataset_add(c->dm, d_r, corr, S.ds_in, S.ds_target, S.count, S.cap, S.ds_count, c->W.grid,
                               c->stream, mean_block_of(c)))
    return ctx_fail(c, rc, cup_last_error(nullptr));
  S.count = std::min(S.cap, S.count + c->mesh.nb);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return ctx_fail(c, set_cuda_error(e, "dataset_add", __FILE__, __LINE__), cup_last_error(nullptr));
  return 0;
}

int32_t cup_cnn_dataset_size(const cup_ctx* c) { return c ? c->cnn.count : 0; }

int cup_cnn_train(cup_ctx* c, int32_t steps, int32_t batch, float lr, uint64_t seed, float* loss_out) {
  ProfBind pb_(c);
  if (!c || c->host_only || steps < 0 || batch <= 0) return ctx_fail(c, CUP_ERR_ARG, "cup_cnn_train: bad arguments");
  CnnState& S = c->cnn;
  if (!S.ready) return ctx_fail(c, CUP_ERR_STATE, "cup_cnn_train: no weights (cup_cnn_init)");
  if (S.count <= 0) return ctx_fail(c, CUP_ERR_STATE, "cup_cnn_train: empty dataset");
  if (S.idx_cap < batch) {
    int* p = nullptr;
    if (int rc = S.arena.alloc(&p, batch)) return ctx_fail(c, rc, cup_last_error(nullptr));
    S.idx = p;
    S.idx_cap = batch;
  }
  // Train in normalised units: targets read divided by their RMS and the
  // output layer expressed in the same units during the steps, then scaled
  // back, so the stored network keeps predicting raw targets.  The reported
  // losses are relative to the targets' mean square.
  double rms = 0.0;
  if (int rc = target_rms(c, &rms)) return ctx_fail(c, rc, cup_last_error(nullptr));
  if (!(rms > 0.0)) rms = 1.0;
  if (int rc = scale_output_layer(c, float(1.0 / rms))) return ctx_fail(c, rc, cup_last_error(nullptr));
  int train_rc = 0;
  std::mt19937_64 g(seed);
  const int ntrain = S.count - std::min(S.ntest, S.count - 1);
  std::uniform_int_distribution<int> pick(0, ntrain - 1);
  std::vector<int> idx(batch);
  for (int it = 0; it < steps && !train_rc; ++it) {
    for (int i = 0; i < batch; ++i) idx[i] = pick(g);
    cudaError_t e = cudaMemcpyAsync(S.idx, idx.data(), batch * sizeof(int), cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) {
      train_rc = set_cuda_error(e, "train idx", __FILE__, __LINE__);
      break;
    }
    S.adam_t += 1;
    if ((train_rc = cnn_train_step(S.W, S.adam_m, S.adam_v, S.adam_t, lr, S.ds_in, S.ds_target, float(1.0 / rms),
                                   S.idx, batch, S.gpart, S.grad, S.loss, S.train_grid, c->stream)))
      break;
    if (loss_out) {
      e = cudaMemcpyAsync(&loss_out[it], S.loss, sizeof(float), cudaMemcpyDeviceToHost, c->stream);
      if (e != cudaSuccess) {
        train_rc = set_cuda_error(e, "train loss", __FILE__, __LINE__);
        break;
      }
    }
    // the host index buffer is reused next iteration: wait for its copy
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) train_rc = set_cuda_error(e, "train", __FILE__, __LINE__);
  }
  c->cnn.folded = false;
  const int back_rc = scale_output_layer(c, float(rms));
  if (train_rc || back_rc) return ctx_fail(c, train_rc ? train_rc : back_rc, cup_last_error(nullptr));
  if (int rc = cnn_pack(S.W, c->stream)) return ctx_fail(c, rc, cup_last_error(nullptr));
  if (cudaError_t e = cudaStreamSynchronize(c->stream))
    return ctx_fail(c, set_cuda_error(e, "train", __FILE__, __LINE__), cup_last_error(nullptr));
  return 0;
}

int cup_cnn_holdout(cup_ctx* c, int32_t ntest) {
  if (!c || ntest < 0) return ctx_fail(c, CUP_ERR_ARG, "cup_cnn_holdout: bad arguments");
  c->cnn.ntest = ntest;
  return 0;
}

int cup_cnn_eval(cup_ctx* c, float* rel_loss) {
  ProfBind pb_(c);
  if (!c || !rel_loss || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_cnn_eval: bad arguments");
  CnnState& S = c->cnn;
  if (!S.ready) return ctx_fail(c, CUP_ERR_STATE, "cup_cnn_eval: no weights");
  const int nt = std::min(S.ntest, S.count);
  if (nt <= 0) return ctx_fail(c, CUP_ERR_STATE, "cup_cnn_eval: no held-out samples (cup_cnn_holdout)");
  const int first = S.count - nt;
  const float* in = S.ds_in + size_t(first) * 1000;
  const float* tg = S.ds_target + size_t(first) * BN;
  // the residual-norm loss of the network and of the zero prediction over them
  double err = 0.0, ms = 0.0;
  for (int b0 = 0; b0 < nt; b0 += S.train_grid) {
    const int nb_ = std::min(S.train_grid, nt - b0);
    for (int zero = 0; zero < 2; ++zero) {
      if (int rc = cnn_residual_loss(S.W, in + size_t(b0) * 1000, tg + size_t(b0) * BN, nb_, zero, S.gpart, S.loss,
                                     S.train_grid, c->stream))
        return ctx_fail(c, rc, cup_last_error(nullptr));
      float l = 0.f;
      CUP_CUDA_TRY(stream_d2h(c->stream, &l, S.loss, sizeof(float)));
      (zero ? ms : err) += double(l) * nb_;
    }
  }
  *rel_loss = float(ms > 0 ? err / ms : 0.0);
  return 0;
}

int cup_cnn_forward_host(cup_ctx* c, const float* in, float* out, int32_t n) {
  if (!c || c->host_only || !in || !out || n <= 0) return ctx_fail(c, CUP_ERR_ARG, "cup_cnn_forward_host: bad arguments");
  CnnState& S = c->cnn;
  if (!S.ready) return ctx_fail(c, CUP_ERR_STATE, "no weights");
  DevArena tmp;
  float *din, *dout;
  int rc = tmp.alloc(&din, size_t(n) * 1000);
  if (!rc) rc = tmp.alloc(&dout, size_t(n) * BN);
  if (rc) return ctx_fail(c, rc, cup_last_error(nullptr));
  if (cudaError_t e = stream_h2d(c->stream, din, in, size_t(n) * 1000 * sizeof(float)))
    return ctx_fail(c, set_cuda_error(e, "cnn_forward in", __FILE__, __LINE__), cup_last_error(nullptr));
  if ((rc = cnn_forward_batch(S.W, din, dout, n, S.gpart, S.train_grid, c->stream)))
    return ctx_fail(c, rc, cup_last_error(nullptr));
  cudaError_t e = cudaMemcpyAsync(out, dout, size_t(n) * BN * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return ctx_fail(c, set_cuda_error(e, "cnn_forward", __FILE__, __LINE__), cup_last_error(nullptr));
  return 0;
}

int cup_cnn_grad_host(cup_ctx* c, const float* in, const float* target, int32_t n, float* grad, float* loss) {
  if (!c || c->host_only || !in || !target || !grad || n <= 0)
    return ctx_fail(c, CUP_ERR_ARG, "cup_cnn_grad_host: bad arguments");
  CnnState& S = c->cnn;
  if (!S.ready) return ctx_fail(c, CUP_ERR_STATE, "no weights");
  DevArena tmp;
  float *din, *dt;
  int rc = tmp.alloc(&din, size_t(n) * 1000);
  if (!rc) rc = tmp.alloc(&dt, size_t(n) * BN);
  if (rc) return ctx_fail(c, rc, cup_last_error(nullptr));
  cudaError_t e = stream_h2d(c->stream, din, in, size_t(n) * 1000 * sizeof(float));
  if (e == cudaSuccess) e = stream_h2d(c->stream, dt, target, size_t(n) * BN * sizeof(float));
  if (e != cudaSuccess) return ctx_fail(c, set_cuda_error(e, "cnn_grad in", __FILE__, __LINE__), cup_last_error(nullptr));
  if ((rc = cnn_grad_batch(S.W, din, dt, n, S.gpart, S.grad, S.loss, S.train_grid, c->stream)))
    return ctx_fail(c, rc, cup_last_error(nullptr));
  e = cudaMemcpyAsync(grad, S.grad, CNN_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && loss) e = cudaMemcpyAsync(loss, S.loss, sizeof(float), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return ctx_fail(c, set_cuda_error(e, "cnn_grad", __FILE__, __LINE__), cup_last_error(nullptr));
  return 0;
}

int cup_cnn_precond_dev(cup_ctx* c, const double* d_r, double* d_z) {
  ProfBind pb_(c);
  if (!dev_ok(c) || !d_r || !d_z) return ctx_fail(c, CUP_ERR_ARG, "cup_cnn_precond_dev: bad arguments");
  if (!c->cnn.ready) return ctx_fail(c, CUP_ERR_STATE, "no weights");
  GridReduce g{c->W.partial, c->W.counters + 15};
  if (int rc = cnn_apply<double>(c->dm, d_r, d_z, c->cnn.W, c->W.grid, c->stream, g, nullptr, mean_block_of(c)))
    return ctx_fail(c, rc, cup_last_error(nullptr));
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return ctx_fail(c, set_cuda_error(e, "cnn_precond", __FILE__, __LINE__), cup_last_error(nullptr));
  return 0;
}

int cup_cnn_map_apply_dev(cup_ctx* c, const double* d_r, double* d_z) {
  ProfBind pb_(c);
  if (!dev_ok(c) || !d_r || !d_z) return ctx_fail(c, CUP_ERR_ARG, "cup_cnn_map_apply_dev: bad arguments");
  LocalMap lm{};
  if (int rc = lmap_prepare(c, &lm)) return ctx_fail(c, rc, cup_last_error(nullptr));
  if (int rc = map_apply(c, lm, d_r, d_z)) return ctx_fail(c, rc, cup_last_error(nullptr));
  return 0;
}

int cup_schwarz_apply_dev(cup_ctx* c, const double* d_r, double* d_z) {
  ProfBind pb_(c);
  if (!dev_ok(c) || !d_r || !d_z) return ctx_fail(c, CUP_ERR_ARG, "cup_schwarz_apply_dev: bad arguments");
  LocalMap lm{};
  if (int rc = schwarz_prepare(c, &lm)) return ctx_fail(c, rc, cup_last_error(nullptr));
  if (int rc = map_apply(c, lm, d_r, d_z)) return ctx_fail(c, rc, cup_last_error(nullptr));
  return 0;
}

int cup_set_poisson(cup_ctx* c, int32_t solver, double tol_abs, double tol_rel, int32_t max_iter) {
  if (!c || solver < 0 || solver > CUP_POISSON_B200_TWOLEVEL_MIXED || max_iter < 0)
    return ctx_fail(c, CUP_ERR_ARG, "cup_set_poisson: bad arguments");
  c->cfg.poisson_solver = solver;
  c->cfg.poisson_tol = tol_abs;
  c->cfg.poisson_tol_rel = tol_rel;
  c->cfg.poisson_max_iter = max_iter;
  graph_reset(c);  // captured steps hold the old settings
  return 0;
}

int cup_set_barrier_limit(cup_ctx* c, int64_t cycles) {
  if (!c || cycles < 0) return ctx_fail(c, CUP_ERR_ARG, "cup_set_barrier_limit: bad arguments");
  c->W.barrier_cycles = cycles;
  graph_reset(c);  // captured steps hold the old limit
  return 0;
}

}  // extern "C"
