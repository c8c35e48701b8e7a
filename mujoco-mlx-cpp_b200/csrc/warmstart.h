// Learned Newton warm start: a 3 x 256 GELU MLP that predicts the change of
// the converged acceleration from the previous substep's.  The prediction
// qacc_prev + mean + std * y enters the Newton solver as a third warm-start
// candidate next to qacc_smooth and the previous qacc; the solver keeps the
// cheapest by the Gauss cost and iterates to the same tolerance, so a poor
// prediction costs nothing but the inference.  No counterpart in the
// reference (its solver cold-starts, solver.hpp:592).
//
// Per-env models: the step kernel evaluates the net itself after the
// constraint build of every substep, on that substep's features (state,
// unconstrained acceleration, previous converged acceleration, controls,
// contacts; dev_nn.cuh), with bf16 mma.sync tiles shared by the CTA's warps.
// Per-body models (free bodies only, nv > 64): one row per body from the end
// of the previous substep, inferred by a separate tcgen05 launch.
//
// Training, and the per-body inference, run on the GPU through BF16 tcgen05
// GEMMs with FP32 accumulation (mlp_kernels.cu); parameters are kept in FP32
// with Adam.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "engine.h"
#include "mlp_kernels.cuh"
#include "step_params.h"

namespace mjb {

class WarmStartNet {
 public:
  static constexpr int kHidden = 256;
  static constexpr int kLayers = 4;  // three hidden GELU layers and the output layer
  static constexpr int kOutPad = 64;

  WarmStartNet(int in_raw, int nout, uint64_t seed);
  ~WarmStartNet();

  int in_raw() const { return in_raw_; }
  int in_pad() const { return in_pad_; }
  int nout() const { return nout_; }
  int num_params() const { return nparam_; }
  int rows(int l) const { return rows_[l]; }
  int cols(int l) const { return cols_[l]; }

  void get_params(float* host) const;
  void set_params(const float* host);
  // Normalisation of the raw inputs and of the targets (host arrays).
  void set_normalization(const float* in_mean, const float* in_std, const float* out_mean, const float* out_std);
  void get_normalization(float* in_mean, float* in_std, float* out_mean, float* out_std) const;
  // Mean / standard deviation of device data xraw[n][in_raw], traw[n][nout].
  void fit_normalization(const float* xraw, const float* traw, int n);

  // y[n][nout] (device): network output in normalised target units.
  void forward(const float* xraw, int n, float* y);
  // Loss (mean over rows of the squared normalised error summed over the
  // outputs / nout) and its gradient with respect to every parameter
  // (host, parameter layout), for one batch taken in order.
  float gradients(const float* xraw, const float* traw, int n, float* grads_host);
  // Adam training on device data; epoch_loss (host, may be null) receives the
  // mean batch loss of each epoch.  Returns the number of optimiser steps.
  int train(const float* xraw, const float* traw, int n, int epochs, int batch, float lr, uint64_t seed, float* epoch_loss);

  // Inference for a sim: features feat[B][fstride] (first nfeat used) and
  // controls ctrl[B][nu] form the raw input; pred[B][nout] = prev + mean +
  // std * y.  Runs on stream s (capturable: buffers are fixed per B).
  // fused: one kernel (gather + 4 layers + prediction); otherwise the gather
  // kernel and 4 GEMM launches.  Both compute the same arithmetic.
  void infer(const float* feat, int fstride, int nfeat, const float* ctrl, int nu, const float* prev, float* pred, int B, cudaStream_t s,
             bool fused = true);
  // Allocates the inference buffers for batches of B envs (separate from the
  // training buffers, so captured inference graphs stay valid while the net
  // trains); a net serves one inference batch size.
  void prepare_inference(int B);

  int error_word();

  // Device pointers of the weights (bf16 [rows][cols] per layer), biases and
  // normalisation for the step kernel's fused inference (StepParams nn_*).
  void fill_fused(StepParams& P) const;

 private:
  void ensure_batch(int n);
  void split_k(GemmArgs& g);
  void build_weight_maps();
  const CUtensorMap& pick_b(GemmArgs& g, const CUtensorMap& wide, const CUtensorMap& narrow, bool has_narrow) const;
  void build_maps(int n);
  void forward_batch(int n, bool train, const float* target, float* loss, float* y_f32, const float* prev, float* pred, cudaStream_t s,
                     bool inference_buffers = false);
  void backward_batch(int n, cudaStream_t s);
  float* P(int l) { return params_.p + woff_[l]; }
  float* Bias(int l) { return params_.p + boff_[l]; }
  __nv_bfloat16* W(int l) { return reinterpret_cast<__nv_bfloat16*>(wb_.p) + woff_[l] - layer_base_[l]; }
  __nv_bfloat16* WT(int l) { return reinterpret_cast<__nv_bfloat16*>(wtb_.p) + woff_[l] - layer_base_[l]; }

  int in_raw_, in_pad_, nout_;
  int rows_[kLayers], cols_[kLayers];
  size_t woff_[kLayers], boff_[kLayers], layer_base_[kLayers];
  int nparam_ = 0, nweight_ = 0;
  cudaStream_t stream_ = nullptr;

  DevBuf<float> params_, grads_, adam_m_, adam_v_;
  DevBuf<uint16_t> wb_, wtb_;  // bf16 weights [rows][cols] and transposes, packed by layer (weights only)
  DevBuf<float> in_mean_, in_istd_, out_mean_, out_std_, out_istd_;
  std::vector<float> h_in_mean_, h_in_std_, h_out_mean_, h_out_std_;
  DevBuf<int> err_;
  DevBuf<float> loss_;
  DevBuf<float> splitk_;   // split-K partial tiles of the weight-gradient GEMMs

  // batch scratch (capacity cap_)
  int cap_ = 0, maps_n_ = -1;
  DevBuf<uint16_t> x_, xt_, z_[3], h_[3], ht_[3], dy_, dyt_, dza_, dzb_, dzat_, dzbt_;
  DevBuf<float> t_, yf_, zero_prev_;
  DevBuf<int> idx_;
  CUtensorMap m_x_, m_h_[3], m_w_[kLayers], m_wt_[kLayers], m_dy_, m_dyt_, m_xt_, m_ht_[3], m_dza_, m_dzb_, m_dzat_, m_dzbt_;
  // the same weights with 64-row boxes, for GEMMs whose M is too small to
  // fill the GPU with one CTA per 256 output columns (w64_ / wt64_: which exist)
  CUtensorMap m_w64_[kLayers], m_wt64_[kLayers];
  bool w64_[kLayers] = {}, wt64_[kLayers] = {};
  int adam_t_ = 0;
  // inference buffers (batch inf_B_)
  int inf_B_ = 0;
  DevBuf<uint16_t> xi_, hi_[3];
  CUtensorMap m_xi_, m_hi_[3];
};

}  // namespace mjb
