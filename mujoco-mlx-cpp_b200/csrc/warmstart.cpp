// Host side of the learned warm start: parameter storage, normalisation,
// training loop (forward, backward, Adam on the GPU), inference for a sim.
#include "warmstart.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>

#include "mlp_kernels.cuh"

namespace mjb {

namespace {

__nv_bfloat16* bf(DevBuf<uint16_t>& b) { return reinterpret_cast<__nv_bfloat16*>(b.p); }

void map_or_throw(CUtensorMap* m, const void* base, int rows, int cols, int box_rows) {
  if (!make_tmap_bf16(m, base, rows, cols, box_rows))
    throw std::runtime_error("warm start: tensor map encode failed (rows " + std::to_string(rows) + ", cols " + std::to_string(cols) + ")");
}

GemmArgs gemm_args(int M, int N, int K, int mode, int ldo, int* err) {
  GemmArgs a{};
  a.M = M;
  a.N = N;
  a.K = K;
  a.mode = mode;
  a.ldo = ldo;
  a.err = err;
  return a;
}

}  // namespace

WarmStartNet::WarmStartNet(int in_raw, int nout, uint64_t seed) : in_raw_(in_raw), nout_(nout) {
  if (in_raw <= 0 || in_raw > 256 || nout <= 0 || nout > kOutPad) throw std::runtime_error("warm start: input width must be 1..256 and outputs 1..64");
  in_pad_ = (in_raw + 63) / 64 * 64;
  rows_[0] = kHidden;
  cols_[0] = in_pad_;
  rows_[1] = rows_[2] = kHidden;
  cols_[1] = cols_[2] = kHidden;
  rows_[3] = kOutPad;
  cols_[3] = kHidden;
  size_t off = 0, woff = 0;
  for (int l = 0; l < kLayers; l++) {
    woff_[l] = off;
    layer_base_[l] = off - woff;
    off += (size_t)rows_[l] * cols_[l];
    woff += (size_t)rows_[l] * cols_[l];
    boff_[l] = off;
    off += rows_[l];
  }
  nparam_ = (int)off;
  nweight_ = (int)woff;
  check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "warm start stream");
  params_.alloc(nparam_);
  grads_.alloc(nparam_);
  adam_m_.alloc(nparam_);
  adam_v_.alloc(nparam_);
  wb_.alloc(nweight_);
  wtb_.alloc(nweight_);
  err_.alloc(1);
  loss_.alloc(1);
  check(cudaMemsetAsync(err_.p, 0, sizeof(int), stream_), "warm start err");
  check(cudaStreamSynchronize(stream_), "warm start sync");
  // initial parameters: U(+-1/sqrt(fan_in)) on real inputs, output layer x0.1,
  // zero biases, zero weights on padded inputs / outputs
  std::vector<float> h(nparam_, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < kLayers; l++) {
    const int fan_in = l == 0 ? in_raw_ : cols_[l];
    const int real_rows = l == kLayers - 1 ? nout_ : rows_[l];
    const float bound = (l == kLayers - 1 ? 0.1f : 1.f) / std::sqrt((float)fan_in);
    std::uniform_real_distribution<float> U(-bound, bound);
    for (int r = 0; r < real_rows; r++)
      for (int c = 0; c < fan_in; c++) h[woff_[l] + (size_t)r * cols_[l] + c] = U(rng);
  }
  set_params(h.data());
  std::vector<float> zi(in_raw_, 0.f), oi(in_raw_, 1.f), zo(nout_, 0.f), oo(nout_, 1.f);
  set_normalization(zi.data(), oi.data(), zo.data(), oo.data());
}

WarmStartNet::~WarmStartNet() {
  if (stream_) cudaStreamDestroy(stream_);
}

// Copies and fills run on the net's own stream and are waited for (the
// stream is non-blocking, so legacy-stream copies would not be ordered with
// its kernels).
int WarmStartNet::error_word() {
  int e = 0;
  if (cudaMemcpyAsync(&e, err_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_) != cudaSuccess) return -1;
  cudaStreamSynchronize(stream_);
  return e;
}

void WarmStartNet::get_params(float* host) const {
  check(cudaMemcpyAsync(host, params_.p, sizeof(float) * nparam_, cudaMemcpyDeviceToHost, stream_), "warm start get params");
  check(cudaStreamSynchronize(stream_), "warm start sync");
}

void WarmStartNet::set_params(const float* host) {
  check(cudaMemcpyAsync(params_.p, host, sizeof(float) * nparam_, cudaMemcpyHostToDevice, stream_), "warm start set params");
  check(cudaMemsetAsync(adam_m_.p, 0, sizeof(float) * nparam_, stream_), "adam m");
  check(cudaMemsetAsync(adam_v_.p, 0, sizeof(float) * nparam_, stream_), "adam v");
  adam_t_ = 0;
  for (int l = 0; l < kLayers; l++) check(cast_weights(rows_[l], cols_[l], P(l), W(l), WT(l), stream_), "cast weights");
  check(cudaStreamSynchronize(stream_), "warm start sync");
}

void WarmStartNet::fill_fused(StepParams& P) const {
  for (int l = 0; l < kLayers; l++) {
    P.nn_w[l] = wb_.p + woff_[l] - layer_base_[l];
    P.nn_b[l] = params_.p + boff_[l];
    P.nn_rows[l] = rows_[l];
    P.nn_cols[l] = cols_[l];
  }
  P.nn_in_mean = in_mean_.p;
  P.nn_in_istd = in_istd_.p;
  P.nn_out_mean = out_mean_.p;
  P.nn_out_std = out_std_.p;
  P.nn_in_raw = in_raw_;
  P.nn_nout = nout_;
}

void WarmStartNet::set_normalization(const float* in_mean, const float* in_std, const float* out_mean, const float* out_std) {
  h_in_mean_.assign(in_mean, in_mean + in_raw_);
  h_in_std_.assign(in_std, in_std + in_raw_);
  h_out_mean_.assign(out_mean, out_mean + nout_);
  h_out_std_.assign(out_std, out_std + nout_);
  std::vector<float> iis(in_raw_), ois(nout_), os(nout_);
  for (int j = 0; j < in_raw_; j++) iis[j] = h_in_std_[j] > 1e-6f ? 1.f / h_in_std_[j] : 0.f;
  for (int k = 0; k < nout_; k++) {
    os[k] = std::max(h_out_std_[k], 1e-6f);
    ois[k] = 1.f / os[k];
  }
  in_mean_.upload(h_in_mean_, stream_);
  in_istd_.upload(iis, stream_);
  out_mean_.upload(h_out_mean_, stream_);
  out_std_.upload(os, stream_);
  out_istd_.upload(ois, stream_);
  check(cudaStreamSynchronize(stream_), "warm start sync");
}

void WarmStartNet::get_normalization(float* in_mean, float* in_std, float* out_mean, float* out_std) const {
  if (in_mean) std::copy(h_in_mean_.begin(), h_in_mean_.end(), in_mean);
  if (in_std) std::copy(h_in_std_.begin(), h_in_std_.end(), in_std);
  if (out_mean) std::copy(h_out_mean_.begin(), h_out_mean_.end(), out_mean);
  if (out_std) std::copy(h_out_std_.begin(), h_out_std_.end(), out_std);
}

void WarmStartNet::fit_normalization(const float* xraw, const float* traw, int n) {
  if (n <= 1) throw std::runtime_error("warm start: need at least 2 samples");
  DevBuf<double> s, q;
  const int c = std::max(in_raw_, nout_);
  s.alloc(c);
  q.alloc(c);
  std::vector<double> hs(c), hq(c);
  std::vector<float> im(in_raw_), is(in_raw_), om(nout_), os(nout_);
  auto stats = [&](const float* x, int cols, float* mean, float* sd) {
    check(column_stats(x, n, cols, cols, s.p, q.p, stream_), "column stats");
    check(cudaMemcpyAsync(hs.data(), s.p, sizeof(double) * cols, cudaMemcpyDeviceToHost, stream_), "stats copy");
    check(cudaMemcpyAsync(hq.data(), q.p, sizeof(double) * cols, cudaMemcpyDeviceToHost, stream_), "stats copy");
    check(cudaStreamSynchronize(stream_), "stats sync");
    for (int j = 0; j < cols; j++) {
      const double m = hs[j] / n;
      mean[j] = (float)m;
      sd[j] = (float)std::sqrt(std::max(hq[j] / n - m * m, 0.0));
    }
  };
  stats(xraw, in_raw_, im.data(), is.data());
  stats(traw, nout_, om.data(), os.data());
  set_normalization(im.data(), is.data(), om.data(), os.data());
}

void WarmStartNet::ensure_batch(int n) {
  if (n <= cap_) return;
  const int cap = (n + 127) / 128 * 128;
  const size_t H = kHidden;
  x_.alloc((size_t)cap * in_pad_);
  xt_.alloc((size_t)cap * in_pad_);
  for (int i = 0; i < 3; i++) {
    z_[i].alloc(cap * H);
    h_[i].alloc(cap * H);
    ht_[i].alloc(cap * H);
  }
  dy_.alloc((size_t)cap * kOutPad);
  dyt_.alloc((size_t)cap * 128);
  dza_.alloc(cap * H);
  dzb_.alloc(cap * H);
  dzat_.alloc(cap * H);
  dzbt_.alloc(cap * H);
  t_.alloc((size_t)cap * nout_);
  yf_.alloc((size_t)cap * kOutPad);
  zero_prev_.alloc((size_t)cap * nout_);
  check(cudaMemsetAsync(zero_prev_.p, 0, sizeof(float) * cap * nout_, stream_), "zero prev");
  check(cudaStreamSynchronize(stream_), "warm start sync");
  cap_ = cap;
  maps_n_ = -1;
}

void WarmStartNet::build_weight_maps() {
  for (int l = 0; l < kLayers; l++) {
    map_or_throw(&m_w_[l], W(l), rows_[l], cols_[l], rows_[l]);
    w64_[l] = rows_[l] > 64 && rows_[l] % 64 == 0;
    if (w64_[l]) map_or_throw(&m_w64_[l], W(l), rows_[l], cols_[l], 64);
  }
  for (int l = 1; l < kLayers; l++) {
    map_or_throw(&m_wt_[l], WT(l), cols_[l], rows_[l], cols_[l]);
    wt64_[l] = cols_[l] > 64 && cols_[l] % 64 == 0;
    if (wt64_[l]) map_or_throw(&m_wt64_[l], WT(l), cols_[l], rows_[l], 64);
  }
}

// B operand of a GEMM whose N is the weight's row count: 64-column tiles
// (four CTAs per 256 columns) when one CTA per 256 columns would use under
// half the SMs, as for a 4096-row training batch (32 row tiles).
const CUtensorMap& WarmStartNet::pick_b(GemmArgs& g, const CUtensorMap& wide, const CUtensorMap& narrow, bool has_narrow) const {
  const int ctas = (g.M + 127) / 128 * ((g.N + 255) / 256);
  if (has_narrow && g.N > 64 && g.N % 64 == 0 && 2 * ctas <= 148) {
    g.bn = 64;
    return narrow;
  }
  return wide;
}

void WarmStartNet::build_maps(int n) {
  if (n == maps_n_) return;
  const int H = kHidden;
  map_or_throw(&m_x_, x_.p, n, in_pad_, 128);
  for (int i = 0; i < 3; i++) map_or_throw(&m_h_[i], h_[i].p, n, H, 128);
  build_weight_maps();
  map_or_throw(&m_dy_, dy_.p, n, kOutPad, 128);
  map_or_throw(&m_dza_, dza_.p, n, H, 128);
  map_or_throw(&m_dzb_, dzb_.p, n, H, 128);
  if (n % 64 == 0) {
    // transposed operands of the weight-gradient GEMMs (K = batch)
    map_or_throw(&m_dyt_, dyt_.p, 128, n, 128);
    map_or_throw(&m_xt_, xt_.p, in_pad_, n, in_pad_);
    for (int i = 0; i < 3; i++) map_or_throw(&m_ht_[i], ht_[i].p, H, n, H);
    map_or_throw(&m_dzat_, dzat_.p, H, n, 128);
    map_or_throw(&m_dzbt_, dzbt_.p, H, n, 128);
    check(cudaMemsetAsync(dyt_.p, 0, sizeof(uint16_t) * 128 * (size_t)n, stream_), "dyt zero");
  }
  maps_n_ = n;
}

// Forward pass of n rows already gathered into x_.  train: keeps the
// pre-activations and transposes and writes the loss gradient of the output;
// y_f32: network output (with bias) to yf_; pred: the sim prediction.
void WarmStartNet::forward_batch(int n, bool train, const float* target, float* loss, float* y_f32, const float* prev, float* pred, cudaStream_t s,
                                 bool inference_buffers) {
  const int H = kHidden;
  const CUtensorMap* a_map = inference_buffers ? &m_xi_ : &m_x_;
  int K = in_pad_;
  for (int l = 0; l < 3; l++) {
    GemmArgs a = gemm_args(n, H, K, EPI_HIDDEN, H, err_.p);
    a.bias = Bias(l);
    a.out = bf(inference_buffers ? hi_[l] : h_[l]);
    if (train) {
      a.pre = bf(z_[l]);
      a.out_t = bf(ht_[l]);
      a.ldt = n;
    }
    check(gemm_tn(*a_map, pick_b(a, m_w_[l], m_w64_[l], w64_[l]), a, s), "warm start forward gemm");
    a_map = inference_buffers ? &m_hi_[l] : &m_h_[l];
    K = H;
  }
  GemmArgs a = gemm_args(n, kOutPad, H, EPI_F32, kOutPad, err_.p);
  a.bias = Bias(3);
  a.nvalid = nout_;
  if (train) {
    a.mode = EPI_OUT_LOSS;
    a.target = target;
    a.loss = loss;
    a.scale = 2.f / ((float)n * (float)nout_);
    a.out = bf(dy_);
    a.out_t = bf(dyt_);
    a.ldt = n;
  } else if (pred) {
    a.mode = EPI_OUT_PRED;
    a.prev = prev;
    a.omean = out_mean_.p;
    a.ostd = out_std_.p;
    a.pred = pred;
  } else {
    a.out_f32 = y_f32;
  }
  check(gemm_tn(*a_map, m_w_[3], a, s), "warm start output gemm");
}

// Weight gradients have K = the batch (thousands) and only one or two
// output tiles: split K over enough CTAs to spread the loop over the SMs.
void WarmStartNet::split_k(GemmArgs& g) {
  const int ks = gemm_ksplit(g.M, g.N, g.K);
  if (ks <= 1) return;
  const size_t need = (size_t)ks * g.M * g.ldo;
  if (splitk_.n < need) splitk_.alloc(need);
  g.ksplit = ks;
  g.split_ws = splitk_.p;
}

void WarmStartNet::backward_batch(int n, cudaStream_t s) {
  const int H = kHidden;
  // output layer: dW3 = dY^T H2, db3 = colsum dY, dZ2 = (dY W3) * gelu'(Z2)
  {
    GemmArgs a = gemm_args(kOutPad, H, n, EPI_F32, H, err_.p);
    a.out_f32 = grads_.p + woff_[3];
    split_k(a);
    check(gemm_tn(m_dyt_, m_ht_[2], a, s), "dW3");
    check(rowsum_bf16(bf(dyt_), kOutPad, n, n, grads_.p + boff_[3], s), "db3");
    GemmArgs b = gemm_args(n, H, kOutPad, EPI_BWD_GELU, H, err_.p);
    b.pre_in = bf(z_[2]);
    b.out = bf(dza_);
    b.out_t = bf(dzat_);
    b.ldt = n;
    check(gemm_tn(m_dy_, pick_b(b, m_wt_[3], m_wt64_[3], wt64_[3]), b, s), "dH2");
  }
  // hidden layers 2, 1 (dZ ping-pongs between the a and b buffers)
  DevBuf<uint16_t>* dz = &dza_;
  DevBuf<uint16_t>* dzt = &dzat_;
  DevBuf<uint16_t>* nz = &dzb_;
  DevBuf<uint16_t>* nzt = &dzbt_;
  const CUtensorMap* m_dz = &m_dza_;
  const CUtensorMap* m_dzt = &m_dzat_;
  const CUtensorMap* m_nz = &m_dzb_;
  const CUtensorMap* m_nzt = &m_dzbt_;
  for (int l = 2; l >= 1; l--) {
    GemmArgs a = gemm_args(H, H, n, EPI_F32, H, err_.p);
    a.out_f32 = grads_.p + woff_[l];
    split_k(a);
    check(gemm_tn(*m_dzt, m_ht_[l - 1], a, s), "dW hidden");
    check(rowsum_bf16(bf(*dzt), H, n, n, grads_.p + boff_[l], s), "db hidden");
    GemmArgs b = gemm_args(n, H, H, EPI_BWD_GELU, H, err_.p);
    b.pre_in = bf(z_[l - 1]);
    b.out = bf(*nz);
    b.out_t = bf(*nzt);
    b.ldt = n;
    check(gemm_tn(*m_dz, pick_b(b, m_wt_[l], m_wt64_[l], wt64_[l]), b, s), "dH hidden");
    std::swap(dz, nz);
    std::swap(dzt, nzt);
    std::swap(m_dz, m_nz);
    std::swap(m_dzt, m_nzt);
  }
  // input layer: dW0 = dZ0^T X, db0
  GemmArgs a = gemm_args(H, in_pad_, n, EPI_F32, in_pad_, err_.p);
  a.out_f32 = grads_.p + woff_[0];
  split_k(a);
  check(gemm_tn(*m_dzt, m_xt_, a, s), "dW0");
  check(rowsum_bf16(bf(*dzt), H, n, n, grads_.p + boff_[0], s), "db0");
}

void WarmStartNet::forward(const float* xraw, int n, float* y) {
  if (n <= 0) return;
  ensure_batch(n);
  build_maps(n);
  check(gather_rows(n, nullptr, xraw, in_raw_, in_raw_, nullptr, 0, 0, in_mean_.p, in_istd_.p, bf(x_), in_pad_, nullptr, 0, nullptr, 0, nullptr,
                    nullptr, nullptr, stream_),
        "gather");
  forward_batch(n, false, nullptr, nullptr, yf_.p, nullptr, nullptr, stream_);
  check(cudaMemcpy2DAsync(y, sizeof(float) * nout_, yf_.p, sizeof(float) * kOutPad, sizeof(float) * nout_, n, cudaMemcpyDeviceToDevice, stream_),
        "forward copy");
  check(cudaStreamSynchronize(stream_), "forward sync");
  if (error_word()) throw std::runtime_error("warm start: a GEMM wait timed out");
}

float WarmStartNet::gradients(const float* xraw, const float* traw, int n, float* grads_host) {
  if (n <= 0 || n % 64 != 0) throw std::runtime_error("warm start: gradient batch must be a positive multiple of 64");
  ensure_batch(n);
  build_maps(n);
  check(cudaMemsetAsync(loss_.p, 0, sizeof(float), stream_), "loss zero");
  check(gather_rows(n, nullptr, xraw, in_raw_, in_raw_, nullptr, 0, 0, in_mean_.p, in_istd_.p, bf(x_), in_pad_, bf(xt_), n, traw, nout_,
                    out_mean_.p, out_istd_.p, t_.p, stream_),
        "gather");
  forward_batch(n, true, t_.p, loss_.p, nullptr, nullptr, nullptr, stream_);
  backward_batch(n, stream_);
  float loss = 0;
  check(cudaMemcpyAsync(&loss, loss_.p, sizeof(float), cudaMemcpyDeviceToHost, stream_), "loss copy");
  if (grads_host) check(cudaMemcpyAsync(grads_host, grads_.p, sizeof(float) * nparam_, cudaMemcpyDeviceToHost, stream_), "grad copy");
  check(cudaStreamSynchronize(stream_), "gradients sync");
  if (error_word()) throw std::runtime_error("warm start: a GEMM wait timed out");
  return loss / ((float)n * (float)nout_);
}

int WarmStartNet::train(const float* xraw, const float* traw, int n, int epochs, int batch, float lr, uint64_t seed, float* epoch_loss) {
  if (batch <= 0 || batch % 64 != 0) throw std::runtime_error("warm start: batch must be a positive multiple of 64");
  const int steps = n / batch;
  if (steps <= 0 || epochs <= 0) return 0;
  ensure_batch(batch);
  build_maps(batch);
  idx_.alloc((size_t)steps * batch);
  std::vector<int> perm(n);
  std::mt19937_64 rng(seed);
  const int total = steps * epochs;
  int step = 0;
  for (int e = 0; e < epochs; e++) {
    std::iota(perm.begin(), perm.end(), 0);
    std::shuffle(perm.begin(), perm.end(), rng);
    check(cudaMemcpyAsync(idx_.p, perm.data(), sizeof(int) * (size_t)steps * batch, cudaMemcpyHostToDevice, stream_), "perm upload");
    check(cudaMemsetAsync(loss_.p, 0, sizeof(float), stream_), "loss zero");
    for (int k = 0; k < steps; k++, step++) {
      check(gather_rows(batch, idx_.p + (size_t)k * batch, xraw, in_raw_, in_raw_, nullptr, 0, 0, in_mean_.p, in_istd_.p, bf(x_), in_pad_, bf(xt_),
                        batch, traw, nout_, out_mean_.p, out_istd_.p, t_.p, stream_),
            "gather");
      forward_batch(batch, true, t_.p, loss_.p, nullptr, nullptr, nullptr, stream_);
      backward_batch(batch, stream_);
      // cosine decay to 5 % of the initial rate
      const float rate = lr * (0.05f + 0.95f * 0.5f * (1.f + std::cos(3.14159265f * (float)step / (float)total)));
      adam_t_++;
      for (int l = 0; l < kLayers; l++) {
        check(adam_step(rows_[l] * cols_[l], P(l), grads_.p + woff_[l], adam_m_.p + woff_[l], adam_v_.p + woff_[l], rate, 0.9f, 0.999f, 1e-8f, adam_t_,
                        0.f, rows_[l], cols_[l], W(l), WT(l), stream_),
              "adam W");
        check(adam_step(rows_[l], Bias(l), grads_.p + boff_[l], adam_m_.p + boff_[l], adam_v_.p + boff_[l], rate, 0.9f, 0.999f, 1e-8f, adam_t_, 0.f,
                        1, rows_[l], nullptr, nullptr, stream_),
              "adam b");
      }
    }
    float l = 0;
    check(cudaMemcpyAsync(&l, loss_.p, sizeof(float), cudaMemcpyDeviceToHost, stream_), "loss copy");
    check(cudaStreamSynchronize(stream_), "epoch sync");
    if (epoch_loss) epoch_loss[e] = l / ((float)steps * batch * nout_);
  }
  if (error_word()) throw std::runtime_error("warm start: a GEMM wait timed out");
  return step;
}

void WarmStartNet::prepare_inference(int B) {
  if (B == inf_B_) return;
  if (inf_B_ != 0) throw std::runtime_error("warm start: this net already serves another batch size");
  if (B <= 0) throw std::runtime_error("warm start: bad inference batch");
  xi_.alloc((size_t)B * in_pad_);
  for (int i = 0; i < 3; i++) hi_[i].alloc((size_t)B * kHidden);
  map_or_throw(&m_xi_, xi_.p, B, in_pad_, 128);
  for (int i = 0; i < 3; i++) map_or_throw(&m_hi_[i], hi_[i].p, B, kHidden, 128);
  if (maps_n_ < 0) build_weight_maps();
  inf_B_ = B;
}

void WarmStartNet::infer(const float* feat, int fstride, int nfeat, const float* ctrl, int nu, const float* prev, float* pred, int B, cudaStream_t s,
                         bool fused) {
  if (nfeat + nu != in_raw_) throw std::runtime_error("warm start: features + controls do not match the network input width");
  prepare_inference(B);
  if (fused) {
    InferArgs a{};
    a.B = B;
    a.feat = feat;
    a.fstride = fstride;
    a.nfeat = nfeat;
    a.ctrl = ctrl;
    a.nu = nu;
    a.in_pad = in_pad_;
    a.mean = in_mean_.p;
    a.istd = in_istd_.p;
    for (int l = 0; l < kLayers; l++) {
      a.rows[l] = rows_[l];
      a.cols[l] = cols_[l];
      a.bias[l] = Bias(l);
    }
    a.nout = nout_;
    a.prev = prev;
    a.omean = out_mean_.p;
    a.ostd = out_std_.p;
    a.pred = pred;
    a.err = err_.p;
    check(mlp_infer(m_w_, a, s), "warm start fused inference");
    return;
  }
  check(gather_rows(B, nullptr, feat, fstride, nfeat, ctrl, nu, nu, in_mean_.p, in_istd_.p, bf(xi_), in_pad_, nullptr, 0, nullptr, 0, nullptr, nullptr,
                    nullptr, s),
        "gather");
  forward_batch(B, false, nullptr, nullptr, nullptr, prev, pred, s, true);
}

}  // namespace mjb
