// C ABI of the learned warm start (mjb200_warmstart.h).
#include <memory>
#include <stdexcept>
#include <string>

#include "../../include/mjmlx/mjb200_warmstart.h"
#include "capi_internal.h"
#include "engine.h"
#include "mlp_kernels.cuh"
#include "warmstart.h"

using mjb::set_error;

struct MjbWarmStart {
  std::unique_ptr<mjb::WarmStartNet> net;
};

namespace {

template <class F>
int guarded(const char* fn, F&& f) {
  try {
    return f();
  } catch (const std::exception& e) {
    set_error(std::string(fn) + ": " + e.what());
    return -1;
  }
}

}  // namespace

extern "C" {

MJMLX_API MjbWarmStart* mjb200_warmstart_create(int in_raw, int nout, unsigned long long seed) {
  try {
    auto* w = new MjbWarmStart();
    w->net = std::make_unique<mjb::WarmStartNet>(in_raw, nout, seed);
    return w;
  } catch (const std::exception& e) {
    set_error(std::string("mjb200_warmstart_create: ") + e.what());
    return nullptr;
  }
}

MJMLX_API void mjb200_warmstart_free(MjbWarmStart* net) { delete net; }

MJMLX_API int mjb200_warmstart_input_width(const MjmlxBatchedSim* sim) {
  if (!sim || !sim->engine) return -1;
  return guarded("mjb200_warmstart_input_width", [&] {
    if (!sim->engine->uniform()) throw std::runtime_error("needs a single-model batch");
    return sim->engine->warmstart_input_width();
  });
}

MJMLX_API int mjb200_warmstart_layout(const MjmlxBatchedSim* sim, int* in_raw, int* nout, int* rows_per_env) {
  if (!sim || !sim->engine) return -1;
  return guarded("mjb200_warmstart_layout", [&] {
    const auto& e = *sim->engine;
    if (!e.uniform()) throw std::runtime_error("needs a single-model batch");
    if (in_raw) *in_raw = e.warmstart_input_width();
    if (nout) *nout = e.warmstart_outputs();
    if (rows_per_env) *rows_per_env = e.rows_per_env();
    return 0;
  });
}

MJMLX_API int mjb200_warmstart_dims(const MjbWarmStart* w, int* in_raw, int* in_pad, int* hidden, int* nout, int* out_pad, int* nparams) {
  if (!w) return -1;
  const auto& n = *w->net;
  if (in_raw) *in_raw = n.in_raw();
  if (in_pad) *in_pad = n.in_pad();
  if (hidden) *hidden = mjb::WarmStartNet::kHidden;
  if (nout) *nout = n.nout();
  if (out_pad) *out_pad = mjb::WarmStartNet::kOutPad;
  if (nparams) *nparams = n.num_params();
  return 0;
}

MJMLX_API int mjb200_warmstart_get_params(const MjbWarmStart* w, float* params) {
  if (!w || !params) return -1;
  return guarded("mjb200_warmstart_get_params", [&] {
    w->net->get_params(params);
    return 0;
  });
}

MJMLX_API int mjb200_warmstart_set_params(MjbWarmStart* w, const float* params) {
  if (!w || !params) return -1;
  return guarded("mjb200_warmstart_set_params", [&] {
    w->net->set_params(params);
    return 0;
  });
}

MJMLX_API int mjb200_warmstart_set_normalization(MjbWarmStart* w, const float* in_mean, const float* in_std, const float* out_mean, const float* out_std) {
  if (!w || !in_mean || !in_std || !out_mean || !out_std) return -1;
  return guarded("mjb200_warmstart_set_normalization", [&] {
    w->net->set_normalization(in_mean, in_std, out_mean, out_std);
    return 0;
  });
}

MJMLX_API int mjb200_warmstart_get_normalization(const MjbWarmStart* w, float* in_mean, float* in_std, float* out_mean, float* out_std) {
  if (!w) return -1;
  w->net->get_normalization(in_mean, in_std, out_mean, out_std);
  return 0;
}

MJMLX_API int mjb200_warmstart_fit_normalization(MjbWarmStart* w, const float* xraw, const float* traw, int n) {
  if (!w || !xraw || !traw) return -1;
  return guarded("mjb200_warmstart_fit_normalization", [&] {
    w->net->fit_normalization(xraw, traw, n);
    return 0;
  });
}

MJMLX_API int mjb200_warmstart_forward(MjbWarmStart* w, const float* xraw, int n, float* y) {
  if (!w || !xraw || !y || n < 0) return -1;
  return guarded("mjb200_warmstart_forward", [&] {
    w->net->forward(xraw, n, y);
    return 0;
  });
}

MJMLX_API int mjb200_warmstart_gradients(MjbWarmStart* w, const float* xraw, const float* traw, int n, float* grads, float* loss) {
  if (!w || !xraw || !traw) return -1;
  return guarded("mjb200_warmstart_gradients", [&] {
    float l = w->net->gradients(xraw, traw, n, grads);
    if (loss) *loss = l;
    return 0;
  });
}

MJMLX_API int mjb200_warmstart_train(MjbWarmStart* w, const float* xraw, const float* traw, int n, int epochs, int batch, float lr, unsigned long long seed,
                                     float* epoch_loss) {
  if (!w || !xraw || !traw || n <= 0) return -1;
  return guarded("mjb200_warmstart_train", [&] { return w->net->train(xraw, traw, n, epochs, batch, lr, seed, epoch_loss); });
}

MJMLX_API int mjb200_batched_warmstart_collect(MjmlxBatchedSim* sim, const float* ctrl, int nctrl, int sub, float* xraw, float* traw, int max_rows) {
  if (!sim || !sim->engine || !xraw || !traw || nctrl < 0 || sub <= 0 || max_rows < 0) return -1;
  if (sim->engine->total_u() > 0 && !ctrl) return -1;
  return guarded("mjb200_batched_warmstart_collect", [&] { return sim->engine->collect(ctrl, nctrl, sub, xraw, traw, max_rows); });
}

MJMLX_API int mjb200_batched_set_warmstart(MjmlxBatchedSim* sim, MjbWarmStart* w) {
  if (!sim || !sim->engine) return -1;
  return guarded("mjb200_batched_set_warmstart", [&] {
    sim->engine->set_warmstart(w ? w->net.get() : nullptr);
    return 0;
  });
}

MJMLX_API int mjb200_batched_get_warmstart_debug(MjmlxBatchedSim* sim, float* features, float* pred) {
  if (!sim || !sim->engine) return -1;
  return guarded("mjb200_batched_get_warmstart_debug", [&] { return sim->engine->get_warmstart_debug(features, pred); });
}

MJMLX_API int mjb200_warmstart_predict(MjbWarmStart* w, const float* feat, int fstride, int nfeat, const float* ctrl, int nu, const float* prev,
                                       float* pred, int B, int fused) {
  if (!w || !feat || !prev || !pred || B <= 0 || (nu > 0 && !ctrl)) return -1;
  return guarded("mjb200_warmstart_predict", [&] {
    w->net->infer(feat, fstride, nfeat, ctrl, nu, prev, pred, B, nullptr, fused != 0);
    mjb::check(cudaStreamSynchronize(nullptr), "predict sync");
    if (w->net->error_word()) throw std::runtime_error("a bounded wait in an inference kernel timed out");
    return 0;
  });
}

MJMLX_API int mjb200_gemm_bf16(const void* A, const void* B, float* C, int M, int N, int K, void* stream) {
  if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0 || K % 64 != 0) {
    set_error("mjb200_gemm_bf16: bad arguments");
    return -1;
  }
  const int bn = N <= 256 ? N : 256;
  if (!(N == 64 || N == 128 || N == 192 || N % 256 == 0)) {
    set_error("mjb200_gemm_bf16: N must be 64, 128, 192 or a multiple of 256");
    return -1;
  }
  CUtensorMap ma, mb;
  if (!mjb::make_tmap_bf16(&ma, A, M, K, 128) || !mjb::make_tmap_bf16(&mb, B, N, K, bn)) {
    set_error("mjb200_gemm_bf16: tensor map encode failed (alignment or driver)");
    return -1;
  }
  mjb::GemmArgs a{};
  a.M = M;
  a.N = N;
  a.K = K;
  a.mode = mjb::EPI_F32;
  a.ldo = N;
  a.out_f32 = C;
  cudaError_t e = mjb::gemm_tn(ma, mb, a, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    set_error(std::string("mjb200_gemm_bf16: ") + cudaGetErrorString(e));
    return -3;
  }
  return 0;
}

MJMLX_API int mjb200_gemm_bf16_gated(const void* A, const void* B, float* C, int M, int N, int K, const int* gate_dev, double wait_limit_s,
                                     int* err_dev, void* stream) {
  if (!A || !B || !C || !gate_dev || !err_dev || M <= 0 || K <= 0 || K % 64 != 0 || !(wait_limit_s > 0) || wait_limit_s > 2.0 ||
      !(N == 64 || N == 128 || N == 192 || N == 256)) {
    set_error("mjb200_gemm_bf16_gated: bad arguments");
    return -1;
  }
  CUtensorMap ma, mb;
  if (!mjb::make_tmap_bf16(&ma, A, M, K, 128) || !mjb::make_tmap_bf16(&mb, B, N, K, N)) {
    set_error("mjb200_gemm_bf16_gated: tensor map encode failed (alignment or driver)");
    return -1;
  }
  mjb::GemmArgs a{};
  a.M = M;
  a.N = N;
  a.K = K;
  a.mode = mjb::EPI_F32;
  a.ldo = N;
  a.out_f32 = C;
  a.err = err_dev;
  a.gate = gate_dev;
  a.wait_limit_ns = (unsigned long long)(wait_limit_s * 1e9);
  cudaError_t e = mjb::gemm_tn(ma, mb, a, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    set_error(std::string("mjb200_gemm_bf16_gated: ") + cudaGetErrorString(e));
    return -3;
  }
  return 0;
}

}  // extern "C"
