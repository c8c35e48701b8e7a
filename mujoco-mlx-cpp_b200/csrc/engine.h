// Host runtime of the batched step: device model tables, HBM state buffers,
// launch configuration, CUDA graphs, getters.  Replaces the reference's
// BatchedSim + make_batched_step pipeline (src/batched.cpp:891-1247,
// src/internal.h:520-612) with explicit CUDA buffers and one fused launch.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "devmodel.h"
#include "model.h"
#include "step_params.h"

namespace mjb {

struct EngineConfig {
  int warps_per_block = 0;   // 0: autotuned / default
  int persistent = -1;       // -1 auto, 0 static env mapping, 1 persistent work queue
  int blocks_per_sm = 0;     // persistent grid: 0 = occupancy limit
  int ncon_max = 0;          // 0 = auto per model
  int nefc_max = 0;          // 0 = auto per model
  int use_graph = 1;
  int record = 1;            // write derived quantities (xpos, cvel, ...) on the last substep
  int warmstart = 0;         // 0 previous-step (MuJoCo), 1 learned prediction + fallback
  double tolerance = -1;     // > 0 overrides the model tolerance
  int max_iter = 0;          // > 0 overrides the model / config iteration count
  int lockstep = 1;          // warps of a CTA run the stages together (instruction-cache locality)
  int predict_every = 1;     // learned warm start: predict at substeps s % predict_every == 0 of a call
};

class CudaError : public std::runtime_error {
 public:
  using std::runtime_error::runtime_error;
};

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count);
  void upload(const std::vector<T>& v, cudaStream_t s);
};

struct ModelLayout {
  DevModelDesc desc;
  int nq, nv, nu, nbody;
};

class Engine {
 public:
  Engine(const std::vector<const Model*>& models, const std::vector<int>& counts, int solver_iterations, int domain_rand, const EngineConfig& cfg);
  ~Engine();

  int num_envs() const { return B_; }
  int nmodels() const { return (int)models_.size(); }
  const Model& model(int i) const { return *models_[i]; }
  int total_q() const { return tot_q_; }
  int total_v() const { return tot_v_; }
  int total_u() const { return tot_u_; }
  bool convex() const { return convex_; }
  bool hbm_workspace() const { return gws_mode_; }
  int total_sensordata() const { return tot_s_; }
  float* sensordata_device() { return sensordata_.p; }
  int total_b() const { return tot_b_; }
  bool uniform() const { return models_.size() == 1; }

  void step(const float* ctrl_host, int n);    // host ctrl, async
  void step_device(int n);                      // ctrl already on device
  void step_device_ctrl(const float* dctrl, int n);  // ctrl copied from another device buffer
  void sync();
  cudaStream_t stream() const { return stream_; }

  void get_state(float* qpos, float* qvel);
  void set_state(const float* qpos, const float* qvel);
  void set_env_state(int env, const float* qpos, const float* qvel);
  void reset(const int* mask);
  const float* get_host(const char* what, int* n);  // staging copies of recorded quantities

  // per-env stats of the last launch
  void stats(int* status, int* niter_sum, int* niter_max, int* ncon, int* nefc, int* choice);
  void set_debug(int ncon_max, int nefc_max);
  void get_debug(float* contacts, float* efc, float* vec);
  // Debug capture of the fused learned warm start (last substep of the last
  // recorded step): input features [B][warmstart_input_width()] and
  // predictions [total_v].  Returns the feature width, or -1 when nothing
  // was captured.
  int get_warmstart_debug(float* features, float* pred);
  int dbg_ncon_max() const { return dbg_ncon_; }
  int dbg_nefc_max() const { return dbg_nefc_; }
  int dbg_nv_max() const { return nv_max_; }

  // domain randomisation
  int set_env_params(const int* env_idx, int n, const float* mass_scale, const float* com_delta, const float* friction_scale, const float* gain_scale);
  // per-env quadratic drag F = -k |v| v on each free joint (domain_rand sims)
  int set_free_drag(const int* env_idx, int n, const float* drag_k);
  // d(qvel after one step) / d(ctrl) by central differences, out[env][nv][nu]
  void grad_step(float* out);
  bool domain_rand() const { return rand_on_; }

  // learned warm start
  // Input width of the net for this sim: per-env models, the fused layout of
  // the substep after its constraint build (qpos minus the leading free-joint
  // x, y; qvel; qacc_smooth; previous converged qacc; ctrl; 16 x contact
  // normal and distance); per-body models, MJB_FEAT_BODY.
  int warmstart_input_width() const;
  // Per-body mode: floats per body row written after each substep.
  int feature_count() const;
  int feature_qskip() const;
  // A per-env net is attached: the step kernel runs it (lockstep CTAs of 8
  // or 16 warps, workspaces in shared memory, nv * nv >= 256).
  bool fused_warmstart() const { return net_ && !feature_per_body(); }
  // Per-body mode: models made only of free bodies (children of the world)
  // with more dofs than a per-env net serves (nv > 64) and no controls get
  // one feature row and 6 outputs per body (rows_per_env = nbody - 1);
  // otherwise one row of nv outputs per env.
  bool feature_per_body() const;
  int rows_per_env() const { return feature_per_body() ? models_[0]->nbody - 1 : 1; }
  int warmstart_outputs() const { return feature_per_body() ? 6 : models_[0]->nv; }
  // Attaches a trained net (null detaches): every substep then offers the
  // net's prediction to the Newton solver as a warm-start candidate.  Per-env
  // models switch the sim to 8-warp lockstep CTAs when its launch shape
  // cannot run the fused inference; throws when no shape can.
  void set_warmstart(class WarmStartNet* net);
  class WarmStartNet* warmstart() const { return net_; }
  // Plain rollout that records training pairs.  Per-env models: for every
  // substep, B rows of xraw = the fused input features of the substep and
  // traw = its converged qacc minus the previous one (written by the step
  // kernel).  Per-body models: for each substep after the first, B *
  // (nbody - 1) body rows of the previous substep's features and the
  // change of the bodies' converged accelerations.  ctrl_seq: nctrl device
  // control sets of total_u floats, each held for sub_per_ctrl substeps.
  // Returns the number of rows written (<= max_rows).
  int collect(const float* ctrl_seq, int nctrl, int sub_per_ctrl, float* xraw, float* traw, int max_rows);
  // n substeps; the first offers qacc[total_v] (device) to the Newton
  // solver as an extra warm-start candidate (kept when its cost is lowest).
  void step_with_warmstart(const float* qacc, int n);
  // Host copies of the previous-step acceleration the solver warm-starts
  // from (checkpoint / resume of the full solver state).
  void get_qacc_warmstart(float* out);
  void set_qacc_warmstart(const float* in);
  const float* features_device() const { return feat_.p; }
  float* qacc_pred_device() { return pred_.p; }

  void configure(const EngineConfig& cfg);
  // Launch-shape autotuner: times each candidate (envs per CTA 2/4/8/16,
  // lockstep CTAs or the independent-warp work queue) on `reps` launches of
  // `nsub` substeps from the sim's current state, restoring the state before
  // every candidate and at the end, then keeps the fastest.  Results do not
  // depend on the launch shape (the same stage code runs per env).
  struct TuneCandidate {
    int warps_per_block, lockstep, blocks_per_sm;
    float ms;  // mean per launch; < 0 when the shape cannot launch
  };
  std::vector<TuneCandidate> autotune(int nsub, int reps);
  // The autotuner's choice for this sim's batch, from a process-wide cache
  // keyed by the compiled model tables, the per-model env counts and the
  // contact / row capacities (a learned net attached counts too); tunes and
  // stores it on a miss.  Returns true when the cached choice was applied.
  bool autotune_cached(int nsub, int reps);
  const EngineConfig& config() const { return cfg_; }
  void launch_shape(int* grid, int* warps, int* smem_bytes, int* persistent) const;
  int lockstep() const { return lockstep_; }
  void stage_timing(int enable, unsigned long long* out8);
  std::vector<int> env_qadr() const { return h_qadr_; }
  std::vector<int> env_vadr() const { return h_vadr_; }
  std::vector<int> env_uadr() const { return h_uadr_; }

  float* d_qpos() { return qpos_.p; }
  float* d_qvel() { return qvel_.p; }
  float* d_ctrl() { return ctrl_.p; }
  float* d_qacc_warm() { return warm_.p; }

  // Launch parameters that read and write caller-owned buffers (state in the
  // sim's layout, work-queue head, six per-env statistics arrays of num_envs
  // ints each) instead of the engine's own; used by the allocation-free entry.
  StepParams external_params(float* qpos, float* qvel, const float* ctrl, float* qacc_warm, int n, int* work_counter, int* stats6) const;
  int desc_words() const { return desc_words_; }
  int ws_stride() const { return ws_stride_; }
  int sm_count() const { return sm_count_; }

  int pack_spec(const int* body_ids, int nsel, int dof_lo, int ndof);
  int get_pack(float* out);
  // Runs the pack kernel on the sim's stream and returns the device buffer
  // (num_envs x stride floats, valid until the next pack call).
  int pack_device(float** out_dev);
  int raycast(const float* pnt, const float* vec, int nray, int bodyexclude, const unsigned char* geomgroup, int flg_static, float* dist, int* geomid);

 private:
  void build_tables(const EngineConfig& cfg, int solver_iterations);
  void alloc_state();
  void choose_launch();
  void launch(int n, bool record);
  void launch_learned(int n, bool record);
  void ensure_features();
  void invalidate_graphs();
  StepParams params(int n, bool record);
  // why the current launch shape cannot run the fused inference ("" = it can)
  std::string fused_blocker() const;

  std::vector<const Model*> models_;
  std::vector<int> counts_;
  int B_ = 0, tot_q_ = 0, tot_v_ = 0, tot_u_ = 0, tot_b_ = 0, nv_max_ = 0;
  EngineConfig cfg_;
  bool rand_on_ = false;
  bool convex_ = false;   // some model has a pair for the GJK / EPA collider or an elliptic cone (extended kernel instance)
  bool gws_mode_ = false; // workspaces in HBM (too large for shared memory)
  int itab_smem_ = 0;      // words of the int table the step kernel copies into shared memory (0: none)
  DevBuf<float> gws_;
  cudaStream_t stream_ = nullptr;

  std::vector<ModelLayout> layouts_;
  std::vector<int> h_itab_;
  std::vector<float> h_ftab_;
  std::vector<int> h_model_, h_qadr_, h_vadr_, h_uadr_, h_badr_, h_sadr_, h_aadr_;
  int tot_s_ = 0, tot_a_ = 0;   // sensordata floats, accelerometer history floats
  DevBuf<int> d_sadr_, d_aadr_, sens_valid_;
  DevBuf<float> sensordata_, sens_prev_;
  DevBuf<DevModelDesc> d_models_;
  DevBuf<int> d_itab_, d_model_, d_qadr_, d_vadr_, d_uadr_, d_badr_;
  DevBuf<float> d_ftab_;

  DevBuf<float> qpos_, qvel_, ctrl_, warm_, pred_, qpos0_;
  DevBuf<int> status_, niter_sum_, niter_max_, ncon_, nefc_, choice_, counter_;
  DevBuf<float> rec_xpos_, rec_xquat_, rec_scom_, rec_cinert_, rec_cvel_, rec_qfa_, rec_cfrc_, rec_qacc_;
  DevBuf<float> dbg_con_, dbg_efc_, dbg_vec_, dbg_feat_, dbg_pred_;
  int dbg_ncon_ = 0, dbg_nefc_ = 0;
  DevBuf<float> rand_mass_, rand_fric_, rand_gain_, rand_com_, rand_drag_;
  std::vector<float> h_rand_mass_, h_rand_fric_, h_rand_gain_, h_rand_com_, h_rand_drag_;
  std::vector<int> h_fadr_;
  DevBuf<int> d_fadr_;
  int tot_f_ = 0;                            // free joints over all envs
  bool com_on_ = false, drag_on_ = false;    // COM offsets / drag set at least once
  DevBuf<float> feat_, tmp_prev_;
  DevBuf<unsigned long long> stage_cycles_;
  bool timing_ = false;
  int poison_ = 0;   // MJB200_POISON_WORKSPACE=1 at creation: NaN-fill shared workspaces (test aid)
  int feat_stride_ = 0;
  bool feat_valid_ = false;   // features of the last substep are in feat_ (cleared by state changes)
  class WarmStartNet* net_ = nullptr;

  float* h_ctrl_pinned_ = nullptr;
  cudaEvent_t ctrl_done_ = nullptr;   // set after a direct upload from a page-locked ctrl buffer
  std::map<std::string, float*> h_stage_;
  std::map<std::string, size_t> h_stage_n_;

  int ws_stride_ = 0, desc_words_ = 0, warps_ = 4, grid_ = 1, smem_ = 0, persistent_ = 0, lockstep_ = 0, sm_count_ = 148;

  std::map<std::pair<int, int>, cudaGraphExec_t> graphs_;

  // packed read-back
  std::vector<int> pack_bodies_;
  int pack_dof_lo_ = 0, pack_ndof_ = 0, pack_stride_ = -1;
  DevBuf<int> d_pack_bodies_;
  DevBuf<float> d_pack_;
};

void check(cudaError_t e, const char* what);

}  // namespace mjb
