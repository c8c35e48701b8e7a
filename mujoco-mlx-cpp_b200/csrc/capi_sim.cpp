// C ABI: batched simulation (libmjmlx), the libmjb backend layer and the
// mjb200 extensions.  Bodies replace src/batched.cpp:1368-1934 (mjmlx_batched_*)
// and src/mjb.cpp:135-883 (mjb_*) of the reference; a CUDA failure returns
// NULL / -1 with a stderr message and never falls back to a CPU path.
#include <cstdio>
#include <cstring>
#include <string>

#include "capi_internal.h"
#include "engine.h"

using mjb::Engine;
using mjb::set_error;

namespace {

mjb::EngineConfig to_cfg(const MjbEngineConfig* e) {
  mjb::EngineConfig c;
  if (!e) return c;
  c.warps_per_block = e->warps_per_block;
  c.persistent = e->persistent;
  c.blocks_per_sm = e->blocks_per_sm;
  c.ncon_max = e->ncon_max;
  c.nefc_max = e->nefc_max;
  c.use_graph = e->use_graph;
  c.record = e->record;
  c.warmstart = e->warmstart;
  c.tolerance = e->tolerance;
  c.max_iter = e->max_iter;
  c.lockstep = e->lockstep;
  c.predict_every = e->predict_every > 0 ? e->predict_every : 1;
  return c;
}

MjbEngineConfig from_cfg(const mjb::EngineConfig& c) {
  MjbEngineConfig e;
  e.warps_per_block = c.warps_per_block;
  e.persistent = c.persistent;
  e.blocks_per_sm = c.blocks_per_sm;
  e.ncon_max = c.ncon_max;
  e.nefc_max = c.nefc_max;
  e.use_graph = c.use_graph;
  e.record = c.record;
  e.warmstart = c.warmstart;
  e.tolerance = c.tolerance;
  e.max_iter = c.max_iter;
  e.lockstep = c.lockstep;
  e.predict_every = c.predict_every;
  return e;
}

template <class F>
auto guard(const char* fn, F&& f, decltype(f()) on_error) -> decltype(f()) {
  try {
    return f();
  } catch (const std::exception& e) {
    set_error(std::string(fn) + ": " + e.what());
    return on_error;
  }
}

MjmlxBatchedSim* create(const MjmlxModel* const* models, const int* counts, int nmodels, const MjmlxBatchedConfig* config, const MjbEngineConfig* ecfg) {
  if (!models || !counts || nmodels <= 0 || !config) {
    set_error("mjmlx_batched_create: bad arguments");
    return nullptr;
  }
  if (config->use_gpu == 0) {
    set_error("mjmlx_batched_create: use_gpu = 0 requested, but this library has no CPU backend");
    return nullptr;
  }
  if (config->integrator != MJMLX_INTEGRATOR_EULER && config->integrator != MJMLX_INTEGRATOR_IMPLICITFAST && config->integrator != MJMLX_INTEGRATOR_IMPLICIT) {
    set_error("mjmlx_batched_create: only the Euler and implicit(fast) integrators are supported");
    return nullptr;
  }
  return guard("mjmlx_batched_create", [&]() -> MjmlxBatchedSim* {
    std::vector<const mjb::Model*> ms;
    std::vector<int> cs;
    for (int i = 0; i < nmodels; i++) {
      if (!models[i]) throw std::runtime_error("NULL model");
      ms.push_back(&models[i]->model);
      cs.push_back(counts[i]);
    }
    mjb::EngineConfig c = to_cfg(ecfg);
    if (!ecfg) c = mjb::EngineConfig();
    auto* h = new MjmlxBatchedSim();
    h->engine = std::make_unique<Engine>(ms, cs, config->solver_iterations, config->domain_rand, c);
    return h;
  }, nullptr);
}

}  // namespace

extern "C" {

// ------------------------------------------------------------------ mjmlx
MJMLX_API MjmlxBatchedSim* mjmlx_batched_create(const MjmlxModel* model, const MjmlxBatchedConfig* config) {
  if (!config) {
    set_error("mjmlx_batched_create: NULL config");
    return nullptr;
  }
  int n = config->num_envs;
  return create(&model, &n, 1, config, nullptr);
}

MJMLX_API void mjmlx_batched_free(MjmlxBatchedSim* sim) {
  if (!sim) return;
  try {
    delete sim;
  } catch (...) {
  }
}

MJMLX_API void mjmlx_batched_step_n(MjmlxBatchedSim* sim, const float* ctrl, int n) {
  if (!sim || n <= 0) return;
  guard("mjmlx_batched_step_n", [&]() { sim->engine->step(ctrl, n); return 0; }, 0);
}

MJMLX_API void mjmlx_batched_step(MjmlxBatchedSim* sim, const float* ctrl) { mjmlx_batched_step_n(sim, ctrl, 1); }

MJMLX_API void mjmlx_batched_reset(MjmlxBatchedSim* sim, const int* mask) {
  if (!sim || !mask) return;
  guard("mjmlx_batched_reset", [&]() { sim->engine->reset(mask); return 0; }, 0);
}

MJMLX_API void mjmlx_batched_get_state(const MjmlxBatchedSim* sim, float* qpos_out, float* qvel_out, int* nq_out, int* nv_out) {
  if (!sim) return;
  Engine& e = *sim->engine;
  if (nq_out) *nq_out = e.uniform() ? e.model(0).nq : -1;
  if (nv_out) *nv_out = e.uniform() ? e.model(0).nv : -1;
  guard("mjmlx_batched_get_state", [&]() { e.get_state(qpos_out, qvel_out); return 0; }, 0);
}

MJMLX_API void mjmlx_batched_set_state(MjmlxBatchedSim* sim, const float* qpos, const float* qvel) {
  if (!sim) return;
  guard("mjmlx_batched_set_state", [&]() { sim->engine->set_state(qpos, qvel); return 0; }, 0);
}

static const float* getter(const MjmlxBatchedSim* sim, const char* what, int* n_out) {
  if (!sim) return nullptr;
  return guard("mjmlx_batched_get", [&]() { return sim->engine->get_host(what, n_out); }, (const float*)nullptr);
}

MJMLX_API const float* mjmlx_batched_get_qpos(const MjmlxBatchedSim* sim, int* n) { return getter(sim, "qpos", n); }
MJMLX_API const float* mjmlx_batched_get_qvel(const MjmlxBatchedSim* sim, int* n) { return getter(sim, "qvel", n); }
MJMLX_API const float* mjmlx_batched_get_xpos(const MjmlxBatchedSim* sim, int* n) { return getter(sim, "xpos", n); }
MJMLX_API const float* mjmlx_batched_get_xquat(const MjmlxBatchedSim* sim, int* n) { return getter(sim, "xquat", n); }
MJMLX_API const float* mjmlx_batched_get_subtree_com(const MjmlxBatchedSim* sim, int* n) { return getter(sim, "subtree_com", n); }
MJMLX_API const float* mjmlx_batched_get_cinert(const MjmlxBatchedSim* sim, int* n) { return getter(sim, "cinert", n); }
MJMLX_API const float* mjmlx_batched_get_cvel(const MjmlxBatchedSim* sim, int* n) { return getter(sim, "cvel", n); }
MJMLX_API const float* mjmlx_batched_get_qfrc_actuator(const MjmlxBatchedSim* sim, int* n) { return getter(sim, "qfrc_actuator", n); }
MJMLX_API const float* mjmlx_batched_get_cfrc_ext(const MjmlxBatchedSim* sim, int* n) { return getter(sim, "cfrc_ext", n); }

MJMLX_API int mjmlx_batched_nsensordata(const MjmlxBatchedSim* sim) {
  if (!sim || !sim->engine) return 0;
  if (!sim->engine->uniform()) return -1;
  return sim->engine->model(0).nsensordata;
}
MJMLX_API const float* mjmlx_batched_get_sensordata(const MjmlxBatchedSim* sim, int* n) { return getter(sim, "sensordata", n); }

MJMLX_API int mjb200_batched_sensordata_device(MjmlxBatchedSim* sim, float** sensordata_dev, int* n) {
  if (!sim || !sim->engine) return -1;
  if (n) *n = sim->engine->total_sensordata();
  if (sensordata_dev) *sensordata_dev = sim->engine->total_sensordata() ? sim->engine->sensordata_device() : nullptr;
  return 0;
}

MJMLX_API void mjmlx_batched_set_env_qpos(MjmlxBatchedSim* sim, int env_idx, const float* qpos, int nq) {
  if (!sim || !qpos || env_idx < 0 || env_idx >= sim->engine->num_envs()) return;
  (void)nq;
  guard("mjmlx_batched_set_env_qpos", [&]() { sim->engine->set_env_state(env_idx, qpos, nullptr); return 0; }, 0);
}

MJMLX_API void mjmlx_batched_set_env_qvel(MjmlxBatchedSim* sim, int env_idx, const float* qvel, int nv) {
  if (!sim || !qvel || env_idx < 0 || env_idx >= sim->engine->num_envs()) return;
  (void)nv;
  guard("mjmlx_batched_set_env_qvel", [&]() { sim->engine->set_env_state(env_idx, nullptr, qvel); return 0; }, 0);
}

MJMLX_API int mjmlx_batched_set_env_params(MjmlxBatchedSim* sim, const int* env_idx, int n, const float* mass_scale, const float* com_delta,
                                           const float* friction_scale, const float* gain_scale) {
  if (!sim || !sim->engine->domain_rand()) return -1;
  return guard("mjmlx_batched_set_env_params", [&]() { return sim->engine->set_env_params(env_idx, n, mass_scale, com_delta, friction_scale, gain_scale); }, -1);
}

MJMLX_API int mjmlx_batched_set_free_drag(MjmlxBatchedSim* sim, const int* env_idx, int n, const float* drag_k) {
  if (!sim || !sim->engine) return -1;
  return guard("mjmlx_batched_set_free_drag", [&]() { return sim->engine->set_free_drag(env_idx, n, drag_k); }, -1);
}

MJMLX_API void mjmlx_batched_grad_step(MjmlxBatchedSim* sim, float* grad_out) {
  if (!sim || !sim->engine || !grad_out) return;
  guard("mjmlx_batched_grad_step", [&]() { sim->engine->grad_step(grad_out); return 0; }, 0);
}

MJMLX_API int mjmlx_batched_num_free_joints(const MjmlxBatchedSim* sim) {
  if (!sim || !sim->engine->uniform()) return 0;
  const auto& m = sim->engine->model(0);
  int n = 0;
  for (int t : m.jnt_type) n += t == mjb::JNT_FREE;
  return n;
}

MJMLX_API int mjmlx_batched_set_pack_spec(MjmlxBatchedSim* sim, const int* body_ids, int nbody_sel, int dof_lo, int ndof) {
  if (!sim) return -1;
  return guard("mjmlx_batched_set_pack_spec", [&]() { return sim->engine->pack_spec(body_ids, nbody_sel, dof_lo, ndof); }, -1);
}

MJMLX_API int mjmlx_batched_get_pack(MjmlxBatchedSim* sim, float* out) {
  if (!sim || !out) return -1;
  return guard("mjmlx_batched_get_pack", [&]() { return sim->engine->get_pack(out); }, -1);
}

MJMLX_API int mjmlx_batched_raycast(MjmlxBatchedSim* sim, const float* pnt, const float* vec, int nray, int bodyexclude, const unsigned char* geomgroup,
                                    int flg_static, float* dist_out, int* geomid_out) {
  if (!sim || !pnt || !vec || nray <= 0 || !dist_out || !geomid_out) return -1;
  return guard("mjmlx_batched_raycast", [&]() { return sim->engine->raycast(pnt, vec, nray, bodyexclude, geomgroup, flg_static, dist_out, geomid_out); }, -1);
}

MJMLX_API void mjmlx_batched_eval_state(const MjmlxBatchedSim* sim) {
  if (!sim) return;
  guard("mjmlx_batched_eval_state", [&]() { sim->engine->sync(); return 0; }, 0);
}

// ------------------------------------------------------------------ mjb200
MJMLX_API MjbEngineConfig mjb200_default_engine_config(void) { return from_cfg(mjb::EngineConfig()); }

MJMLX_API MjmlxBatchedSim* mjb200_batched_create_multi(const MjmlxModel* const* models, const int* counts, int nmodels, const MjmlxBatchedConfig* config,
                                                       const MjbEngineConfig* ecfg) {
  return create(models, counts, nmodels, config, ecfg);
}

MJMLX_API int mjb200_batched_configure(MjmlxBatchedSim* sim, const MjbEngineConfig* ecfg) {
  if (!sim || !ecfg) return -1;
  return guard("mjb200_batched_configure", [&]() { sim->engine->configure(to_cfg(ecfg)); return 0; }, -1);
}

MJMLX_API int mjb200_batched_get_config(const MjmlxBatchedSim* sim, MjbEngineConfig* out) {
  if (!sim || !out) return -1;
  *out = from_cfg(sim->engine->config());
  return 0;
}

MJMLX_API int mjb200_batched_pack_device(MjmlxBatchedSim* sim, float** pack_dev) {
  if (!sim || !sim->engine || !pack_dev) return -1;
  return guard("mjb200_batched_pack_device", [&]() { return sim->engine->pack_device(pack_dev); }, -1);
}

MJMLX_API int mjb200_batched_autotune(MjmlxBatchedSim* sim, int nsub, int reps, int max_candidates, int* warps, int* lockstep, float* ms) {
  if (!sim || !sim->engine || nsub <= 0 || reps <= 0) return -1;
  return guard("mjb200_batched_autotune", [&]() {
    auto res = sim->engine->autotune(nsub, reps);
    for (int i = 0; i < (int)res.size() && i < max_candidates; i++) {
      if (warps) warps[i] = res[i].warps_per_block;
      if (lockstep) lockstep[i] = res[i].lockstep;
      if (ms) ms[i] = res[i].ms;
    }
    return (int)res.size();
  }, -1);
}

MJMLX_API int mjb200_batched_autotune_cached(MjmlxBatchedSim* sim, int nsub, int reps) {
  if (!sim || !sim->engine || nsub <= 0 || reps <= 0) return -1;
  return guard("mjb200_batched_autotune_cached", [&]() { return sim->engine->autotune_cached(nsub, reps) ? 1 : 0; }, -1);
}

MJMLX_API int mjb200_batched_layout(const MjmlxBatchedSim* sim, int* num_envs, int* total_q, int* total_v, int* total_u, int* qadr, int* vadr, int* uadr) {
  if (!sim) return -1;
  Engine& e = *sim->engine;
  if (num_envs) *num_envs = e.num_envs();
  if (total_q) *total_q = e.total_q();
  if (total_v) *total_v = e.total_v();
  if (total_u) *total_u = e.total_u();
  auto cp = [&](int* dst, const std::vector<int>& v) {
    if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(int));
  };
  cp(qadr, e.env_qadr());
  cp(vadr, e.env_vadr());
  cp(uadr, e.env_uadr());
  return 0;
}

MJMLX_API int mjb200_batched_step_device(MjmlxBatchedSim* sim, int n) {
  if (!sim || n <= 0) return -1;
  return guard("mjb200_batched_step_device", [&]() { sim->engine->step_device(n); return 0; }, -1);
}

MJMLX_API int mjb200_batched_step_device_ctrl(MjmlxBatchedSim* sim, const float* ctrl_dev, int n) {
  if (!sim || n < 0) return -1;
  return guard("mjb200_batched_step_device_ctrl", [&]() { sim->engine->step_device_ctrl(ctrl_dev, n); return 0; }, -1);
}

MJMLX_API int mjb200_batched_step_warmstart(MjmlxBatchedSim* sim, const float* qacc_dev, int n) {
  if (!sim || !sim->engine || !qacc_dev || n < 0) {
    set_error("mjb200_batched_step_warmstart: bad arguments");
    return -1;
  }
  try {
    sim->engine->step_with_warmstart(qacc_dev, n);
    return 0;
  } catch (const std::exception& e) {
    set_error(std::string("mjb200_batched_step_warmstart: ") + e.what());
    return -3;
  }
}

MJMLX_API int mjb200_batched_get_qacc_warmstart(MjmlxBatchedSim* sim, float* qacc) {
  if (!sim || !sim->engine || !qacc) return -1;
  return guard("mjb200_batched_get_qacc_warmstart", [&]() { sim->engine->get_qacc_warmstart(qacc); return 0; }, -1);
}

MJMLX_API int mjb200_batched_set_qacc_warmstart(MjmlxBatchedSim* sim, const float* qacc) {
  if (!sim || !sim->engine || !qacc) return -1;
  return guard("mjb200_batched_set_qacc_warmstart", [&]() { sim->engine->set_qacc_warmstart(qacc); return 0; }, -1);
}

MJMLX_API int mjb200_batched_device_state(MjmlxBatchedSim* sim, float** qpos, float** qvel, float** ctrl, float** qacc) {
  if (!sim) return -1;
  Engine& e = *sim->engine;
  if (qpos) *qpos = e.d_qpos();
  if (qvel) *qvel = e.d_qvel();
  if (ctrl) *ctrl = e.d_ctrl();
  if (qacc) *qacc = e.d_qacc_warm();
  return 0;
}

MJMLX_API void* mjb200_batched_stream(MjmlxBatchedSim* sim) { return sim ? (void*)sim->engine->stream() : nullptr; }

MJMLX_API int mjb200_batched_launch_shape(const MjmlxBatchedSim* sim, int* grid, int* warps, int* smem, int* persistent) {
  if (!sim) return -1;
  sim->engine->launch_shape(grid, warps, smem, persistent);
  return 0;
}

MJMLX_API int mjb200_batched_stats(MjmlxBatchedSim* sim, int* status, int* niter_sum, int* niter_max, int* ncon, int* nefc, int* warm_choice) {
  if (!sim) return -1;
  return guard("mjb200_batched_stats", [&]() { sim->engine->stats(status, niter_sum, niter_max, ncon, nefc, warm_choice); return 0; }, -1);
}

MJMLX_API const float* mjb200_batched_get_qacc(MjmlxBatchedSim* sim, int* n) { return getter(sim, "qacc", n); }

MJMLX_API int mjb200_batched_stage_timing(MjmlxBatchedSim* sim, int enable, unsigned long long* cycles8) {
  if (!sim) return -1;
  return guard("mjb200_batched_stage_timing", [&]() { sim->engine->stage_timing(enable, cycles8); return 0; }, -1);
}

MJMLX_API int mjb200_batched_set_debug(MjmlxBatchedSim* sim, int ncon_max, int nefc_max) {
  if (!sim) return -1;
  return guard("mjb200_batched_set_debug", [&]() { sim->engine->set_debug(ncon_max, nefc_max); return 0; }, -1);
}

MJMLX_API int mjb200_batched_get_debug(MjmlxBatchedSim* sim, float* contacts, float* efc, float* vec) {
  if (!sim) return -1;
  return guard("mjb200_batched_get_debug", [&]() { sim->engine->get_debug(contacts, efc, vec); return sim->engine->dbg_nv_max(); }, -1);
}

}  // extern "C"
