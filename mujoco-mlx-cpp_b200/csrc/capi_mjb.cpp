// C ABI: libmjb backend layer (reference: include/mjmlx/mjb.h, src/mjb.cpp).
// MJB_BACKEND_CUDA and MJB_BACKEND_MLX ("the GPU engine") forward to the
// libmjmlx CUDA engine; MJB_BACKEND_CPU (MuJoCo C) is not part of this
// library and is refused at mjb_create_backend.
#include <cstring>

#include "../../include/mjmlx/mjb.h"
#include "capi_internal.h"

struct MjbBackend {
  MjbBackendType type;
};
struct MjbModel {
  MjbBackendType type;
  MjmlxModel* m;
};
struct MjbBatchedSim {
  MjmlxBatchedSim* s;
};

using mjb::set_error;

extern "C" {

MJB_API MjbBackend* mjb_create_backend(MjbBackendType type) {
  if (type == MJB_BACKEND_CPU) {
    set_error("mjb_create_backend: MJB_BACKEND_CPU is MuJoCo C, which this library does not contain; use MJB_BACKEND_CUDA");
    return nullptr;
  }
  if (type != MJB_BACKEND_MLX && type != MJB_BACKEND_CUDA) {
    set_error("mjb_create_backend: unknown backend type");
    return nullptr;
  }
  auto* b = new MjbBackend();
  b->type = type;
  return b;
}

MJB_API void mjb_free_backend(MjbBackend* backend) { delete backend; }
MJB_API MjbBackendType mjb_backend_type(const MjbBackend* backend) { return backend ? backend->type : MJB_BACKEND_CPU; }

static MjbModel* wrap(MjbBackend* b, MjmlxModel* m) {
  if (!m) return nullptr;
  auto* h = new MjbModel();
  h->type = b->type;
  h->m = m;
  return h;
}

MJB_API MjbModel* mjb_load_model(MjbBackend* b, const char* xml_path) {
  if (!b) return nullptr;
  return wrap(b, mjmlx_load_model(xml_path));
}

MJB_API MjbModel* mjb_load_model_from_string(MjbBackend* b, const char* xml) {
  if (!b) return nullptr;
  return wrap(b, mjmlx_load_model_from_string(xml));
}

MJB_API void mjb_free_model(MjbModel* model) {
  if (!model) return;
  mjmlx_free_model(model->m);
  delete model;
}

MJB_API MjbModelInfo mjb_model_info(const MjbModel* model) {
  MjbModelInfo i;
  std::memset(&i, 0, sizeof(i));
  if (!model) return i;
  const auto& m = model->m->model;
  i.nq = m.nq;
  i.nv = m.nv;
  i.nu = m.nu;
  i.nbody = m.nbody;
  i.njnt = m.njnt;
  i.ngeom = m.ngeom;
  return i;
}

MJB_API float mjb_model_opt_timestep(const MjbModel* model) { return model ? mjmlx_model_opt_timestep(model->m) : 0.f; }
MJB_API void mjb_model_set_opt_timestep(MjbModel* model, float dt) {
  if (model) mjmlx_model_set_opt_timestep(model->m, dt);
}
MJB_API float mjb_model_body_mass(const MjbModel* model, int body_id) { return model ? mjmlx_model_body_mass(model->m, body_id) : 0.f; }
MJB_API int mjb_name2id(const MjbModel* model, int obj_type, const char* name) { return model ? mjmlx_name2id(model->m, obj_type, name) : -1; }

MJB_API int mjb_model_jnt_qposadr(const MjbModel* model, int j) {
  if (!model || j < 0 || j >= model->m->model.njnt) return -1;
  return model->m->model.jnt_qposadr[j];
}
MJB_API int mjb_model_jnt_dofadr(const MjbModel* model, int j) {
  if (!model || j < 0 || j >= model->m->model.njnt) return -1;
  return model->m->model.jnt_dofadr[j];
}
MJB_API int mjb_model_jnt_type(const MjbModel* model, int j) {
  if (!model || j < 0 || j >= model->m->model.njnt) return -1;
  return model->m->model.jnt_type[j];
}
MJB_API int mjb_model_nconmax(const MjbModel* model) { return model ? model->m->model.max_contacts_bound : 0; }
MJB_API int mjb_model_geom_type(const MjbModel* model, int g) {
  if (!model || g < 0 || g >= model->m->model.ngeom) return -1;
  return model->m->model.geom_type[g];
}

MJB_API MjbBatchedSim* mjb_batched_create(MjbModel* model, const MjbBatchedConfig* config) {
  if (!model || !config) return nullptr;
  MjmlxBatchedConfig c;
  c.num_envs = config->num_envs;
  c.integrator = MJMLX_INTEGRATOR_EULER;
  c.use_gpu = 1;
  c.solver_iterations = config->solver_iterations;
  c.domain_rand = 0;
  MjmlxBatchedSim* s = mjmlx_batched_create(model->m, &c);
  if (!s) return nullptr;
  auto* h = new MjbBatchedSim();
  h->s = s;
  return h;
}

MJB_API void mjb_batched_free(MjbBatchedSim* sim) {
  if (!sim) return;
  mjmlx_batched_free(sim->s);
  delete sim;
}

MJB_API int mjb_batched_is_gpu(const MjbBatchedSim* sim) { return sim ? 1 : 0; }
MJB_API void mjb_batched_step(MjbBatchedSim* sim, const float* ctrl) {
  if (sim) mjmlx_batched_step(sim->s, ctrl);
}
MJB_API void mjb_batched_reset(MjbBatchedSim* sim, const int* mask) {
  if (sim) mjmlx_batched_reset(sim->s, mask);
}
MJB_API const float* mjb_batched_get_qpos(const MjbBatchedSim* sim, int* n) { return sim ? mjmlx_batched_get_qpos(sim->s, n) : nullptr; }
MJB_API void mjb_batched_get_state(const MjbBatchedSim* sim, float* qpos, float* qvel, int* nq, int* nv) {
  if (sim) mjmlx_batched_get_state(sim->s, qpos, qvel, nq, nv);
}
MJB_API void mjb_batched_set_state(MjbBatchedSim* sim, const float* qpos, const float* qvel) {
  if (sim) mjmlx_batched_set_state(sim->s, qpos, qvel);
}
MJB_API const float* mjb_batched_get_qvel(const MjbBatchedSim* sim, int* n) { return sim ? mjmlx_batched_get_qvel(sim->s, n) : nullptr; }
MJB_API const float* mjb_batched_get_xpos(const MjbBatchedSim* sim, int* n) { return sim ? mjmlx_batched_get_xpos(sim->s, n) : nullptr; }
MJB_API const float* mjb_batched_get_xquat(const MjbBatchedSim* sim, int* n) { return sim ? mjmlx_batched_get_xquat(sim->s, n) : nullptr; }
MJB_API const float* mjb_batched_get_subtree_com(const MjbBatchedSim* sim, int* n) { return sim ? mjmlx_batched_get_subtree_com(sim->s, n) : nullptr; }
MJB_API const float* mjb_batched_get_cinert(const MjbBatchedSim* sim, int* n) { return sim ? mjmlx_batched_get_cinert(sim->s, n) : nullptr; }
MJB_API const float* mjb_batched_get_cvel(const MjbBatchedSim* sim, int* n) { return sim ? mjmlx_batched_get_cvel(sim->s, n) : nullptr; }
MJB_API const float* mjb_batched_get_qfrc_actuator(const MjbBatchedSim* sim, int* n) { return sim ? mjmlx_batched_get_qfrc_actuator(sim->s, n) : nullptr; }
MJB_API const float* mjb_batched_get_cfrc_ext(const MjbBatchedSim* sim, int* n) { return sim ? mjmlx_batched_get_cfrc_ext(sim->s, n) : nullptr; }
MJB_API void mjb_batched_set_env_qpos(MjbBatchedSim* sim, int env, const float* qpos, int nq) {
  if (sim) mjmlx_batched_set_env_qpos(sim->s, env, qpos, nq);
}
MJB_API void mjb_batched_set_env_qvel(MjbBatchedSim* sim, int env, const float* qvel, int nv) {
  if (sim) mjmlx_batched_set_env_qvel(sim->s, env, qvel, nv);
}
MJB_API void mjb_batched_eval_state(const MjbBatchedSim* sim) {
  if (sim) mjmlx_batched_eval_state(sim->s);
}

}  // extern "C"
