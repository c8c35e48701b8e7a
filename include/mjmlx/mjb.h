/*
 * libmjb: one physics API over several backends.
 *
 * Same entry points as the reference's include/mjmlx/mjb.h for the batched
 * path.  MJB_BACKEND_CUDA (and MJB_BACKEND_MLX, the reference's "GPU engine"
 * value) dispatch to the B200 CUDA engine of libmjmlx.  MJB_BACKEND_CPU is
 * MuJoCo C in the reference; MuJoCo C is not part of this library, so
 * mjb_create_backend(MJB_BACKEND_CPU) returns NULL with a stderr message.
 * A CUDA failure at create time returns NULL instead of silently falling back
 * to a CPU thread pool (reference: mjb.cpp:771-786).
 */
#ifndef MJB_H
#define MJB_H

#include "mjb_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Replace mjb.h:38-40. */
MJB_API MjbBackend* mjb_create_backend(MjbBackendType type);
MJB_API void mjb_free_backend(MjbBackend* backend);
MJB_API MjbBackendType mjb_backend_type(const MjbBackend* backend);

/* Replace mjb.h:46-48. */
MJB_API MjbModel* mjb_load_model(MjbBackend* b, const char* xml_path);
MJB_API MjbModel* mjb_load_model_from_string(MjbBackend* b, const char* xml_string);
MJB_API void mjb_free_model(MjbModel* model);

/* Replace mjb.h:54-58, mjb.h:60-64. */
MJB_API MjbModelInfo mjb_model_info(const MjbModel* model);
MJB_API float mjb_model_opt_timestep(const MjbModel* model);
MJB_API void mjb_model_set_opt_timestep(MjbModel* model, float dt);
MJB_API float mjb_model_body_mass(const MjbModel* model, int body_id);
MJB_API int mjb_name2id(const MjbModel* model, int obj_type, const char* name);
MJB_API int mjb_model_jnt_qposadr(const MjbModel* model, int jnt_id);
MJB_API int mjb_model_jnt_dofadr(const MjbModel* model, int jnt_id);
MJB_API int mjb_model_jnt_type(const MjbModel* model, int jnt_id);
MJB_API int mjb_model_nconmax(const MjbModel* model);
MJB_API int mjb_model_geom_type(const MjbModel* model, int geom_id);

/* Batched simulation.  Replace mjb.h:197-233. */
MJB_API MjbBatchedSim* mjb_batched_create(MjbModel* model, const MjbBatchedConfig* config);
MJB_API void mjb_batched_free(MjbBatchedSim* sim);
/* 1 when the sim runs on the CUDA engine (always, for this library). */
MJB_API int mjb_batched_is_gpu(const MjbBatchedSim* sim);
MJB_API void mjb_batched_step(MjbBatchedSim* sim, const float* ctrl);
MJB_API void mjb_batched_reset(MjbBatchedSim* sim, const int* reset_mask);
MJB_API const float* mjb_batched_get_qpos(const MjbBatchedSim* sim, int* n_out);
MJB_API void mjb_batched_get_state(const MjbBatchedSim* sim, float* qpos_out, float* qvel_out, int* nq_out, int* nv_out);
MJB_API void mjb_batched_set_state(MjbBatchedSim* sim, const float* qpos, const float* qvel);
MJB_API const float* mjb_batched_get_qvel(const MjbBatchedSim* sim, int* n_out);
MJB_API const float* mjb_batched_get_xpos(const MjbBatchedSim* sim, int* n_out);
MJB_API const float* mjb_batched_get_xquat(const MjbBatchedSim* sim, int* n_out);
MJB_API const float* mjb_batched_get_subtree_com(const MjbBatchedSim* sim, int* n_out);
MJB_API const float* mjb_batched_get_cinert(const MjbBatchedSim* sim, int* n_out);
MJB_API const float* mjb_batched_get_cvel(const MjbBatchedSim* sim, int* n_out);
MJB_API const float* mjb_batched_get_qfrc_actuator(const MjbBatchedSim* sim, int* n_out);
MJB_API const float* mjb_batched_get_cfrc_ext(const MjbBatchedSim* sim, int* n_out);
MJB_API void mjb_batched_set_env_qpos(MjbBatchedSim* sim, int env_idx, const float* qpos, int nq);
MJB_API void mjb_batched_set_env_qvel(MjbBatchedSim* sim, int env_idx, const float* qvel, int nv);
MJB_API void mjb_batched_eval_state(const MjbBatchedSim* sim);

#ifdef __cplusplus
}
#endif

#endif /* MJB_H */
