/*
 * libmjmlx: batched MuJoCo physics step, B200 CUDA engine.
 *
 * This header keeps the batched-simulation entry points of the reference's
 * include/mjmlx/mjmlx.h with the same names, argument meaning and error
 * behaviour, so an existing caller relinks against this library unchanged.
 * Every declaration cites the reference declaration it replaces.
 *
 * Differences a caller can observe (all deliberate):
 *  - There is no CPU fallback.  mjmlx_batched_create returns NULL and prints
 *    to stderr when the CUDA engine cannot be built (reference: batched.cpp
 *    falls back to a MuJoCo C thread pool when use_gpu == 0).
 *  - Getter pointers point into host staging buffers owned by the sim; they
 *    stay valid until the next getter call of the same quantity or the next
 *    step (reference: mjmlx.h:137-138, same lifetime rule).
 *  - Arrays at this boundary are env-major: qpos is float[num_envs * nq], etc.
 */
#ifndef MJMLX_H
#define MJMLX_H

#include "mjmlx_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Library version string.  Replaces mjmlx.h:37. */
MJMLX_API const char* mjmlx_version(void);

/* Load an MJCF model from a file / string.  NULL + stderr message on error.
 * Replaces mjmlx.h:44 and mjmlx.h:47.  The built-in compiler reads the MJCF
 * subset: option, compiler(angle), default (unnamed), worldbody/body/
 * inertial/joint/freejoint/geom, asset/mesh(vertex), actuator/position|motor|
 * general, contact/exclude|pair.  Unknown elements are an error. */
MJMLX_API MjmlxModel* mjmlx_load_model(const char* xml_path);
MJMLX_API MjmlxModel* mjmlx_load_model_from_string(const char* xml_string);

/* Load-time options: self_collision = 0 clears conaffinity of the robot's
 * geoms (bodies with joints and their descendants); max_condim > 0 caps the
 * robot geoms' condim.  Replaces mjmlx.h:53-59. */
typedef struct MjmlxModelOptions {
    int self_collision;
    int max_condim;
} MjmlxModelOptions;
MJMLX_API MjmlxModelOptions mjmlx_default_model_options(void);
MJMLX_API MjmlxModel* mjmlx_load_model_ex(const char* xml_path, const MjmlxModelOptions* options);
MJMLX_API MjmlxModel* mjmlx_load_model_from_string_ex(const char* xml_string, const MjmlxModelOptions* options);

/* Replaces mjmlx.h:62. */
MJMLX_API void mjmlx_free_model(MjmlxModel* model);
/* Replaces mjmlx.h:65. */
MJMLX_API MjmlxModelInfo mjmlx_model_info(const MjmlxModel* model);
/* Replaces mjmlx.h:72 / mjmlx.h:75. */
MJMLX_API float mjmlx_model_opt_timestep(const MjmlxModel* model);
MJMLX_API void mjmlx_model_set_opt_timestep(MjmlxModel* model, float dt);
/* Replaces mjmlx.h:78.  Returns 0 for an out-of-range id. */
MJMLX_API float mjmlx_model_body_mass(const MjmlxModel* model, int body_id);
/* Replaces mjmlx.h:83.  obj_type: 1 body, 3 joint, 5 geom, 6 site,
 * 18 tendon, 19 actuator, 20 sensor (MuJoCo mjtObj numbering).  Returns -1
 * if not found. */
MJMLX_API int mjmlx_name2id(const MjmlxModel* model, int obj_type, const char* name);

/* MJCF <sensor> metadata: MuJoCo's sensor_type (mjtSensor code), sensor_adr
 * and sensor_dim, and the name (NULL when unnamed).  -1 / NULL for an
 * out-of-range id.  Replaces mjmlx.h:86-91. */
MJMLX_API int mjmlx_model_nsensor(const MjmlxModel* model);
MJMLX_API int mjmlx_model_nsensordata(const MjmlxModel* model);
MJMLX_API const char* mjmlx_model_sensor_name(const MjmlxModel* model, int sensor_id);
MJMLX_API int mjmlx_model_sensor_type(const MjmlxModel* model, int sensor_id);
MJMLX_API int mjmlx_model_sensor_adr(const MjmlxModel* model, int sensor_id);
MJMLX_API int mjmlx_model_sensor_dim(const MjmlxModel* model, int sensor_id);

/* ---------------------------------------------------------------- batched */

/* Create a batched simulation of config->num_envs copies of the model, all
 * at qpos0 with zero velocity.  Replaces mjmlx.h:171. */
MJMLX_API MjmlxBatchedSim* mjmlx_batched_create(const MjmlxModel* model, const MjmlxBatchedConfig* config);
/* Replaces mjmlx.h:176. */
MJMLX_API void mjmlx_batched_free(MjmlxBatchedSim* sim);
/* One physics step of every env with ctrl float[num_envs * nu] (NULL = zero
 * controls).  Asynchronous: getters synchronise.  Replaces mjmlx.h:181. */
MJMLX_API void mjmlx_batched_step(MjmlxBatchedSim* sim, const float* ctrl);
/* n physics steps with the same ctrl; ctrl crosses host->device once.
 * Replaces mjmlx.h:186. */
MJMLX_API void mjmlx_batched_step_n(MjmlxBatchedSim* sim, const float* ctrl, int n);
/* Reset envs with mask[i] != 0 to qpos0 / zero velocity.  Replaces mjmlx.h:193. */
MJMLX_API void mjmlx_batched_reset(MjmlxBatchedSim* sim, const int* reset_mask);
/* Copy qpos / qvel of all envs out with one synchronisation.  Replaces mjmlx.h:198. */
MJMLX_API void mjmlx_batched_get_state(const MjmlxBatchedSim* sim, float* qpos_out, float* qvel_out, int* nq_out, int* nv_out);
/* Overwrite the whole qpos / qvel batch (either may be NULL).  Replaces mjmlx.h:203. */
MJMLX_API void mjmlx_batched_set_state(MjmlxBatchedSim* sim, const float* qpos, const float* qvel);

/* Batched getters, float[num_envs * dim].  Replace mjmlx.h:208-216.
 * xpos/xquat/subtree_com/cinert/cvel/qfrc_actuator/cfrc_ext are the values
 * computed during the last physics step (from the state at its start, as in
 * the reference and in MuJoCo's mj_step). */
MJMLX_API const float* mjmlx_batched_get_qpos(const MjmlxBatchedSim* sim, int* n_out);
MJMLX_API const float* mjmlx_batched_get_qvel(const MjmlxBatchedSim* sim, int* n_out);
MJMLX_API const float* mjmlx_batched_get_xpos(const MjmlxBatchedSim* sim, int* n_out);
MJMLX_API const float* mjmlx_batched_get_xquat(const MjmlxBatchedSim* sim, int* n_out);
MJMLX_API const float* mjmlx_batched_get_subtree_com(const MjmlxBatchedSim* sim, int* n_out);
MJMLX_API const float* mjmlx_batched_get_cinert(const MjmlxBatchedSim* sim, int* n_out);
MJMLX_API const float* mjmlx_batched_get_cvel(const MjmlxBatchedSim* sim, int* n_out);
MJMLX_API const float* mjmlx_batched_get_qfrc_actuator(const MjmlxBatchedSim* sim, int* n_out);
MJMLX_API const float* mjmlx_batched_get_cfrc_ext(const MjmlxBatchedSim* sim, int* n_out);

/* Sensor values float[num_envs * nsensordata], each env laid out as MuJoCo's
 * d->sensordata (sensor_adr).  Like the other getters they belong to the
 * start state of the last physics step, i.e. MuJoCo's sensordata after
 * mj_step.  Computed on the device inside the step (no extra launch):
 * joint / tendon / actuator positions and velocities, joint actuator force,
 * ball joints, subtree COM, frame pose / axes / velocities (world frame),
 * gyro, velocimeter, magnetometer, and the accelerometer as the one-step
 * difference of the site's world velocity minus gravity, in the site frame
 * (zero difference on the first step after creation or reset).  Other
 * sensor types, and frame sensors relative to another frame, read 0.
 * nsensordata: per env; -1 for a mixed-model sim (get_sensordata then
 * returns every env's values back to back).  NULL / 0 without sensors.
 * Replace mjmlx.h:220-221. */
MJMLX_API int mjmlx_batched_nsensordata(const MjmlxBatchedSim* sim);
MJMLX_API const float* mjmlx_batched_get_sensordata(const MjmlxBatchedSim* sim, int* n_out);

/* Jacobian d(qvel after one physics step) / d(ctrl) of every env at the
 * current state and the controls of the last step, grad_out float[num_envs
 * * nv * nu] (row-major per env), by central differences of perturbed
 * steps from the saved state, which is restored afterwards (single-model
 * sims; the statistics reflect the probe steps).  The reference declares
 * this entry point with an empty body.  Replaces mjmlx.h:268-270. */
MJMLX_API void mjmlx_batched_grad_step(MjmlxBatchedSim* sim, float* grad_out);

/* Per-env state setters.  Replace mjmlx.h:224-225. */
MJMLX_API void mjmlx_batched_set_env_qpos(MjmlxBatchedSim* sim, int env_idx, const float* qpos, int nq);
MJMLX_API void mjmlx_batched_set_env_qvel(MjmlxBatchedSim* sim, int env_idx, const float* qvel, int nv);

/* Per-env physics randomisation (config->domain_rand == 1 only).  For each
 * env_idx[i] (env_idx == NULL: n == num_envs, all envs) update the non-NULL
 * arrays: mass_scale[n*nbody] (mass and inertia), com_delta[n*nbody*3] (COM
 * offset in the body frame), friction_scale[n] (pair friction),
 * gain_scale[n*nu] (actuator force).  Returns 0 ok, -1 bad handle /
 * domain_rand off / bad n, -2 env index out of range.  Replaces
 * mjmlx.h:233. */
MJMLX_API int mjmlx_batched_set_env_params(MjmlxBatchedSim* sim, const int* env_idx, int n, const float* mass_scale, const float* com_delta, const float* friction_scale, const float* gain_scale);
/* Quadratic drag F = -k|v|v [N s^2/m^2] on the translational dofs of each
 * free joint (MJCF order), drag_k[n * nfree]; 0 (no drag) until set.
 * Returns as above, -3 if no model of the sim has a free joint.  Replaces
 * mjmlx.h:237-238. */
MJMLX_API int mjmlx_batched_set_free_drag(MjmlxBatchedSim* sim, const int* env_idx, int n, const float* drag_k);
MJMLX_API int mjmlx_batched_num_free_joints(const MjmlxBatchedSim* sim);

/* Packed read-back: one row per env of [qpos(nq), qvel(nv), |contact force|
 * of each selected body (nbody_sel), sum of qfrc_actuator^2 over dofs
 * [dof_lo, dof_lo+ndof), sum of |qfrc_actuator| over the same dofs].
 * set_pack_spec returns the row stride (or -1); get_pack fills
 * out[num_envs * stride] and returns 0 (or -1).  Replaces mjmlx.h:241-242. */
MJMLX_API int mjmlx_batched_set_pack_spec(MjmlxBatchedSim* sim, const int* body_ids, int nbody_sel, int dof_lo, int ndof);
MJMLX_API int mjmlx_batched_get_pack(MjmlxBatchedSim* sim, float* out);

/* Batched ray casting against the geoms of every env at the pose of the last
 * step (mj_ray semantics).  pnt/vec float[B*nray*3]; dist_out float[B*nray]
 * (-1 = no hit), geomid_out int[B*nray] (-1 = no hit).  Plane, sphere,
 * capsule, ellipsoid, cylinder and box geoms are hit.  Returns 0 / -1.
 * Replaces mjmlx.h:248. */
MJMLX_API int mjmlx_batched_raycast(MjmlxBatchedSim* sim, const float* pnt, const float* vec, int nray, int bodyexclude, const unsigned char* geomgroup, int flg_static, float* dist_out, int* geomid_out);

/* Wait for the last step.  Replaces mjmlx.h:252. */
MJMLX_API void mjmlx_batched_eval_state(const MjmlxBatchedSim* sim);

/* Camera sensor (replaces mjmlx.h:272-295, the reference's Vulkan renderer).
 * Rendering needs a graphics stack, which this CUDA engine does not have:
 * the functions are exported so that callers built against the reference's
 * API (its Python RL binding among them) link unchanged, and they refuse at
 * run time.  mjmlx_camera_create returns NULL with a message
 * (mjb200_last_error); the int functions return -1 (count, draw-call count
 * and gpu_supported return 0); free accepts NULL. */
typedef struct MjmlxCameraRenderer MjmlxCameraRenderer;
MJMLX_API MjmlxCameraRenderer* mjmlx_camera_create(MjmlxBatchedSim* sim, int width, int height);
MJMLX_API void mjmlx_camera_free(MjmlxCameraRenderer* r);
MJMLX_API int mjmlx_camera_count(const MjmlxCameraRenderer* r);
MJMLX_API int mjmlx_camera_render(MjmlxCameraRenderer* r);
MJMLX_API int mjmlx_camera_draw_call_count(const MjmlxCameraRenderer* r);
MJMLX_API int mjmlx_camera_get_rgb(MjmlxCameraRenderer* r, uint8_t* out);
MJMLX_API int mjmlx_camera_get_depth(MjmlxCameraRenderer* r, float* out);
MJMLX_API int mjmlx_camera_gpu_supported(const MjmlxCameraRenderer* r);
MJMLX_API int mjmlx_camera_gpu_copy(MjmlxCameraRenderer* r);
MJMLX_API int mjmlx_camera_gpu_export_fd(MjmlxCameraRenderer* r, int which, uint64_t* alloc_size);

#ifdef __cplusplus
}
#endif

#endif /* MJMLX_H */
