/*
 * mjb200: extensions of libmjmlx that have no counterpart in the reference's
 * public headers.  They expose what the B200 engine adds to the method
 * (engine configuration, solver statistics, device-resident stepping,
 * mixed-model batches, the learned Newton warm start) and the compiled-model
 * dump that the FP64 test oracle reads.  Plain C types only.
 */
#ifndef MJB200_H
#define MJB200_H

#include <stddef.h>
#include <stdint.h>

#include "mjmlx.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ model dump */

/* Writes a text dump of the compiled model ("name kind n values..." per line)
 * into buf (NUL-terminated) when bufsize is large enough; returns the number
 * of bytes needed including the NUL, or -1 on a bad handle.  No reference
 * counterpart (the reference hands out the MuJoCo mjModel instead,
 * mjmlx.h:95 mjmlx_get_mj_model). */
MJMLX_API int mjb200_model_dump(const MjmlxModel* model, char* buf, int bufsize);

/* Last error message of the calling thread ("" if none). */
MJMLX_API const char* mjb200_last_error(void);

/* ------------------------------------------------------ engine configuration */

typedef struct MjbEngineConfig {
    int warps_per_block;   /* envs per CTA (one warp each); 0 = default */
    int persistent;        /* -1 auto, 0 one warp per env, 1 persistent work queue */
    int blocks_per_sm;     /* persistent grid size per SM; 0 = occupancy limit */
    int ncon_max;          /* per-env contact capacity; 0 = automatic */
    int nefc_max;          /* per-env constraint-row capacity; 0 = automatic */
    int use_graph;         /* replay launches from captured CUDA graphs */
    int record;            /* write xpos/xquat/cvel/cinert/... on the last substep */
    int warmstart;         /* 0 previous-step qacc (MuJoCo), 1 learned prediction with fallback */
    double tolerance;      /* > 0 overrides the model's solver tolerance */
    int max_iter;          /* > 0 overrides the Newton iteration cap */
    int lockstep;          /* 1: the warps of a CTA run each stage together */
    int predict_every;     /* learned warm start: predict at every k-th substep of a step call (1 = every substep);
                              the substeps between run in one launch with the previous-step warm start */
} MjbEngineConfig;

/* Defaults of MjbEngineConfig. */
MJMLX_API MjbEngineConfig mjb200_default_engine_config(void);

/* Mixed-model batch: counts[i] envs of models[i], stored model by model
 * (env-major records of varying size; see mjb200_batched_layout).  All envs
 * step in one launch.  ecfg may be NULL.  NULL + stderr on failure. */
MJMLX_API MjmlxBatchedSim* mjb200_batched_create_multi(const MjmlxModel* const* models, const int* counts, int nmodels,
                                                       const MjmlxBatchedConfig* config, const MjbEngineConfig* ecfg);
MJMLX_API int mjb200_batched_configure(MjmlxBatchedSim* sim, const MjbEngineConfig* ecfg);
MJMLX_API int mjb200_batched_get_config(const MjmlxBatchedSim* sim, MjbEngineConfig* out);
/* Launch-shape autotuner: times envs-per-CTA 2/4/8/16 with lockstep CTAs and
 * with the independent-warp work queue (CTAs per SM at the occupancy
 * limit), and lockstep CTAs of 4 and 8 warps at one CTA per SM; reps
 * launches of nsub substeps each, from the sim's current state (restored
 * before every candidate and at the end), and keeps the fastest.  Per
 * candidate i (at most max_candidates): warps[i], lockstep[i], ms[i] (mean
 * per launch, -1 if it cannot launch); any array may be NULL.  Returns the
 * number of candidates, or -1.  No counterpart in the reference (its
 * per-kernel workgroup sizes are fixed, src/batched.cpp:53-57). */
MJMLX_API int mjb200_batched_autotune(MjmlxBatchedSim* sim, int nsub, int reps, int max_candidates, int* warps, int* lockstep, float* ms);
/* The autotuner's choice for the sim, cached per process by the compiled
 * model tables, per-model env counts and capacities (and whether a learned
 * net is attached): a sim of an already tuned batch takes the cached launch
 * shape without timing anything.  Returns 1 when the cached choice was
 * applied, 0 when it tuned now and stored the choice, -1 on error. */
MJMLX_API int mjb200_batched_autotune_cached(MjmlxBatchedSim* sim, int nsub, int reps);

/* Record layout: num_envs, sum of nq / nv / nu over envs, and the per-env
 * offsets (arrays of num_envs, each may be NULL). */
MJMLX_API int mjb200_batched_layout(const MjmlxBatchedSim* sim, int* num_envs, int* total_q, int* total_v, int* total_u,
                                    int* qadr, int* vadr, int* uadr);

/* n physics steps with the controls already in device memory (no host copy). */
MJMLX_API int mjb200_batched_step_device(MjmlxBatchedSim* sim, int n);
/* n physics steps with controls read from device memory ctrl_dev[total_u]
 * (copied on the sim's stream, device to device); n = 0 only copies. */
MJMLX_API int mjb200_batched_step_device_ctrl(MjmlxBatchedSim* sim, const float* ctrl_dev, int n);
/* n physics steps with controls already in device memory, where the first
 * step offers qacc_dev[total_v] (device, the sim's layout) to the Newton
 * solver as an extra warm-start candidate, kept when its Gauss cost is lowest
 * (e.g. a model-predictive controller's guess).  The solver still iterates to
 * its tolerance.  No counterpart in the reference. */
MJMLX_API int mjb200_batched_step_warmstart(MjmlxBatchedSim* sim, const float* qacc_dev, int n);
/* The previous-step acceleration qacc[total_v] the solver warm-starts from
 * (host arrays); with get/set_state it checkpoints the whole solver state so
 * a resumed run repeats the original bit for bit.  No counterpart in the
 * reference (its solver starts from zero). */
MJMLX_API int mjb200_batched_get_qacc_warmstart(MjmlxBatchedSim* sim, float* qacc);
MJMLX_API int mjb200_batched_set_qacc_warmstart(MjmlxBatchedSim* sim, const float* qacc);
/* Allocation-free step.  No counterpart in the reference.
 *
 * For callers that cannot let a library allocate device memory while they
 * step: a trainer that hands all free device memory to its own caching
 * allocator at start-up (cudaMalloc then fails or fragments its pool), a
 * real-time control loop that cannot wait on cudaMalloc / cudaFree (they may
 * synchronise the device), a host that fixes its device-memory budget when it
 * starts.  Runs n physics steps of the sim's model(s) on state held in the
 * caller's device buffers, laid out like the sim's own (mjb200_batched_layout
 * offsets): qpos[total_q], qvel[total_v], ctrl[total_u] (may be NULL when
 * total_u == 0) and qacc_warmstart[total_v] (zeros for a cold start), all
 * updated in place, with the sim's own launch shape, so the results equal
 * the regular step's.  The launch is ordered on `stream` (cudaStream_t;
 * NULL = legacy default stream).
 *
 * What it leaves out: per-env statistics of the call are not kept
 * (mjb200_batched_stats still reports the sim's own last step); sensors are
 * not computed (sensordata and the accelerometer history keep the sim's own
 * last step); a learned warm-start net attached to the sim is not used (the
 * previous-step warm start in qacc_warmstart is); recorded quantities (xpos,
 * cfrc_ext, ...) are not written.  A model whose workspace needs the HBM
 * workspace of the regular step (too large for shared memory) is refused
 * with -1.
 *
 * Scratch comes from a fixed area inside the library, sized for at most
 * 65536 envs; a larger sim is rejected (return -2, mjb200_last_error says
 * why).  The first call on each device looks up the scratch area's device
 * address and caches it; make that first call before any stream capture.
 * The scratch is shared by every sim on a device and keeps the last call's
 * contents, so calls whose kernels may overlap on the GPU race; order them
 * on one stream.
 *
 * Returns 0 on success, -1 bad arguments or refused model, -2 too many envs,
 * -3 CUDA error. */
MJMLX_API int mjb200_batched_step_noalloc(MjmlxBatchedSim* sim, float* qpos, float* qvel, const float* ctrl, float* qacc_warmstart, int n,
                                          void* stream);
/* Device pointers of the HBM-resident state (float, env-major records). */
MJMLX_API int mjb200_batched_device_state(MjmlxBatchedSim* sim, float** qpos, float** qvel, float** ctrl, float** qacc_warmstart);
/* The CUDA stream (cudaStream_t) every launch of the sim is ordered on. */
MJMLX_API void* mjb200_batched_stream(MjmlxBatchedSim* sim);
/* Launch shape chosen for the step kernel. */
MJMLX_API int mjb200_batched_launch_shape(const MjmlxBatchedSim* sim, int* grid, int* warps_per_block, int* smem_bytes, int* persistent);

/* Per-env statistics of the last step call (arrays of num_envs, each may be
 * NULL): status bits (1 bad state reset, 2 bad acceleration reset, 4 contact
 * overflow, 8 constraint-row overflow, 16 unsupported pair), Newton
 * iterations summed / maximum over the substeps, contacts and rows of the
 * last substep, warm-start choice (0 smooth, 1 previous, 2 predicted). */
MJMLX_API int mjb200_batched_stats(MjmlxBatchedSim* sim, int* status, int* niter_sum, int* niter_max, int* ncon, int* nefc, int* warm_choice);

/* Solver acceleration qacc of the last substep, float[total_v]. */
MJMLX_API const float* mjb200_batched_get_qacc(MjmlxBatchedSim* sim, int* n_out);

/* Packed read-back without a host copy: runs the pack kernel for the spec
 * set by mjmlx_batched_set_pack_spec on the sim's stream and returns its
 * device buffer (num_envs x stride floats, owned by the sim, valid until the
 * next pack or free).  Order reads after it on the sim's stream.  No
 * counterpart in the reference (its get_pack copies to the host).  0 / -1. */
MJMLX_API int mjb200_batched_pack_device(MjmlxBatchedSim* sim, float** pack_dev);

/* Device pointer to the sensordata of all envs (layout of
 * mjmlx_batched_get_sensordata; valid until the sim is freed, rewritten by
 * each step) and its float count; NULL / 0 without sensors. */
MJMLX_API int mjb200_batched_sensordata_device(MjmlxBatchedSim* sim, float** sensordata_dev, int* n);

/* Per-stage SM clock totals of the lockstep step kernel, summed over CTAs.
 * A stage runs from one stage barrier to the next and ends when the CTA's
 * last warp arrives: 0 constraint force, integration, state check and the
 * next substep's kinematics, 1 collision, 2 COM + CRB, 3 RNE + forces, 4
 * unconstrained solve, 5 constraint build, 6 the fused learned warm start
 * (features and MLP, when a per-env net is attached), 7 the Newton solve
 * (until the CTA's slowest solve ends).  enable 1 starts (and zeroes) the
 * counters, 0 stops them, -1 leaves them; cycles8 (may be NULL) receives the
 * totals accumulated so far.  Returns 0 / -1. */
MJMLX_API int mjb200_batched_stage_timing(MjmlxBatchedSim* sim, int enable, unsigned long long* cycles8);

/* Capture contacts / constraint rows / solver vectors of the last substep.
 * set_debug(ncon_max, nefc_max) enables capture (0 disables); get_debug fills
 * contacts[num_envs*ncon_max*16] (pos3 frame9 dist pair dim includemargin),
 * efc[num_envs*nefc_max*4] (type force D aref), vec[num_envs*4*nv_max]
 * (qacc_smooth, qfrc_smooth, qacc, qfrc_constraint); returns nv_max. */
MJMLX_API int mjb200_batched_set_debug(MjmlxBatchedSim* sim, int ncon_max, int nefc_max);
MJMLX_API int mjb200_batched_get_debug(MjmlxBatchedSim* sim, float* contacts, float* efc, float* vec);

#ifdef __cplusplus
}
#endif

#endif /* MJB200_H */
