/*
 * mjb200 learned Newton warm start.  No counterpart in the reference, whose
 * Newton solver starts from qacc = 0 (src/compat/mkx_kernels/solver.hpp:592).
 *
 * A 3 x 256 GELU MLP predicts the converged acceleration of a substep as a
 * change from the previous substep's.  Per-env models: the step kernel runs
 * the net itself, after the constraint build of every substep, on that
 * substep's features (qpos without the free root's x, y; qvel; qacc_smooth;
 * the previous converged qacc; ctrl; normal and distance of up to 16
 * contacts), with bf16 tensor-core tiles shared by the warps of a lockstep
 * CTA (8 or 16 warps).  Models made only of free bodies with nv > 64: one
 * feature row per body from the end of the previous substep, inferred by a
 * separate launch.  Attached to a sim, the prediction is a third warm-start
 * candidate of the Newton solver next to qacc_smooth and the previous qacc;
 * the solver keeps the lowest Gauss cost and iterates to the same tolerance
 * as without it.
 *
 * All arrays named *_dev are device pointers (float, row-major).  Functions
 * return 0 on success and -1 on error (message in mjb200_last_error), unless
 * stated otherwise.
 */
#ifndef MJB200_WARMSTART_H
#define MJB200_WARMSTART_H

#include "mjb200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct MjbWarmStart MjbWarmStart;

/* Network for in_raw inputs and nout outputs (the model's nv).  in_raw for a
 * sim is mjb200_warmstart_input_width(sim).  NULL on failure. */
MJMLX_API MjbWarmStart* mjb200_warmstart_create(int in_raw, int nout, unsigned long long seed);
MJMLX_API void mjb200_warmstart_free(MjbWarmStart* net);

/* Input width the sim's learned warm start expects, or -1. */
MJMLX_API int mjb200_warmstart_input_width(const MjmlxBatchedSim* sim);

/* The net shape a sim expects: input width, output width and rows per env.
 * One row of nv outputs per env, except for models made only of free bodies
 * (children of the world) with nv > 64 and no controls: one row per body of
 * 45 features (height, orientation quaternion, the body's 6 velocities and 6
 * converged accelerations, its first 4 contacts as normal along the force on
 * the body, distance and contact point minus body position) and 6 outputs,
 * rows_per_env = nbody - 1.  Any pointer may be NULL; 0 or -1. */
MJMLX_API int mjb200_warmstart_layout(const MjmlxBatchedSim* sim, int* in_raw, int* nout, int* rows_per_env);

/* Sizes: input width, padded input width, hidden width, output width, padded
 * output width, total parameter count.  Any pointer may be NULL. */
MJMLX_API int mjb200_warmstart_dims(const MjbWarmStart* net, int* in_raw, int* in_pad, int* hidden, int* nout, int* out_pad, int* nparams);

/* FP32 parameters in the order W0[hidden][in_pad], b0[hidden], W1[hidden][hidden],
 * b1, W2[hidden][hidden], b2, W3[out_pad][hidden], b3[out_pad] (host arrays). */
MJMLX_API int mjb200_warmstart_get_params(const MjbWarmStart* net, float* params);
MJMLX_API int mjb200_warmstart_set_params(MjbWarmStart* net, const float* params);

/* Input / target normalisation (host arrays of in_raw and nout floats). */
MJMLX_API int mjb200_warmstart_set_normalization(MjbWarmStart* net, const float* in_mean, const float* in_std, const float* out_mean, const float* out_std);
MJMLX_API int mjb200_warmstart_get_normalization(const MjbWarmStart* net, float* in_mean, float* in_std, float* out_mean, float* out_std);
/* Mean and standard deviation of training data xraw_dev[n][in_raw], traw_dev[n][nout]. */
MJMLX_API int mjb200_warmstart_fit_normalization(MjbWarmStart* net, const float* xraw_dev, const float* traw_dev, int n);

/* Network output y_dev[n][nout] (normalised target units) for raw inputs. */
MJMLX_API int mjb200_warmstart_forward(MjbWarmStart* net, const float* xraw_dev, int n, float* y_dev);
/* Loss and gradient of one batch of n rows (n a multiple of 64): loss = mean
 * over rows and outputs of the squared error in normalised units; grads
 * (host, parameter layout) may be NULL. */
MJMLX_API int mjb200_warmstart_gradients(MjbWarmStart* net, const float* xraw_dev, const float* traw_dev, int n, float* grads, float* loss);
/* Adam training, batch a multiple of 64, cosine-decayed learning rate;
 * epoch_loss (host, epochs floats) may be NULL.  Returns the number of
 * optimiser steps, or -1. */
MJMLX_API int mjb200_warmstart_train(MjbWarmStart* net, const float* xraw_dev, const float* traw_dev, int n, int epochs, int batch, float lr,
                                     unsigned long long seed, float* epoch_loss);

/* Training data from a plain rollout of the sim (learned warm start off):
 * ctrl_dev holds nctrl control sets of total_u floats, each applied for
 * substeps_per_ctrl substeps.  Per-env models: every substep writes num_envs
 * rows xraw_dev[.][in_raw] (the features the fused inference sees) and
 * traw_dev[.][nv] (the substep's converged qacc minus the previous one);
 * per-body models: every substep after the first writes num_envs x
 * rows_per_env rows (mjb200_warmstart_layout).  Rows are written while
 * max_rows allows.  Returns the number of rows written, or -1. */
MJMLX_API int mjb200_batched_warmstart_collect(MjmlxBatchedSim* sim, const float* ctrl_dev, int nctrl, int substeps_per_ctrl, float* xraw_dev,
                                               float* traw_dev, int max_rows);
/* Attaches a net to the sim (NULL detaches).  The net must outlive the
 * attachment and serves one sim batch size.  Per-env models need lockstep
 * CTAs of 8 or 16 warps with the workspaces in shared memory and nv * nv >=
 * 256; the sim switches to 8-warp CTAs when it can, else -1. */
MJMLX_API int mjb200_batched_set_warmstart(MjmlxBatchedSim* sim, MjbWarmStart* net);
/* Debug capture of the fused warm start (mjb200_batched_set_debug enabled, a
 * per-env net attached): the input features features[num_envs][in_raw] and
 * the predictions pred[total_v] of the last substep of the last step (either
 * may be NULL).  Returns in_raw, or -1 when nothing was captured. */
MJMLX_API int mjb200_batched_get_warmstart_debug(MjmlxBatchedSim* sim, float* features, float* pred);

/* Prediction for B envs from device arrays feat_dev[B][fstride] (first nfeat
 * used), ctrl_dev[B][nu] and the previous qacc prev_dev[B][nout]:
 * pred_dev = prev + mean + std * net(...).  fused = 1 runs the single fused
 * kernel the sims use, 0 the gather kernel plus four GEMM launches (same
 * arithmetic).  Runs on the legacy default stream and waits for it. */
MJMLX_API int mjb200_warmstart_predict(MjbWarmStart* net, const float* feat_dev, int fstride, int nfeat, const float* ctrl_dev, int nu,
                                       const float* prev_dev, float* pred_dev, int B, int fused);

/* C[M][N] (float, device) = A[M][K] * B[N][K]^T with bf16 device operands, on
 * the tcgen05 GEMM the network uses.  K a multiple of 64; N 64, 128, 192 or a
 * multiple of 256.  stream: cudaStream_t (NULL = legacy default).  Returns
 * 0, -1 bad arguments, -3 CUDA error. */
MJMLX_API int mjb200_gemm_bf16(const void* A, const void* B, float* C, int M, int N, int K, void* stream);

/* The same GEMM with its failure path exposed, for tests of the bounded
 * waits (no counterpart in the reference).  Before its first MMA each CTA
 * waits for the device word *gate_dev to become nonzero; every wait of the
 * kernel gives up after wait_limit_s seconds (0 < wait_limit_s <= 2).  A
 * CTA whose wait gave up writes nothing to C, sets *err_dev (device int) to
 * 1, lets its own TMA copies and MMAs finish, frees its TMEM and returns, so
 * the context stays usable.  N 64, 128, 192 or 256.  Returns 0, -1 bad
 * arguments, -3 CUDA error (the launch, not the wait: read *err_dev). */
MJMLX_API int mjb200_gemm_bf16_gated(const void* A, const void* B, float* C, int M, int N, int K, const int* gate_dev, double wait_limit_s,
                                     int* err_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MJB200_WARMSTART_H */
