/*
 * Public types of the libmjmlx C API (batched physics step on B200).
 *
 * Layout-compatible with the reference's include/mjmlx/mjmlx_types.h so that an
 * existing caller recompiles against this header without source changes:
 *   MjmlxIntegrator      <- mjmlx_types.h:37-42
 *   MjmlxSolver          <- mjmlx_types.h:45-49
 *   MjmlxDisableFlag     <- mjmlx_types.h:52-64
 *   MjmlxModelInfo       <- mjmlx_types.h:67-77
 *   MjmlxBatchedConfig   <- mjmlx_types.h:83-89
 */
#ifndef MJMLX_TYPES_H
#define MJMLX_TYPES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifdef _WIN32
#define MJMLX_API __declspec(dllexport)
#else
#define MJMLX_API __attribute__((visibility("default")))
#endif

typedef struct MjmlxModel MjmlxModel;
typedef struct MjmlxBatchedSim MjmlxBatchedSim;

typedef enum {
    MJMLX_INTEGRATOR_EULER = 0,
    MJMLX_INTEGRATOR_RK4 = 1,
    MJMLX_INTEGRATOR_IMPLICIT = 2,
    MJMLX_INTEGRATOR_IMPLICITFAST = 3,
} MjmlxIntegrator;

typedef enum {
    MJMLX_SOLVER_PGS = 0,
    MJMLX_SOLVER_CG = 1,
    MJMLX_SOLVER_NEWTON = 2,
} MjmlxSolver;

typedef enum {
    MJMLX_DISABLE_CONSTRAINT = 1 << 0,
    MJMLX_DISABLE_EQUALITY = 1 << 1,
    MJMLX_DISABLE_FRICTIONLOSS = 1 << 2,
    MJMLX_DISABLE_LIMIT = 1 << 3,
    MJMLX_DISABLE_CONTACT = 1 << 4,
    MJMLX_DISABLE_PASSIVE = 1 << 5,
    MJMLX_DISABLE_GRAVITY = 1 << 6,
    MJMLX_DISABLE_CLAMPCTRL = 1 << 7,
    MJMLX_DISABLE_WARMSTART = 1 << 8,
    MJMLX_DISABLE_FILTERPARENT = 1 << 9,
    MJMLX_DISABLE_ACTUATION = 1 << 10,
    MJMLX_DISABLE_REFSAFE = 1 << 11,
    MJMLX_DISABLE_EULERDAMP = 1 << 15,
} MjmlxDisableFlag;

typedef struct {
    int nq;
    int nv;
    int nu;
    int na;
    int nbody;
    int njnt;
    int ngeom;
    int nsite;
    int ncon;     /* collision candidate pairs (upper bound on contacts is the per-env contact cap) */
} MjmlxModelInfo;

typedef struct {
    int num_envs;
    MjmlxIntegrator integrator;
    int use_gpu;              /* must be 1: this library has no CPU fallback */
    int solver_iterations;    /* 0 = model default, >0 = override */
    int domain_rand;          /* 1 = enable per-env mass/friction/gain scaling */
} MjmlxBatchedConfig;

#ifdef __cplusplus
}
#endif

#endif /* MJMLX_TYPES_H */
