/*
 * Types of the libmjb unified backend API.
 *
 * Layout-compatible with the reference's include/mjmlx/mjb_types.h.  The one
 * addition is MJB_BACKEND_CUDA: a caller switches to the B200 engine by
 * changing only the backend enum passed to mjb_create_backend.
 *   MjbBackendType   <- mjb_types.h:34-37 (+ MJB_BACKEND_CUDA)
 *   MjbModelInfo     <- mjb_types.h:46-59
 *   MjbBatchedConfig <- mjb_types.h:62-65
 */
#ifndef MJB_TYPES_H
#define MJB_TYPES_H

#ifdef __cplusplus
extern "C" {
#endif

#ifdef _WIN32
#define MJB_API __declspec(dllexport)
#else
#define MJB_API __attribute__((visibility("default")))
#endif

typedef enum {
    MJB_BACKEND_CPU = 0,   /* MuJoCo C (double).  Not part of this library: create returns NULL. */
    MJB_BACKEND_MLX = 1,   /* "the GPU engine": served by the CUDA engine in this library */
    MJB_BACKEND_CUDA = 2,  /* B200 CUDA engine (float32) */
} MjbBackendType;

typedef struct MjbBackend MjbBackend;
typedef struct MjbModel MjbModel;
typedef struct MjbBatchedSim MjbBatchedSim;

typedef struct {
    int nq;
    int nv;
    int nu;
    int nbody;
    int njnt;
    int ngeom;
    int nsite;
    int nmocap;
    int ntendon;
    int nsensor;
    int nsensordata;
    int neq;
} MjbModelInfo;

typedef struct {
    int num_envs;
    int solver_iterations;    /* 0 = model default, >0 = override */
} MjbBatchedConfig;

#ifdef __cplusplus
}
#endif

#endif /* MJB_TYPES_H */
