/*
 * FP64 CPU oracle of the batched MuJoCo physics step -- TEST INFRASTRUCTURE.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg (and
 * bench.py --impl reference) may load this code, and only as the checker or
 * the timed CPU baseline; the product (libmjb200.so) never links it.
 *
 * What it restates: the reference's batched step (src/batched.cpp:980-1228)
 * stage by stage -- kinematics (src/compat/mkx_kernels/kinematics.hpp:75-183),
 * smooth dynamics (forward.hpp:143-469), collision (collision.hpp:235-501),
 * constraint rows and impedance (solver.hpp:122-138, 259-587), Newton solve
 * (solver.hpp:592-854), Euler integration (euler.hpp:26-110) -- in double
 * precision, with MuJoCo C's published semantics where the reference's GPU
 * kernels deviate from MuJoCo (multi-contact plane rules, contact frame,
 * previous-step warm start, tolerance-scaled termination, exact line search).
 *
 * Parity status: UNPINNED.  MuJoCo C 3.5.0 (the reference's CPU backend,
 * pyproject.toml:2) is not installed here and the reference ships no golden
 * vectors for this path; the oracle is pinned only by analytic known answers
 * and structural rules (tests/test_oracle.py) and every MuJoCo semantic it
 * encodes is unverified against MuJoCo C until cross-checked.
 */
#ifndef MJORACLE_H
#define MJORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OModel {
  int nq, nv, nu, nbody, njnt, ngeom, nmesh, npair;
  int iterations, ls_iterations, cone, integrator, disableflags;
  double timestep, gravity[3], tolerance, ls_tolerance, impratio, meaninertia;
  const int *body_parentid, *body_rootid, *body_weldid, *body_jntnum, *body_jntadr, *body_dofnum, *body_dofadr, *body_subtreesize;
  const double *body_pos, *body_quat, *body_ipos, *body_iquat, *body_mass, *body_inertia, *body_invweight0;
  const int *jnt_type, *jnt_qposadr, *jnt_dofadr, *jnt_bodyid, *jnt_limited;
  const double *jnt_pos, *jnt_axis, *jnt_range, *jnt_margin, *jnt_solref, *jnt_solimp, *jnt_stiffness;
  const int *dof_bodyid, *dof_jntid, *dof_parentid;
  const double *dof_armature, *dof_damping, *dof_frictionloss, *dof_invweight0, *dof_solref, *dof_solimp;
  const double *qpos0, *qpos_spring;
  const int *geom_type, *geom_bodyid, *geom_dataid;
  const double *geom_pos, *geom_quat, *geom_size, *geom_rbound;
  const int *mesh_vertadr, *mesh_vertnum;
  const double *mesh_vert;
  const int *actuator_trnid, *actuator_gaintype, *actuator_biastype, *actuator_ctrllimited, *actuator_forcelimited;
  const double *actuator_gear, *actuator_gainprm, *actuator_biasprm, *actuator_ctrlrange, *actuator_forcerange;
  /* collision candidates: pair_int[6*p] = g1 g2 b1 b2 condim explicit,
     pair_real[16*p] = margin gap friction(5) solref(2) solimp(5) invw_t invw_r */
  const int* pair_int;
  const double* pair_real;
  /* equality constraints (type 2 = joint: q1 - q1_0 = poly(q2 - q2_0)) */
  int neq;
  const int *eq_type, *eq_obj1, *eq_obj2, *eq_active;
  const double *eq_data, *eq_solref, *eq_solimp, *eq_invweight;
  /* fixed tendons: length = sum over wraps of coef * qpos (hinge / slide
     joints); actuator_trntype 0 = joint, 3 = tendon (actuator_trnid) */
  int ntendon;
  const int *tendon_adr, *tendon_num, *tendon_limited, *wrap_objid, *actuator_trntype;
  const double *wrap_prm, *tendon_range, *tendon_margin, *tendon_frictionloss, *tendon_stiffness, *tendon_damping, *tendon_lengthspring;
  const double *tendon_solref_lim, *tendon_solimp_lim, *tendon_solref_fri, *tendon_solimp_fri, *tendon_length0, *tendon_invweight0;
  /* sites and sensors (sensor_type: MuJoCo mjtSensor code; objtype: mjtObj
     code 1 body, 2 xbody, 3 joint, 5 geom, 6 site, 18 tendon, 19 actuator) */
  int nsite, nsensor;
  const int *site_bodyid, *sensor_type, *sensor_objtype, *sensor_objid, *sensor_dim, *sensor_adr, *sensor_supported;
  const double *site_pos, *site_quat, *magnetic;
  /* gravity compensation per body (fraction of its weight) */
  const double* body_gravcomp;
  /* tendon wrap element types (mjtWrap: 1 joint, 2 pulley, 3 site, 4 sphere,
     5 cylinder); wrap_objid / wrap_prm: joint, site or geom id / joint
     coef, pulley divisor or the geom's side site (-1 none) */
  const int* wrap_type;
} OModel;

/* per-env randomisation (NULL pointers = identity) */
typedef struct ORand {
  const double* mass_scale;     /* [nbody] */
  double friction_scale;
  const double* gain_scale;     /* [nu] */
  const double* com_delta;      /* [nbody][3]: COM offset in the body frame */
  const double* drag_k;         /* [free joints]: quadratic drag F = -k |v| v */
} ORand;

#define ORACLE_CONTACT_STRIDE 20  /* pos3 frame9 dist pair g1 g2 dim mu0 includemargin efc_adr */

typedef struct OData {
  int ncon_max, nefc_max;
  /* state in / out */
  double *qpos, *qvel, *ctrl, *qacc_warmstart;
  /* optional predicted warm start (NULL = none) */
  const double* qacc_predicted;
  /* outputs of the last step (sizes from the model) */
  double *xpos, *xquat, *xmat, *xipos, *ximat, *xanchor, *xaxis, *geom_xpos, *geom_xmat;
  double *subtree_com, *cinert, *cdof, *cvel, *cdof_dot, *cacc, *cfrc;
  double *M, *qLD, *qfrc_bias, *qfrc_passive, *qfrc_actuator, *qfrc_smooth, *qacc_smooth;
  double *contact;              /* [ncon_max * ORACLE_CONTACT_STRIDE] */
  double *efc_J, *efc_aref, *efc_D, *efc_R, *efc_floss, *efc_force, *efc_jar;  /* [nefc_max(*nv)] */
  int *efc_type;                /* 0 friction 1 limit 2 contact-pyramid 3 contact-frictionless 5 equality */
  double *qacc, *qfrc_constraint, *cfrc_ext;
  double *work;                 /* >= 6*nv*nv + 16*nv + 8*nefc_max doubles */
  /* scalars */
  int ncon, nefc, niter, status, warm_choice;   /* warm_choice 0 smooth 1 previous 2 predicted */
  int ncon_dropped, nefc_dropped;
  double cost_initial, cost_final;
} OData;

/* status bits */
#define ORACLE_BADSTATE 1
#define ORACLE_BADQACC 2
#define ORACLE_CONTACT_OVERFLOW 4
#define ORACLE_EFC_OVERFLOW 8

/* stages (usable alone by tests) */
void oracle_kinematics(const OModel* m, OData* d);
void oracle_com(const OModel* m, OData* d, const ORand* r);
void oracle_crb(const OModel* m, OData* d, const ORand* r);
void oracle_rne(const OModel* m, OData* d, const ORand* r);   /* cvel, cdof_dot, qfrc_bias */
void oracle_smooth_forces(const OModel* m, OData* d, const ORand* r);  /* passive, actuation, smooth, qacc_smooth */
/* length, velocity and Jacobian (J: nv doubles, may be NULL) of fixed tendon t */
void oracle_tendon(const OModel* m, const OData* d, int t, double* len, double* vel, double* J);
void oracle_collide(const OModel* m, OData* d);
void oracle_make_constraints(const OModel* m, OData* d, const ORand* r);
void oracle_solve(const OModel* m, OData* d, int max_iter);
void oracle_integrate(const OModel* m, OData* d);
/* contact wrench per body (cfrc_ext) from the solved contact rows */
void oracle_cfrc_ext(const OModel* m, OData* d, const ORand* r);

/* one full physics step (mj_step with the Euler integrator); max_iter <= 0
 * uses the model's iteration count */
void oracle_step(const OModel* m, OData* d, const ORand* r, int max_iter);

/* Sensor values of one env after oracle_step, from the quantities that step
 * computed at its start state (q0, v0): sensordata[nsensordata].  Frame
 * linear velocities (3 per sensor, world frame) go to linvel_out when not
 * NULL; accelerometers difference them against prev_linvel (the previous
 * step's, NULL when there is none) over one timestep. */
void oracle_sensors(const OModel* m, const OData* d, const double* q0, const double* v0, const double* prev_linvel, double* linvel_out,
                    double* sensordata);

/* nearest ray hit t (pnt + t vec) among the geoms with include[g] != 0 at
 * the poses of the last oracle_kinematics call; -1 and geomid -1 when none */
double oracle_ray(const OModel* m, const OData* d, const double* pnt, const double* vec, const int* include, int* geomid);

/* step B envs (state arrays env-major) over nthread host threads; each env
 * uses its own OData built from the per-env pointer tables */
void oracle_step_batch(const OModel* m, OData* const* d, int B, int nsub, int max_iter, int nthread);

#ifdef __cplusplus
}
#endif

#endif
