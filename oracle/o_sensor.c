/*
 * FP64 oracle of the batched sensors -- TEST INFRASTRUCTURE (see mjoracle.h).
 *
 * Restates the reference's batched sensordata (src/sensor.cpp:265-356):
 * values at the start state of the last substep, i.e. MuJoCo's d->sensordata
 * after mj_step.  Position / velocity stage sensors follow MuJoCo's
 * formulas: frames from the body pose and the object's local frame, frame
 * velocity from cvel moved from the root subtree COM to the frame origin,
 * gyro / velocimeter / magnetometer rotated into the site frame.  The
 * accelerometer is the reference's: the one-step difference of the site's
 * world linear velocity, minus gravity, in the site frame (zero difference
 * after a reset), not MuJoCo's exact rne_post_constraint acceleration.
 * framequat has w >= 0, as in the reference.  Unverified against MuJoCo C.
 */
#include <math.h>
#include <string.h>

#include "mjoracle.h"
#include "o_util.h"

/* world pose of a sensor's object frame */
static void object_frame(const OModel* m, const OData* d, int objtype, int id, double pos[3], double quat[4], int* body) {
  const double* lp = NULL;
  const double* lq = NULL;
  int b = 0;
  if (objtype == 6) { b = m->site_bodyid[id]; lp = m->site_pos + 3 * id; lq = m->site_quat + 4 * id; }
  else if (objtype == 5) { b = m->geom_bodyid[id]; lp = m->geom_pos + 3 * id; lq = m->geom_quat + 4 * id; }
  else if (objtype == 1) { b = id; lp = m->body_ipos + 3 * id; lq = m->body_iquat + 4 * id; }
  else b = id;  /* xbody: the body frame itself */
  const double* bp = d->xpos + 3 * b;
  const double* bq = d->xquat + 4 * b;
  if (lp) {
    double off[3];
    o_quat_rot(bq, lp, off);
    for (int k = 0; k < 3; k++) pos[k] = bp[k] + off[k];
    o_quat_mul(bq, lq, quat);
  } else {
    memcpy(pos, bp, 3 * sizeof(double));
    memcpy(quat, bq, 4 * sizeof(double));
  }
  *body = b;
}

void oracle_sensors(const OModel* m, const OData* d, const double* q0, const double* v0, const double* prev_linvel, double* linvel_out,
                    double* out) {
  OData at = *d;  /* the start state, for tendon lengths */
  at.qpos = (double*)q0;
  at.qvel = (double*)v0;
  for (int s = 0; s < m->nsensor; s++) {
    double* y = out + m->sensor_adr[s];
    const int type = m->sensor_type[s], ot = m->sensor_objtype[s], id = m->sensor_objid[s];
    for (int k = 0; k < m->sensor_dim[s]; k++) y[k] = 0;
    if (linvel_out) memset(linvel_out + 3 * s, 0, 3 * sizeof(double));
    if (!m->sensor_supported[s]) continue;
    if (type == 9) { y[0] = q0[m->jnt_qposadr[id]]; continue; }                    /* jointpos */
    if (type == 10) { y[0] = v0[m->jnt_dofadr[id]]; continue; }                    /* jointvel */
    if (type == 16) { y[0] = d->qfrc_actuator[m->jnt_dofadr[id]]; continue; }      /* jointactuatorfrc */
    if (type == 11 || type == 12) {                                               /* tendonpos / tendonvel */
      double len, vel;
      oracle_tendon(m, &at, id, &len, &vel, NULL);
      y[0] = type == 11 ? len : vel;
      continue;
    }
    if (type == 13 || type == 14) {                                               /* actuatorpos / actuatorvel */
      double len, vel, g = m->actuator_gear[id];
      if (m->actuator_trntype[id] == 3) {
        oracle_tendon(m, &at, m->actuator_trnid[id], &len, &vel, NULL);
      } else {
        len = q0[m->jnt_qposadr[m->actuator_trnid[id]]];
        vel = v0[m->jnt_dofadr[m->actuator_trnid[id]]];
      }
      y[0] = g * (type == 13 ? len : vel);
      continue;
    }
    if (type == 18) {                                                             /* ballquat */
      const double* q = q0 + m->jnt_qposadr[id];
      double n = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
      for (int k = 0; k < 4; k++) y[k] = q[k] / n;
      continue;
    }
    if (type == 19) { for (int k = 0; k < 3; k++) y[k] = v0[m->jnt_dofadr[id] + k]; continue; }  /* ballangvel */
    if (type == 35) { for (int k = 0; k < 3; k++) y[k] = d->subtree_com[3 * id + k]; continue; } /* subtreecom */
    /* frame-based: site sensors (accelerometer 1, velocimeter 2, gyro 3,
       magnetometer 6) and frame sensors (26-32) */
    double pos[3], quat[4], R[9];
    int body;
    object_frame(m, d, ot, id, pos, quat, &body);
    o_quat2mat(quat, R);
    const double* cv = d->cvel + 6 * body;
    const double* c = d->subtree_com + 3 * m->body_rootid[body];
    double r[3] = {pos[0] - c[0], pos[1] - c[1], pos[2] - c[2]}, wxr[3], w[3] = {cv[0], cv[1], cv[2]}, v[3];
    o_cross(w, r, wxr);
    for (int k = 0; k < 3; k++) v[k] = cv[3 + k] + wxr[k];
    if (linvel_out) memcpy(linvel_out + 3 * s, v, 3 * sizeof(double));
    switch (type) {
      case 26: memcpy(y, pos, 3 * sizeof(double)); break;
      case 27: { double sg = quat[0] < 0 ? -1 : 1; for (int k = 0; k < 4; k++) y[k] = sg * quat[k]; break; }
      case 28: case 29: case 30: for (int k = 0; k < 3; k++) y[k] = R[3 * k + (type - 28)]; break;
      case 31: memcpy(y, v, 3 * sizeof(double)); break;
      case 32: memcpy(y, w, 3 * sizeof(double)); break;
      case 3: o_mulmatT(R, w, y); break;
      case 2: o_mulmatT(R, v, y); break;
      case 6: o_mulmatT(R, m->magnetic, y); break;
      case 1: {
        double a[3] = {0, 0, 0};
        if (prev_linvel)
          for (int k = 0; k < 3; k++) a[k] = (v[k] - prev_linvel[3 * s + k]) / m->timestep;
        for (int k = 0; k < 3; k++) a[k] -= m->gravity[k];
        o_mulmatT(R, a, y);
        break;
      }
      default: break;
    }
  }
}
