/*
 * Oracle (test infrastructure): kinematics and smooth dynamics in FP64.
 *   oracle_kinematics   <- kinematics.hpp:75-183 (mj_kinematics)
 *   oracle_com          <- forward.hpp:143-233   (Phase A: subtree COM, cinert, cdof)
 *   oracle_crb          <- forward.hpp:237-279   (Phase B: CRB mass matrix)
 *   oracle_rne          <- forward.hpp:281-397   (Phases C, D: cvel, cdof_dot, RNE bias)
 *   oracle_smooth_forces<- forward.hpp:399-469   (Phase E: passive, actuation, qfrc_smooth)
 */
#include "mjoracle.h"
#include "o_util.h"

void oracle_kinematics(const OModel* m, OData* d) {
  int nb = m->nbody;
  d->xpos[0] = d->xpos[1] = d->xpos[2] = 0;
  d->xquat[0] = 1; d->xquat[1] = d->xquat[2] = d->xquat[3] = 0;
  for (int b = 1; b < nb; b++) {
    int p = m->body_parentid[b];
    double pos[3], quat[4], r[3];
    o_quat_rot(&d->xquat[4 * p], &m->body_pos[3 * b], r);
    for (int k = 0; k < 3; k++) pos[k] = d->xpos[3 * p + k] + r[k];
    o_quat_mul(&d->xquat[4 * p], &m->body_quat[4 * b], quat);
    for (int j = m->body_jntadr[b]; j >= 0 && j < m->body_jntadr[b] + m->body_jntnum[b]; j++) {
      int qa = m->jnt_qposadr[j];
      const double* q = d->qpos + qa;
      double* an = &d->xanchor[3 * j];
      double* ax = &d->xaxis[3 * j];
      if (m->jnt_type[j] == 0) {  /* free */
        for (int k = 0; k < 3; k++) pos[k] = q[k];
        for (int k = 0; k < 4; k++) quat[k] = q[3 + k];
        o_quat_normalize(quat);
        for (int k = 0; k < 3; k++) an[k] = pos[k];
        ax[0] = 0; ax[1] = 0; ax[2] = 1;
        continue;
      }
      double rj[3];
      o_quat_rot(quat, &m->jnt_pos[3 * j], rj);
      for (int k = 0; k < 3; k++) an[k] = pos[k] + rj[k];
      o_quat_rot(quat, &m->jnt_axis[3 * j], ax);
      if (m->jnt_type[j] == 3 || m->jnt_type[j] == 1) {  /* hinge / ball rotate about the anchor */
        double ql[4];
        if (m->jnt_type[j] == 3) {
          double ang = q[0] - m->qpos0[qa];
          double s = sin(0.5 * ang);
          const double* a = &m->jnt_axis[3 * j];
          ql[0] = cos(0.5 * ang); ql[1] = a[0] * s; ql[2] = a[1] * s; ql[3] = a[2] * s;
        } else {
          for (int k = 0; k < 4; k++) ql[k] = q[k];
          o_quat_normalize(ql);
        }
        o_quat_mul(quat, ql, quat);
        o_quat_rot(quat, &m->jnt_pos[3 * j], rj);
        for (int k = 0; k < 3; k++) pos[k] = an[k] - rj[k];
      } else {  /* slide */
        double dist = q[0] - m->qpos0[qa];
        for (int k = 0; k < 3; k++) pos[k] += ax[k] * dist;
      }
    }
    o_quat_normalize(quat);
    for (int k = 0; k < 3; k++) d->xpos[3 * b + k] = pos[k];
    for (int k = 0; k < 4; k++) d->xquat[4 * b + k] = quat[k];
  }
  for (int b = 0; b < nb; b++) {
    o_quat2mat(&d->xquat[4 * b], &d->xmat[9 * b]);
    double r[3], q[4];
    o_quat_rot(&d->xquat[4 * b], &m->body_ipos[3 * b], r);
    for (int k = 0; k < 3; k++) d->xipos[3 * b + k] = d->xpos[3 * b + k] + r[k];
    o_quat_mul(&d->xquat[4 * b], &m->body_iquat[4 * b], q);
    o_quat2mat(q, &d->ximat[9 * b]);
  }
  for (int g = 0; g < m->ngeom; g++) {
    int b = m->geom_bodyid[g];
    double r[3], q[4];
    o_quat_rot(&d->xquat[4 * b], &m->geom_pos[3 * g], r);
    for (int k = 0; k < 3; k++) d->geom_xpos[3 * g + k] = d->xpos[3 * b + k] + r[k];
    o_quat_mul(&d->xquat[4 * b], &m->geom_quat[4 * g], q);
    o_quat2mat(q, &d->geom_xmat[9 * g]);
  }
}

static double msc(const ORand* r, int b) { return (r && r->mass_scale) ? r->mass_scale[b] : 1.0; }

void oracle_com(const OModel* m, OData* d, const ORand* rnd) {
  int nb = m->nbody, nv = m->nv;
  double* mass = d->work;           /* nb */
  double* mc = d->work + nb;        /* 3 nb */
  /* per-env COM offset, body frame (reference: forward.hpp:110-115 XIP) */
  if (rnd && rnd->com_delta)
    for (int b = 1; b < nb; b++) {
      double w[3];
      o_mulmat(&d->xmat[9 * b], &rnd->com_delta[3 * b], w);
      for (int k = 0; k < 3; k++) d->xipos[3 * b + k] += w[k];
    }
  for (int b = 0; b < nb; b++) {
    mass[b] = m->body_mass[b] * msc(rnd, b);
    for (int k = 0; k < 3; k++) mc[3 * b + k] = mass[b] * d->xipos[3 * b + k];
  }
  for (int b = nb - 1; b > 0; b--) {
    int p = m->body_parentid[b];
    mass[p] += mass[b];
    for (int k = 0; k < 3; k++) mc[3 * p + k] += mc[3 * b + k];
  }
  for (int b = 0; b < nb; b++)
    for (int k = 0; k < 3; k++) d->subtree_com[3 * b + k] = mass[b] > 1e-8 ? mc[3 * b + k] / mass[b] : d->xipos[3 * b + k];
  /* cinert about the subtree COM of the body's root: (I00 I11 I22 I01 I02 I12, m*off, m) */
  for (int b = 0; b < nb; b++) {
    double* ci = &d->cinert[10 * b];
    if (b == 0) { memset(ci, 0, 10 * sizeof(double)); continue; }
    double s = msc(rnd, b);
    double mb = m->body_mass[b] * s;
    const double* R = &d->ximat[9 * b];
    const double* I = &m->body_inertia[3 * b];
    double Ig[9];
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) Ig[r * 3 + c] = s * (R[r * 3] * I[0] * R[c * 3] + R[r * 3 + 1] * I[1] * R[c * 3 + 1] + R[r * 3 + 2] * I[2] * R[c * 3 + 2]);
    const double* rc = &d->subtree_com[3 * m->body_rootid[b]];
    double off[3] = {d->xipos[3 * b] - rc[0], d->xipos[3 * b + 1] - rc[1], d->xipos[3 * b + 2] - rc[2]};
    double d2 = o_dot3(off, off);
    ci[0] = Ig[0] + mb * (d2 - off[0] * off[0]);
    ci[1] = Ig[4] + mb * (d2 - off[1] * off[1]);
    ci[2] = Ig[8] + mb * (d2 - off[2] * off[2]);
    ci[3] = Ig[1] - mb * off[0] * off[1];
    ci[4] = Ig[2] - mb * off[0] * off[2];
    ci[5] = Ig[5] - mb * off[1] * off[2];
    ci[6] = mb * off[0]; ci[7] = mb * off[1]; ci[8] = mb * off[2];
    ci[9] = mb;
  }
  /* cdof = [axis; axis x (subtree_com[root] - anchor)] for rotations, [0; axis] for translations */
  for (int i = 0; i < nv; i++) {
    int b = m->dof_bodyid[i], j = m->dof_jntid[i], t = m->jnt_type[j];
    int sub = i - m->jnt_dofadr[j];
    double* c = &d->cdof[6 * i];
    const double* rc = &d->subtree_com[3 * m->body_rootid[b]];
    double ax[3];
    int rot = 1;
    if (t == 3) { ax[0] = d->xaxis[3 * j]; ax[1] = d->xaxis[3 * j + 1]; ax[2] = d->xaxis[3 * j + 2]; }
    else if (t == 2) { rot = 0; ax[0] = d->xaxis[3 * j]; ax[1] = d->xaxis[3 * j + 1]; ax[2] = d->xaxis[3 * j + 2]; }
    else if (t == 0 && sub < 3) { rot = 0; ax[0] = ax[1] = ax[2] = 0; ax[sub] = 1; }
    else {
      int col = (t == 0) ? sub - 3 : sub;
      for (int k = 0; k < 3; k++) ax[k] = d->xmat[9 * b + 3 * k + col];
    }
    if (rot) {
      double off[3] = {rc[0] - d->xanchor[3 * j], rc[1] - d->xanchor[3 * j + 1], rc[2] - d->xanchor[3 * j + 2]};
      c[0] = ax[0]; c[1] = ax[1]; c[2] = ax[2];
      o_cross(ax, off, c + 3);
    } else {
      c[0] = c[1] = c[2] = 0;
      c[3] = ax[0]; c[4] = ax[1]; c[5] = ax[2];
    }
  }
}

/* f = cinert * v (spatial inertia times motion vector) */
static void cinert_mul(const double* ci, const double* v, double* f) {
  const double *w = v, *l = v + 3;
  f[0] = ci[0] * w[0] + ci[3] * w[1] + ci[4] * w[2] + (ci[7] * l[2] - ci[8] * l[1]);
  f[1] = ci[3] * w[0] + ci[1] * w[1] + ci[5] * w[2] + (ci[8] * l[0] - ci[6] * l[2]);
  f[2] = ci[4] * w[0] + ci[5] * w[1] + ci[2] * w[2] + (ci[6] * l[1] - ci[7] * l[0]);
  f[3] = ci[9] * l[0] - (ci[7] * w[2] - ci[8] * w[1]);
  f[4] = ci[9] * l[1] - (ci[8] * w[0] - ci[6] * w[2]);
  f[5] = ci[9] * l[2] - (ci[6] * w[1] - ci[7] * w[0]);
}

void oracle_crb(const OModel* m, OData* d, const ORand* rnd) {
  (void)rnd;
  int nb = m->nbody, nv = m->nv;
  double* crb = d->work;  /* 10 nb */
  memcpy(crb, d->cinert, 10 * nb * sizeof(double));
  for (int k = 0; k < 10; k++) crb[k] = 0;
  for (int b = nb - 1; b > 0; b--) {
    int p = m->body_parentid[b];
    for (int k = 0; k < 10; k++) crb[10 * p + k] += crb[10 * b + k];
  }
  memset(d->M, 0, nv * nv * sizeof(double));
  for (int i = 0; i < nv; i++) {
    double f[6];
    cinert_mul(&crb[10 * m->dof_bodyid[i]], &d->cdof[6 * i], f);
    for (int j = i; j >= 0; j = m->dof_parentid[j]) {
      const double* cj = &d->cdof[6 * j];
      double s = 0;
      for (int k = 0; k < 6; k++) s += f[k] * cj[k];
      d->M[i * nv + j] = s;
      d->M[j * nv + i] = s;
    }
    d->M[i * nv + i] += m->dof_armature[i];
  }
  memcpy(d->qLD, d->M, nv * nv * sizeof(double));
  o_chol(d->qLD, nv);
}

/* motion cross product v x u, v = [w; vl] */
static void cross_motion(const double* v, const double* u, double* r) {
  double a[3], b[3];
  o_cross(v, u, r);
  o_cross(v + 3, u, a);
  o_cross(v, u + 3, b);
  for (int k = 0; k < 3; k++) r[3 + k] = a[k] + b[k];
}
/* force cross product v x* f */
static void cross_force(const double* v, const double* f, double* r) {
  double a[3], b[3];
  o_cross(v, f, a);
  o_cross(v + 3, f + 3, b);
  for (int k = 0; k < 3; k++) r[k] = a[k] + b[k];
  o_cross(v, f + 3, r + 3);
}

void oracle_rne(const OModel* m, OData* d, const ORand* rnd) {
  (void)rnd;
  int nb = m->nbody, nv = m->nv;
  const double* qv = d->qvel;
  memset(d->cvel, 0, 6 * sizeof(double));
  for (int b = 1; b < nb; b++) {
    double cv[6];
    memcpy(cv, &d->cvel[6 * m->body_parentid[b]], sizeof(cv));
    int a = m->body_dofadr[b], n = m->body_dofnum[b];
    for (int k = 0; k < n;) {
      int i = a + k;
      int t = m->jnt_type[m->dof_jntid[i]];
      if (t == 0) {  /* free: translations (cdof_dot 0), then rotations with a common cvel */
        for (int s = 0; s < 3; s++) {
          memset(&d->cdof_dot[6 * (i + s)], 0, 6 * sizeof(double));
          for (int c = 0; c < 6; c++) cv[c] += d->cdof[6 * (i + s) + c] * qv[i + s];
        }
        for (int s = 3; s < 6; s++) cross_motion(cv, &d->cdof[6 * (i + s)], &d->cdof_dot[6 * (i + s)]);
        for (int s = 3; s < 6; s++)
          for (int c = 0; c < 6; c++) cv[c] += d->cdof[6 * (i + s) + c] * qv[i + s];
        k += 6;
      } else if (t == 1) {  /* ball: three rotations with a common cvel */
        for (int s = 0; s < 3; s++) cross_motion(cv, &d->cdof[6 * (i + s)], &d->cdof_dot[6 * (i + s)]);
        for (int s = 0; s < 3; s++)
          for (int c = 0; c < 6; c++) cv[c] += d->cdof[6 * (i + s) + c] * qv[i + s];
        k += 3;
      } else {
        cross_motion(cv, &d->cdof[6 * i], &d->cdof_dot[6 * i]);
        for (int c = 0; c < 6; c++) cv[c] += d->cdof[6 * i + c] * qv[i];
        k += 1;
      }
    }
    memcpy(&d->cvel[6 * b], cv, sizeof(cv));
  }
  /* RNE with qacc = 0: cacc, cfrc, backward sum, projection */
  memset(d->cacc, 0, 6 * sizeof(double));
  if (!(m->disableflags & (1 << 6)))
    for (int k = 0; k < 3; k++) d->cacc[3 + k] = -m->gravity[k];
  for (int b = 1; b < nb; b++) {
    double* ca = &d->cacc[6 * b];
    memcpy(ca, &d->cacc[6 * m->body_parentid[b]], 6 * sizeof(double));
    for (int i = m->body_dofadr[b]; i < m->body_dofadr[b] + m->body_dofnum[b]; i++)
      for (int c = 0; c < 6; c++) ca[c] += d->cdof_dot[6 * i + c] * qv[i];
  }
  for (int b = 0; b < nb; b++) {
    double Ia[6], Iv[6], vf[6];
    cinert_mul(&d->cinert[10 * b], &d->cacc[6 * b], Ia);
    cinert_mul(&d->cinert[10 * b], &d->cvel[6 * b], Iv);
    cross_force(&d->cvel[6 * b], Iv, vf);
    for (int c = 0; c < 6; c++) d->cfrc[6 * b + c] = Ia[c] + vf[c];
  }
  for (int b = nb - 1; b > 0; b--) {
    int p = m->body_parentid[b];
    for (int c = 0; c < 6; c++) d->cfrc[6 * p + c] += d->cfrc[6 * b + c];
  }
  for (int i = 0; i < nv; i++) {
    const double* f = &d->cfrc[6 * m->dof_bodyid[i]];
    double s = 0;
    for (int c = 0; c < 6; c++) s += d->cdof[6 * i + c] * f[c];
    d->qfrc_bias[i] = s;
  }
}

/* Fixed tendon (reference: tendon.hpp emit_tendon_phase; MuJoCo
 * mj_tendon): length = sum coef * qpos, J = sum coef * e_dof. */
void oracle_tendon(const OModel* m, const OData* d, int t, double* len, double* vel, double* J) {
  double l = 0, v = 0;
  if (J) memset(J, 0, m->nv * sizeof(double));
  for (int w = m->tendon_adr[t]; w < m->tendon_adr[t] + m->tendon_num[t]; w++) {
    int j = m->wrap_joint[w];
    double c = m->wrap_coef[w];
    l += c * d->qpos[m->jnt_qposadr[j]];
    v += c * d->qvel[m->jnt_dofadr[j]];
    if (J) J[m->jnt_dofadr[j]] += c;
  }
  *len = l;
  *vel = v;
}

void oracle_smooth_forces(const OModel* m, OData* d, const ORand* rnd) {
  int nv = m->nv;
  memset(d->qfrc_passive, 0, nv * sizeof(double));
  double* tJ = d->work;  /* nv */
  if (!(m->disableflags & (1 << 5))) {
    for (int j = 0; j < m->njnt; j++) {
      int t = m->jnt_type[j];
      if ((t == 2 || t == 3) && m->jnt_stiffness[j] != 0) {
        int qa = m->jnt_qposadr[j], da = m->jnt_dofadr[j];
        d->qfrc_passive[da] -= m->jnt_stiffness[j] * (d->qpos[qa] - m->qpos_spring[qa]);
      }
    }
    for (int i = 0; i < nv; i++) d->qfrc_passive[i] -= m->dof_damping[i] * d->qvel[i];
    /* gravity compensation: -gravcomp * m * gravity at the body's COM,
       through cdof (reference: forward.hpp:438-452) */
    for (int b = 1; b < m->nbody && !(m->disableflags & (1 << 6)); b++) {
      double gc = m->body_gravcomp[b];
      if (gc == 0) continue;
      double mb = m->body_mass[b] * gc * msc(rnd, b), f[3], o[3], w[6];
      const double* rc = &d->subtree_com[3 * m->body_rootid[b]];
      for (int k = 0; k < 3; k++) { f[k] = -mb * m->gravity[k]; o[k] = d->xipos[3 * b + k] - rc[k]; }
      o_cross(o, f, w);
      w[3] = f[0]; w[4] = f[1]; w[5] = f[2];
      for (int i = 0; i < nv; i++) {
        int db = m->dof_bodyid[i];
        if (!(db <= b && b < db + m->body_subtreesize[db])) continue;
        double s = 0;
        for (int k = 0; k < 6; k++) s += d->cdof[6 * i + k] * w[k];
        d->qfrc_passive[i] += s;
      }
    }
    /* quadratic drag on free joints, per env (reference: forward.hpp:455-464) */
    if (rnd && rnd->drag_k) {
      int f = 0;
      for (int j = 0; j < m->njnt; j++) {
        if (m->jnt_type[j] != 0) continue;
        int da = m->jnt_dofadr[j];
        const double* v = &d->qvel[da];
        double kd = -rnd->drag_k[f++] * sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int k = 0; k < 3; k++) d->qfrc_passive[da + k] += kd * v[k];
      }
    }
    /* tendon spring with a dead band [lengthspring lo, hi] and damper
       (reference: tendon.hpp:360-377) */
    for (int t = 0; t < m->ntendon; t++) {
      double k = m->tendon_stiffness[t], c = m->tendon_damping[t];
      if (k == 0 && c == 0) continue;
      double len, vel, f = 0;
      oracle_tendon(m, d, t, &len, &vel, tJ);
      double lo = m->tendon_lengthspring[2 * t], hi = m->tendon_lengthspring[2 * t + 1];
      if (len > hi) f += k * (hi - len);
      else if (len < lo) f += k * (lo - len);
      f -= c * vel;
      for (int i = 0; i < nv; i++) d->qfrc_passive[i] += tJ[i] * f;
    }
  }
  memset(d->qfrc_actuator, 0, nv * sizeof(double));
  if (!(m->disableflags & (1 << 10))) {
    for (int a = 0; a < m->nu; a++) {
      const int tendon = m->actuator_trntype[a] == 3;
      double gear = m->actuator_gear[a];
      double tl = 0, tv = 0;
      int qa = 0, da = 0;
      if (tendon) {
        oracle_tendon(m, d, m->actuator_trnid[a], &tl, &tv, tJ);
      } else {
        int j = m->actuator_trnid[a];
        qa = m->jnt_qposadr[j];
        da = m->jnt_dofadr[j];
      }
      double ctrl = d->ctrl[a];
      if (m->actuator_ctrllimited[a] && !(m->disableflags & (1 << 7))) {
        double lo = m->actuator_ctrlrange[2 * a], hi = m->actuator_ctrlrange[2 * a + 1];
        ctrl = ctrl < lo ? lo : ctrl > hi ? hi : ctrl;
      }
      double len = gear * (tendon ? tl : d->qpos[qa]), vel = gear * (tendon ? tv : d->qvel[da]);
      const double* g = &m->actuator_gainprm[3 * a];
      const double* bp = &m->actuator_biasprm[3 * a];
      double gain = g[0] + (m->actuator_gaintype[a] ? g[1] * len + g[2] * vel : 0);
      double bias = m->actuator_biastype[a] ? bp[0] + bp[1] * len + bp[2] * vel : 0;
      double force = gain * ctrl + bias;
      if (rnd && rnd->gain_scale) force *= rnd->gain_scale[a];
      if (m->actuator_forcelimited[a]) {
        double lo = m->actuator_forcerange[2 * a], hi = m->actuator_forcerange[2 * a + 1];
        force = force < lo ? lo : force > hi ? hi : force;
      }
      if (tendon)
        for (int i = 0; i < nv; i++) d->qfrc_actuator[i] += gear * force * tJ[i];
      else
        d->qfrc_actuator[da] += gear * force;
    }
  }
  for (int i = 0; i < nv; i++) {
    d->qfrc_smooth[i] = d->qfrc_passive[i] - d->qfrc_bias[i] + d->qfrc_actuator[i];
    d->qacc_smooth[i] = d->qfrc_smooth[i];
  }
  o_chol_solve(d->qLD, nv, d->qacc_smooth);
}
