/*
 * Oracle (test infrastructure): kinematics and smooth dynamics in FP64.
 *   oracle_kinematics   <- kinematics.hpp:75-183 (mj_kinematics)
 *   oracle_com          <- forward.hpp:143-233   (Phase A: subtree COM, cinert, cdof)
 *   oracle_crb          <- forward.hpp:237-279   (Phase B: CRB mass matrix)
 *   oracle_rne          <- forward.hpp:281-397   (Phases C, D: cvel, cdof_dot, RNE bias)
 *   oracle_smooth_forces<- forward.hpp:399-469   (Phase E: passive, actuation, qfrc_smooth)
 */
#include <math.h>
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
/* ---- spatial tendon wrapping (MuJoCo's sphere / cylinder wrapping; the
 * geometry of tangent lines to a circle, restated for the oracle) */

static int seg_cross(const double* p1, const double* p2, const double* p3, const double* p4) {
  double det = (p4[1] - p3[1]) * (p2[0] - p1[0]) - (p4[0] - p3[0]) * (p2[1] - p1[1]);
  if (fabs(det) < 1e-15) return 0;
  double a = ((p4[0] - p3[0]) * (p1[1] - p3[1]) - (p4[1] - p3[1]) * (p1[0] - p3[0])) / det;
  double b = ((p2[0] - p1[0]) * (p1[1] - p3[1]) - (p2[1] - p1[1]) * (p1[0] - p3[0])) / det;
  return a >= 0 && a <= 1 && b >= 0 && b <= 1;
}

/* 2D wrap of the path p0 -> p1 around the circle |x| = r; returns the arc
 * length and the tangent points, or -1 when the straight segment is the
 * path (it stays outside the circle, on the side point's side if given) */
static double wrap_circle(const double* p0, const double* p1, double r, const double* side, double* t0, double* t1) {
  double l0 = p0[0] * p0[0] + p0[1] * p0[1], l1 = p1[0] * p1[0] + p1[1] * p1[1];
  if (r <= 0 || l0 <= r * r || l1 <= r * r) return -1;
  double e[2] = {p1[0] - p0[0], p1[1] - p0[1]}, ee = e[0] * e[0] + e[1] * e[1];
  double a = ee > 0 ? -(p0[0] * e[0] + p0[1] * e[1]) / ee : 0;
  a = a < 0 ? 0 : a > 1 ? 1 : a;
  double q[2] = {p0[0] + a * e[0], p0[1] + a * e[1]};
  if (q[0] * q[0] + q[1] * q[1] > r * r && (!side || side[0] * q[0] + side[1] * q[1] >= 0)) return -1;
  double ta[2][2], tb[2][2], arc[2], best_g = 0;
  int best = -1;
  for (int k = 0; k < 2; k++) {
    double sg = k == 0 ? 1 : -1;   /* counter-clockwise, clockwise */
    const double* pp[2] = {p0, p1};
    for (int e2 = 0; e2 < 2; e2++) {
      const double* p = pp[e2];
      double dd = sqrt(p[0] * p[0] + p[1] * p[1]), c = r / dd, s = sqrt(1 - c * c) * (e2 == 0 ? sg : -sg);
      double u[2] = {p[0] / dd, p[1] / dd}, *t = e2 == 0 ? ta[k] : tb[k];
      t[0] = r * (c * u[0] - s * u[1]);
      t[1] = r * (c * u[1] + s * u[0]);
    }
    double ang = atan2(ta[k][0] * tb[k][1] - ta[k][1] * tb[k][0], ta[k][0] * tb[k][0] + ta[k][1] * tb[k][1]) * sg;
    if (ang < 0) ang += 6.283185307179586;
    arc[k] = r * ang;
    double g;
    if (side) {
      double mid[2] = {ta[k][0] + tb[k][0], ta[k][1] + tb[k][1]}, lm = sqrt(mid[0] * mid[0] + mid[1] * mid[1]);
      if (lm > 1e-12) { mid[0] /= lm; mid[1] /= lm; } else { mid[0] = 1; mid[1] = 0; }
      g = mid[0] * side[0] + mid[1] * side[1];
    } else {
      double dx = ta[k][0] - tb[k][0], dy = ta[k][1] - tb[k][1];
      g = -(dx * dx + dy * dy);
    }
    if (seg_cross(p0, ta[k], p1, tb[k])) g = -1e4;
    if (best < 0 || g > best_g) { best = k; best_g = g; }
  }
  if (seg_cross(p0, ta[best], p1, tb[best])) return -1;
  t0[0] = ta[best][0]; t0[1] = ta[best][1];
  t1[0] = tb[best][0]; t1[1] = tb[best][1];
  return arc[best];
}

/* path s0 -> s1 around a sphere (type 2) or cylinder (type 5) at c with
 * rotation R and radius r; returns its length; *wrapped and the tangent
 * points t0, t1 when it leaves the straight line */
static double wrap_geom(int type, const double* c, const double* R, double r, const double* s0, const double* s1, const double* side, double* t0,
                        double* t1, int* wrapped) {
  double d0[3], d1[3], e1[3], e2[3], ax[3] = {R[2], R[5], R[8]}, z0 = 0, z1 = 0;
  for (int k = 0; k < 3; k++) { d0[k] = s0[k] - c[k]; d1[k] = s1[k] - c[k]; }
  double sv[3] = {s1[0] - s0[0], s1[1] - s0[1], s1[2] - s0[2]}, straight = o_norm3(sv);
  *wrapped = 0;
  if (type == 5) {
    for (int k = 0; k < 3; k++) { e1[k] = R[3 * k]; e2[k] = R[3 * k + 1]; }
    z0 = o_dot3(d0, ax);
    z1 = o_dot3(d1, ax);
  } else {
    double l0 = o_norm3(d0);
    if (l0 < 1e-12) return straight;
    for (int k = 0; k < 3; k++) e1[k] = d0[k] / l0;
    double p = o_dot3(d1, e1), w[3];
    for (int k = 0; k < 3; k++) w[k] = d1[k] - p * e1[k];
    double lw = o_norm3(w);
    if (lw < 1e-12 * (1 + o_norm3(d1))) {
      if (side) {
        double ds[3] = {side[0] - c[0], side[1] - c[1], side[2] - c[2]}, ps = o_dot3(ds, e1);
        for (int k = 0; k < 3; k++) w[k] = ds[k] - ps * e1[k];
        lw = o_norm3(w);
      }
      if (lw < 1e-12) {
        double a[3] = {fabs(e1[0]) < 0.6 ? 1 : 0, fabs(e1[0]) < 0.6 ? 0 : 1, 0}, pa = o_dot3(a, e1);
        for (int k = 0; k < 3; k++) w[k] = a[k] - pa * e1[k];
        lw = o_norm3(w);
      }
    }
    for (int k = 0; k < 3; k++) e2[k] = w[k] / lw;
  }
  double p0[2] = {o_dot3(d0, e1), o_dot3(d0, e2)}, p1[2] = {o_dot3(d1, e1), o_dot3(d1, e2)}, sd[2], a2[2], b2[2];
  const double* sdp = NULL;
  if (side) {
    double ds[3] = {side[0] - c[0], side[1] - c[1], side[2] - c[2]};
    sd[0] = o_dot3(ds, e1);
    sd[1] = o_dot3(ds, e2);
    sdp = sd;
  }
  double arc = wrap_circle(p0, p1, r, sdp, a2, b2);
  if (arc < 0) return straight;
  *wrapped = 1;
  double la = hypot(a2[0] - p0[0], a2[1] - p0[1]), lb = hypot(p1[0] - b2[0], p1[1] - b2[1]), L2 = la + arc + lb, len = L2, za = 0, zb = 0;
  if (type == 5) {
    double dz = z1 - z0;
    za = z0 + (L2 > 0 ? dz * la / L2 : 0);
    zb = z0 + (L2 > 0 ? dz * (la + arc) / L2 : 0);
    len = sqrt(L2 * L2 + dz * dz);
  }
  for (int k = 0; k < 3; k++) {
    t0[k] = c[k] + a2[0] * e1[k] + a2[1] * e2[k] + (type == 5 ? za * ax[k] : 0);
    t1[k] = c[k] + b2[0] * e1[k] + b2[1] * e2[k] + (type == 5 ? zb * ax[k] : 0);
  }
  return len;
}

static void site_world(const OModel* m, const OData* d, int s, double* p) {
  int b = m->site_bodyid[s];
  double r[3];
  o_quat_rot(&d->xquat[4 * b], &m->site_pos[3 * s], r);
  for (int k = 0; k < 3; k++) p[k] = d->xpos[3 * b + k] + r[k];
}

/* J += scale * dir' (point Jacobian of body b at world point p) */
static void point_jac(const OModel* m, const OData* d, int b, const double* p, const double* dir, double scale, double* J) {
  const double* rc = &d->subtree_com[3 * m->body_rootid[b]];
  double off[3] = {p[0] - rc[0], p[1] - rc[1], p[2] - rc[2]};
  for (int i = 0; i < m->nv; i++) {
    int db = m->dof_bodyid[i];
    if (!(db <= b && b < db + m->body_subtreesize[db])) continue;
    const double* c = &d->cdof[6 * i];
    double jp[3] = {c[3] + (c[1] * off[2] - c[2] * off[1]), c[4] + (c[2] * off[0] - c[0] * off[2]), c[5] + (c[0] * off[1] - c[1] * off[0])};
    J[i] += scale * o_dot3(dir, jp);
  }
}

static void piece(const OModel* m, const OData* d, const double* p0, int b0, const double* p1, int b1, double scale, double* len, double* J) {
  double e[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]}, l = o_norm3(e);
  *len += scale * l;
  if (l < 1e-12) return;
  for (int k = 0; k < 3; k++) e[k] /= l;
  point_jac(m, d, b1, p1, e, scale, J);
  point_jac(m, d, b0, p0, e, -scale, J);
}

/* Fixed tendons (reference: tendon.hpp emit_tendon_phase; MuJoCo
 * mj_tendon): length = sum coef * qpos, J = sum coef * e_dof.  Spatial
 * tendons: the path length through the sites (around wrapping geoms, scaled
 * by 1 / divisor after each pulley), J = sum over straight pieces of the
 * piece direction times the difference of the end points' Jacobians, the
 * tangent points moving with the wrapping geom; velocity = J qvel.  The
 * kinematic quantities are those of the last oracle_kinematics / oracle_com. */
void oracle_tendon(const OModel* m, const OData* d, int t, double* len, double* vel, double* J) {
  int nv = m->nv;
  double Jl[nv > 0 ? nv : 1];
  double* JJ = J ? J : Jl;
  double l = 0, scale = 1;
  memset(JJ, 0, nv * sizeof(double));
  int a0 = m->tendon_adr[t], a1 = a0 + m->tendon_num[t];
  for (int w = a0; w < a1; w++) {
    int ty = m->wrap_type[w];
    if (ty == 1) {
      int j = m->wrap_objid[w];
      double c = m->wrap_prm[w];
      l += c * d->qpos[m->jnt_qposadr[j]];
      JJ[m->jnt_dofadr[j]] += c;
    } else if (ty == 2) {
      scale = 1 / m->wrap_prm[w];
    } else if (ty == 3 && w + 1 < a1 && m->wrap_type[w + 1] == 3) {
      double p0[3], p1[3];
      int s0 = m->wrap_objid[w], s1 = m->wrap_objid[w + 1];
      site_world(m, d, s0, p0);
      site_world(m, d, s1, p1);
      piece(m, d, p0, m->site_bodyid[s0], p1, m->site_bodyid[s1], scale, &l, JJ);
    } else if (ty == 3 && w + 2 < a1 && (m->wrap_type[w + 1] == 4 || m->wrap_type[w + 1] == 5)) {
      int s0 = m->wrap_objid[w], g = m->wrap_objid[w + 1], s1 = m->wrap_objid[w + 2], ss = (int)m->wrap_prm[w + 1];
      double p0[3], p1[3], sp[3], t0[3], t1[3];
      site_world(m, d, s0, p0);
      site_world(m, d, s1, p1);
      if (ss >= 0) site_world(m, d, ss, sp);
      int wrapped = 0, gb = m->geom_bodyid[g];
      double full = wrap_geom(m->wrap_type[w + 1] == 4 ? 2 : 5, &d->geom_xpos[3 * g], &d->geom_xmat[9 * g], m->geom_size[3 * g], p0, p1,
                              ss >= 0 ? sp : NULL, t0, t1, &wrapped);
      if (!wrapped) {
        piece(m, d, p0, m->site_bodyid[s0], p1, m->site_bodyid[s1], scale, &l, JJ);
      } else {
        double dummy = 0;
        piece(m, d, p0, m->site_bodyid[s0], t0, gb, scale, &dummy, JJ);
        piece(m, d, t1, gb, p1, m->site_bodyid[s1], scale, &dummy, JJ);
        l += scale * full;
      }
      w += 1;
    }
  }
  double v = 0;
  for (int i = 0; i < nv; i++) v += JJ[i] * d->qvel[i];
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
