/*
 * Oracle (test infrastructure): constraint rows, Newton solver, Euler.
 *   oracle_make_constraints <- solver.hpp:259-587 (rows in the order
 *        frictionloss -> limits -> contacts; impedance efc_kbi solver.hpp:122-138;
 *        pyramid rows J_n +- mu_k J_k with R = 2 mu0^2 / impratio * R_first,
 *        R_first from invw_t (1 + mu0^2), solver.hpp:536-571)
 *   oracle_solve            <- solver.hpp:592-854 (Newton on the primal cost,
 *        Cholesky of H = M + J' D J), here with MuJoCo's previous-step warm
 *        start (smooth vs warm by total cost), an exact line search on the
 *        piecewise-quadratic cost, and termination by improvement or gradient
 *        below tolerance scaled by 1/(meaninertia * nv)
 *   oracle_integrate        <- euler.hpp:26-110 (semi-implicit Euler,
 *        quaternion exp-map for free/ball joints), batched.cpp:712-745 for the
 *        implicit joint-damping fold
 */
#include <pthread.h>
#include <stdlib.h>

#include "mjoracle.h"
#include "o_util.h"

enum { T_FRICTION = 0, T_LIMIT = 1, T_PYRAMID = 2, T_FRICTIONLESS = 3, T_ELLIPTIC = 4, T_EQUALITY = 5, T_ELLFRIC = 6 };

static void impedance(const OModel* m, const double* solref, const double* solimp, double pos, double* k, double* b, double* imp) {
  double tc = solref[0], dr = solref[1];
  if (!(m->disableflags & (1 << 11)) && tc > 0 && tc < 2 * m->timestep) tc = 2 * m->timestep;
  double dmin = solimp[0] < 1e-4 ? 1e-4 : solimp[0] > 0.9999 ? 0.9999 : solimp[0];
  double dmax = solimp[1] < 1e-4 ? 1e-4 : solimp[1] > 0.9999 ? 0.9999 : solimp[1];
  double width = solimp[2] < 1e-12 ? 1e-12 : solimp[2];
  double mid = solimp[3] < 1e-4 ? 1e-4 : solimp[3] > 0.9999 ? 0.9999 : solimp[3];
  double power = solimp[4] < 1 ? 1 : solimp[4];
  *k = tc > 0 ? 1.0 / (dmax * dmax * tc * tc * dr * dr) : -tc / (dmax * dmax);
  *b = dr > 0 ? 2.0 / (dmax * tc) : -dr / dmax;
  double x = fabs(pos) / width;
  if (x >= 1) { *imp = dmax; return; }
  double y = x < mid ? pow(x, power) / pow(mid, power - 1) : 1 - pow(1 - x, power) / pow(1 - mid, power - 1);
  double v = dmin + y * (dmax - dmin);
  *imp = v < dmin ? dmin : v > dmax ? dmax : v;
}

static int add_row(OData* d, int nv, int type) {
  int r = d->nefc++;
  memset(&d->efc_J[r * nv], 0, nv * sizeof(double));
  d->efc_type[r] = type;
  d->efc_floss[r] = 0;
  return r;
}

static double rowdot(const double* J, const double* v, int nv) {
  double s = 0;
  for (int i = 0; i < nv; i++) s += J[i] * v[i];
  return s;
}

void oracle_make_constraints(const OModel* m, OData* d, const ORand* rnd) {
  int nv = m->nv;
  d->nefc = 0;
  d->nefc_dropped = 0;
  int stop = 0;  /* set when a row group does not fit: it and every later group are dropped */
  if (m->disableflags & 1) return;
  /* joint equalities first (reference: solver.hpp:259-289; bilateral) */
  if (!(m->disableflags & (1 << 1))) {
    double* J2 = d->work;  /* nv */
    for (int e = 0; e < m->neq; e++) {
      if (!m->eq_active[e] || (m->eq_type[e] != 2 && m->eq_type[e] != 3)) continue;
      if (stop || d->nefc + 1 > d->nefc_max) { stop = 1; d->nefc_dropped++; d->status |= ORACLE_EFC_OVERFLOW; continue; }
      const int ten = m->eq_type[e] == 3;
      int o1 = m->eq_obj1[e], o2 = m->eq_obj2[e];
      /* joint: q - qpos0 / tendon: length - length0, and its rate */
      double x1, v1, x2 = 0, v2 = 0;
      int r = add_row(d, nv, T_EQUALITY);
      double* J = &d->efc_J[r * nv];
      if (ten) {
        oracle_tendon(m, d, o1, &x1, &v1, J);
        x1 -= m->tendon_length0[o1];
        if (o2 >= 0) {
          oracle_tendon(m, d, o2, &x2, &v2, J2);
          x2 -= m->tendon_length0[o2];
        }
      } else {
        x1 = d->qpos[m->jnt_qposadr[o1]] - m->qpos0[m->jnt_qposadr[o1]];
        v1 = d->qvel[m->jnt_dofadr[o1]];
        J[m->jnt_dofadr[o1]] = 1;
        if (o2 >= 0) {
          memset(J2, 0, nv * sizeof(double));
          x2 = d->qpos[m->jnt_qposadr[o2]] - m->qpos0[m->jnt_qposadr[o2]];
          v2 = d->qvel[m->jnt_dofadr[o2]];
          J2[m->jnt_dofadr[o2]] = 1;
        }
      }
      const double* c = &m->eq_data[5 * e];
      double poly = c[0], dpoly = 0;
      if (o2 >= 0) {
        poly = c[0] + x2 * (c[1] + x2 * (c[2] + x2 * (c[3] + x2 * c[4])));
        dpoly = c[1] + x2 * (2 * c[2] + x2 * (3 * c[3] + x2 * 4 * c[4]));
        for (int i = 0; i < nv; i++) J[i] -= dpoly * J2[i];
      }
      double pos = x1 - poly;
      double vel = v1 - dpoly * v2;
      double k, b, imp;
      impedance(m, &m->eq_solref[2 * e], &m->eq_solimp[5 * e], pos, &k, &b, &imp);
      double R = (1 - imp) / imp * m->eq_invweight[e];
      d->efc_R[r] = R < O_MINVAL ? O_MINVAL : R;
      d->efc_D[r] = 1 / d->efc_R[r];
      d->efc_aref[r] = -b * vel - k * imp * pos;
    }
  }
  if (!(m->disableflags & (1 << 2))) {
    for (int i = 0; i < nv; i++) {
      if (m->dof_frictionloss[i] <= 0) continue;
      if (stop || d->nefc + 1 > d->nefc_max) { stop = 1; d->nefc_dropped++; d->status |= ORACLE_EFC_OVERFLOW; continue; }
      double k, b, imp;
      impedance(m, &m->dof_solref[2 * i], &m->dof_solimp[5 * i], 0, &k, &b, &imp);
      int r = add_row(d, nv, T_FRICTION);
      d->efc_J[r * nv + i] = 1;
      double R = (1 - imp) / imp * m->dof_invweight0[i];
      d->efc_R[r] = R < O_MINVAL ? O_MINVAL : R;
      d->efc_D[r] = 1 / d->efc_R[r];
      d->efc_aref[r] = -b * d->qvel[i];
      d->efc_floss[r] = m->dof_frictionloss[i];
    }
    /* tendon frictionloss rows after the dof ones (reference: solver.hpp:320-342) */
    for (int t = 0; t < m->ntendon; t++) {
      if (m->tendon_frictionloss[t] <= 0) continue;
      if (stop || d->nefc + 1 > d->nefc_max) { stop = 1; d->nefc_dropped++; d->status |= ORACLE_EFC_OVERFLOW; continue; }
      double k, b, imp, len, vel;
      impedance(m, &m->tendon_solref_fri[2 * t], &m->tendon_solimp_fri[5 * t], 0, &k, &b, &imp);
      int r = add_row(d, nv, T_FRICTION);
      oracle_tendon(m, d, t, &len, &vel, &d->efc_J[r * nv]);
      double R = (1 - imp) / imp * m->tendon_invweight0[t];
      d->efc_R[r] = R < O_MINVAL ? O_MINVAL : R;
      d->efc_D[r] = 1 / d->efc_R[r];
      d->efc_aref[r] = -b * vel;
      d->efc_floss[r] = m->tendon_frictionloss[t];
    }
  }
  if (!(m->disableflags & (1 << 3))) {
    for (int j = 0; j < m->njnt; j++) {
      if (!m->jnt_limited[j] || (m->jnt_type[j] != 2 && m->jnt_type[j] != 3)) continue;
      int qa = m->jnt_qposadr[j], da = m->jnt_dofadr[j];
      for (int side = 0; side < 2; side++) {
        double dist = side == 0 ? d->qpos[qa] - m->jnt_range[2 * j] : m->jnt_range[2 * j + 1] - d->qpos[qa];
        double margin = m->jnt_margin[j];
        if (!(dist < margin)) continue;
        if (stop || d->nefc + 1 > d->nefc_max) { stop = 1; d->nefc_dropped++; d->status |= ORACLE_EFC_OVERFLOW; continue; }
        double k, b, imp, pos = dist - margin;
        impedance(m, &m->jnt_solref[2 * j], &m->jnt_solimp[5 * j], pos, &k, &b, &imp);
        int r = add_row(d, nv, T_LIMIT);
        double sg = side == 0 ? 1.0 : -1.0;
        d->efc_J[r * nv + da] = sg;
        double R = (1 - imp) / imp * m->dof_invweight0[da];
        d->efc_R[r] = R < O_MINVAL ? O_MINVAL : R;
        d->efc_D[r] = 1 / d->efc_R[r];
        d->efc_aref[r] = -b * sg * d->qvel[da] - k * imp * pos;
      }
    }
    /* tendon limits after the joint limits, lower side then upper side
       (reference: solver.hpp:370-395) */
    for (int t = 0; t < m->ntendon; t++) {
      if (!m->tendon_limited[t]) continue;
      double len, vel;
      oracle_tendon(m, d, t, &len, &vel, NULL);
      for (int side = 0; side < 2; side++) {
        double dist = side == 0 ? len - m->tendon_range[2 * t] : m->tendon_range[2 * t + 1] - len;
        double margin = m->tendon_margin[t];
        if (!(dist < margin)) continue;
        if (stop || d->nefc + 1 > d->nefc_max) { stop = 1; d->nefc_dropped++; d->status |= ORACLE_EFC_OVERFLOW; continue; }
        double k, b, imp, pos = dist - margin;
        impedance(m, &m->tendon_solref_lim[2 * t], &m->tendon_solimp_lim[5 * t], pos, &k, &b, &imp);
        int r = add_row(d, nv, T_LIMIT);
        double sg = side == 0 ? 1.0 : -1.0;
        oracle_tendon(m, d, t, &len, &vel, &d->efc_J[r * nv]);
        for (int i = 0; i < nv; i++) d->efc_J[r * nv + i] *= sg;
        double R = (1 - imp) / imp * m->tendon_invweight0[t];
        d->efc_R[r] = R < O_MINVAL ? O_MINVAL : R;
        d->efc_D[r] = 1 / d->efc_R[r];
        d->efc_aref[r] = -b * sg * vel - k * imp * pos;
      }
    }
  }
  if (m->disableflags & (1 << 4)) return;
  double* jacp = d->work;           /* 3 nv */
  double* jacr = d->work + 3 * nv;  /* 3 nv */
  for (int c = 0; c < d->ncon; c++) {
    double* con = &d->contact[ORACLE_CONTACT_STRIDE * c];
    con[19] = -1;
    double dist = con[12], incl = con[18];
    if (!(dist < incl)) continue;
    int pair = (int)con[13];
    const int* pi = &m->pair_int[6 * pair];
    const double* pr = &m->pair_real[16 * pair];
    int dim = pi[4];
    const int elliptic = m->cone == 1 && dim > 1;
    int nrow = dim == 1 ? 1 : elliptic ? dim : 2 * (dim - 1);
    if (stop || d->nefc + nrow > d->nefc_max) { stop = 1; d->nefc_dropped += nrow; d->status |= ORACLE_EFC_OVERFLOW; continue; }
    double fs = (rnd ? rnd->friction_scale : 1.0);
    double mu[5];
    for (int k = 0; k < 5; k++) mu[k] = pr[2 + k] * fs;
    double pos = dist - incl, k, b, imp;
    impedance(m, pr + 7, pr + 9, pos, &k, &b, &imp);
    /* Jacobian difference body2 - body1 at the contact point */
    memset(jacp, 0, 6 * nv * sizeof(double));
    for (int side = 0; side < 2; side++) {
      int body = side == 0 ? pi[3] : pi[2];
      double sg = side == 0 ? 1.0 : -1.0;
      const double* rc = &d->subtree_com[3 * m->body_rootid[body]];
      double off[3] = {con[0] - rc[0], con[1] - rc[1], con[2] - rc[2]};
      for (int i = 0; i < nv; i++) {
        int db = m->dof_bodyid[i];
        if (!(db <= body && body < db + m->body_subtreesize[db])) continue;
        const double* cd = &d->cdof[6 * i];
        double x[3];
        o_cross(cd, off, x);
        for (int a = 0; a < 3; a++) {
          jacp[a * nv + i] += sg * (cd[3 + a] + x[a]);
          jacr[a * nv + i] += sg * cd[a];
        }
      }
    }
    const double* fr = con + 3;  /* n, t1, t2 */
    con[19] = d->nefc;
    double* Jn = d->work + 6 * nv;  /* nv */
    for (int i = 0; i < nv; i++) Jn[i] = fr[0] * jacp[i] + fr[1] * jacp[nv + i] + fr[2] * jacp[2 * nv + i];
    if (dim == 1) {
      int r = add_row(d, nv, T_FRICTIONLESS);
      memcpy(&d->efc_J[r * nv], Jn, nv * sizeof(double));
      double R = (1 - imp) / imp * pr[14];
      d->efc_R[r] = R < O_MINVAL ? O_MINVAL : R;
      d->efc_D[r] = 1 / d->efc_R[r];
      d->efc_aref[r] = -b * rowdot(Jn, d->qvel, nv) - k * imp * pos;
      continue;
    }
    if (elliptic) {
      /* elliptic cone (MuJoCo's model): the normal row and dim - 1 friction
         rows along t1, t2 (translation), n (torsion), t1, t2 (rolling).
         R_n from the translational invweight; friction R_j = R_n (mu_0 /
         mu_j)^2 / impratio, so the cone's aspect in the solver is
         mu = mu_0 / sqrt(impratio) (stored in the normal row's floss slot;
         each friction row stores its own coefficient mu_j) */
      double Rn = (1 - imp) / imp * pr[14];
      if (Rn < O_MINVAL) Rn = O_MINVAL;
      int r = add_row(d, nv, T_ELLIPTIC);
      memcpy(&d->efc_J[r * nv], Jn, nv * sizeof(double));
      d->efc_R[r] = Rn;
      d->efc_D[r] = 1 / Rn;
      d->efc_aref[r] = -b * rowdot(Jn, d->qvel, nv) - k * imp * pos;
      d->efc_floss[r] = mu[0] / sqrt(m->impratio);
      for (int dir = 0; dir < dim - 1; dir++) {
        const double* ax = dir == 0 || dir == 3 ? fr + 3 : dir == 1 || dir == 4 ? fr + 6 : fr;
        const double* src = dir < 2 ? jacp : jacr;
        int rf = add_row(d, nv, T_ELLFRIC);
        double* J = &d->efc_J[rf * nv];
        for (int i = 0; i < nv; i++) J[i] = ax[0] * src[i] + ax[1] * src[nv + i] + ax[2] * src[2 * nv + i];
        double Rf = Rn * (mu[0] * mu[0]) / (mu[dir] * mu[dir]) / m->impratio;
        d->efc_R[rf] = Rf < O_MINVAL ? O_MINVAL : Rf;
        d->efc_D[rf] = 1 / d->efc_R[rf];
        d->efc_aref[rf] = -b * rowdot(J, d->qvel, nv);
        d->efc_floss[rf] = mu[dir];
      }
      continue;
    }
    double mu0 = mu[0];
    double Rfirst = (1 - imp) / imp * pr[14] * (1 + mu0 * mu0);
    if (Rfirst < O_MINVAL) Rfirst = O_MINVAL;
    double Rpy = 2 * mu0 * mu0 / m->impratio * Rfirst;
    if (Rpy < O_MINVAL) Rpy = O_MINVAL;
    for (int dir = 0; dir < dim - 1; dir++) {
      /* directions: t1, t2 (translation), n (spin), t1, t2 (rolling) */
      const double* ax = dir == 0 || dir == 3 ? fr + 3 : dir == 1 || dir == 4 ? fr + 6 : fr;
      const double* src = dir < 2 ? jacp : jacr;
      for (int sgi = 0; sgi < 2; sgi++) {
        double sg = sgi == 0 ? 1.0 : -1.0;
        int r = add_row(d, nv, T_PYRAMID);
        double* J = &d->efc_J[r * nv];
        for (int i = 0; i < nv; i++) {
          double jt = ax[0] * src[i] + ax[1] * src[nv + i] + ax[2] * src[2 * nv + i];
          J[i] = Jn[i] + sg * mu[dir] * jt;
        }
        d->efc_R[r] = Rpy;
        d->efc_D[r] = 1 / Rpy;
        d->efc_aref[r] = -b * rowdot(J, d->qvel, nv) - k * imp * pos;
      }
    }
  }
}

/* ------------------------------------------------------------------ Newton */

/* row cost s(y) and force -s'(y) */
static double row_cost(int type, double D, double fl, double y) {
  if (type == T_FRICTION) {
    double R = 1 / D;
    if (fabs(y) < fl * R) return 0.5 * D * y * y;
    return fl * fabs(y) - 0.5 * fl * fl * R;
  }
  if (type == T_EQUALITY) return 0.5 * D * y * y;
  return y < 0 ? 0.5 * D * y * y : 0;
}
static double row_force(int type, double D, double fl, double y) {
  if (type == T_FRICTION) {
    double f = -D * y;
    return f > fl ? fl : f < -fl ? -fl : f;
  }
  if (type == T_EQUALITY) return -D * y;
  return y < 0 ? -D * y : 0;
}
static int row_quadratic(int type, double D, double fl, double y) {
  if (type == T_FRICTION) return fabs(y) < fl / D;
  if (type == T_EQUALITY) return 1;
  return y < 0;
}
/* s(y + dy) - s(y), written to keep precision when dy is small */
static double row_cost_delta(int type, double D, double fl, double y, double dy) {
  int q0 = row_quadratic(type, D, fl, y), q1 = row_quadratic(type, D, fl, y + dy);
  if (q0 && q1) return 0.5 * D * dy * (2 * y + dy);
  if (type != T_FRICTION && !q0 && !q1) return 0;
  if (type == T_FRICTION && !q0 && !q1 && (y > 0) == (y + dy > 0)) return fl * (fabs(y + dy) - fabs(y));
  return row_cost(type, D, fl, y + dy) - row_cost(type, D, fl, y);
}

/* Elliptic contact group (rows r0 = normal, r0+1 .. r0+dim-1 = friction)
 * with jar y[0..dim): MuJoCo's three zones in the cone space U_0 = mu y_0,
 * U_j = mu_j y_j, N = U_0, T = |U_t|:
 *  top (N >= mu T): no force;
 *  bottom (mu N + T <= 0): every row quadratic, f_j = -D_j y_j;
 *  middle: cost 0.5 Dm (N - mu T)^2 with Dm = D_0 / (mu^2 (1 + mu^2)).
 * Returns the cost; fills the forces, the zone (0 top, 1 bottom, 2 middle)
 * and, if H is not NULL, the dim x dim Hessian in jar space. */
static double cone_eval(int dim, const double* D, const double* fl, const double* y, double* f, int* zone, double* H) {
  double mu = fl[0], U[6], T = 0;
  U[0] = mu * y[0];
  for (int j = 1; j < dim; j++) { U[j] = fl[j] * y[j]; T += U[j] * U[j]; }
  T = sqrt(T);
  double N = U[0], cost = 0;
  if (H) memset(H, 0, dim * dim * sizeof(double));
  if (N >= mu * T || (T <= 0 && N >= 0)) {
    for (int j = 0; j < dim; j++) f[j] = 0;
    *zone = 0;
  } else if (mu * N + T <= 0 || (T <= 0 && N < 0)) {
    for (int j = 0; j < dim; j++) {
      f[j] = -D[j] * y[j];
      cost += 0.5 * D[j] * y[j] * y[j];
      if (H) H[j * dim + j] = D[j];
    }
    *zone = 1;
  } else {
    double Dm = D[0] / (mu * mu * (1 + mu * mu)), NmT = N - mu * T;
    cost = 0.5 * Dm * NmT * NmT;
    f[0] = -Dm * NmT * mu;
    for (int j = 1; j < dim; j++) f[j] = Dm * NmT * mu * U[j] / T * fl[j];
    if (H) {
      /* Dm (a a' + NmT S' grad^2(N - mu T) S), a = S' grad(N - mu T),
         S = diag(mu, mu_1..) */
      double a[6];
      a[0] = mu;
      for (int j = 1; j < dim; j++) a[j] = -mu * U[j] / T * fl[j];
      for (int i = 0; i < dim; i++)
        for (int j = 0; j < dim; j++) H[i * dim + j] = Dm * a[i] * a[j];
      double c = -Dm * NmT * mu / T;   /* > 0 in the middle zone */
      for (int i = 1; i < dim; i++)
        for (int j = 1; j < dim; j++) H[i * dim + j] += c * fl[i] * fl[j] * ((i == j ? 1.0 : 0.0) - U[i] * U[j] / (T * T));
    }
    *zone = 2;
  }
  return cost;
}

static int group_dim(const int* type, int r, int ne) {
  int dim = 1;
  while (r + dim < ne && type[r + dim] == T_ELLFRIC) dim++;
  return dim;
}

typedef struct {
  int nv, nefc;
  const double *M, *qfrc_smooth, *qacc_smooth, *J, *aref, *D, *floss;
  const int* type;
} Prob;

/* total cost at x with d = x - qacc_smooth: 0.5 d'Md + sum of row costs;
 * fills y (jar), force, Md = M d, grad = Md - J'force */
static double eval_point(const Prob* P, const double* x, double* y, double* force, double* Md, double* grad) {
  int nv = P->nv;
  double cost = 0;
  for (int i = 0; i < nv; i++) {
    double s = 0;
    for (int j = 0; j < nv; j++) s += P->M[i * nv + j] * (x[j] - P->qacc_smooth[j]);
    Md[i] = s;
  }
  for (int i = 0; i < nv; i++) cost += 0.5 * (x[i] - P->qacc_smooth[i]) * Md[i];
  for (int r = 0; r < P->nefc; r++) y[r] = rowdot(&P->J[r * nv], x, nv) - P->aref[r];
  for (int r = 0; r < P->nefc; r++) {
    if (P->type[r] == T_ELLFRIC) continue;
    if (P->type[r] == T_ELLIPTIC) {
      int dim = group_dim(P->type, r, P->nefc), zone;
      cost += cone_eval(dim, &P->D[r], &P->floss[r], &y[r], &force[r], &zone, NULL);
      continue;
    }
    force[r] = row_force(P->type[r], P->D[r], P->floss[r], y[r]);
    cost += row_cost(P->type[r], P->D[r], P->floss[r], y[r]);
  }
  for (int i = 0; i < nv; i++) {
    double s = Md[i];
    for (int r = 0; r < P->nefc; r++) s -= P->J[r * nv + i] * force[r];
    grad[i] = s;
  }
  return cost;
}

/* f'(a), f''(a) of the cost along p from the current point */
static void ls_deriv(const Prob* P, double A, double B, const double* y, const double* q, double a, double* d1, double* d2) {
  double g1 = a * A + B, g2 = A;
  for (int r = 0; r < P->nefc; r++) {
    if (P->type[r] == T_ELLFRIC) continue;
    if (P->type[r] == T_ELLIPTIC) {
      /* d/da and d2/da2 of the group cost along q, from its jar-space
         gradient (-force) and Hessian */
      int dim = group_dim(P->type, r, P->nefc), zone;
      double yy[6], f[6], H[36];
      for (int j = 0; j < dim; j++) yy[j] = y[r + j] + a * q[r + j];
      cone_eval(dim, &P->D[r], &P->floss[r], yy, f, &zone, H);
      for (int i = 0; i < dim; i++) {
        g1 -= q[r + i] * f[i];
        for (int j = 0; j < dim; j++) g2 += q[r + i] * H[i * dim + j] * q[r + j];
      }
      continue;
    }
    double yr = y[r] + a * q[r];
    double f = row_force(P->type[r], P->D[r], P->floss[r], yr);
    g1 -= q[r] * f;
    if (row_quadratic(P->type[r], P->D[r], P->floss[r], yr)) g2 += P->D[r] * q[r] * q[r];
  }
  *d1 = g1;
  *d2 = g2;
}

/* exact minimiser of the piecewise-quadratic cost along p (safeguarded Newton
 * on the monotone derivative); returns alpha and the cost change */
static double linesearch(const Prob* P, const double* y, const double* q, double A, double B, int maxit, double* dcost) {
  double d0, h0;
  ls_deriv(P, A, B, y, q, 0, &d0, &h0);
  *dcost = 0;
  if (!(d0 < 0)) return 0;
  double lo = 0, dlo = d0, hi = -1, dhi = 0;
  double a = -d0 / h0;
  for (int it = 0; it < maxit; it++) {
    double dd, hh;
    ls_deriv(P, A, B, y, q, a, &dd, &hh);
    if (dd < 0) { lo = a; dlo = dd; } else { hi = a; dhi = dd; }
    if (fabs(dd) <= 1e-10 * fabs(d0)) break;
    double an = a - dd / hh;
    if (hi >= 0 && !(an > lo && an < hi)) {
      an = (dlo * hi - dhi * lo) / (dlo - dhi);
      if (!(an > lo && an < hi)) an = 0.5 * (lo + hi);
    }
    if (fabs(an - a) <= 1e-12 * fabs(a)) { a = an; break; }
    a = an;
  }
  double dc = 0.5 * a * a * A + a * B;
  for (int r = 0; r < P->nefc; r++) {
    if (P->type[r] == T_ELLFRIC) continue;
    if (P->type[r] == T_ELLIPTIC) {
      int dim = group_dim(P->type, r, P->nefc), zone;
      double yy[6], f[6];
      for (int j = 0; j < dim; j++) yy[j] = y[r + j] + a * q[r + j];
      dc += cone_eval(dim, &P->D[r], &P->floss[r], yy, f, &zone, NULL) - cone_eval(dim, &P->D[r], &P->floss[r], &y[r], f, &zone, NULL);
      continue;
    }
    dc += row_cost_delta(P->type[r], P->D[r], P->floss[r], y[r], a * q[r]);
  }
  *dcost = dc;
  return a;
}

void oracle_solve(const OModel* m, OData* d, int max_iter) {
  int nv = m->nv, ne = d->nefc;
  Prob P = {nv, ne, d->M, d->qfrc_smooth, d->qacc_smooth, d->efc_J, d->efc_aref, d->efc_D, d->efc_floss, d->efc_type};
  double* w = d->work;
  double *x = w, *Ma = w + nv, *grad = w + 2 * nv, *p = w + 3 * nv, *Mp = w + 4 * nv, *xc = w + 5 * nv, *tmp = w + 6 * nv;
  double* H = w + 8 * nv;
  double* q = H + nv * nv;
  double* yc = q + d->nefc_max;
  double* fc = yc + d->nefc_max;
  double scale = 1.0 / (m->meaninertia * (nv > 1 ? nv : 1));
  /* warm start: the lowest-cost candidate of smooth / previous / predicted */
  double best;
  memcpy(x, d->qacc_smooth, nv * sizeof(double));
  best = eval_point(&P, x, d->efc_jar, d->efc_force, Ma, grad);
  d->warm_choice = 0;
  if (!(m->disableflags & (1 << 8))) {
    double c = eval_point(&P, d->qacc_warmstart, yc, fc, tmp, tmp + nv);
    if (c < best) { best = c; memcpy(x, d->qacc_warmstart, nv * sizeof(double)); d->warm_choice = 1; }
    if (d->qacc_predicted) {
      double cp = eval_point(&P, d->qacc_predicted, yc, fc, tmp, tmp + nv);
      if (cp <= best) { best = cp; memcpy(x, d->qacc_predicted, nv * sizeof(double)); d->warm_choice = 2; }
    }
  }
  double cost = eval_point(&P, x, d->efc_jar, d->efc_force, Ma, grad);
  d->cost_initial = cost;
  d->niter = 0;
  double gn = 0;
  for (int i = 0; i < nv; i++) gn += grad[i] * grad[i];
  if (ne > 0 && scale * sqrt(gn) >= m->tolerance) {
    for (int it = 0; it < max_iter; it++) {
      /* H = M + sum_quadratic D J'J */
      memcpy(H, d->M, nv * nv * sizeof(double));
      for (int r = 0; r < ne; r++) {
        if (d->efc_type[r] == T_ELLFRIC) continue;
        if (d->efc_type[r] == T_ELLIPTIC) {
          /* cone Hessian: J_c' Hc J_c over the group's rows */
          int dim = group_dim(d->efc_type, r, ne), zone;
          double f[6], Hc[36];
          cone_eval(dim, &d->efc_D[r], &d->efc_floss[r], &d->efc_jar[r], f, &zone, Hc);
          if (zone == 0) continue;
          for (int a = 0; a < dim; a++)
            for (int bb = 0; bb < dim; bb++) {
              double hab = Hc[a * dim + bb];
              if (hab == 0) continue;
              const double* Ja = &d->efc_J[(r + a) * nv];
              const double* Jb = &d->efc_J[(r + bb) * nv];
              for (int i = 0; i < nv; i++) {
                if (Ja[i] == 0) continue;
                for (int j = 0; j <= i; j++) H[i * nv + j] += Ja[i] * hab * Jb[j];
              }
            }
          continue;
        }
        if (!row_quadratic(d->efc_type[r], d->efc_D[r], d->efc_floss[r], d->efc_jar[r])) continue;
        const double* J = &d->efc_J[r * nv];
        double Dr = d->efc_D[r];
        for (int i = 0; i < nv; i++) {
          if (J[i] == 0) continue;
          for (int j = 0; j <= i; j++) H[i * nv + j] += Dr * J[i] * J[j];
        }
      }
      for (int i = 0; i < nv; i++)
        for (int j = i + 1; j < nv; j++) H[i * nv + j] = H[j * nv + i];
      o_chol(H, nv);
      for (int i = 0; i < nv; i++) p[i] = -grad[i];
      o_chol_solve(H, nv, p);
      double gp = 0;
      for (int i = 0; i < nv; i++) gp += grad[i] * p[i];
      if (!(gp < 0)) break;
      /* line search coefficients */
      double A = 0, B = 0;
      for (int i = 0; i < nv; i++) {
        double s = 0;
        for (int j = 0; j < nv; j++) s += d->M[i * nv + j] * p[j];
        Mp[i] = s;
        A += p[i] * s;
        B += p[i] * Ma[i];
      }
      for (int r = 0; r < ne; r++) q[r] = rowdot(&d->efc_J[r * nv], p, nv);
      double dcost;
      double alpha = linesearch(&P, d->efc_jar, q, A, B, m->ls_iterations, &dcost);
      d->niter++;
      if (alpha == 0) break;
      for (int i = 0; i < nv; i++) x[i] += alpha * p[i];
      cost = eval_point(&P, x, d->efc_jar, d->efc_force, Ma, grad);
      double improvement = -scale * dcost;
      gn = 0;
      for (int i = 0; i < nv; i++) gn += grad[i] * grad[i];
      if (improvement < m->tolerance || scale * sqrt(gn) < m->tolerance) break;
    }
  }
  (void)xc;
  d->cost_final = cost;
  memcpy(d->qacc, x, nv * sizeof(double));
  for (int i = 0; i < nv; i++) {
    double s = 0;
    for (int r = 0; r < ne; r++) s += d->efc_J[r * nv + i] * d->efc_force[r];
    d->qfrc_constraint[i] = s;
  }
}

void oracle_integrate(const OModel* m, OData* d) {
  int nv = m->nv;
  double h = m->timestep;
  double* acc = d->work;  /* nv */
  memcpy(acc, d->qacc, nv * sizeof(double));
  /* implicit damping: (M + h D) qacc = qfrc_smooth + qfrc_constraint */
  int implicit = 0;
  double* damp = d->work + nv;
  for (int i = 0; i < nv; i++) damp[i] = m->dof_damping[i];
  if (m->integrator == 2 || m->integrator == 3) {
    for (int a = 0; a < m->nu; a++) {
      if (!m->actuator_biastype[a] || m->actuator_trntype[a] != 0) continue;
      double gv = m->actuator_gaintype[a] ? m->actuator_gainprm[3 * a + 2] : 0;
      double bv = m->actuator_biasprm[3 * a + 2];
      if (gv != 0 || bv == 0) continue;
      double g = m->actuator_gear[a];
      damp[m->jnt_dofadr[m->actuator_trnid[a]]] += -bv * g * g;
    }
  } else if (m->disableflags & (1 << 15)) {
    for (int i = 0; i < nv; i++) damp[i] = 0;
  }
  for (int i = 0; i < nv; i++)
    if (damp[i] != 0) implicit = 1;
  if (implicit) {
    double* Md = d->work + 2 * nv;
    memcpy(Md, d->M, nv * nv * sizeof(double));
    for (int i = 0; i < nv; i++) Md[i * nv + i] += h * damp[i];
    o_chol(Md, nv);
    for (int i = 0; i < nv; i++) acc[i] = d->qfrc_smooth[i] + d->qfrc_constraint[i];
    o_chol_solve(Md, nv, acc);
  }
  for (int i = 0; i < nv; i++) d->qvel[i] += h * acc[i];
  for (int j = 0; j < m->njnt; j++) {
    int qa = m->jnt_qposadr[j], da = m->jnt_dofadr[j], t = m->jnt_type[j];
    double* q = d->qpos + qa;
    const double* v = d->qvel + da;
    if (t == 2 || t == 3) { q[0] += h * v[0]; continue; }
    const double* w = v;
    double* qq = q;
    if (t == 0) {
      for (int k = 0; k < 3; k++) q[k] += h * v[k];
      w = v + 3;
      qq = q + 3;
    }
    double wn = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    double ha = 0.5 * h * wn;
    double s = wn > 1e-12 ? sin(ha) / wn : 0.5 * h;
    double dq[4] = {cos(ha), s * w[0], s * w[1], s * w[2]};
    o_quat_mul(qq, dq, qq);
    o_quat_normalize(qq);
  }
}

static int bad(double x) { return !(fabs(x) <= 1e10); }

static void reset_env(const OModel* m, OData* d) {
  memcpy(d->qpos, m->qpos0, m->nq * sizeof(double));
  memset(d->qvel, 0, m->nv * sizeof(double));
  memset(d->qacc_warmstart, 0, m->nv * sizeof(double));
}

/* Contact wrench per body after the solve, cfrc_ext[6 nb] = (torque, force)
 * in com-based coordinates: torque about the subtree COM of the body's root.
 * Follows the reference's mjmlx_cfrc_ext aggregation
 * (src/compat/mkx_kernels/solver.hpp:906-929: per contact, geom 2's body gets
 * +F and geom 1's body -F) with MuJoCo's contact wrench (mj_contactForce /
 * mj_rnePostConstraint semantics, unverified vs MuJoCo C until
 * cross-checked) where the reference keeps only the normal force and no
 * torque: pyramidal rows decode to the normal force sum f_n = sum_k f_k and
 * per direction mu_d (f_2d - f_2d+1); elliptic rows are the normal and
 * friction forces themselves; world force F = f_n n + f_1 t1 + f_2 t2,
 * torsional / rolling torque T = f_3 n + f_4 t1 + f_5 t2; each side adds
 * (p - subtree_com[root]) x F + T to the torque. */
void oracle_cfrc_ext(const OModel* m, OData* d, const ORand* rnd) {
  memset(d->cfrc_ext, 0, 6 * m->nbody * sizeof(double));
  const double fs = rnd ? rnd->friction_scale : 1.0;
  for (int c = 0; c < d->ncon; c++) {
    const double* con = &d->contact[ORACLE_CONTACT_STRIDE * c];
    const int r = (int)con[19];
    if (r < 0) continue;
    const int pair = (int)con[13];
    const int* pi = &m->pair_int[6 * pair];
    const double* pr = &m->pair_real[16 * pair];
    const int dim = pi[4];
    double f[6] = {0, 0, 0, 0, 0, 0};
    if (d->efc_type[r] == T_ELLIPTIC) {
      for (int k = 0; k < dim; k++) f[k] = d->efc_force[r + k];
    } else if (dim == 1) {
      f[0] = d->efc_force[r];
    } else {
      for (int k = 0; k < 2 * (dim - 1); k++) f[0] += d->efc_force[r + k];
      for (int k = 0; k + 1 < dim; k++) f[1 + k] = pr[2 + k] * fs * (d->efc_force[r + 2 * k] - d->efc_force[r + 2 * k + 1]);
    }
    const double* n = con + 3;
    const double* t1 = con + 6;
    const double* t2 = con + 9;
    double F[3], T[3];
    for (int k = 0; k < 3; k++) {
      F[k] = f[0] * n[k] + f[1] * t1[k] + f[2] * t2[k];
      T[k] = f[3] * n[k] + f[4] * t1[k] + f[5] * t2[k];
    }
    for (int side = 0; side < 2; side++) {
      const int body = side == 0 ? pi[3] : pi[2];
      const double sg = side == 0 ? 1.0 : -1.0;
      const double* rc = &d->subtree_com[3 * m->body_rootid[body]];
      double off[3] = {con[0] - rc[0], con[1] - rc[1], con[2] - rc[2]}, tq[3];
      o_cross(off, F, tq);
      for (int k = 0; k < 3; k++) {
        d->cfrc_ext[6 * body + k] += sg * (tq[k] + T[k]);
        d->cfrc_ext[6 * body + 3 + k] += sg * F[k];
      }
    }
  }
}

void oracle_step(const OModel* m, OData* d, const ORand* r, int max_iter) {
  if (max_iter <= 0) max_iter = m->iterations;
  d->status = 0;
  for (int i = 0; i < m->nq; i++)
    if (bad(d->qpos[i])) { reset_env(m, d); d->status |= ORACLE_BADSTATE; break; }
  for (int i = 0; i < m->nv; i++)
    if (bad(d->qvel[i])) { reset_env(m, d); d->status |= ORACLE_BADSTATE; break; }
  oracle_kinematics(m, d);
  oracle_com(m, d, r);
  oracle_crb(m, d, r);
  oracle_rne(m, d, r);
  oracle_smooth_forces(m, d, r);
  oracle_collide(m, d);
  oracle_make_constraints(m, d, r);
  oracle_solve(m, d, max_iter);
  oracle_cfrc_ext(m, d, r);
  for (int i = 0; i < m->nv; i++)
    if (bad(d->qacc[i])) {
      reset_env(m, d);
      memset(d->qacc, 0, m->nv * sizeof(double));
      d->status |= ORACLE_BADQACC;
      return;
    }
  memcpy(d->qacc_warmstart, d->qacc, m->nv * sizeof(double));
  oracle_integrate(m, d);
}

typedef struct {
  const OModel* m;
  OData* const* d;
  int B, nsub, max_iter, tid, nthread;
} Job;

static void* worker(void* arg) {
  Job* j = (Job*)arg;
  for (int e = j->tid; e < j->B; e += j->nthread)
    for (int s = 0; s < j->nsub; s++) oracle_step(j->m, j->d[e], NULL, j->max_iter);
  return NULL;
}

void oracle_step_batch(const OModel* m, OData* const* d, int B, int nsub, int max_iter, int nthread) {
  if (nthread < 1) nthread = 1;
  if (nthread > B) nthread = B;
  pthread_t th[256];
  Job jobs[256];
  if (nthread > 256) nthread = 256;
  for (int t = 0; t < nthread; t++) {
    jobs[t] = (Job){m, d, B, nsub, max_iter, t, nthread};
    if (t > 0) pthread_create(&th[t], NULL, worker, &jobs[t]);
  }
  worker(&jobs[0]);
  for (int t = 1; t < nthread; t++) pthread_join(th[t], NULL);
}
