// MJCF -> Model compiler.
//
// Restates, for the MJCF subset used by the batched path, what the reference
// obtains from MuJoCo C at load time (src/io.cpp:563-601 mj_loadXML/mj_compile,
// src/io.cpp:255 convert_model) and its own collision-pair cache
// (src/io.cpp:913-1165 Model::init_cache).  Conventions are MuJoCo's:
// quaternions (w,x,y,z), geom size triples, qpos0 from the body frames,
// compiler angle unit "degree" unless <compiler angle="radian">, autolimits.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <stdexcept>

#include "hull.h"
#include "model.h"
#include "tendon_wrap.h"
#include "xml.h"

namespace mjb {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kMinVal = 1e-15;

[[noreturn]] void fail(const std::string& msg) { throw std::runtime_error("MJCF compile error: " + msg); }

std::vector<double> parse_nums(const std::string& s, const std::string& what) {
  std::vector<double> v;
  const char* p = s.c_str();
  char* end = nullptr;
  for (;;) {
    while (*p && (std::isspace(static_cast<unsigned char>(*p)) || *p == ',')) p++;
    if (!*p) break;
    double x = std::strtod(p, &end);
    if (end == p) fail("bad number list for '" + what + "': " + s);
    v.push_back(x);
    p = end;
  }
  return v;
}

// ---------------------------------------------------------------- math
void quat_mul(const double a[4], const double b[4], double r[4]) {
  double t[4] = {a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3], a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2],
                 a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1], a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0]};
  std::memcpy(r, t, sizeof(t));
}
void quat_normalize(double q[4]) {
  double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (n < kMinVal) { q[0] = 1; q[1] = q[2] = q[3] = 0; return; }
  for (int k = 0; k < 4; k++) q[k] /= n;
}
void quat_rot(const double q[4], const double v[3], double r[3]) {
  double w = q[0], x = q[1], y = q[2], z = q[3];
  double t0 = 2 * (x * v[0] + y * v[1] + z * v[2]);
  double t1 = w * w - (x * x + y * y + z * z);
  double o[3] = {t1 * v[0] + t0 * x + 2 * w * (y * v[2] - z * v[1]), t1 * v[1] + t0 * y + 2 * w * (z * v[0] - x * v[2]),
                 t1 * v[2] + t0 * z + 2 * w * (x * v[1] - y * v[0])};
  std::memcpy(r, o, sizeof(o));
}
void quat2mat(const double q[4], double m[9]) {
  double w = q[0], x = q[1], y = q[2], z = q[3];
  m[0] = 1 - 2 * (y * y + z * z); m[1] = 2 * (x * y - w * z); m[2] = 2 * (x * z + w * y);
  m[3] = 2 * (x * y + w * z); m[4] = 1 - 2 * (x * x + z * z); m[5] = 2 * (y * z - w * x);
  m[6] = 2 * (x * z - w * y); m[7] = 2 * (y * z + w * x); m[8] = 1 - 2 * (x * x + y * y);
}
// Rotation matrix (columns = frame axes) to quaternion (Shepperd's method).
void mat2quat(const double m[9], double q[4]) {
  double tr = m[0] + m[4] + m[8];
  if (tr > 0) {
    double s = std::sqrt(tr + 1.0) * 2;
    q[0] = 0.25 * s; q[1] = (m[7] - m[5]) / s; q[2] = (m[2] - m[6]) / s; q[3] = (m[3] - m[1]) / s;
  } else if (m[0] > m[4] && m[0] > m[8]) {
    double s = std::sqrt(1.0 + m[0] - m[4] - m[8]) * 2;
    q[0] = (m[7] - m[5]) / s; q[1] = 0.25 * s; q[2] = (m[1] + m[3]) / s; q[3] = (m[2] + m[6]) / s;
  } else if (m[4] > m[8]) {
    double s = std::sqrt(1.0 + m[4] - m[0] - m[8]) * 2;
    q[0] = (m[2] - m[6]) / s; q[1] = (m[1] + m[3]) / s; q[2] = 0.25 * s; q[3] = (m[5] + m[7]) / s;
  } else {
    double s = std::sqrt(1.0 + m[8] - m[0] - m[4]) * 2;
    q[0] = (m[3] - m[1]) / s; q[1] = (m[2] + m[6]) / s; q[2] = (m[5] + m[7]) / s; q[3] = 0.25 * s;
  }
  if (q[0] < 0) for (int k = 0; k < 4; k++) q[k] = -q[k];
  quat_normalize(q);
}
void axisangle2quat(const double ax[3], double ang, double q[4]) {
  double n = std::sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]);
  if (n < kMinVal) fail("zero-length rotation axis");
  double s = std::sin(ang / 2) / n;
  q[0] = std::cos(ang / 2); q[1] = ax[0] * s; q[2] = ax[1] * s; q[3] = ax[2] * s;
}
// Minimal rotation taking +z to direction v.
void z2vec_quat(const double v[3], double q[4]) {
  double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if (n < kMinVal) fail("fromto with coincident end points");
  double d[3] = {v[0] / n, v[1] / n, v[2] / n};
  double c = d[2];  // dot(z, d)
  double ax[3] = {-d[1], d[0], 0};  // z x d
  double s = std::sqrt(ax[0] * ax[0] + ax[1] * ax[1]);
  if (s < 1e-12) {
    if (c > 0) { q[0] = 1; q[1] = q[2] = q[3] = 0; }
    else { q[0] = 0; q[1] = 1; q[2] = q[3] = 0; }
    return;
  }
  double ang = std::atan2(s, c);
  axisangle2quat(ax, ang, q);
}
// Symmetric 3x3 eigen-decomposition by cyclic Jacobi; columns of V are
// eigenvectors; eigenvalues sorted in decreasing order (MuJoCo orders the
// principal moments the same way).
void eig3(const double A[9], double w[3], double V[9]) {
  double a[9];
  std::memcpy(a, A, sizeof(a));
  double v[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int sweep = 0; sweep < 50; sweep++) {
    double off = a[1] * a[1] + a[2] * a[2] + a[5] * a[5];
    if (off < 1e-30) break;
    for (int p = 0; p < 2; p++)
      for (int q = p + 1; q < 3; q++) {
        double apq = a[p * 3 + q];
        if (std::fabs(apq) < 1e-300) continue;
        double theta = (a[q * 3 + q] - a[p * 3 + p]) / (2 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < 3; k++) {  // A = J^T A J
          double akp = a[k * 3 + p], akq = a[k * 3 + q];
          a[k * 3 + p] = c * akp - s * akq;
          a[k * 3 + q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; k++) {
          double apk = a[p * 3 + k], aqk = a[q * 3 + k];
          a[p * 3 + k] = c * apk - s * aqk;
          a[q * 3 + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; k++) {
          double vkp = v[k * 3 + p], vkq = v[k * 3 + q];
          v[k * 3 + p] = c * vkp - s * vkq;
          v[k * 3 + q] = s * vkp + c * vkq;
        }
      }
  }
  int idx[3] = {0, 1, 2};
  double ev[3] = {a[0], a[4], a[8]};
  std::sort(idx, idx + 3, [&](int i, int j) { return ev[i] > ev[j]; });
  for (int c = 0; c < 3; c++) {
    w[c] = ev[idx[c]];
    for (int r = 0; r < 3; r++) V[r * 3 + c] = v[r * 3 + idx[c]];
  }
  // right-handed frame
  double det = V[0] * (V[4] * V[8] - V[5] * V[7]) - V[1] * (V[3] * V[8] - V[5] * V[6]) + V[2] * (V[3] * V[7] - V[4] * V[6]);
  if (det < 0)
    for (int r = 0; r < 3; r++) V[r * 3 + 2] = -V[r * 3 + 2];
}

// ---------------------------------------------------------------- defaults
struct DefaultClass {
  std::string name;
  int parent = -1;
  std::map<std::string, std::map<std::string, std::string>> elems;  // tag -> attrs
};

struct Compiler {
  Model m;
  LoadOptions opt;
  std::string base_dir;
  bool degrees = true;
  bool autolimits = true;
  std::string inertiafromgeom = "auto";
  std::vector<DefaultClass> classes;
  std::map<std::string, int> class_index;

  // per-geom bookkeeping for inertia and mesh references
  std::vector<std::string> geom_meshname;
  struct MeshAsset {
    std::string name;
    std::vector<double> verts;  // raw vertices
    double scale[3] = {1, 1, 1};
  };
  std::vector<MeshAsset> mesh_assets;
  struct MeshProps {
    std::vector<double> hull;  // hull vertices in mesh frame (after centring/alignment)
    double volume = 0;
    double inertia_unit[3] = {0, 0, 0};  // principal inertia per unit density
    double pos[3] = {0, 0, 0}, quat[4] = {1, 0, 0, 0};  // hull frame in the mesh asset frame
  };
  std::vector<MeshProps> mesh_props;

  // pending actuator / contact references resolved after the body pass
  struct PendingActuator {
    std::map<std::string, std::string> a;
    std::string kind;
  };
  std::vector<PendingActuator> pending_act;

  // attribute lookup: element attribute, else class default
  std::string get(const XmlNode& n, const char* key, const std::string& cls, const char* def_tag = nullptr) const {
    if (auto v = n.attr(key)) return *v;
    std::string tag = def_tag ? def_tag : n.tag;
    int ci = class_of(n, cls);
    auto it = classes[ci].elems.find(tag);
    if (it != classes[ci].elems.end()) {
      auto jt = it->second.find(key);
      if (jt != it->second.end()) return jt->second;
    }
    return std::string();
  }
  int class_of(const XmlNode& n, const std::string& cls) const {
    std::string c = cls;
    if (auto v = n.attr("class")) c = *v;
    if (c.empty()) return 0;
    auto it = class_index.find(c);
    if (it == class_index.end()) fail("unknown default class '" + c + "'");
    return it->second;
  }
  bool has(const XmlNode& n, const char* key, const std::string& cls, const char* def_tag = nullptr) const {
    return !get(n, key, cls, def_tag).empty();
  }
  double num(const XmlNode& n, const char* key, const std::string& cls, double def, const char* def_tag = nullptr) const {
    std::string s = get(n, key, cls, def_tag);
    if (s.empty()) return def;
    auto v = parse_nums(s, key);
    if (v.size() != 1) fail(std::string("attribute '") + key + "' expects one number");
    return v[0];
  }
  std::vector<double> nums(const XmlNode& n, const char* key, const std::string& cls, std::vector<double> def, const char* def_tag = nullptr) const {
    std::string s = get(n, key, cls, def_tag);
    if (s.empty()) return def;
    return parse_nums(s, key);
  }

  void parse_defaults(const XmlNode& d, int parent) {
    DefaultClass c;
    c.parent = parent;
    if (parent < 0) c.name = "main";
    else {
      auto v = d.attr("class");
      if (!v) fail("nested <default> needs a class attribute");
      c.name = *v;
      c.elems = classes[parent].elems;
    }
    for (auto& ch : d.children) {
      if (ch.tag == "default") continue;
      auto& dst = c.elems[ch.tag];
      for (auto& kv : ch.attrs) dst[kv.first] = kv.second;
    }
    int idx = (int)classes.size();
    if (class_index.count(c.name)) fail("duplicate default class '" + c.name + "'");
    class_index[c.name] = idx;
    classes.push_back(c);
    for (auto& ch : d.children)
      if (ch.tag == "default") parse_defaults(ch, idx);
  }

  // frame from pos + one of quat / euler / axisangle / zaxis
  void read_frame(const XmlNode& n, const std::string& cls, double pos[3], double quat[4], const char* def_tag = nullptr) {
    auto p = nums(n, "pos", cls, {0, 0, 0}, def_tag);
    if (p.size() != 3) fail("pos needs 3 numbers");
    for (int k = 0; k < 3; k++) pos[k] = p[k];
    quat[0] = 1; quat[1] = quat[2] = quat[3] = 0;
    if (n.attr("quat")) {
      auto q = parse_nums(*n.attr("quat"), "quat");
      if (q.size() != 4) fail("quat needs 4 numbers");
      for (int k = 0; k < 4; k++) quat[k] = q[k];
      quat_normalize(quat);
    } else if (n.attr("euler")) {
      auto e = parse_nums(*n.attr("euler"), "euler");
      if (e.size() != 3) fail("euler needs 3 numbers");
      double s = degrees ? kPi / 180 : 1;
      double q[4] = {1, 0, 0, 0};
      const double axes[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
      for (int k = 0; k < 3; k++) {  // intrinsic x-y-z (MuJoCo default eulerseq)
        double r[4];
        axisangle2quat(axes[k], e[k] * s, r);
        quat_mul(q, r, q);
      }
      std::memcpy(quat, q, sizeof(q));
    } else if (n.attr("axisangle")) {
      auto a = parse_nums(*n.attr("axisangle"), "axisangle");
      if (a.size() != 4) fail("axisangle needs 4 numbers");
      axisangle2quat(a.data(), a[3] * (degrees ? kPi / 180 : 1), quat);
    } else if (n.attr("zaxis")) {
      auto z = parse_nums(*n.attr("zaxis"), "zaxis");
      if (z.size() != 3) fail("zaxis needs 3 numbers");
      z2vec_quat(z.data(), quat);
    }
  }

  // ------------------------------------------------------------ bodies
  struct BodyInertiaAcc {
    bool explicit_inertial = false;
    double mass = 0;
    double com[3] = {0, 0, 0};
    double I[9] = {0};  // about body origin, body frame
    std::vector<std::array<double, 16>> geom_parts;  // mass, pos(3), R(9), diag(3)
  };
  std::vector<BodyInertiaAcc> inert;

  int add_body(const std::string& name, int parent) {
    int id = m.nbody++;
    m.body_name.push_back(name);
    m.body_parentid.push_back(parent);
    m.body_jntnum.push_back(0);
    m.body_jntadr.push_back(-1);
    m.body_dofnum.push_back(0);
    m.body_dofadr.push_back(-1);
    for (int k = 0; k < 3; k++) m.body_pos.push_back(0);
    m.body_quat.insert(m.body_quat.end(), {1, 0, 0, 0});
    for (int k = 0; k < 3; k++) m.body_ipos.push_back(0);
    m.body_iquat.insert(m.body_iquat.end(), {1, 0, 0, 0});
    m.body_mass.push_back(0);
    for (int k = 0; k < 3; k++) m.body_inertia.push_back(0);
    m.body_gravcomp.push_back(0);
    inert.emplace_back();
    return id;
  }

  void add_joint(const XmlNode& n, const std::string& cls, int body, bool is_free) {
    int type = JNT_HINGE;
    if (is_free) type = JNT_FREE;
    else {
      std::string t = get(n, "type", cls);
      if (t.empty() || t == "hinge") type = JNT_HINGE;
      else if (t == "slide") type = JNT_SLIDE;
      else if (t == "ball") type = JNT_BALL;
      else if (t == "free") type = JNT_FREE;
      else fail("unknown joint type '" + t + "'");
    }
    if (type == JNT_FREE && m.body_parentid[body] != 0) fail("free joint allowed only in top-level bodies");
    int j = m.njnt++;
    auto nm = n.attr("name");
    m.jnt_name.push_back(nm ? *nm : std::string());
    m.jnt_type.push_back(type);
    m.jnt_bodyid.push_back(body);
    m.jnt_qposadr.push_back(m.nq);
    m.jnt_dofadr.push_back(m.nv);
    auto pos = is_free ? std::vector<double>{0, 0, 0} : nums(n, "pos", cls, {0, 0, 0}, "joint");
    auto axis = is_free ? std::vector<double>{0, 0, 1} : nums(n, "axis", cls, {0, 0, 1}, "joint");
    if (pos.size() != 3 || axis.size() != 3) fail("joint pos/axis need 3 numbers");
    double an = std::sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
    if (an < kMinVal) fail("joint axis has zero length");
    for (int k = 0; k < 3; k++) { m.jnt_pos.push_back(pos[k]); m.jnt_axis.push_back(axis[k] / an); }
    auto range = is_free ? std::vector<double>{0, 0} : nums(n, "range", cls, {0, 0}, "joint");
    if (range.size() != 2) fail("joint range needs 2 numbers");
    std::string lim = is_free ? std::string("false") : get(n, "limited", cls, "joint");
    int limited = 0;
    if (lim == "true") limited = 1;
    else if (lim == "false") limited = 0;
    else if (lim.empty() || lim == "auto") limited = (autolimits && !is_free && n.attr("range") != nullptr) || (autolimits && !is_free && has(n, "range", cls, "joint"));
    else fail("bad joint limited value '" + lim + "'");
    if (limited && range[0] >= range[1] && type != JNT_BALL) fail("joint range must satisfy lo < hi");
    double rs = (degrees && (type == JNT_HINGE || type == JNT_BALL)) ? kPi / 180 : 1;
    m.jnt_limited.push_back(limited);
    m.jnt_range.push_back(range[0] * rs);
    m.jnt_range.push_back(range[1] * rs);
    m.jnt_margin.push_back(is_free ? 0 : num(n, "margin", cls, 0, "joint"));
    auto sr = is_free ? std::vector<double>{0.02, 1} : nums(n, "solreflimit", cls, {0.02, 1}, "joint");
    auto si = is_free ? std::vector<double>{0.9, 0.95, 0.001, 0.5, 2} : nums(n, "solimplimit", cls, {0.9, 0.95, 0.001, 0.5, 2}, "joint");
    if (sr.size() != 2 || si.size() < 3) fail("bad solreflimit/solimplimit");
    while (si.size() < 5) si.push_back(si.size() == 3 ? 0.5 : 2);
    m.jnt_solref.insert(m.jnt_solref.end(), sr.begin(), sr.end());
    m.jnt_solimp.insert(m.jnt_solimp.end(), si.begin(), si.begin() + 5);
    double stiff = is_free ? 0 : num(n, "stiffness", cls, 0, "joint");
    m.jnt_stiffness.push_back(stiff);
    double ref = is_free ? 0 : num(n, "ref", cls, 0, "joint") * ((type == JNT_HINGE && degrees) ? kPi / 180 : 1);
    double springref = is_free ? 0 : num(n, "springref", cls, 0, "joint") * ((type == JNT_HINGE && degrees) ? kPi / 180 : 1);

    int ndof = type == JNT_FREE ? 6 : type == JNT_BALL ? 3 : 1;
    int nqj = type == JNT_FREE ? 7 : type == JNT_BALL ? 4 : 1;
    double arm = is_free ? 0 : num(n, "armature", cls, 0, "joint");
    double damp = is_free ? 0 : num(n, "damping", cls, 0, "joint");
    double floss = is_free ? 0 : num(n, "frictionloss", cls, 0, "joint");
    auto srf = is_free ? std::vector<double>{0.02, 1} : nums(n, "solreffriction", cls, {0.02, 1}, "joint");
    auto sif = is_free ? std::vector<double>{0.9, 0.95, 0.001, 0.5, 2} : nums(n, "solimpfriction", cls, {0.9, 0.95, 0.001, 0.5, 2}, "joint");
    while (sif.size() < 5) sif.push_back(sif.size() == 3 ? 0.5 : 2);
    for (int d = 0; d < ndof; d++) {
      m.dof_bodyid.push_back(body);
      m.dof_jntid.push_back(j);
      m.dof_armature.push_back(arm);
      m.dof_damping.push_back(damp);
      m.dof_frictionloss.push_back(floss);
      m.dof_solref.insert(m.dof_solref.end(), srf.begin(), srf.begin() + 2);
      m.dof_solimp.insert(m.dof_solimp.end(), sif.begin(), sif.begin() + 5);
    }
    // qpos0 / qpos_spring
    if (type == JNT_FREE) {
      const double* bp = &m.body_pos[3 * body];
      const double* bq = &m.body_quat[4 * body];
      for (int k = 0; k < 3; k++) m.qpos0.push_back(bp[k]);
      for (int k = 0; k < 4; k++) m.qpos0.push_back(bq[k]);
      for (int k = 0; k < 3; k++) m.qpos_spring.push_back(bp[k]);
      for (int k = 0; k < 4; k++) m.qpos_spring.push_back(bq[k]);
    } else if (type == JNT_BALL) {
      m.qpos0.insert(m.qpos0.end(), {1, 0, 0, 0});
      m.qpos_spring.insert(m.qpos_spring.end(), {1, 0, 0, 0});
    } else {
      m.qpos0.push_back(ref);
      m.qpos_spring.push_back(springref);
    }
    if (m.body_jntnum[body] == 0) m.body_jntadr[body] = j;
    m.body_jntnum[body]++;
    if (m.body_dofnum[body] == 0) m.body_dofadr[body] = m.nv;
    m.body_dofnum[body] += ndof;
    m.nq += nqj;
    m.nv += ndof;
  }

  // Geom volume and principal inertia per unit mass in the geom frame.
  void geom_mass_props(int type, const double* size, int mesh, double& volume, double I_unit[3], double& caps_cyl_frac) const {
    caps_cyl_frac = 0;
    double r = size[0];
    switch (type) {
      case GEOM_SPHERE:
        volume = 4.0 / 3.0 * kPi * r * r * r;
        I_unit[0] = I_unit[1] = I_unit[2] = 0.4 * r * r;
        break;
      case GEOM_CAPSULE: {
        double h = size[1];
        double vc = kPi * r * r * 2 * h, vs = 4.0 / 3.0 * kPi * r * r * r;
        volume = vc + vs;
        double fc = vc / volume, fs = vs / volume;
        caps_cyl_frac = fc;
        I_unit[2] = fc * r * r / 2 + fs * 0.4 * r * r;
        I_unit[0] = I_unit[1] = fc * (r * r / 4 + (2 * h) * (2 * h) / 12) + fs * (0.4 * r * r + h * h + 0.75 * h * r);
        break;
      }
      case GEOM_CYLINDER: {
        double h = size[1];
        volume = kPi * r * r * 2 * h;
        I_unit[2] = r * r / 2;
        I_unit[0] = I_unit[1] = (3 * r * r + 4 * h * h) / 12;
        break;
      }
      case GEOM_BOX: {
        double a = size[0], b = size[1], c = size[2];
        volume = 8 * a * b * c;
        I_unit[0] = (b * b + c * c) / 3;
        I_unit[1] = (a * a + c * c) / 3;
        I_unit[2] = (a * a + b * b) / 3;
        break;
      }
      case GEOM_ELLIPSOID: {
        double a = size[0], b = size[1], c = size[2];
        volume = 4.0 / 3.0 * kPi * a * b * c;
        I_unit[0] = (b * b + c * c) / 5;
        I_unit[1] = (a * a + c * c) / 5;
        I_unit[2] = (a * a + b * b) / 5;
        break;
      }
      case GEOM_MESH: {
        const MeshProps& mp = mesh_props[mesh];
        volume = mp.volume;
        for (int k = 0; k < 3; k++) I_unit[k] = mp.volume > 0 ? mp.inertia_unit[k] / mp.volume : 0;
        break;
      }
      default:
        volume = 0;
        I_unit[0] = I_unit[1] = I_unit[2] = 0;
    }
  }

  void add_geom(const XmlNode& n, const std::string& cls, int body) {
    m.ngeom++;
    auto nm = n.attr("name");
    m.geom_name.push_back(nm ? *nm : std::string());
    std::string t = get(n, "type", cls, "geom");
    int type;
    if (t.empty() || t == "sphere") type = GEOM_SPHERE;
    else if (t == "plane") type = GEOM_PLANE;
    else if (t == "capsule") type = GEOM_CAPSULE;
    else if (t == "ellipsoid") type = GEOM_ELLIPSOID;
    else if (t == "cylinder") type = GEOM_CYLINDER;
    else if (t == "box") type = GEOM_BOX;
    else if (t == "mesh") type = GEOM_MESH;
    else fail("unsupported geom type '" + t + "'");
    m.geom_type.push_back(type);
    m.geom_bodyid.push_back(body);
    double pos[3], quat[4];
    read_frame(n, cls, pos, quat, "geom");
    auto size = nums(n, "size", cls, {}, "geom");
    double sz[3] = {0, 0, 0};
    for (size_t k = 0; k < size.size() && k < 3; k++) sz[k] = size[k];
    std::string ft = get(n, "fromto", cls, "geom");
    if (!ft.empty()) {
      auto f = parse_nums(ft, "fromto");
      if (f.size() != 6) fail("fromto needs 6 numbers");
      if (type != GEOM_CAPSULE && type != GEOM_CYLINDER) fail("fromto is supported for capsule and cylinder geoms");
      double d[3] = {f[3] - f[0], f[4] - f[1], f[5] - f[2]};
      for (int k = 0; k < 3; k++) pos[k] = 0.5 * (f[k] + f[k + 3]);
      z2vec_quat(d, quat);
      sz[1] = 0.5 * std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    }
    int mesh = -1;
    if (type == GEOM_MESH) {
      std::string mn = get(n, "mesh", cls, "geom");
      for (size_t k = 0; k < mesh_assets.size(); k++)
        if (mesh_assets[k].name == mn) mesh = (int)k;
      if (mesh < 0) fail("geom references unknown mesh '" + mn + "'");
      // the hull frame is centred/aligned; fold it into the geom frame
      const MeshProps& mp = mesh_props[mesh];
      double rp[3];
      quat_rot(quat, mp.pos, rp);
      for (int k = 0; k < 3; k++) pos[k] += rp[k];
      quat_mul(quat, mp.quat, quat);
    } else {
      int need = type == GEOM_SPHERE ? 1 : (type == GEOM_CAPSULE || type == GEOM_CYLINDER) ? 2 : type == GEOM_PLANE ? 0 : 3;
      if ((int)size.size() < need && ft.empty()) fail("geom '" + m.geom_name.back() + "' needs " + std::to_string(need) + " size values");
      if (type == GEOM_CAPSULE || type == GEOM_CYLINDER) {
        if (!ft.empty() && size.size() < 1) fail("capsule/cylinder fromto needs size radius");
      }
    }
    m.geom_dataid.push_back(mesh);
    for (int k = 0; k < 3; k++) { m.geom_pos.push_back(pos[k]); m.geom_size.push_back(sz[k]); }
    for (int k = 0; k < 4; k++) m.geom_quat.push_back(quat[k]);
    m.geom_contype.push_back((int)num(n, "contype", cls, 1, "geom"));
    m.geom_conaffinity.push_back((int)num(n, "conaffinity", cls, 1, "geom"));
    m.geom_condim.push_back((int)num(n, "condim", cls, 3, "geom"));
    m.geom_priority.push_back((int)num(n, "priority", cls, 0, "geom"));
    m.geom_group.push_back((int)num(n, "group", cls, 0, "geom"));
    auto fr = nums(n, "friction", cls, {1, 0.005, 0.0001}, "geom");
    while (fr.size() < 3) fr.push_back(fr.size() == 1 ? 0.005 : 0.0001);
    m.geom_friction.insert(m.geom_friction.end(), fr.begin(), fr.begin() + 3);
    auto sr = nums(n, "solref", cls, {0.02, 1}, "geom");
    if (sr.size() != 2) fail("geom solref needs 2 numbers");
    m.geom_solref.insert(m.geom_solref.end(), sr.begin(), sr.end());
    auto si = nums(n, "solimp", cls, {0.9, 0.95, 0.001, 0.5, 2}, "geom");
    while (si.size() < 5) si.push_back(si.size() == 3 ? 0.5 : 2);
    m.geom_solimp.insert(m.geom_solimp.end(), si.begin(), si.begin() + 5);
    m.geom_solmix.push_back(num(n, "solmix", cls, 1, "geom"));
    m.geom_margin.push_back(num(n, "margin", cls, 0, "geom"));
    m.geom_gap.push_back(num(n, "gap", cls, 0, "geom"));
    m.geom_rbound.push_back(0);

    // mass contribution to the body
    double gmass = 0;
    if (type != GEOM_PLANE && inertiafromgeom != "false") {
      double vol, Iu[3], fc;
      geom_mass_props(type, sz, mesh, vol, Iu, fc);
      if (has(n, "mass", cls, "geom")) gmass = num(n, "mass", cls, 0, "geom");
      else gmass = num(n, "density", cls, 1000, "geom") * vol;
      if (gmass > 0) {
        std::array<double, 16> part{};
        part[0] = gmass;
        for (int k = 0; k < 3; k++) part[1 + k] = pos[k];
        double R[9];
        quat2mat(quat, R);
        for (int k = 0; k < 9; k++) part[4 + k] = R[k];
        for (int k = 0; k < 3; k++) part[13 + k] = gmass * Iu[k];
        inert[body].geom_parts.push_back(part);
      }
    }
    m.geom_mass.push_back(gmass);
  }

  void add_site(const XmlNode& n, const std::string& cls, int body) {
    m.nsite++;
    auto nm = n.attr("name");
    m.site_name.push_back(nm ? *nm : std::string());
    m.site_bodyid.push_back(body);
    double pos[3], quat[4];
    read_frame(n, cls, pos, quat, "site");
    m.site_pos.insert(m.site_pos.end(), pos, pos + 3);
    m.site_quat.insert(m.site_quat.end(), quat, quat + 4);
  }

  void parse_body(const XmlNode& n, int parent, const std::string& childclass) {
    std::string cls = childclass;
    if (auto v = n.attr("childclass")) cls = *v;
    auto nm = n.attr("name");
    int b = add_body(nm ? *nm : std::string(), parent);
    double pos[3], quat[4];
    read_frame(n, std::string(), pos, quat, "body");
    for (int k = 0; k < 3; k++) m.body_pos[3 * b + k] = pos[k];
    for (int k = 0; k < 4; k++) m.body_quat[4 * b + k] = quat[k];
    if (auto gc = n.attr("gravcomp")) m.body_gravcomp[b] = parse_nums(*gc, "gravcomp").at(0);
    // element order inside a body: joints first in document order, then the
    // rest; MuJoCo assigns dofs in joint order, which is document order.
    for (auto& ch : n.children) {
      if (ch.tag == "joint") add_joint(ch, cls, b, false);
      else if (ch.tag == "freejoint") add_joint(ch, cls, b, true);
    }
    for (auto& ch : n.children) {
      if (ch.tag == "inertial") {
        auto& acc = inert[b];
        acc.explicit_inertial = true;
        double ip[3], iq[4];
        read_frame(ch, std::string(), ip, iq, "inertial");
        double mass = parse_nums(ch.attr("mass") ? *ch.attr("mass") : "0", "mass").at(0);
        double I[3];
        if (ch.attr("diaginertia")) {
          auto d = parse_nums(*ch.attr("diaginertia"), "diaginertia");
          if (d.size() != 3) fail("diaginertia needs 3 numbers");
          for (int k = 0; k < 3; k++) I[k] = d[k];
        } else if (ch.attr("fullinertia")) {
          auto f = parse_nums(*ch.attr("fullinertia"), "fullinertia");
          if (f.size() != 6) fail("fullinertia needs 6 numbers");
          double A[9] = {f[0], f[3], f[4], f[3], f[1], f[5], f[4], f[5], f[2]}, V[9];
          eig3(A, I, V);
          double R[9], Rq[9], q2[4];
          mat2quat(V, q2);
          quat_mul(iq, q2, iq);
          (void)R; (void)Rq;
        } else fail("inertial needs diaginertia or fullinertia");
        acc.mass = mass;
        for (int k = 0; k < 3; k++) {
          m.body_ipos[3 * b + k] = ip[k];
          m.body_inertia[3 * b + k] = I[k];
        }
        for (int k = 0; k < 4; k++) m.body_iquat[4 * b + k] = iq[k];
        m.body_mass[b] = mass;
      } else if (ch.tag == "geom") {
        add_geom(ch, cls, b);
      } else if (ch.tag == "body") {
        parse_body(ch, b, cls);
      } else if (ch.tag == "site") {
        add_site(ch, cls, b);
      } else if (ch.tag == "joint" || ch.tag == "freejoint" || ch.tag == "camera" || ch.tag == "light") {
        // joints handled above; cameras/lights are not used by the step
      } else {
        fail("unsupported element <" + ch.tag + "> inside <body> (line " + std::to_string(ch.line) + ")");
      }
    }
  }

  void finish_inertia() {
    for (int b = 1; b < m.nbody; b++) {
      auto& acc = inert[b];
      bool use_geoms = inertiafromgeom == "true" || (inertiafromgeom == "auto" && !acc.explicit_inertial);
      if (!use_geoms) continue;
      double M = 0, com[3] = {0, 0, 0};
      for (auto& p : acc.geom_parts) {
        M += p[0];
        for (int k = 0; k < 3; k++) com[k] += p[0] * p[1 + k];
      }
      if (M < kMinVal) {
        m.body_mass[b] = 0;
        continue;
      }
      for (int k = 0; k < 3; k++) com[k] /= M;
      double I[9] = {0};
      for (auto& p : acc.geom_parts) {
        const double* R = &p[4];
        const double* Id = &p[13];
        // R diag(Id) R^T
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) {
            double s = 0;
            for (int k = 0; k < 3; k++) s += R[r * 3 + k] * Id[k] * R[c * 3 + k];
            I[r * 3 + c] += s;
          }
        double d[3] = {p[1] - com[0], p[2] - com[1], p[3] - com[2]};
        double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) I[r * 3 + c] += p[0] * ((r == c ? d2 : 0) - d[r] * d[c]);
      }
      double w[3], V[9], q[4];
      eig3(I, w, V);
      mat2quat(V, q);
      m.body_mass[b] = M;
      for (int k = 0; k < 3; k++) {
        m.body_ipos[3 * b + k] = com[k];
        m.body_inertia[3 * b + k] = std::max(w[k], 0.0);
      }
      for (int k = 0; k < 4; k++) m.body_iquat[4 * b + k] = q[k];
    }
  }

  void parse_actuator(const XmlNode& n) {
    for (auto& a : n.children) {
      std::string cls;
      std::string kind = a.tag;
      if (kind != "position" && kind != "motor" && kind != "velocity" && kind != "general")
        fail("unsupported actuator <" + kind + ">");
      m.nu++;
      auto nm = a.attr("name");
      m.actuator_name.push_back(nm ? *nm : std::string());
      std::string jn = get(a, "joint", cls), tn = get(a, "tendon", cls);
      if (jn.empty() == tn.empty()) fail("actuator needs exactly one transmission: joint= or tendon=");
      if (!tn.empty()) {
        m.actuator_trntype.push_back(3);
        m.actuator_trnid.push_back(tendon_by_name(tn));
      } else {
        int jid = -1;
        for (int j = 0; j < m.njnt; j++)
          if (m.jnt_name[j] == jn) jid = j;
        if (jid < 0) fail("actuator references unknown joint '" + jn + "'");
        if (m.jnt_type[jid] != JNT_HINGE && m.jnt_type[jid] != JNT_SLIDE) fail("actuator transmission must be a hinge or slide joint");
        m.actuator_trntype.push_back(0);
        m.actuator_trnid.push_back(jid);
      }
      auto gear = nums(a, "gear", cls, {1});
      m.actuator_gear.push_back(gear.at(0));
      double g[3] = {0, 0, 0}, bsp[3] = {0, 0, 0};
      int gaintype = 0, biastype = 0;
      if (kind == "position") {
        double kp = num(a, "kp", cls, 1), kv = num(a, "kv", cls, 0);
        g[0] = kp; bsp[1] = -kp; bsp[2] = -kv; biastype = 1;
      } else if (kind == "motor") {
        g[0] = 1;
      } else if (kind == "velocity") {
        double kv = num(a, "kv", cls, 1);
        g[0] = kv; bsp[2] = -kv; biastype = 1;
      } else {
        auto gp = nums(a, "gainprm", cls, {1, 0, 0});
        auto bp = nums(a, "biasprm", cls, {0, 0, 0});
        for (size_t k = 0; k < 3 && k < gp.size(); k++) g[k] = gp[k];
        for (size_t k = 0; k < 3 && k < bp.size(); k++) bsp[k] = bp[k];
        std::string gt = get(a, "gaintype", cls), bt = get(a, "biastype", cls);
        gaintype = (gt == "affine") ? 1 : 0;
        biastype = (bt == "affine") ? 1 : 0;
        if (!gt.empty() && gt != "fixed" && gt != "affine") fail("unsupported gaintype " + gt);
        if (!bt.empty() && bt != "none" && bt != "affine") fail("unsupported biastype " + bt);
        if (gaintype == 0) { g[1] = g[2] = 0; }
        if (biastype == 0) { bsp[0] = bsp[1] = bsp[2] = 0; }
      }
      m.actuator_gaintype.push_back(gaintype);
      m.actuator_biastype.push_back(biastype);
      for (int k = 0; k < 3; k++) { m.actuator_gainprm.push_back(g[k]); m.actuator_biasprm.push_back(bsp[k]); }
      auto cr = nums(a, "ctrlrange", cls, {0, 0});
      auto fr = nums(a, "forcerange", cls, {0, 0});
      std::string cl = get(a, "ctrllimited", cls), fl = get(a, "forcelimited", cls);
      int ctrllim = cl == "true" ? 1 : cl == "false" ? 0 : (autolimits && has(a, "ctrlrange", cls));
      int forcelim = fl == "true" ? 1 : fl == "false" ? 0 : (autolimits && has(a, "forcerange", cls));
      m.actuator_ctrllimited.push_back(ctrllim);
      m.actuator_forcelimited.push_back(forcelim);
      m.actuator_ctrlrange.insert(m.actuator_ctrlrange.end(), {cr.at(0), cr.at(1)});
      m.actuator_forcerange.insert(m.actuator_forcerange.end(), {fr.at(0), fr.at(1)});
    }
  }

  int body_by_name(const std::string& s) const {
    for (int b = 0; b < m.nbody; b++)
      if (m.body_name[b] == s) return b;
    fail("unknown body '" + s + "'");
  }
  int geom_by_name(const std::string& s) const {
    for (int g = 0; g < m.ngeom; g++)
      if (m.geom_name[g] == s) return g;
    fail("unknown geom '" + s + "'");
  }

  void parse_contact(const XmlNode& n) {
    for (auto& c : n.children) {
      if (c.tag == "exclude") {
        auto b1 = c.attr("body1"), b2 = c.attr("body2");
        if (!b1 || !b2) fail("exclude needs body1 and body2");
        m.exclude_body1.push_back(body_by_name(*b1));
        m.exclude_body2.push_back(body_by_name(*b2));
      } else if (c.tag == "pair") {
        auto g1 = c.attr("geom1"), g2 = c.attr("geom2");
        if (!g1 || !g2) fail("pair needs geom1 and geom2");
        Model::ExplicitPair p;
        p.g1 = geom_by_name(*g1);
        p.g2 = geom_by_name(*g2);
        std::string cls;
        p.condim = (int)num(c, "condim", cls, 3);
        auto fr = nums(c, "friction", cls, {1, 1, 0.005, 0.0001, 0.0001});
        while (fr.size() < 5) fr.push_back(0);
        for (int k = 0; k < 5; k++) p.friction[k] = fr[k];
        auto sr = nums(c, "solref", cls, {0.02, 1});
        auto si = nums(c, "solimp", cls, {0.9, 0.95, 0.001, 0.5, 2});
        while (si.size() < 5) si.push_back(si.size() == 3 ? 0.5 : 2);
        for (int k = 0; k < 2; k++) p.solref[k] = sr.at(k);
        for (int k = 0; k < 5; k++) p.solimp[k] = si[k];
        p.margin = num(c, "margin", cls, 0);
        p.gap = num(c, "gap", cls, 0);
        m.explicit_pairs.push_back(p);
      } else fail("unsupported element <" + c.tag + "> inside <contact>");
    }
  }

  void parse_tendon(const XmlNode& n) {
    for (auto& t : n.children) {
      if (t.tag != "fixed" && t.tag != "spatial") fail("unsupported element <" + t.tag + "> inside <tendon>");
      std::string cls;
      auto nm = t.attr("name");
      m.tendon_name.push_back(nm ? *nm : std::string());
      m.tendon_adr.push_back((int)m.wrap_objid.size());
      if (t.tag == "fixed") {
        for (auto& w : t.children) {
          if (w.tag != "joint") fail("fixed tendon elements must be <joint>");
          auto jn = w.attr("joint");
          if (!jn) fail("tendon joint needs joint=");
          int j = joint_by_name(*jn);
          if (m.jnt_type[j] != JNT_HINGE && m.jnt_type[j] != JNT_SLIDE) fail("fixed tendons use hinge or slide joints");
          m.wrap_type.push_back(1);
          m.wrap_objid.push_back(j);
          m.wrap_prm.push_back(num(w, "coef", cls, 1));
        }
      } else {
        // spatial path: branches of sites separated by pulleys; a sphere or
        // cylinder geom may sit between two sites of a branch
        int prev = 0;   // 0 branch start, 3 site, 4 geom
        for (auto& w : t.children) {
          if (w.tag == "site") {
            auto sn = w.attr("site");
            if (!sn) fail("spatial tendon site needs site=");
            m.wrap_type.push_back(3);
            m.wrap_objid.push_back(index_of(m.site_name, *sn, "site"));
            m.wrap_prm.push_back(0);
            prev = 3;
          } else if (w.tag == "geom") {
            auto gn = w.attr("geom");
            if (!gn) fail("spatial tendon geom needs geom=");
            if (prev != 3) fail("a wrapping geom must follow a site in a spatial tendon");
            const int g = geom_by_name(*gn);
            if (m.geom_type[g] != GEOM_SPHERE && m.geom_type[g] != GEOM_CYLINDER) fail("spatial tendons wrap around sphere and cylinder geoms only");
            m.wrap_type.push_back(m.geom_type[g] == GEOM_SPHERE ? 4 : 5);
            m.wrap_objid.push_back(g);
            auto ss = w.attr("sidesite");
            m.wrap_prm.push_back(ss ? index_of(m.site_name, *ss, "site") : -1);
            prev = 4;
          } else if (w.tag == "pulley") {
            if (prev != 3) fail("a pulley must follow a site in a spatial tendon");
            const double dv = num(w, "divisor", cls, 0);
            if (!(dv > 0)) fail("pulley divisor must be positive");
            m.wrap_type.push_back(2);
            m.wrap_objid.push_back(-1);
            m.wrap_prm.push_back(dv);
            prev = 0;
          } else {
            fail("spatial tendon elements must be <site>, <geom> or <pulley>");
          }
        }
        if (prev != 3) fail("a spatial tendon (and each pulley branch) must end with a site");
      }
      m.tendon_num.push_back((int)m.wrap_objid.size() - m.tendon_adr.back());
      auto rng = nums(t, "range", cls, {0, 0});
      auto lim = t.attr("limited");
      const bool auto_lim = !lim || *lim == "auto";
      if (lim && !auto_lim && *lim != "true" && *lim != "false") fail("tendon limited= must be true, false or auto");
      bool limited = auto_lim ? (rng.size() == 2 && rng[0] < rng[1]) : (*lim == "true");
      m.tendon_limited.push_back(limited);
      m.tendon_range.push_back(rng.at(0));
      m.tendon_range.push_back(rng.at(1));
      m.tendon_margin.push_back(num(t, "margin", cls, 0));
      m.tendon_frictionloss.push_back(num(t, "frictionloss", cls, 0));
      m.tendon_stiffness.push_back(num(t, "stiffness", cls, 0));
      m.tendon_damping.push_back(num(t, "damping", cls, 0));
      auto sl = nums(t, "springlength", cls, {-1, -1});
      m.tendon_lengthspring.push_back(sl.at(0));
      m.tendon_lengthspring.push_back(sl.size() > 1 ? sl[1] : sl[0]);
      auto srl = nums(t, "solreflimit", cls, {0.02, 1});
      auto sil = nums(t, "solimplimit", cls, {0.9, 0.95, 0.001, 0.5, 2});
      auto srf = nums(t, "solreffriction", cls, {0.02, 1});
      auto sif = nums(t, "solimpfriction", cls, {0.9, 0.95, 0.001, 0.5, 2});
      while (sil.size() < 5) sil.push_back(sil.size() == 3 ? 0.5 : 2);
      while (sif.size() < 5) sif.push_back(sif.size() == 3 ? 0.5 : 2);
      for (int k = 0; k < 2; k++) { m.tendon_solref_lim.push_back(srl.at(k)); m.tendon_solref_fri.push_back(srf.at(k)); }
      for (int k = 0; k < 5; k++) { m.tendon_solimp_lim.push_back(sil[k]); m.tendon_solimp_fri.push_back(sif[k]); }
      m.ntendon++;
    }
  }

  static int index_of(const std::vector<std::string>& names, const std::string& s, const char* what) {
    for (size_t i = 0; i < names.size(); i++)
      if (names[i] == s) return (int)i;
    fail(std::string("unknown ") + what + " '" + s + "'");
  }

  // <sensor> (reference: sensor.cpp make_sensor_ctx; MuJoCo's sensor list).
  // Types outside the batched set compile with their MuJoCo dimension and
  // read as zeros, with a warning, as in the reference.
  void parse_sensor(const XmlNode& n) {
    struct Kind { int type, dim; const char* obj; };
    static const std::map<std::string, Kind> kinds = {
        {"touch", {SENS_TOUCH, 1, "site"}}, {"accelerometer", {SENS_ACCELEROMETER, 3, "site"}}, {"velocimeter", {SENS_VELOCIMETER, 3, "site"}},
        {"gyro", {SENS_GYRO, 3, "site"}}, {"force", {SENS_FORCE, 3, "site"}}, {"torque", {SENS_TORQUE, 3, "site"}},
        {"magnetometer", {SENS_MAGNETOMETER, 3, "site"}}, {"rangefinder", {SENS_RANGEFINDER, 1, "site"}},
        {"jointpos", {SENS_JOINTPOS, 1, "joint"}}, {"jointvel", {SENS_JOINTVEL, 1, "joint"}}, {"tendonpos", {SENS_TENDONPOS, 1, "tendon"}},
        {"tendonvel", {SENS_TENDONVEL, 1, "tendon"}}, {"actuatorpos", {SENS_ACTUATORPOS, 1, "actuator"}},
        {"actuatorvel", {SENS_ACTUATORVEL, 1, "actuator"}}, {"actuatorfrc", {SENS_ACTUATORFRC, 1, "actuator"}},
        {"jointactuatorfrc", {SENS_JOINTACTFRC, 1, "joint"}}, {"tendonactuatorfrc", {SENS_TENDONACTFRC, 1, "tendon"}},
        {"ballquat", {SENS_BALLQUAT, 4, "joint"}}, {"ballangvel", {SENS_BALLANGVEL, 3, "joint"}},
        {"jointlimitpos", {SENS_JOINTLIMITPOS, 1, "joint"}}, {"jointlimitvel", {SENS_JOINTLIMITVEL, 1, "joint"}},
        {"jointlimitfrc", {SENS_JOINTLIMITFRC, 1, "joint"}}, {"tendonlimitpos", {SENS_TENDONLIMITPOS, 1, "tendon"}},
        {"tendonlimitvel", {SENS_TENDONLIMITVEL, 1, "tendon"}}, {"tendonlimitfrc", {SENS_TENDONLIMITFRC, 1, "tendon"}},
        {"framepos", {SENS_FRAMEPOS, 3, "frame"}}, {"framequat", {SENS_FRAMEQUAT, 4, "frame"}}, {"framexaxis", {SENS_FRAMEXAXIS, 3, "frame"}},
        {"frameyaxis", {SENS_FRAMEYAXIS, 3, "frame"}}, {"framezaxis", {SENS_FRAMEZAXIS, 3, "frame"}},
        {"framelinvel", {SENS_FRAMELINVEL, 3, "frame"}}, {"frameangvel", {SENS_FRAMEANGVEL, 3, "frame"}},
        {"framelinacc", {SENS_FRAMELINACC, 3, "frame"}}, {"frameangacc", {SENS_FRAMEANGACC, 3, "frame"}},
        {"subtreecom", {SENS_SUBTREECOM, 3, "body"}}, {"subtreelinvel", {SENS_SUBTREELINVEL, 3, "body"}},
        {"subtreeangmom", {SENS_SUBTREEANGMOM, 3, "body"}}};
    for (auto& c : n.children) {
      auto it = kinds.find(c.tag);
      if (it == kinds.end()) fail("unsupported sensor <" + c.tag + ">");
      const Kind& k = it->second;
      const std::string obj = k.obj;
      auto need = [&](const char* attr) {
        auto v = c.attr(attr);
        if (!v) fail("sensor <" + c.tag + "> needs " + attr + "=");
        return *v;
      };
      int objtype = OBJ_UNKNOWN, objid = -1;
      bool supported = true;
      if (obj == "site") {
        objtype = OBJ_SITE;
        objid = index_of(m.site_name, need("site"), "site");
      } else if (obj == "joint") {
        objtype = OBJ_JOINT;
        objid = joint_by_name(need("joint"));
        const int jt = m.jnt_type[objid];
        const bool ball = k.type == SENS_BALLQUAT || k.type == SENS_BALLANGVEL;
        if (ball != (jt == JNT_BALL) || jt == JNT_FREE) fail("sensor <" + c.tag + "> on a joint of the wrong type");
      } else if (obj == "tendon") {
        objtype = OBJ_TENDON;
        objid = tendon_by_name(need("tendon"));
      } else if (obj == "actuator") {
        objtype = OBJ_ACTUATOR;
        objid = index_of(m.actuator_name, need("actuator"), "actuator");
      } else if (obj == "body") {
        objtype = OBJ_BODY;
        objid = body_by_name(need("body"));
      } else {  // frame sensors: objtype body / xbody / geom / site
        const std::string ot = need("objtype"), on = need("objname");
        if (ot == "body") { objtype = OBJ_BODY; objid = body_by_name(on); }
        else if (ot == "xbody") { objtype = OBJ_XBODY; objid = body_by_name(on); }
        else if (ot == "geom") { objtype = OBJ_GEOM; objid = geom_by_name(on); }
        else if (ot == "site") { objtype = OBJ_SITE; objid = index_of(m.site_name, on, "site"); }
        else fail("frame sensor objtype must be body, xbody, geom or site");
        if (c.attr("reftype") || c.attr("refname")) supported = false;  // relative frames: not in the batched set
      }
      switch (k.type) {
        case SENS_ACCELEROMETER: case SENS_VELOCIMETER: case SENS_GYRO: case SENS_MAGNETOMETER: case SENS_JOINTPOS: case SENS_JOINTVEL:
        case SENS_TENDONPOS: case SENS_TENDONVEL: case SENS_ACTUATORPOS: case SENS_ACTUATORVEL: case SENS_JOINTACTFRC: case SENS_BALLQUAT:
        case SENS_BALLANGVEL: case SENS_FRAMEPOS: case SENS_FRAMEQUAT: case SENS_FRAMEXAXIS: case SENS_FRAMEYAXIS: case SENS_FRAMEZAXIS:
        case SENS_FRAMELINVEL: case SENS_FRAMEANGVEL: case SENS_SUBTREECOM:
          break;
        default:
          supported = false;
      }
      auto nm = c.attr("name");
      if (!supported)
        std::fprintf(stderr, "mjb200: sensor '%s' (<%s>) is outside the batched sensor set; its sensordata stays 0\n", nm ? nm->c_str() : "",
                     c.tag.c_str());
      m.sensor_name.push_back(nm ? *nm : std::string());
      m.sensor_type.push_back(k.type);
      m.sensor_objtype.push_back(objtype);
      m.sensor_objid.push_back(objid);
      m.sensor_dim.push_back(k.dim);
      m.sensor_adr.push_back(m.nsensordata);
      m.sensor_supported.push_back(supported);
      m.nsensordata += k.dim;
      m.nsensor++;
    }
  }

  int tendon_by_name(const std::string& s) const {
    for (int t = 0; t < m.ntendon; t++)
      if (m.tendon_name[t] == s) return t;
    fail("unknown tendon '" + s + "'");
  }

  void parse_equality(const XmlNode& n) {
    static const std::map<std::string, int> kinds = {{"connect", 0}, {"weld", 1}, {"joint", 2}, {"tendon", 3}};
    for (auto& c : n.children) {
      auto it = kinds.find(c.tag);
      if (it == kinds.end()) fail("unsupported element <" + c.tag + "> inside <equality>");
      std::string cls;
      int o1 = -1, o2 = -1;
      if (it->second == 3) {
        auto t1 = c.attr("tendon1"), t2 = c.attr("tendon2");
        if (!t1) fail("equality tendon needs tendon1");
        o1 = tendon_by_name(*t1);
        if (t2) o2 = tendon_by_name(*t2);
      }
      if (it->second == 2) {
        auto j1 = c.attr("joint1"), j2 = c.attr("joint2");
        if (!j1) fail("equality joint needs joint1");
        o1 = joint_by_name(*j1);
        if (j2) o2 = joint_by_name(*j2);
        for (int j : {o1, o2})
          if (j >= 0 && m.jnt_type[j] != JNT_HINGE && m.jnt_type[j] != JNT_SLIDE) fail("equality joint couples hinge or slide joints only");
      }
      m.eq_type.push_back(it->second);
      m.eq_obj1.push_back(o1);
      m.eq_obj2.push_back(o2);
      auto act = c.attr("active");
      m.eq_active.push_back(!act || *act != "false");
      auto pc = nums(c, "polycoef", cls, {0, 1, 0, 0, 0});
      while (pc.size() < 5) pc.push_back(0);
      auto sr = nums(c, "solref", cls, {0.02, 1});
      auto si = nums(c, "solimp", cls, {0.9, 0.95, 0.001, 0.5, 2});
      while (si.size() < 5) si.push_back(si.size() == 3 ? 0.5 : 2);
      for (int k = 0; k < 5; k++) m.eq_data.push_back(pc[k]);
      for (int k = 0; k < 2; k++) m.eq_solref.push_back(sr.at(k));
      for (int k = 0; k < 5; k++) m.eq_solimp.push_back(si[k]);
      m.eq_invweight.push_back(0);
    }
  }

  int joint_by_name(const std::string& s) const {
    for (int j = 0; j < m.njnt; j++)
      if (m.jnt_name[j] == s) return j;
    fail("unknown joint '" + s + "'");
  }

  void parse_asset(const XmlNode& n) {
    for (auto& a : n.children) {
      if (a.tag != "mesh") fail("unsupported asset <" + a.tag + "> (only inline-vertex meshes are supported)");
      MeshAsset ma;
      auto nm = a.attr("name");
      if (!nm) fail("mesh needs a name");
      ma.name = *nm;
      if (!a.attr("vertex")) fail("mesh '" + ma.name + "' needs inline vertex data");
      ma.verts = parse_nums(*a.attr("vertex"), "vertex");
      if (ma.verts.size() < 12 || ma.verts.size() % 3) fail("mesh '" + ma.name + "' needs at least 4 vertices");
      if (a.attr("scale")) {
        auto s = parse_nums(*a.attr("scale"), "scale");
        for (int k = 0; k < 3; k++) ma.scale[k] = s.at(k);
      }
      for (size_t v = 0; v < ma.verts.size() / 3; v++)
        for (int k = 0; k < 3; k++) ma.verts[3 * v + k] *= ma.scale[k];
      mesh_assets.push_back(ma);
      // hull and mass properties (unit density)
      MeshProps mp;
      ConvexHull h = convex_hull(ma.verts);
      if (h.faces.empty()) fail("mesh '" + ma.name + "' is degenerate (no 3-D hull)");
      double vol, com[3], I[9];
      hull_mass_properties(h, vol, com, I);
      if (vol <= kMinVal) fail("mesh '" + ma.name + "' has zero volume");
      double w[3], V[9];
      eig3(I, w, V);
      mat2quat(V, mp.quat);
      for (int k = 0; k < 3; k++) { mp.pos[k] = com[k]; mp.inertia_unit[k] = w[k]; }
      mp.volume = vol;
      // hull vertices in the centred, principal frame: R^T (v - com)
      for (int idx : h.vertex_ids) {
        double d[3] = {ma.verts[3 * idx] - com[0], ma.verts[3 * idx + 1] - com[1], ma.verts[3 * idx + 2] - com[2]};
        for (int c = 0; c < 3; c++) mp.hull.push_back(V[0 * 3 + c] * d[0] + V[1 * 3 + c] * d[1] + V[2 * 3 + c] * d[2]);
      }
      mesh_props.push_back(mp);
    }
  }

  void parse_option(const XmlNode& n) {
    std::string cls;
    m.timestep = num(n, "timestep", cls, m.timestep);
    auto g = nums(n, "gravity", cls, {m.gravity[0], m.gravity[1], m.gravity[2]});
    for (int k = 0; k < 3; k++) m.gravity[k] = g.at(k);
    auto mg = nums(n, "magnetic", cls, {m.magnetic[0], m.magnetic[1], m.magnetic[2]});
    for (int k = 0; k < 3; k++) m.magnetic[k] = mg.at(k);
    m.iterations = (int)num(n, "iterations", cls, m.iterations);
    m.tolerance = num(n, "tolerance", cls, m.tolerance);
    m.ls_iterations = (int)num(n, "ls_iterations", cls, m.ls_iterations);
    m.ls_tolerance = num(n, "ls_tolerance", cls, m.ls_tolerance);
    m.impratio = num(n, "impratio", cls, m.impratio);
    std::string cone = get(n, "cone", cls);
    if (cone == "elliptic") m.cone = CONE_ELLIPTIC;
    else if (cone.empty() || cone == "pyramidal") m.cone = CONE_PYRAMIDAL;
    else fail("unknown cone " + cone);
    std::string integ = get(n, "integrator", cls);
    if (integ.empty() || integ == "Euler") m.integrator = 0;
    else if (integ == "implicitfast") m.integrator = 3;
    else if (integ == "implicit") m.integrator = 2;
    else fail("unsupported integrator '" + integ + "' (Euler, implicit, implicitfast)");
    std::string solver = get(n, "solver", cls);
    if (!solver.empty() && solver != "Newton") fail("only the Newton solver is supported");
    for (auto& f : n.children) {
      if (f.tag != "flag") fail("unsupported element <" + f.tag + "> inside <option>");
      static const std::pair<const char*, int> flags[] = {
          {"constraint", DSBL_CONSTRAINT}, {"equality", DSBL_EQUALITY}, {"frictionloss", DSBL_FRICTIONLOSS}, {"limit", DSBL_LIMIT},
          {"contact", DSBL_CONTACT}, {"passive", DSBL_PASSIVE}, {"gravity", DSBL_GRAVITY}, {"clampctrl", DSBL_CLAMPCTRL},
          {"warmstart", DSBL_WARMSTART}, {"filterparent", DSBL_FILTERPARENT}, {"actuation", DSBL_ACTUATION}, {"refsafe", DSBL_REFSAFE},
          {"eulerdamp", DSBL_EULERDAMP}};
      for (auto& kv : f.attrs) {
        bool found = false;
        for (auto& fl : flags)
          if (kv.first == fl.first) {
            found = true;
            if (kv.second == "disable") m.disableflags |= fl.second;
            else if (kv.second == "enable") m.disableflags &= ~fl.second;
            else fail("flag value must be enable/disable");
          }
        if (!found) fail("unsupported option flag '" + kv.first + "'");
      }
    }
  }

  void compile(const XmlNode& root) {
    if (root.tag != "mujoco") fail("root element must be <mujoco>");
    if (auto v = root.attr("model")) m.name = *v;
    classes.clear();
    // pass 1: compiler, defaults, assets, option
    bool have_default = false;
    for (auto& c : root.children) {
      if (c.tag == "compiler") {
        if (auto a = c.attr("angle")) degrees = (*a != "radian");
        if (auto a = c.attr("autolimits")) autolimits = (*a == "true");
        if (auto a = c.attr("inertiafromgeom")) inertiafromgeom = *a;
      } else if (c.tag == "default") {
        if (have_default) fail("only one top-level <default> is supported");
        have_default = true;
        parse_defaults(c, -1);
      }
    }
    if (!have_default) {
      DefaultClass d;
      d.name = "main";
      classes.push_back(d);
      class_index["main"] = 0;
    }
    for (auto& c : root.children) {
      if (c.tag == "asset") parse_asset(c);
      else if (c.tag == "option") parse_option(c);
    }
    // world body
    add_body("world", -1);
    m.body_parentid[0] = 0;
    for (auto& c : root.children) {
      if (c.tag == "worldbody") {
        for (auto& ch : c.children) {
          if (ch.tag == "body") parse_body(ch, 0, std::string());
          else if (ch.tag == "geom") add_geom(ch, std::string(), 0);
          else if (ch.tag == "site") add_site(ch, std::string(), 0);
          else if (ch.tag == "camera" || ch.tag == "light") continue;
          else fail("unsupported element <" + ch.tag + "> inside <worldbody>");
        }
      }
    }
    // tendons before the actuators and equalities that name them
    for (auto& c : root.children)
      if (c.tag == "tendon") parse_tendon(c);
    for (auto& c : root.children) {
      if (c.tag == "actuator") parse_actuator(c);
      else if (c.tag == "contact") parse_contact(c);
      else if (c.tag == "equality") parse_equality(c);
      else if (c.tag == "tendon" || c.tag == "sensor" || c.tag == "compiler" || c.tag == "default" || c.tag == "asset" || c.tag == "option" || c.tag == "worldbody" || c.tag == "size" ||
               c.tag == "visual" || c.tag == "statistic" || c.tag == "keyframe")
        continue;
      else fail("unsupported top-level element <" + c.tag + ">");
    }
    // sensors last: they name joints, tendons, actuators, bodies, geoms and sites
    for (auto& c : root.children)
      if (c.tag == "sensor") parse_sensor(c);
    finish_inertia();
    // meshes into the model
    m.nmesh = (int)mesh_props.size();
    for (auto& mp : mesh_props) {
      m.mesh_vertadr.push_back((int)m.mesh_vert.size() / 3);
      m.mesh_vertnum.push_back((int)mp.hull.size() / 3);
      m.mesh_vert.insert(m.mesh_vert.end(), mp.hull.begin(), mp.hull.end());
    }
    for (auto& a : mesh_assets) m.mesh_name.push_back(a.name);
    for (int b = 1; b < m.nbody; b++) {
      bool moving = false;
      for (int a = b; a > 0; a = m.body_parentid[a])
        if (m.body_jntnum[a] > 0) moving = true;
      if (moving && m.body_mass[b] < kMinVal && m.body_jntnum[b] > 0)
        fail("body '" + m.body_name[b] + "' has joints but no mass");
    }
  }
};

// ------------------------------------------------------------ finalize
// Forward kinematics, composite-rigid-body mass matrix and invweights at
// qpos0 in double precision (MuJoCo computes the same quantities in
// mj_setConst; the reference reads them from mjModel).
struct QposZeroData {
  std::vector<double> xpos, xquat, xmat, xipos, xanchor, xaxis, subtree_com, cdof, M;
};

void kinematics_qpos0(const Model& m, QposZeroData& d) {
  int nb = m.nbody;
  d.xpos.assign(3 * nb, 0);
  d.xquat.assign(4 * nb, 0);
  d.xmat.assign(9 * nb, 0);
  d.xipos.assign(3 * nb, 0);
  d.xanchor.assign(3 * m.njnt, 0);
  d.xaxis.assign(3 * m.njnt, 0);
  d.xquat[0] = 1;
  quat2mat(&d.xquat[0], &d.xmat[0]);
  for (int b = 1; b < nb; b++) {
    int p = m.body_parentid[b];
    double pos[3], quat[4], r[3];
    quat_rot(&d.xquat[4 * p], &m.body_pos[3 * b], r);
    for (int k = 0; k < 3; k++) pos[k] = d.xpos[3 * p + k] + r[k];
    quat_mul(&d.xquat[4 * p], &m.body_quat[4 * b], quat);
    for (int j = m.body_jntadr[b]; j >= 0 && j < m.body_jntadr[b] + m.body_jntnum[b]; j++) {
      // at qpos0 hinge/slide displacements are zero and free joints equal the body frame
      double a[3], ax[3];
      quat_rot(quat, &m.jnt_pos[3 * j], a);
      for (int k = 0; k < 3; k++) a[k] += pos[k];
      quat_rot(quat, &m.jnt_axis[3 * j], ax);
      if (m.jnt_type[j] == JNT_FREE) {
        ax[0] = 0; ax[1] = 0; ax[2] = 1;
        for (int k = 0; k < 3; k++) a[k] = pos[k];
      }
      for (int k = 0; k < 3; k++) { d.xanchor[3 * j + k] = a[k]; d.xaxis[3 * j + k] = ax[k]; }
    }
    quat_normalize(quat);
    for (int k = 0; k < 3; k++) d.xpos[3 * b + k] = pos[k];
    for (int k = 0; k < 4; k++) d.xquat[4 * b + k] = quat[k];
    quat2mat(quat, &d.xmat[9 * b]);
  }
  for (int b = 0; b < nb; b++) {
    double r[3];
    quat_rot(&d.xquat[4 * b], &m.body_ipos[3 * b], r);
    for (int k = 0; k < 3; k++) d.xipos[3 * b + k] = d.xpos[3 * b + k] + r[k];
  }
  // subtree COM
  std::vector<double> mass(nb), mc(3 * nb);
  for (int b = 0; b < nb; b++) {
    mass[b] = m.body_mass[b];
    for (int k = 0; k < 3; k++) mc[3 * b + k] = m.body_mass[b] * d.xipos[3 * b + k];
  }
  for (int b = nb - 1; b > 0; b--) {
    int p = m.body_parentid[b];
    mass[p] += mass[b];
    for (int k = 0; k < 3; k++) mc[3 * p + k] += mc[3 * b + k];
  }
  d.subtree_com.assign(3 * nb, 0);
  for (int b = 0; b < nb; b++)
    for (int k = 0; k < 3; k++) d.subtree_com[3 * b + k] = mass[b] > kMinVal ? mc[3 * b + k] / mass[b] : d.xipos[3 * b + k];
  // cdof
  int nv = m.nv;
  d.cdof.assign(6 * nv, 0);
  for (int i = 0; i < nv; i++) {
    int b = m.dof_bodyid[i], j = m.dof_jntid[i];
    const double* rc = &d.subtree_com[3 * m.body_rootid[b]];
    double* c = &d.cdof[6 * i];
    int t = m.jnt_type[j];
    int sub = i - m.jnt_dofadr[j];
    double ax[3];
    bool rot = true;
    if (t == JNT_HINGE) for (int k = 0; k < 3; k++) ax[k] = d.xaxis[3 * j + k];
    else if (t == JNT_SLIDE) { rot = false; for (int k = 0; k < 3; k++) ax[k] = d.xaxis[3 * j + k]; }
    else if (t == JNT_FREE && sub < 3) { rot = false; ax[0] = ax[1] = ax[2] = 0; ax[sub] = 1; }
    else {
      int col = (t == JNT_FREE) ? sub - 3 : sub;
      for (int k = 0; k < 3; k++) ax[k] = d.xmat[9 * b + 3 * k + col];
    }
    if (rot) {
      double off[3] = {rc[0] - d.xanchor[3 * j], rc[1] - d.xanchor[3 * j + 1], rc[2] - d.xanchor[3 * j + 2]};
      c[0] = ax[0]; c[1] = ax[1]; c[2] = ax[2];
      c[3] = ax[1] * off[2] - ax[2] * off[1];
      c[4] = ax[2] * off[0] - ax[0] * off[2];
      c[5] = ax[0] * off[1] - ax[1] * off[0];
    } else {
      c[3] = ax[0]; c[4] = ax[1]; c[5] = ax[2];
    }
  }
  // cinert and CRB
  std::vector<double> crb(10 * nb, 0);
  for (int b = 1; b < nb; b++) {
    double R[9], q[4];
    quat_mul(&d.xquat[4 * b], &m.body_iquat[4 * b], q);
    quat2mat(q, R);
    const double* I = &m.body_inertia[3 * b];
    double Ig[9];
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) {
        double s = 0;
        for (int k = 0; k < 3; k++) s += R[r * 3 + k] * I[k] * R[c * 3 + k];
        Ig[r * 3 + c] = s;
      }
    const double* rc = &d.subtree_com[3 * m.body_rootid[b]];
    double off[3] = {d.xipos[3 * b] - rc[0], d.xipos[3 * b + 1] - rc[1], d.xipos[3 * b + 2] - rc[2]};
    double mb = m.body_mass[b], d2 = off[0] * off[0] + off[1] * off[1] + off[2] * off[2];
    double* ci = &crb[10 * b];
    ci[0] = Ig[0] + mb * (d2 - off[0] * off[0]);
    ci[1] = Ig[4] + mb * (d2 - off[1] * off[1]);
    ci[2] = Ig[8] + mb * (d2 - off[2] * off[2]);
    ci[3] = Ig[1] - mb * off[0] * off[1];
    ci[4] = Ig[2] - mb * off[0] * off[2];
    ci[5] = Ig[5] - mb * off[1] * off[2];
    ci[6] = mb * off[0]; ci[7] = mb * off[1]; ci[8] = mb * off[2];
    ci[9] = mb;
  }
  for (int b = nb - 1; b > 0; b--) {
    int p = m.body_parentid[b];
    if (p > 0)
      for (int k = 0; k < 10; k++) crb[10 * p + k] += crb[10 * b + k];
  }
  d.M.assign(nv * nv, 0);
  for (int i = 0; i < nv; i++) {
    const double* ci = &crb[10 * m.dof_bodyid[i]];
    const double* c = &d.cdof[6 * i];
    double f[6];
    f[0] = ci[0] * c[0] + ci[3] * c[1] + ci[4] * c[2] + (ci[7] * c[5] - ci[8] * c[4]);
    f[1] = ci[3] * c[0] + ci[1] * c[1] + ci[5] * c[2] + (ci[8] * c[3] - ci[6] * c[5]);
    f[2] = ci[4] * c[0] + ci[5] * c[1] + ci[2] * c[2] + (ci[6] * c[4] - ci[7] * c[3]);
    f[3] = ci[9] * c[3] - (ci[7] * c[2] - ci[8] * c[1]);
    f[4] = ci[9] * c[4] - (ci[8] * c[0] - ci[6] * c[2]);
    f[5] = ci[9] * c[5] - (ci[6] * c[1] - ci[7] * c[0]);
    for (int j = i; j >= 0; j = m.dof_parentid[j]) {
      const double* cj = &d.cdof[6 * j];
      double s = 0;
      for (int k = 0; k < 6; k++) s += f[k] * cj[k];
      d.M[i * nv + j] = s;
      d.M[j * nv + i] = s;
    }
    d.M[i * nv + i] += m.dof_armature[i];
  }
}

// Dense Cholesky solve in place (A is overwritten by L); returns false if not SPD.
bool cholesky(std::vector<double>& A, int n) {
  for (int j = 0; j < n; j++) {
    double s = A[j * n + j];
    for (int k = 0; k < j; k++) s -= A[j * n + k] * A[j * n + k];
    if (s <= 0) return false;
    double d = std::sqrt(s);
    A[j * n + j] = d;
    for (int i = j + 1; i < n; i++) {
      double t = A[i * n + j];
      for (int k = 0; k < j; k++) t -= A[i * n + k] * A[j * n + k];
      A[i * n + j] = t / d;
    }
  }
  return true;
}
void chol_solve(const std::vector<double>& L, int n, double* x) {
  for (int i = 0; i < n; i++) {
    double s = x[i];
    for (int k = 0; k < i; k++) s -= L[i * n + k] * x[k];
    x[i] = s / L[i * n + i];
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = x[i];
    for (int k = i + 1; k < n; k++) s -= L[k * n + i] * x[k];
    x[i] = s / L[i * n + i];
  }
}

void compute_invweights(Model& m) {
  int nv = m.nv, nb = m.nbody;
  m.body_invweight0.assign(2 * nb, 0);
  m.dof_invweight0.assign(nv, 0);
  m.meaninertia = 1;
  if (nv == 0) return;
  QposZeroData d;
  kinematics_qpos0(m, d);
  double tr = 0;
  for (int i = 0; i < nv; i++) tr += d.M[i * nv + i];
  m.meaninertia = tr / nv;
  std::vector<double> L = d.M;
  if (!cholesky(L, nv)) fail("mass matrix at qpos0 is not positive definite (check masses/armature)");
  // dof invweights from diag(M^-1)
  std::vector<double> minv_diag(nv);
  std::vector<double> e(nv);
  for (int i = 0; i < nv; i++) {
    std::fill(e.begin(), e.end(), 0.0);
    e[i] = 1;
    chol_solve(L, nv, e.data());
    minv_diag[i] = e[i];
  }
  for (int j = 0; j < m.njnt; j++) {
    int a = m.jnt_dofadr[j];
    int t = m.jnt_type[j];
    if (t == JNT_FREE) {
      double tt = (minv_diag[a] + minv_diag[a + 1] + minv_diag[a + 2]) / 3;
      double rr = (minv_diag[a + 3] + minv_diag[a + 4] + minv_diag[a + 5]) / 3;
      for (int k = 0; k < 3; k++) { m.dof_invweight0[a + k] = tt; m.dof_invweight0[a + 3 + k] = rr; }
    } else if (t == JNT_BALL) {
      double rr = (minv_diag[a] + minv_diag[a + 1] + minv_diag[a + 2]) / 3;
      for (int k = 0; k < 3; k++) m.dof_invweight0[a + k] = rr;
    } else {
      m.dof_invweight0[a] = minv_diag[a];
    }
  }
  // tendons: rest length and invweight J M^-1 J^T at qpos0
  m.tendon_length0.assign(m.ntendon, 0);
  m.tendon_invweight0.assign(m.ntendon, 0);
  // world point / body of site s and geom poses at qpos0
  auto site_world = [&](int sidx, double* p) {
    const int b = m.site_bodyid[sidx];
    double r[3];
    quat_rot(&d.xquat[4 * b], &m.site_pos[3 * sidx], r);
    for (int k = 0; k < 3; k++) p[k] = d.xpos[3 * b + k] + r[k];
  };
  // add scale * dir' (point Jacobian of body b at world point p) to jt
  auto add_point = [&](std::vector<double>& jt, int b, const double* p, const double* dir, double scale) {
    const double* rc = &d.subtree_com[3 * m.body_rootid[b]];
    const double off[3] = {p[0] - rc[0], p[1] - rc[1], p[2] - rc[2]};
    for (int i = 0; i < nv; i++) {
      const int db = m.dof_bodyid[i];
      if (!(db <= b && b < db + m.body_subtreesize[db])) continue;
      const double* c = &d.cdof[6 * i];
      const double jp[3] = {c[3] + (c[1] * off[2] - c[2] * off[1]), c[4] + (c[2] * off[0] - c[0] * off[2]), c[5] + (c[0] * off[1] - c[1] * off[0])};
      jt[i] += scale * (dir[0] * jp[0] + dir[1] * jp[1] + dir[2] * jp[2]);
    }
  };
  // straight piece from p0 on body b0 to p1 on body b1
  auto add_piece = [&](std::vector<double>& jt, double& len, const double* p0, int b0, const double* p1, int b1, double scale) {
    double e[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    const double l = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
    len += scale * l;
    if (l < 1e-12) return;
    for (int k = 0; k < 3; k++) e[k] /= l;
    add_point(jt, b1, p1, e, scale);
    add_point(jt, b0, p0, e, -scale);
  };
  for (int t = 0; t < m.ntendon; t++) {
    std::vector<double> jt(nv, 0.0);
    double len = 0;
    const int a0 = m.tendon_adr[t], a1 = a0 + m.tendon_num[t];
    double scale = 1;
    for (int w = a0; w < a1; w++) {
      const int ty = m.wrap_type[w];
      if (ty == 1) {
        const int j = m.wrap_objid[w];
        len += m.wrap_prm[w] * m.qpos0[m.jnt_qposadr[j]];
        jt[m.jnt_dofadr[j]] += m.wrap_prm[w];
      } else if (ty == 2) {
        scale = 1.0 / m.wrap_prm[w];
      } else if (ty == 3 && w + 1 < a1 && m.wrap_type[w + 1] == 3) {
        double p0[3], p1[3];
        site_world(m.wrap_objid[w], p0);
        site_world(m.wrap_objid[w + 1], p1);
        add_piece(jt, len, p0, m.site_bodyid[m.wrap_objid[w]], p1, m.site_bodyid[m.wrap_objid[w + 1]], scale);
      } else if (ty == 3 && w + 2 < a1 && (m.wrap_type[w + 1] == 4 || m.wrap_type[w + 1] == 5)) {
        const int s0 = m.wrap_objid[w], g = m.wrap_objid[w + 1], s1 = m.wrap_objid[w + 2], ss = (int)m.wrap_prm[w + 1];
        double p0[3], p1[3], gc[3], gq[4], gR[9], sp[3], t0[3], t1[3], r[3];
        site_world(s0, p0);
        site_world(s1, p1);
        const int gb = m.geom_bodyid[g];
        quat_rot(&d.xquat[4 * gb], &m.geom_pos[3 * g], r);
        for (int k = 0; k < 3; k++) gc[k] = d.xpos[3 * gb + k] + r[k];
        quat_mul(&d.xquat[4 * gb], &m.geom_quat[4 * g], gq);
        quat2mat(gq, gR);
        if (ss >= 0) site_world(ss, sp);
        bool wrapped = false;
        mjbwrap::geom<double>(m.wrap_type[w + 1] == 4 ? 2 : 5, gc, gR, m.geom_size[3 * g], p0, p1, ss >= 0 ? sp : nullptr, t0, t1, wrapped);
        if (!wrapped) {
          add_piece(jt, len, p0, m.site_bodyid[s0], p1, m.site_bodyid[s1], scale);
        } else {
          const double l_before = len;
          add_piece(jt, len, p0, m.site_bodyid[s0], t0, gb, scale);
          add_piece(jt, len, t1, gb, p1, m.site_bodyid[s1], scale);
          // the arc (helix) between the tangent points moves rigidly with the geom
          const double full = mjbwrap::geom<double>(m.wrap_type[w + 1] == 4 ? 2 : 5, gc, gR, m.geom_size[3 * g], p0, p1, ss >= 0 ? sp : nullptr, t0, t1,
                                                    wrapped);
          len = l_before + scale * full;
        }
        w += 1;   // the geom; the next site starts the next piece
      }
    }
    std::vector<double> x = jt;
    chol_solve(L, nv, x.data());
    double iw = 0;
    for (int i = 0; i < nv; i++) iw += jt[i] * x[i];
    m.tendon_length0[t] = len;
    m.tendon_invweight0[t] = iw;
    // springlength "-1 -1" (the default) means the length at qpos0
    if (m.tendon_lengthspring[2 * t] == -1 && m.tendon_lengthspring[2 * t + 1] == -1) m.tendon_lengthspring[2 * t] = m.tendon_lengthspring[2 * t + 1] = len;
  }
  // body invweights: A = J M^-1 J^T at the body COM
  std::vector<double> J(6 * nv), X(6 * nv);
  for (int b = 1; b < nb; b++) {
    if (m.body_weldid[b] == 0) continue;
    std::fill(J.begin(), J.end(), 0.0);
    const double* p = &d.xipos[3 * b];
    const double* rc = &d.subtree_com[3 * m.body_rootid[b]];
    double off[3] = {p[0] - rc[0], p[1] - rc[1], p[2] - rc[2]};
    for (int i = 0; i < nv; i++) {
      int db = m.dof_bodyid[i];
      if (!(db <= b && b < db + m.body_subtreesize[db])) continue;
      const double* c = &d.cdof[6 * i];
      // jacp = lin + ang x off ; jacr = ang
      J[0 * nv + i] = c[3] + (c[1] * off[2] - c[2] * off[1]);
      J[1 * nv + i] = c[4] + (c[2] * off[0] - c[0] * off[2]);
      J[2 * nv + i] = c[5] + (c[0] * off[1] - c[1] * off[0]);
      J[3 * nv + i] = c[0];
      J[4 * nv + i] = c[1];
      J[5 * nv + i] = c[2];
    }
    X = J;
    for (int r = 0; r < 6; r++) chol_solve(L, nv, &X[r * nv]);
    double A[6];
    for (int r = 0; r < 6; r++) {
      double s = 0;
      for (int i = 0; i < nv; i++) s += J[r * nv + i] * X[r * nv + i];
      A[r] = s;
    }
    m.body_invweight0[2 * b] = (A[0] + A[1] + A[2]) / 3;
    m.body_invweight0[2 * b + 1] = (A[3] + A[4] + A[5]) / 3;
  }
}

void mix_params(const Model& m, int g1, int g2, Pair& p) {
  int pr1 = m.geom_priority[g1], pr2 = m.geom_priority[g2];
  const double* f1 = &m.geom_friction[3 * g1];
  const double* f2 = &m.geom_friction[3 * g2];
  double fr[3];
  if (pr1 != pr2) {
    int w = pr1 > pr2 ? g1 : g2;
    p.condim = m.geom_condim[w];
    for (int k = 0; k < 3; k++) fr[k] = m.geom_friction[3 * w + k];
    for (int k = 0; k < 2; k++) p.solref[k] = m.geom_solref[2 * w + k];
    for (int k = 0; k < 5; k++) p.solimp[k] = m.geom_solimp[5 * w + k];
  } else {
    p.condim = std::max(m.geom_condim[g1], m.geom_condim[g2]);
    double m1 = m.geom_solmix[g1], m2 = m.geom_solmix[g2], mix;
    if (m1 >= kMinVal && m2 >= kMinVal) mix = m1 / (m1 + m2);
    else if (m1 < kMinVal && m2 < kMinVal) mix = 0.5;
    else if (m1 < kMinVal) mix = 0;
    else mix = 1;
    const double* s1 = &m.geom_solref[2 * g1];
    const double* s2 = &m.geom_solref[2 * g2];
    if (s1[0] > 0 && s2[0] > 0)
      for (int k = 0; k < 2; k++) p.solref[k] = mix * s1[k] + (1 - mix) * s2[k];
    else
      for (int k = 0; k < 2; k++) p.solref[k] = std::min(s1[k], s2[k]);
    for (int k = 0; k < 5; k++) p.solimp[k] = mix * m.geom_solimp[5 * g1 + k] + (1 - mix) * m.geom_solimp[5 * g2 + k];
    for (int k = 0; k < 3; k++) fr[k] = std::max(f1[k], f2[k]);
  }
  p.friction[0] = fr[0];
  p.friction[1] = fr[0];
  p.friction[2] = fr[1];
  p.friction[3] = fr[2];
  p.friction[4] = fr[2];
}

bool has_collider(int t1, int t2) {
  if (t1 > t2) std::swap(t1, t2);
  if (t1 == GEOM_PLANE && t2 == GEOM_PLANE) return false;
  if (t1 == GEOM_HFIELD || t2 == GEOM_HFIELD) return false;
  return true;
}

void build_pairs(Model& m) {
  m.pairs.clear();
  std::set<int> excl;
  for (size_t i = 0; i < m.exclude_body1.size(); i++) {
    int a = std::min(m.exclude_body1[i], m.exclude_body2[i]);
    int b = std::max(m.exclude_body1[i], m.exclude_body2[i]);
    excl.insert((a << 16) | b);
  }
  for (int ga = 0; ga < m.ngeom; ga++)
    for (int gb = ga + 1; gb < m.ngeom; gb++) {
      int g1 = ga, g2 = gb;
      if (m.geom_type[g1] > m.geom_type[g2]) std::swap(g1, g2);
      int t1 = m.geom_type[g1], t2 = m.geom_type[g2];
      if (!has_collider(t1, t2)) continue;
      int mask = (m.geom_contype[g1] & m.geom_conaffinity[g2]) | (m.geom_contype[g2] & m.geom_conaffinity[g1]);
      if (!mask) continue;
      int b1 = m.geom_bodyid[g1], b2 = m.geom_bodyid[g2];
      int w1 = m.body_weldid[b1], w2 = m.body_weldid[b2];
      if (w1 == w2) continue;
      if (!(m.disableflags & DSBL_FILTERPARENT)) {
        int w1p = w1 > 0 ? m.body_weldid[m.body_parentid[w1]] : 0;
        int w2p = w2 > 0 ? m.body_weldid[m.body_parentid[w2]] : 0;
        if (w1 != 0 && w2 != 0 && (w1 == w2p || w2 == w1p)) continue;
      }
      int sig = (std::min(b1, b2) << 16) | std::max(b1, b2);
      if (excl.count(sig)) continue;
      Pair p;
      p.g1 = g1; p.g2 = g2; p.b1 = b1; p.b2 = b2;
      p.margin = std::max(m.geom_margin[g1], m.geom_margin[g2]);
      p.gap = std::max(m.geom_gap[g1], m.geom_gap[g2]);
      mix_params(m, g1, g2, p);
      m.pairs.push_back(p);
    }
  for (auto& ep : m.explicit_pairs) {
    int g1 = ep.g1, g2 = ep.g2;
    if (m.geom_type[g1] > m.geom_type[g2]) std::swap(g1, g2);
    bool dup = false;
    for (auto& q : m.pairs)
      if ((q.g1 == g1 && q.g2 == g2) || (q.g1 == g2 && q.g2 == g1)) dup = true;
    if (dup || !has_collider(m.geom_type[g1], m.geom_type[g2])) continue;
    Pair p;
    p.g1 = g1; p.g2 = g2;
    p.b1 = m.geom_bodyid[g1]; p.b2 = m.geom_bodyid[g2];
    p.condim = ep.condim;
    p.margin = ep.margin;
    p.gap = ep.gap;
    for (int k = 0; k < 5; k++) p.friction[k] = ep.friction[k];
    for (int k = 0; k < 2; k++) p.solref[k] = ep.solref[k];
    for (int k = 0; k < 5; k++) p.solimp[k] = ep.solimp[k];
    p.is_explicit = 1;
    m.pairs.push_back(p);
  }
  m.max_contacts_bound = 0;
  for (auto& p : m.pairs) {
    p.invw_t = m.body_invweight0[2 * p.b1] + m.body_invweight0[2 * p.b2];
    p.invw_r = m.body_invweight0[2 * p.b1 + 1] + m.body_invweight0[2 * p.b2 + 1];
    m.max_contacts_bound += pair_max_contacts(m.geom_type[p.g1], m.geom_type[p.g2]);
  }
}

}  // namespace

int pair_max_contacts(int t1, int t2) {
  if (t1 > t2) std::swap(t1, t2);
  if (t1 == GEOM_PLANE) {
    if (t2 == GEOM_CAPSULE) return 2;
    if (t2 == GEOM_BOX) return 4;
    return 1;
  }
  if (t1 == GEOM_BOX && t2 == GEOM_BOX) return 4;
  return 1;
}

void finalize_model(Model& m, const LoadOptions& opt) {
  int nb = m.nbody;
  // load options (reference: mjmlx.h:53-56)
  if (!opt.self_collision || opt.max_condim > 0) {
    for (int g = 0; g < m.ngeom; g++) {
      int b = m.geom_bodyid[g];
      bool robot = false;
      for (int a = b; a > 0; a = m.body_parentid[a])
        if (m.body_jntnum[a] > 0) robot = true;
      if (!robot) continue;
      if (!opt.self_collision) m.geom_conaffinity[g] = 0;
      if (opt.max_condim > 0) m.geom_condim[g] = std::min(m.geom_condim[g], opt.max_condim);
    }
  }
  m.body_rootid.assign(nb, 0);
  m.body_weldid.assign(nb, 0);
  m.body_depth.assign(nb, 0);
  m.body_subtreesize.assign(nb, 1);
  for (int b = 1; b < nb; b++) {
    int p = m.body_parentid[b];
    if (p >= b) fail("bodies must be stored parent-first");
    m.body_rootid[b] = (p == 0) ? b : m.body_rootid[p];
    m.body_weldid[b] = m.body_jntnum[b] > 0 ? b : m.body_weldid[p];
    m.body_depth[b] = m.body_depth[p] + 1;
  }
  for (int b = nb - 1; b > 0; b--) m.body_subtreesize[m.body_parentid[b]] += m.body_subtreesize[b];
  // dof parents
  m.dof_parentid.assign(m.nv, -1);
  for (int i = 0; i < m.nv; i++) {
    int b = m.dof_bodyid[i];
    if (i > m.body_dofadr[b]) { m.dof_parentid[i] = i - 1; continue; }
    int p = m.body_parentid[b];
    while (p > 0 && m.body_dofnum[p] == 0) p = m.body_parentid[p];
    m.dof_parentid[i] = (p > 0) ? m.body_dofadr[p] + m.body_dofnum[p] - 1 : -1;
  }
  // geoms per body (geoms are stored grouped by body in document order, which
  // need not be contiguous: record first and count only for contiguous runs)
  m.body_geomnum.assign(nb, 0);
  m.body_geomadr.assign(nb, -1);
  for (int g = 0; g < m.ngeom; g++) {
    int b = m.geom_bodyid[g];
    if (m.body_geomadr[b] < 0) m.body_geomadr[b] = g;
    m.body_geomnum[b]++;
  }
  for (int g = 0; g < m.ngeom; g++) {
    const double* s = &m.geom_size[3 * g];
    double r = 0;
    switch (m.geom_type[g]) {
      case GEOM_PLANE: r = 0; break;
      case GEOM_SPHERE: r = s[0]; break;
      case GEOM_CAPSULE: r = s[0] + s[1]; break;
      case GEOM_CYLINDER: r = std::sqrt(s[0] * s[0] + s[1] * s[1]); break;
      case GEOM_BOX: r = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]); break;
      case GEOM_ELLIPSOID: r = std::max(s[0], std::max(s[1], s[2])); break;
      case GEOM_MESH: {
        int md = m.geom_dataid[g];
        for (int v = 0; v < m.mesh_vertnum[md]; v++) {
          const double* p = &m.mesh_vert[3 * (m.mesh_vertadr[md] + v)];
          r = std::max(r, std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]));
        }
        break;
      }
    }
    m.geom_rbound[g] = r;
  }
  if (m.qpos_spring.size() != (size_t)m.nq) m.qpos_spring = m.qpos0;
  compute_invweights(m);
  // joint equality regulariser: sum of the coupled dofs' invweights
  for (size_t e = 0; e < m.eq_type.size(); e++) {
    if (m.eq_type[e] == 2) {
      double w = m.dof_invweight0[m.jnt_dofadr[m.eq_obj1[e]]];
      if (m.eq_obj2[e] >= 0) w += m.dof_invweight0[m.jnt_dofadr[m.eq_obj2[e]]];
      m.eq_invweight[e] = w;
    } else if (m.eq_type[e] == 3) {
      double w = m.tendon_invweight0[m.eq_obj1[e]];
      if (m.eq_obj2[e] >= 0) w += m.tendon_invweight0[m.eq_obj2[e]];
      m.eq_invweight[e] = w;
    }
  }
  build_pairs(m);
}

Model compile_mjcf(const std::string& xml, const LoadOptions& opt, const std::string& base_dir) {
  XmlNode root = parse_xml(xml);
  Compiler c;
  c.opt = opt;
  c.base_dir = base_dir;
  c.compile(root);
  finalize_model(c.m, opt);
  return c.m;
}

std::string dump_model(const Model& m) {
  std::ostringstream os;
  os.precision(17);
  auto di = [&](const char* name, const std::vector<int>& v) {
    os << name << " i " << v.size();
    for (int x : v) os << ' ' << x;
    os << '\n';
  };
  auto dd = [&](const char* name, const std::vector<double>& v) {
    os << name << " f " << v.size();
    for (double x : v) os << ' ' << x;
    os << '\n';
  };
  di("sizes", {m.nq, m.nv, m.nu, m.nbody, m.njnt, m.ngeom, m.nmesh, (int)m.pairs.size(), m.max_contacts_bound});
  di("opt_int", {m.iterations, m.ls_iterations, m.cone, m.integrator, m.disableflags});
  dd("opt_real", {m.timestep, m.gravity[0], m.gravity[1], m.gravity[2], m.tolerance, m.ls_tolerance, m.impratio, m.meaninertia});
  di("body_parentid", m.body_parentid); di("body_rootid", m.body_rootid); di("body_weldid", m.body_weldid);
  di("body_jntnum", m.body_jntnum); di("body_jntadr", m.body_jntadr); di("body_dofnum", m.body_dofnum);
  di("body_dofadr", m.body_dofadr); di("body_subtreesize", m.body_subtreesize); di("body_depth", m.body_depth);
  dd("body_pos", m.body_pos); dd("body_quat", m.body_quat); dd("body_ipos", m.body_ipos); dd("body_iquat", m.body_iquat);
  dd("body_mass", m.body_mass); dd("body_inertia", m.body_inertia); dd("body_invweight0", m.body_invweight0);
  dd("body_gravcomp", m.body_gravcomp);
  di("jnt_type", m.jnt_type); di("jnt_qposadr", m.jnt_qposadr); di("jnt_dofadr", m.jnt_dofadr); di("jnt_bodyid", m.jnt_bodyid);
  di("jnt_limited", m.jnt_limited);
  dd("jnt_pos", m.jnt_pos); dd("jnt_axis", m.jnt_axis); dd("jnt_range", m.jnt_range); dd("jnt_margin", m.jnt_margin);
  dd("jnt_solref", m.jnt_solref); dd("jnt_solimp", m.jnt_solimp); dd("jnt_stiffness", m.jnt_stiffness);
  di("dof_bodyid", m.dof_bodyid); di("dof_jntid", m.dof_jntid); di("dof_parentid", m.dof_parentid);
  dd("dof_armature", m.dof_armature); dd("dof_damping", m.dof_damping); dd("dof_frictionloss", m.dof_frictionloss);
  dd("dof_invweight0", m.dof_invweight0); dd("dof_solref", m.dof_solref); dd("dof_solimp", m.dof_solimp);
  dd("qpos0", m.qpos0); dd("qpos_spring", m.qpos_spring);
  di("geom_type", m.geom_type); di("geom_bodyid", m.geom_bodyid); di("geom_contype", m.geom_contype);
  di("geom_conaffinity", m.geom_conaffinity); di("geom_condim", m.geom_condim); di("geom_priority", m.geom_priority);
  di("geom_dataid", m.geom_dataid);
  dd("geom_pos", m.geom_pos); dd("geom_quat", m.geom_quat); dd("geom_size", m.geom_size); dd("geom_friction", m.geom_friction);
  dd("geom_solref", m.geom_solref); dd("geom_solimp", m.geom_solimp); dd("geom_solmix", m.geom_solmix);
  dd("geom_margin", m.geom_margin); dd("geom_gap", m.geom_gap); dd("geom_rbound", m.geom_rbound);
  di("mesh_vertadr", m.mesh_vertadr); di("mesh_vertnum", m.mesh_vertnum); dd("mesh_vert", m.mesh_vert);
  di("actuator_trntype", m.actuator_trntype); di("actuator_trnid", m.actuator_trnid); di("actuator_gaintype", m.actuator_gaintype); di("actuator_biastype", m.actuator_biastype);
  di("actuator_ctrllimited", m.actuator_ctrllimited); di("actuator_forcelimited", m.actuator_forcelimited);
  dd("actuator_gear", m.actuator_gear); dd("actuator_gainprm", m.actuator_gainprm); dd("actuator_biasprm", m.actuator_biasprm);
  dd("actuator_ctrlrange", m.actuator_ctrlrange); dd("actuator_forcerange", m.actuator_forcerange);
  di("exclude_body1", m.exclude_body1); di("exclude_body2", m.exclude_body2);
  di("wrap_type", m.wrap_type); di("tendon_adr", m.tendon_adr); di("tendon_num", m.tendon_num); di("tendon_limited", m.tendon_limited); di("wrap_objid", m.wrap_objid);
  dd("wrap_prm", m.wrap_prm); dd("tendon_range", m.tendon_range); dd("tendon_margin", m.tendon_margin);
  dd("tendon_frictionloss", m.tendon_frictionloss); dd("tendon_stiffness", m.tendon_stiffness); dd("tendon_damping", m.tendon_damping);
  dd("tendon_lengthspring", m.tendon_lengthspring); dd("tendon_solref_lim", m.tendon_solref_lim); dd("tendon_solimp_lim", m.tendon_solimp_lim);
  dd("tendon_solref_fri", m.tendon_solref_fri); dd("tendon_solimp_fri", m.tendon_solimp_fri); dd("tendon_length0", m.tendon_length0);
  dd("tendon_invweight0", m.tendon_invweight0);
  di("site_bodyid", m.site_bodyid); dd("site_pos", m.site_pos); dd("site_quat", m.site_quat);
  di("sensor_type", m.sensor_type); di("sensor_objtype", m.sensor_objtype); di("sensor_objid", m.sensor_objid);
  di("sensor_dim", m.sensor_dim); di("sensor_adr", m.sensor_adr); di("sensor_supported", m.sensor_supported);
  dd("magnetic", {m.magnetic[0], m.magnetic[1], m.magnetic[2]});
  di("eq_type", m.eq_type); di("eq_obj1", m.eq_obj1); di("eq_obj2", m.eq_obj2); di("eq_active", m.eq_active);
  dd("eq_data", m.eq_data); dd("eq_solref", m.eq_solref); dd("eq_solimp", m.eq_solimp); dd("eq_invweight", m.eq_invweight);
  std::vector<int> ep_i;
  std::vector<double> ep_f;
  for (auto& e : m.explicit_pairs) {
    ep_i.insert(ep_i.end(), {e.g1, e.g2, e.condim});
    ep_f.insert(ep_f.end(), e.friction, e.friction + 5);
    ep_f.insert(ep_f.end(), e.solref, e.solref + 2);
    ep_f.insert(ep_f.end(), e.solimp, e.solimp + 5);
    ep_f.push_back(e.margin);
    ep_f.push_back(e.gap);
  }
  di("explicit_pair_int", ep_i);
  dd("explicit_pair_real", ep_f);
  std::vector<int> pi;
  std::vector<double> pf;
  for (auto& p : m.pairs) {
    pi.insert(pi.end(), {p.g1, p.g2, p.b1, p.b2, p.condim, p.is_explicit});
    pf.insert(pf.end(), {p.margin, p.gap});
    pf.insert(pf.end(), p.friction, p.friction + 5);
    pf.insert(pf.end(), p.solref, p.solref + 2);
    pf.insert(pf.end(), p.solimp, p.solimp + 5);
    pf.insert(pf.end(), {p.invw_t, p.invw_r});
  }
  di("pair_int", pi);
  dd("pair_real", pf);
  return os.str();
}

}  // namespace mjb
