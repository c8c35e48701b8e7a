#include "engine.h"
#include "warmstart.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>

cudaError_t mjb_launch_step(const StepParams& P, int grid, int warps_per_block, size_t smem_bytes, cudaStream_t stream);
cudaError_t mjb_occupancy(int warps_per_block, size_t smem_bytes, int convex, int* blocks_per_sm);
cudaError_t mjb_sub(int n, const float* a, const float* b, float* out, cudaStream_t s);
cudaError_t mjb_launch_pack(int B, int nq, int nv, int nbody, const float* qpos, const float* qvel, const float* cfrc, const float* qfa, const int* bodies,
                            int nsel, int dof_lo, int ndof, int stride, float* out, cudaStream_t s);
cudaError_t mjb_launch_geom_pose(const StepParams& P, float* gpose, int ng_max, int warps_per_block, size_t smem_bytes, cudaStream_t stream);
cudaError_t mjb_launch_ray(int B, int nray, const int* env_model, const int* geom_base, const int* geom_count, const float* ginfo, const float* gpose,
                           int ng_max, const float* pnt, const float* vec, float* dist, int* geomid, cudaStream_t s);
cudaError_t mjb_launch_reset(const DevModelDesc* models, const int* env_model, const int* qadr, const int* vadr, const float* ftab, const int* mask, int B,
                             float* qpos, float* qvel, float* warm, int* sens_valid, cudaStream_t s);

namespace mjb {

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

// The zero fill runs on the legacy default stream, which the engine's
// non-blocking streams are not ordered after; it is waited for here, so a
// copy or kernel issued next on any stream cannot be overtaken by it.
template <class T>
void DevBuf<T>::alloc(size_t count) {
  release();
  n = count;
  if (count) {
    check(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
    check(cudaMemset(p, 0, count * sizeof(T)), "cudaMemset");
    check(cudaStreamSynchronize(nullptr), "cudaMemset sync");
  }
}
template <class T>
void DevBuf<T>::upload(const std::vector<T>& v, cudaStream_t s) {
  if (n < v.size() || !p) alloc(std::max<size_t>(v.size(), 1));
  if (!v.empty()) check(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
}
template struct DevBuf<float>;
template struct DevBuf<int>;
template struct DevBuf<DevModelDesc>;
template struct DevBuf<uint16_t>;
template struct DevBuf<unsigned long long>;
template struct DevBuf<double>;

namespace {

struct TableBuilder {
  std::vector<int>& it;
  std::vector<float>& ft;
  int ai(const std::vector<int>& v) {
    int o = (int)it.size();
    it.insert(it.end(), v.begin(), v.end());
    if (v.empty()) it.push_back(0);
    return o;
  }
  int af(const std::vector<double>& v) {
    int o = (int)ft.size();
    for (double x : v) ft.push_back((float)x);
    if (v.empty()) ft.push_back(0.f);
    return o;
  }
};

// Supported narrowphase type combinations (type-ordered).
// pair needing the GJK / EPA collider (no analytic one)
bool pair_convex(int t1, int t2) {
  if (t1 > t2) std::swap(t1, t2);
  if (t1 == GEOM_PLANE) return false;
  const bool analytic = (t1 == GEOM_SPHERE && (t2 == GEOM_SPHERE || t2 == GEOM_CAPSULE || t2 == GEOM_BOX)) ||
                        (t1 == GEOM_CAPSULE && (t2 == GEOM_CAPSULE || t2 == GEOM_BOX)) || (t1 == GEOM_BOX && t2 == GEOM_BOX);
  return !analytic;
}

bool pair_supported(int t1, int t2) {
  if (t1 == GEOM_PLANE) return t2 == GEOM_SPHERE || t2 == GEOM_CAPSULE || t2 == GEOM_BOX || t2 == GEOM_ELLIPSOID || t2 == GEOM_CYLINDER || t2 == GEOM_MESH;
  // every pair of convex primitives / meshes: analytic or GJK / EPA
  return t1 >= GEOM_SPHERE && t2 >= GEOM_SPHERE && t1 <= GEOM_MESH && t2 <= GEOM_MESH;
}

}  // namespace

Engine::Engine(const std::vector<const Model*>& models, const std::vector<int>& counts, int solver_iterations, int domain_rand, const EngineConfig& cfg)
    : models_(models), counts_(counts), cfg_(cfg) {
  if (models.empty() || models.size() != counts.size()) throw std::runtime_error("engine: need one count per model");
  for (int c : counts)
    if (c <= 0) throw std::runtime_error("engine: env counts must be positive");
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  cudaDeviceProp prop;
  check(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
  if (prop.major < 10) throw std::runtime_error("engine: this build targets sm_100a (B200); device is sm_" + std::to_string(prop.major * 10 + prop.minor));
  sm_count_ = prop.multiProcessorCount;
  if (const char* pz = std::getenv("MJB200_POISON_WORKSPACE")) poison_ = std::atoi(pz) != 0;
  check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  rand_on_ = domain_rand != 0;
  build_tables(cfg, solver_iterations);
  alloc_state();
  choose_launch();
}

Engine::~Engine() {
  if (stream_) cudaStreamSynchronize(stream_);
  invalidate_graphs();
  if (h_ctrl_pinned_) cudaFreeHost(h_ctrl_pinned_);
  if (ctrl_done_) cudaEventDestroy(ctrl_done_);
  for (auto& kv : h_stage_) cudaFreeHost(kv.second);
  if (stream_) cudaStreamDestroy(stream_);
}

void Engine::build_tables(const EngineConfig& cfg, int solver_iterations) {
  h_itab_.clear();
  h_ftab_.clear();
  layouts_.clear();
  TableBuilder tb{h_itab_, h_ftab_};
  ws_stride_ = 0;
  nv_max_ = 0;
  for (const Model* mp : models_) {
    const Model& m = *mp;
    for (auto& p : m.pairs) {
      int t1 = m.geom_type[p.g1], t2 = m.geom_type[p.g2];
      if (!pair_supported(t1, t2))
        throw std::runtime_error("engine: collision pair of geom types " + std::to_string(t1) + "-" + std::to_string(t2) + " has no collider in this build");
      if (pair_convex(t1, t2)) convex_ = true;
    }
    for (auto& p : m.pairs)
      if (p.condim != 1 && p.condim != 3 && p.condim != 4 && p.condim != 6) throw std::runtime_error("engine: condim must be 1, 3, 4 or 6");
    if (m.cone == CONE_ELLIPTIC) convex_ = true;   // the extended kernel instance carries the elliptic solver
    for (int j = 0; j < m.njnt; j++)
      if (m.jnt_limited[j] && m.jnt_type[j] == JNT_BALL) throw std::runtime_error("engine: limited ball joints are not supported");
    if (m.nv > 1024) throw std::runtime_error("engine: models with more than 1024 dofs are not supported by this build");
    DevModelDesc d;
    std::memset(&d, 0, sizeof(d));
    d.nq = m.nq; d.nv = m.nv; d.nu = m.nu; d.nbody = m.nbody; d.njnt = m.njnt; d.ngeom = m.ngeom;
    d.npair = (int)m.pairs.size(); d.nmesh = m.nmesh;
    d.cone = m.cone; d.disableflags = m.disableflags;
    d.iterations = cfg.max_iter > 0 ? cfg.max_iter : (solver_iterations > 0 ? solver_iterations : m.iterations);
    d.ls_iterations = m.ls_iterations;
    d.timestep = (float)m.timestep;
    for (int k = 0; k < 3; k++) d.gravity[k] = (float)m.gravity[k];
    for (int k = 0; k < 3; k++) d.magnetic[k] = (float)m.magnetic[k];
    d.tolerance = (float)(cfg.tolerance > 0 ? cfg.tolerance : m.tolerance);
    d.impratio = (float)m.impratio;
    d.scale = (float)(1.0 / (m.meaninertia * std::max(1, m.nv)));
    // levels (BFS by depth) and children
    int maxd = 0;
    for (int b = 0; b < m.nbody; b++) maxd = std::max(maxd, m.body_depth[b]);
    std::vector<int> level_start(maxd + 2, 0), level_body;
    for (int l = 0; l <= maxd; l++) {
      level_start[l] = (int)level_body.size();
      for (int b = 0; b < m.nbody; b++)
        if (m.body_depth[b] == l) level_body.push_back(b);
    }
    level_start[maxd + 1] = (int)level_body.size();
    d.nlevel = maxd + 1;
    std::vector<int> child_start(m.nbody + 1, 0), child_list;
    for (int b = 0; b < m.nbody; b++) {
      child_start[b] = (int)child_list.size();
      for (int c = 1; c < m.nbody; c++)
        if (m.body_parentid[c] == b) child_list.push_back(c);
    }
    child_start[m.nbody] = (int)child_list.size();
    d.i_body_parentid = tb.ai(m.body_parentid);
    d.i_body_rootid = tb.ai(m.body_rootid);
    d.i_body_jntadr = tb.ai(m.body_jntadr);
    d.i_body_jntnum = tb.ai(m.body_jntnum);
    d.i_body_dofadr = tb.ai(m.body_dofadr);
    d.i_body_dofnum = tb.ai(m.body_dofnum);
    d.i_body_subtreesize = tb.ai(m.body_subtreesize);
    d.i_level_start = tb.ai(level_start);
    d.i_level_body = tb.ai(level_body);
    d.i_child_start = tb.ai(child_start);
    d.i_child_list = tb.ai(child_list);
    d.i_jnt_type = tb.ai(m.jnt_type);
    d.i_jnt_qposadr = tb.ai(m.jnt_qposadr);
    d.i_jnt_dofadr = tb.ai(m.jnt_dofadr);
    d.i_dof_bodyid = tb.ai(m.dof_bodyid);
    d.i_dof_jntid = tb.ai(m.dof_jntid);
    d.i_dof_parentid = tb.ai(m.dof_parentid);
    d.i_geom_type = tb.ai(m.geom_type);
    d.i_geom_bodyid = tb.ai(m.geom_bodyid);
    d.i_geom_dataid = tb.ai(m.geom_dataid);
    std::vector<int> pi;
    std::vector<double> pf;
    for (auto& p : m.pairs) {
      pi.insert(pi.end(), {p.g1, p.g2, p.b1, p.b2, p.condim, pair_max_contacts(m.geom_type[p.g1], m.geom_type[p.g2])});
      pf.insert(pf.end(), {p.margin, p.margin - p.gap});
      pf.insert(pf.end(), p.friction, p.friction + 5);
      pf.insert(pf.end(), p.solref, p.solref + 2);
      pf.insert(pf.end(), p.solimp, p.solimp + 5);
      pf.insert(pf.end(), {p.invw_t, p.invw_r});
    }
    d.i_pair = tb.ai(pi);
    d.f_pair = tb.af(pf);
    std::vector<int> li;
    std::vector<double> lf;
    for (int j = 0; j < m.njnt; j++) {
      if (!m.jnt_limited[j] || (m.jnt_type[j] != JNT_HINGE && m.jnt_type[j] != JNT_SLIDE)) continue;
      li.insert(li.end(), {j, m.jnt_dofadr[j], m.jnt_qposadr[j]});
      lf.insert(lf.end(), {m.jnt_range[2 * j], m.jnt_range[2 * j + 1], m.jnt_margin[j], m.jnt_solref[2 * j], m.jnt_solref[2 * j + 1]});
      lf.insert(lf.end(), &m.jnt_solimp[5 * j], &m.jnt_solimp[5 * j] + 5);
    }
    d.nlimit = (int)li.size() / 3;
    d.i_limit = tb.ai(li);
    d.f_limit = tb.af(lf);
    std::vector<int> fi;
    std::vector<double> ff;
    for (int i = 0; i < m.nv; i++) {
      if (m.dof_frictionloss[i] <= 0) continue;
      fi.push_back(i);
      ff.insert(ff.end(), {m.dof_frictionloss[i], m.dof_solref[2 * i], m.dof_solref[2 * i + 1]});
      ff.insert(ff.end(), &m.dof_solimp[5 * i], &m.dof_solimp[5 * i] + 5);
    }
    d.nfloss = (int)fi.size();
    d.i_floss = tb.ai(fi);
    d.f_floss = tb.af(ff);
    // fixed tendons (reference: build_tendon_host, batched.cpp:100-136, and
    // the tendon limit / friction tables, batched.cpp:480-530)
    std::vector<int> ti, wi, tfl, tlim, tpas;
    std::vector<double> wf, tf;
    for (int t = 0; t < m.ntendon; t++) {
      ti.insert(ti.end(), {m.tendon_adr[t], m.tendon_num[t], m.tendon_limited[t]});
      tf.insert(tf.end(), {m.tendon_range[2 * t], m.tendon_range[2 * t + 1], m.tendon_margin[t], m.tendon_frictionloss[t], m.tendon_stiffness[t],
                           m.tendon_damping[t], m.tendon_lengthspring[2 * t], m.tendon_lengthspring[2 * t + 1]});
      tf.insert(tf.end(), &m.tendon_solref_lim[2 * t], &m.tendon_solref_lim[2 * t] + 2);
      tf.insert(tf.end(), &m.tendon_solimp_lim[5 * t], &m.tendon_solimp_lim[5 * t] + 5);
      tf.insert(tf.end(), &m.tendon_solref_fri[2 * t], &m.tendon_solref_fri[2 * t] + 2);
      tf.insert(tf.end(), &m.tendon_solimp_fri[5 * t], &m.tendon_solimp_fri[5 * t] + 5);
      tf.insert(tf.end(), {m.tendon_invweight0[t], m.tendon_length0[t]});
      if (m.tendon_frictionloss[t] > 0) tfl.push_back(t);
      if (m.tendon_limited[t]) tlim.push_back(t);
      if (m.tendon_stiffness[t] != 0 || m.tendon_damping[t] != 0) tpas.push_back(t);
    }
    int max_pieces = 1;
    for (int t = 0; t < m.ntendon; t++) max_pieces = std::max(max_pieces, m.tendon_num[t]);
    for (size_t w = 0; w < m.wrap_objid.size(); w++) {
      const int ty = m.wrap_type[w], id = m.wrap_objid[w];
      if (ty == 1) wi.insert(wi.end(), {1, m.jnt_dofadr[id], m.jnt_qposadr[id]});
      else if (ty == 2) wi.insert(wi.end(), {2, 0, 0});
      else if (ty == 3) wi.insert(wi.end(), {3, id, m.site_bodyid[id]});
      else wi.insert(wi.end(), {ty, id, (int)m.wrap_prm[w]});
      wf.push_back(ty == 1 || ty == 2 ? m.wrap_prm[w] : 0.0);
    }
    d.i_site_body = tb.ai(m.site_bodyid);
    d.f_site = tb.af(m.site_pos);
    d.ntendon = m.ntendon;
    d.i_ten = tb.ai(ti);
    d.i_wrap = tb.ai(wi);
    d.f_wrap = tb.af(wf);
    d.f_ten = tb.af(tf);
    d.ntfloss = (int)tfl.size();
    d.i_tfloss = tb.ai(tfl);
    d.ntlimit = (int)tlim.size();
    d.i_tlimit = tb.ai(tlim);
    d.npten = (int)tpas.size();
    d.i_pten = tb.ai(tpas);
    // gravity compensation and free joints (reference: forward.hpp:438-464)
    std::vector<int> gci, fri;
    std::vector<double> gcf;
    for (int b = 1; b < m.nbody; b++)
      if (m.body_gravcomp[b] != 0) { gci.push_back(b); gcf.push_back(m.body_gravcomp[b]); }
    for (int j = 0; j < m.njnt; j++)
      if (m.jnt_type[j] == JNT_FREE) fri.push_back(m.jnt_dofadr[j]);
    d.ngcomp = (int)gci.size();
    d.i_gcomp = tb.ai(gci);
    d.f_gcomp = tb.af(gcf);
    d.nfree = (int)fri.size();
    d.i_free = tb.ai(fri);
    // sensors (reference: make_sensor_ctx, sensor.cpp:99-210): the object
    // frame of frame / site sensors relative to its body, state addresses of
    // joint / actuator / tendon sensors, a slot per accelerometer
    std::vector<int> si;
    std::vector<double> sf;
    int nacc = 0;
    for (int k = 0; k < m.nsensor; k++) {
      const int type = m.sensor_supported[k] ? m.sensor_type[k] : -1, ot = m.sensor_objtype[k], id = m.sensor_objid[k];
      int body = 0, a = 0, b = -1, slot = -1;
      double lp[3] = {0, 0, 0}, lq[4] = {1, 0, 0, 0}, gear = 1;
      if (ot == OBJ_SITE) { body = m.site_bodyid[id]; std::copy_n(&m.site_pos[3 * id], 3, lp); std::copy_n(&m.site_quat[4 * id], 4, lq); }
      else if (ot == OBJ_GEOM) { body = m.geom_bodyid[id]; std::copy_n(&m.geom_pos[3 * id], 3, lp); std::copy_n(&m.geom_quat[4 * id], 4, lq); }
      else if (ot == OBJ_BODY || ot == OBJ_XBODY) {
        body = id;
        if (ot == OBJ_BODY && type != SENS_SUBTREECOM) { std::copy_n(&m.body_ipos[3 * id], 3, lp); std::copy_n(&m.body_iquat[4 * id], 4, lq); }
      }
      switch (type) {
        case SENS_JOINTPOS: case SENS_BALLQUAT: a = m.jnt_qposadr[id]; break;
        case SENS_JOINTVEL: case SENS_JOINTACTFRC: case SENS_BALLANGVEL: a = m.jnt_dofadr[id]; break;
        case SENS_TENDONPOS: case SENS_TENDONVEL: a = id; break;
        case SENS_SUBTREECOM: a = id; break;
        case SENS_ACTUATORPOS: case SENS_ACTUATORVEL:
          gear = m.actuator_gear[id];
          if (m.actuator_trntype[id] == 3) { a = m.actuator_trnid[id]; b = -1; }
          else { a = m.jnt_qposadr[m.actuator_trnid[id]]; b = m.jnt_dofadr[m.actuator_trnid[id]]; }
          break;
        case SENS_ACCELEROMETER: slot = nacc++; break;
        default: break;
      }
      si.insert(si.end(), {type, m.sensor_adr[k], m.sensor_dim[k], body, m.body_rootid[body], a, b, slot});
      sf.insert(sf.end(), lp, lp + 3);
      sf.insert(sf.end(), lq, lq + 4);
      sf.push_back(gear);
    }
    d.nsensor = m.nsensor;
    d.nsensordata = m.nsensordata;
    d.nsens_acc = nacc;
    d.i_sensor = tb.ai(si);
    d.f_sensor = tb.af(sf);
    // joint and tendon equalities (reference: build_solver_equality_table,
    // batched.cpp:411-455; tendon ones measure length - tendon_length0)
    std::vector<int> qi;
    std::vector<double> qf;
    if (!(m.disableflags & DSBL_EQUALITY)) {
      for (size_t e = 0; e < m.eq_type.size(); e++) {
        if (!m.eq_active[e]) continue;
        if (m.eq_type[e] != 2 && m.eq_type[e] != 3)
          throw std::runtime_error("engine: connect / weld equality constraints are not supported (joint and tendon equalities are)");
        const int o1 = m.eq_obj1[e], o2 = m.eq_obj2[e];
        if (m.eq_type[e] == 3) {
          qi.insert(qi.end(), {1, o1, o2, 0, 0});
          qf.push_back(m.tendon_length0[o1]);
          qf.push_back(o2 >= 0 ? m.tendon_length0[o2] : 0.0);
        } else {
          qi.insert(qi.end(), {0, m.jnt_dofadr[o1], o2 >= 0 ? m.jnt_dofadr[o2] : -1, m.jnt_qposadr[o1], o2 >= 0 ? m.jnt_qposadr[o2] : 0});
          qf.push_back(m.qpos0[m.jnt_qposadr[o1]]);
          qf.push_back(o2 >= 0 ? m.qpos0[m.jnt_qposadr[o2]] : 0.0);
        }
        qf.insert(qf.end(), &m.eq_data[5 * e], &m.eq_data[5 * e] + 5);
        qf.insert(qf.end(), &m.eq_solref[2 * e], &m.eq_solref[2 * e] + 2);
        qf.insert(qf.end(), &m.eq_solimp[5 * e], &m.eq_solimp[5 * e] + 5);
        qf.push_back(m.eq_invweight[e]);
      }
    }
    d.neq = (int)(qi.size() / 5);
    d.i_eq = tb.ai(qi);
    d.f_eq = tb.af(qf);
    std::vector<int> ai;
    std::vector<double> af;
    for (int a = 0; a < m.nu; a++) {
      const bool ten = m.actuator_trntype[a] == 3;
      int j = ten ? 0 : m.actuator_trnid[a];
      ai.insert(ai.end(), {ten ? -1 : m.jnt_dofadr[j], ten ? 0 : m.jnt_qposadr[j], m.actuator_gaintype[a], m.actuator_biastype[a],
                           m.actuator_ctrllimited[a], m.actuator_forcelimited[a], ten ? m.actuator_trnid[a] : -1});
      af.push_back(m.actuator_gear[a]);
      af.insert(af.end(), &m.actuator_gainprm[3 * a], &m.actuator_gainprm[3 * a] + 3);
      af.insert(af.end(), &m.actuator_biasprm[3 * a], &m.actuator_biasprm[3 * a] + 3);
      af.insert(af.end(), {m.actuator_ctrlrange[2 * a], m.actuator_ctrlrange[2 * a + 1], m.actuator_forcerange[2 * a], m.actuator_forcerange[2 * a + 1]});
    }
    d.i_act = tb.ai(ai);
    d.f_act = tb.af(af);
    std::vector<int> mi;
    for (int k = 0; k < m.nmesh; k++) mi.insert(mi.end(), {m.mesh_vertadr[k], m.mesh_vertnum[k]});
    d.i_mesh = tb.ai(mi);
    d.f_mesh_vert = tb.af(m.mesh_vert);
    d.f_body_pos = tb.af(m.body_pos);
    d.f_body_quat = tb.af(m.body_quat);
    d.f_body_ipos = tb.af(m.body_ipos);
    d.f_body_iquat = tb.af(m.body_iquat);
    d.f_body_mass = tb.af(m.body_mass);
    d.f_body_inertia = tb.af(m.body_inertia);
    d.f_jnt_pos = tb.af(m.jnt_pos);
    d.f_jnt_axis = tb.af(m.jnt_axis);
    d.f_jnt_stiffness = tb.af(m.jnt_stiffness);
    d.f_qpos0 = tb.af(m.qpos0);
    d.f_qpos_spring = tb.af(m.qpos_spring);
    d.f_dof_armature = tb.af(m.dof_armature);
    d.f_dof_damping = tb.af(m.dof_damping);
    d.f_dof_invweight0 = tb.af(m.dof_invweight0);
    d.f_geom_pos = tb.af(m.geom_pos);
    d.f_geom_quat = tb.af(m.geom_quat);
    d.f_geom_size = tb.af(m.geom_size);
    d.f_geom_rbound = tb.af(m.geom_rbound);
    // implicit damping (Euler with eulerdamp, or the implicit integrators)
    std::vector<double> damp(m.dof_damping);
    if (m.integrator == 2 || m.integrator == 3) {
      for (int a = 0; a < m.nu; a++) {
        if (!m.actuator_biastype[a] || m.actuator_trntype[a] != 0) continue;
        double gv = m.actuator_gaintype[a] ? m.actuator_gainprm[3 * a + 2] : 0;
        double bv = m.actuator_biasprm[3 * a + 2];
        if (gv != 0 || bv == 0) continue;
        double g = m.actuator_gear[a];
        damp[m.jnt_dofadr[m.actuator_trnid[a]]] += -bv * g * g;
      }
    } else if (m.disableflags & DSBL_EULERDAMP) {
      std::fill(damp.begin(), damp.end(), 0.0);
    }
    d.implicit = 0;
    for (double x : damp)
      if (x != 0) d.implicit = 1;
    d.f_dof_damping_implicit = tb.af(damp);
    // contact / row capacity
    int ncb = std::max(1, m.max_contacts_bound);
    d.ncon_max = cfg.ncon_max > 0 ? cfg.ncon_max : std::min(ncb, 24);
    int rows_per_con = 1;
    for (auto& p : m.pairs) rows_per_con = std::max(rows_per_con, p.condim == 1 ? 1 : m.cone == CONE_ELLIPTIC ? p.condim : 2 * (p.condim - 1));
    int rows_bound = d.neq + d.nfloss + d.ntfloss + 2 * (d.nlimit + d.ntlimit) + rows_per_con * d.ncon_max;
    d.nefc_max = cfg.nefc_max > 0 ? cfg.nefc_max : std::max(1, std::min(rows_bound, 64));
    // workspace layout
    int nv = m.nv, nb = m.nbody, nj = std::max(1, m.njnt), ng = std::max(1, m.ngeom), nu = std::max(1, m.nu);
    int off = 0;
    auto take = [&](int n) { int o = off; off += (n + 3) & ~3; return o; };
    d.w_qpos = take(m.nq); d.w_qvel = take(nv); d.w_ctrl = take(nu); d.w_x = take(nv); d.w_xwarm = take(nv);
    d.w_scom = take(3 * nb); d.w_cdof = take(6 * nv); d.w_M = take(nv * nv); d.w_qfs = take(nv); d.w_qas = take(nv); d.w_qfa = take(nv);
    d.w_vec = take(9 * nv); d.w_con = take(MJB_CONTACT_FLOATS * d.ncon_max); d.w_rowcon = 0;
    d.w_ten = take(std::max(1, m.ntendon * (nv + 2)));
    int kbase = off;
    d.w_xpos = take(3 * nb); d.w_xquat = take(4 * nb); d.w_xmat = take(9 * nb); d.w_xipos = take(3 * nb);
    d.w_xanchor = take(3 * nj); d.w_xaxis = take(3 * nj); d.w_gxpos = take(3 * ng); d.w_gxmat = take(9 * ng);
    d.w_cinert = take(10 * nb); d.w_crb = take(10 * nb); d.w_cvel = take(6 * nb); d.w_cdofdot = take(6 * nv);
    d.w_cacc = take(6 * nb); d.w_tmp = take(4 * nb);
    d.w_tseg = take(9 * max_pieces);
    int kend = off;
    off = kbase;
    d.ldh = nv <= 32 ? (nv + 3) & ~3 : nv;
    d.w_J = take(d.nefc_max * nv); d.w_efc = take((m.cone == CONE_ELLIPTIC ? MJB_EFC_FIELDS_ELLIPTIC : MJB_EFC_FIELDS) * d.nefc_max);
    d.w_H = take(nv <= 32 ? nv * d.ldh + 32 : nv * nv); d.w_active = take(d.nefc_max);
    d.w_nz = take(std::max(nv, 8));
    int send = off;
    d.ws_size = std::max(kend, send);
    ws_stride_ = std::max(ws_stride_, d.ws_size);
    nv_max_ = std::max(nv_max_, nv);
    ModelLayout L;
    L.desc = d;
    L.nq = m.nq; L.nv = m.nv; L.nu = m.nu; L.nbody = m.nbody;
    layouts_.push_back(L);
  }
  desc_words_ = MJB_DESC_COPY_WORDS + MJB_ENV_SLOT_WORDS;
  std::vector<DevModelDesc> descs;
  for (auto& L : layouts_) descs.push_back(L.desc);
  // copies ordered on the sim's stream (a blocking cudaMemcpy from pageable
  // memory may return before its DMA lands, and the non-blocking stream is
  // not ordered after the legacy stream it runs on)
  d_models_.alloc(descs.size());
  check(cudaMemcpyAsync(d_models_.p, descs.data(), descs.size() * sizeof(DevModelDesc), cudaMemcpyHostToDevice, stream_), "upload models");
  d_itab_.alloc(h_itab_.size());
  check(cudaMemcpyAsync(d_itab_.p, h_itab_.data(), h_itab_.size() * 4, cudaMemcpyHostToDevice, stream_), "upload itab");
  d_ftab_.alloc(h_ftab_.size());
  check(cudaMemcpyAsync(d_ftab_.p, h_ftab_.data(), h_ftab_.size() * 4, cudaMemcpyHostToDevice, stream_), "upload ftab");
  check(cudaStreamSynchronize(stream_), "upload sync");
}

void Engine::alloc_state() {
  B_ = 0;
  for (int c : counts_) B_ += c;
  h_model_.assign(B_, 0);
  h_qadr_.assign(B_, 0);
  h_vadr_.assign(B_, 0);
  h_uadr_.assign(B_, 0);
  h_badr_.assign(B_, 0);
  int e = 0, q = 0, v = 0, u = 0, b = 0;
  for (size_t mi = 0; mi < models_.size(); mi++)
    for (int k = 0; k < counts_[mi]; k++, e++) {
      const Model& m = *models_[mi];
      h_model_[e] = (int)mi;
      h_qadr_[e] = q; h_vadr_[e] = v; h_uadr_[e] = u; h_badr_[e] = b;
      q += m.nq; v += m.nv; u += std::max(m.nu, 0); b += m.nbody;
    }
  tot_q_ = q; tot_v_ = v; tot_u_ = u; tot_b_ = b;
  h_fadr_.assign(B_, 0);
  int fr = 0;
  for (int i = 0; i < B_; i++) {
    h_fadr_[i] = fr;
    fr += layouts_[h_model_[i]].desc.nfree;
  }
  tot_f_ = fr;
  d_fadr_.upload(h_fadr_, stream_);
  // sensordata and accelerometer history addresses
  h_sadr_.assign(B_, 0);
  h_aadr_.assign(B_, 0);
  int sd = 0, ac = 0;
  for (int i = 0; i < B_; i++) {
    const DevModelDesc& dm = layouts_[h_model_[i]].desc;
    h_sadr_[i] = sd;
    h_aadr_[i] = ac;
    sd += dm.nsensordata;
    ac += 3 * dm.nsens_acc;
  }
  tot_s_ = sd;
  tot_a_ = ac;
  d_sadr_.upload(h_sadr_, stream_);
  d_aadr_.upload(h_aadr_, stream_);
  sensordata_.alloc(std::max(sd, 1));
  check(cudaMemsetAsync(sensordata_.p, 0, sizeof(float) * std::max(sd, 1), stream_), "sensordata zero");
  sens_prev_.alloc(std::max(ac, 1));
  sens_valid_.alloc(B_);
  check(cudaMemsetAsync(sens_valid_.p, 0, sizeof(int) * B_, stream_), "sensor history zero");
  d_model_.upload(h_model_, stream_);
  d_qadr_.upload(h_qadr_, stream_);
  d_vadr_.upload(h_vadr_, stream_);
  d_uadr_.upload(h_uadr_, stream_);
  d_badr_.upload(h_badr_, stream_);
  std::vector<float> q0(q);
  for (int i = 0; i < B_; i++) {
    const Model& m = *models_[h_model_[i]];
    for (int k = 0; k < m.nq; k++) q0[h_qadr_[i] + k] = (float)m.qpos0[k];
  }
  qpos0_.upload(q0, stream_);
  qpos_.upload(q0, stream_);
  qvel_.alloc(std::max(v, 1));
  ctrl_.alloc(std::max(u, 1));
  warm_.alloc(std::max(v, 1));
  pred_.alloc(std::max(v, 1));
  for (auto* buf : {&status_, &niter_sum_, &niter_max_, &ncon_, &nefc_, &choice_}) buf->alloc(B_);
  counter_.alloc(1);
  rec_xpos_.alloc(3 * b); rec_xquat_.alloc(4 * b); rec_scom_.alloc(3 * b); rec_cinert_.alloc(10 * b); rec_cvel_.alloc(6 * b);
  rec_qfa_.alloc(std::max(v, 1)); rec_cfrc_.alloc(6 * b); rec_qacc_.alloc(std::max(v, 1));
  check(cudaMallocHost(&h_ctrl_pinned_, sizeof(float) * std::max(u, 1)), "cudaMallocHost");
  if (rand_on_) {
    h_rand_mass_.assign(b, 1.f);
    h_rand_fric_.assign(B_, 1.f);
    h_rand_gain_.assign(std::max(u, 1), 1.f);
    h_rand_com_.assign(3 * std::max(b, 1), 0.f);
    h_rand_drag_.assign(std::max(tot_f_, 1), 0.f);
    rand_mass_.upload(h_rand_mass_, stream_);
    rand_fric_.upload(h_rand_fric_, stream_);
    rand_gain_.upload(h_rand_gain_, stream_);
    rand_com_.upload(h_rand_com_, stream_);
    rand_drag_.upload(h_rand_drag_, stream_);
  }
  check(cudaStreamSynchronize(stream_), "init sync");
}

// Dynamic shared memory available to one step-kernel CTA: the 227 KB a CTA
// can hold on sm_100, less the kernel's few static bytes (stage-clock slots).
constexpr int kStepSmemMax = 227 * 1024 - 64;

void Engine::choose_launch() {
  lockstep_ = cfg_.lockstep ? 1 : 0;
  // a workspace that does not fit shared memory (large models: the bin of
  // free bodies, nv in the hundreds) lives in HBM, one per resident warp;
  // shared memory then holds the model descriptors only
  gws_mode_ = (desc_words_ + ws_stride_) * 4 > kStepSmemMax;
  const int per_warp = (desc_words_ + (gws_mode_ ? 0 : ws_stride_)) * 4;
  if (cfg_.warps_per_block > 0) warps_ = cfg_.warps_per_block;
  else if (gws_mode_) warps_ = 4;
  else if (lockstep_ && 16 * per_warp <= kStepSmemMax) warps_ = 16;   // one lockstep CTA of 16 warps per SM (measured ~3 % faster than two of 8)
  else if (lockstep_) warps_ = std::max(1, std::min(8, (kStepSmemMax / 2) / per_warp));  // two lockstep CTAs of up to 8 warps per SM
  else warps_ = 4;
  smem_ = warps_ * per_warp;
  if (smem_ > kStepSmemMax) {
    warps_ = std::max(1, kStepSmemMax / per_warp);
    smem_ = warps_ * per_warp;
  }
  if (smem_ > kStepSmemMax) throw std::runtime_error("engine: per-env workspace exceeds shared memory (" + std::to_string(ws_stride_ * 4) + " bytes)");
  // the model int table in shared memory too, when the workspaces are there
  // and the table fits after them without costing a resident CTA: the
  // stages walk it in dependent chains (tree levels, parents, dof and joint
  // indices), and from global memory each link can miss the small L1 left
  // beside the workspaces.  (With HBM workspaces several small CTAs share an
  // SM, and a table copy in each halved the 64-body bin's throughput.)
  const int itab_bytes = (int)((h_itab_.size() * 4 + 15) & ~size_t(15));
  itab_smem_ = 0;
  if (!gws_mode_ && !h_itab_.empty() && smem_ + itab_bytes <= kStepSmemMax) {
    int b0 = 0, b1 = 0;
    check(mjb_occupancy(warps_, smem_, convex_, &b0), "occupancy");
    check(mjb_occupancy(warps_, smem_ + itab_bytes, convex_, &b1), "occupancy");
    if (b1 >= b0) {
      itab_smem_ = (int)h_itab_.size();
      smem_ += itab_bytes;
    }
  }
  int bps = 0;
  check(mjb_occupancy(warps_, smem_, convex_, &bps), "occupancy");
  if (bps < 1) throw std::runtime_error("engine: kernel cannot be resident with this configuration");
  if (cfg_.blocks_per_sm > 0) bps = std::min(bps, cfg_.blocks_per_sm);
  persistent_ = (lockstep_ || gws_mode_) ? 1 : (cfg_.persistent < 0 ? 1 : cfg_.persistent);
  if (persistent_) grid_ = std::min(sm_count_ * bps, (B_ + warps_ - 1) / warps_);
  else grid_ = (B_ + warps_ - 1) / warps_;
  grid_ = std::max(grid_, 1);
  if (gws_mode_) gws_.alloc((size_t)grid_ * warps_ * ws_stride_);
  else gws_.alloc(0);
}

void Engine::configure(const EngineConfig& cfg) {
  bool rebuild = cfg.ncon_max != cfg_.ncon_max || cfg.nefc_max != cfg_.nefc_max || cfg.tolerance != cfg_.tolerance || cfg.max_iter != cfg_.max_iter;
  const EngineConfig old = cfg_;
  cfg_ = cfg;
  sync();
  if (rebuild) build_tables(cfg_, 0);
  choose_launch();
  invalidate_graphs();
  if (fused_warmstart()) {
    const std::string why = fused_blocker();
    if (!why.empty()) {
      cfg_ = old;
      if (rebuild) build_tables(cfg_, 0);
      choose_launch();
      throw std::runtime_error("configure: the attached learned warm start " + why);
    }
  }
}

std::string Engine::fused_blocker() const {
  const Model& m = *models_[0];
  if (!lockstep_) return "needs lockstep CTAs (engine config lockstep = 1)";
  if (warps_ != 8 && warps_ != 16) return "needs CTAs of 8 or 16 warps (engine config warps_per_block)";
  if (gws_mode_) return "needs the workspaces in shared memory";
  if (convex_) return "is not built into the kernel instance for general convex pairs and elliptic cones";
  if (m.nv * m.nv < 256) return "needs nv * nv >= 256 (its activation rows use the Hessian slot of the workspace)";
  return "";
}

std::vector<Engine::TuneCandidate> Engine::autotune(int nsub, int reps) {
  if (nsub <= 0 || reps <= 0) throw std::runtime_error("autotune: nsub and reps must be positive");
  sync();
  DevBuf<float> sq, sv, sw;
  sq.alloc(tot_q_);
  sv.alloc(tot_v_);
  sw.alloc(tot_v_);
  auto copy = [&](float* dst, const float* src, size_t n) { check(cudaMemcpyAsync(dst, src, sizeof(float) * n, cudaMemcpyDeviceToDevice, stream_), "autotune copy"); };
  copy(sq.p, qpos_.p, tot_q_);
  copy(sv.p, qvel_.p, tot_v_);
  copy(sw.p, warm_.p, tot_v_);
  auto restore = [&]() {
    copy(qpos_.p, sq.p, tot_q_);
    copy(qvel_.p, sv.p, tot_v_);
    copy(warm_.p, sw.p, tot_v_);
  };
  const EngineConfig orig = cfg_;
  const int per_warp = (desc_words_ + (gws_mode_ ? 0 : ws_stride_)) * 4;
  std::vector<TuneCandidate> out;
  cudaEvent_t e0, e1;
  check(cudaEventCreate(&e0), "event");
  check(cudaEventCreate(&e1), "event");
  const bool feat_valid = feat_valid_;
  const bool fused = fused_warmstart();
  // CTA shapes: warps per CTA x lockstep, at the occupancy limit of CTAs
  // per SM, plus lockstep CTAs of 4 and 8 warps at one CTA per SM
  struct Shape {
    int w, lock, bps;
  };
  std::vector<Shape> shapes;
  for (int lock : {1, 0})
    for (int w : {2, 4, 8, 16}) shapes.push_back({w, lock, 0});
  shapes.push_back({4, 1, 1});
  shapes.push_back({8, 1, 1});
  for (const Shape& sh : shapes) {
    const int w = sh.w, lock = sh.lock;
    {
      TuneCandidate c{w, lock, sh.bps, -1.f};
      // an attached per-env net runs inside the kernel: lockstep, 8 or 16 warps
      if (w * per_warp > kStepSmemMax || (fused && (!lock || (w != 8 && w != 16)))) {
        out.push_back(c);
        continue;
      }
      EngineConfig cfg = orig;
      cfg.warps_per_block = w;
      cfg.lockstep = lock;
      cfg.persistent = 1;
      cfg.blocks_per_sm = sh.bps;
      try {
        configure(cfg);
      } catch (const std::exception&) {
        out.push_back(c);
        continue;
      }
      restore();
      launch(nsub, false);  // warm-up (and graph capture)
      restore();
      check(cudaEventRecord(e0, stream_), "event");
      for (int r = 0; r < reps; r++) launch(nsub, false);
      check(cudaEventRecord(e1, stream_), "event");
      check(cudaEventSynchronize(e1), "event sync");
      float ms = 0;
      check(cudaEventElapsedTime(&ms, e0, e1), "event time");
      c.ms = ms / reps;
      out.push_back(c);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const TuneCandidate* best = nullptr;
  for (auto& c : out)
    if (c.ms >= 0 && (!best || c.ms < best->ms)) best = &c;
  EngineConfig cfg = orig;
  if (best) {
    cfg.warps_per_block = best->warps_per_block;
    cfg.lockstep = best->lockstep;
    cfg.blocks_per_sm = best->blocks_per_sm;
    cfg.persistent = 1;
  }
  configure(cfg);
  restore();
  sync();
  feat_valid_ = feat_valid;
  return out;
}

namespace {
std::mutex g_tune_mutex;
std::map<uint64_t, Engine::TuneCandidate> g_tune_cache;

uint64_t fnv1a(uint64_t h, const void* p, size_t n) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  for (size_t i = 0; i < n; i++) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}
}  // namespace

bool Engine::autotune_cached(int nsub, int reps) {
  uint64_t key = 1469598103934665603ull;
  key = fnv1a(key, h_itab_.data(), h_itab_.size() * sizeof(int));
  key = fnv1a(key, h_ftab_.data(), h_ftab_.size() * sizeof(float));
  key = fnv1a(key, counts_.data(), counts_.size() * sizeof(int));
  for (const auto& L : layouts_) key = fnv1a(key, &L.desc, sizeof(L.desc));
  const int fused = fused_warmstart() ? 1 : 0;
  key = fnv1a(key, &fused, sizeof(fused));
  TuneCandidate hit{0, 0, 0, -1.f};
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) hit = it->second;
  }
  if (hit.warps_per_block > 0) {
    EngineConfig cfg = cfg_;
    cfg.warps_per_block = hit.warps_per_block;
    cfg.lockstep = hit.lockstep;
    cfg.blocks_per_sm = hit.blocks_per_sm;
    cfg.persistent = 1;
    configure(cfg);
    return true;
  }
  autotune(nsub, reps);
  TuneCandidate chosen{warps_, lockstep_, cfg_.blocks_per_sm, 0.f};
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tune_cache[key] = chosen;
  return false;
}

void Engine::launch_shape(int* grid, int* warps, int* smem, int* persistent) const {
  if (grid) *grid = grid_;
  if (warps) *warps = warps_;
  if (smem) *smem = smem_;
  if (persistent) *persistent = persistent_;
}

StepParams Engine::params(int n, bool record) {
  StepParams P;
  std::memset(&P, 0, sizeof(P));
  P.models = d_models_.p;
  P.itab = d_itab_.p;
  P.ftab = d_ftab_.p;
  P.num_envs = B_;
  P.env_model = d_model_.p;
  P.env_qadr = d_qadr_.p;
  P.env_vadr = d_vadr_.p;
  P.env_uadr = d_uadr_.p;
  P.env_badr = d_badr_.p;
  P.qpos = qpos_.p;
  P.qvel = qvel_.p;
  P.ctrl = ctrl_.p;
  P.qacc_warm = warm_.p;
  P.convex = convex_;
  P.nsub = n;
  P.max_iter = 0;
  P.work_counter = (persistent_ && !lockstep_) ? counter_.p : nullptr;
  P.lockstep = lockstep_;
  P.stage_cycles = timing_ ? stage_cycles_.p : nullptr;
  P.ws_stride = ws_stride_;
  P.desc_words = desc_words_;
  P.itab_smem = itab_smem_;
  if (gws_mode_) {
    P.gws = gws_.p;
    P.gws_blocks = grid_;
  }
  P.poison_workspace = poison_;
  P.status = status_.p;
  P.niter_sum = niter_sum_.p;
  P.niter_max = niter_max_.p;
  P.ncon_out = ncon_.p;
  P.nefc_out = nefc_.p;
  P.warm_choice = choice_.p;
  if (record) {
    P.rec_xpos = rec_xpos_.p;
    P.rec_xquat = rec_xquat_.p;
    P.rec_scom = rec_scom_.p;
    P.rec_cinert = rec_cinert_.p;
    P.rec_cvel = rec_cvel_.p;
    P.rec_qfrc_actuator = rec_qfa_.p;
    P.rec_cfrc_ext = rec_cfrc_.p;
    P.rec_qacc = rec_qacc_.p;
    if (dbg_ncon_ > 0) {
      P.dbg_contacts = dbg_con_.p;
      P.dbg_ncon_max = dbg_ncon_;
      P.dbg_efc = dbg_efc_.p;
      P.dbg_nefc_max = dbg_nefc_;
      P.dbg_vec = dbg_vec_.p;
      P.dbg_nv_max = nv_max_;
    }
  }
  if (rand_on_) {
    P.rand_mass = rand_mass_.p;
    P.rand_friction = rand_fric_.p;
    P.rand_gain = rand_gain_.p;
    if (com_on_) P.rand_com = rand_com_.p;
    if (drag_on_) {
      P.rand_drag = rand_drag_.p;
      P.env_fadr = d_fadr_.p;
    }
  }
  if (fused_warmstart()) {
    net_->fill_fused(P);
    P.feat_qskip = feature_qskip();
    if (record && dbg_ncon_ > 0 && dbg_feat_.p) {
      P.nn_feat_out = dbg_feat_.p;
      P.nn_pred_out = dbg_pred_.p;
    }
  }
  if (tot_s_ > 0) {
    if (record) P.sensordata = sensordata_.p;
    P.env_sadr = d_sadr_.p;
    if (tot_a_ > 0) {
      P.sens_prev = sens_prev_.p;
      P.env_aadr = d_aadr_.p;
      P.sens_valid = sens_valid_.p;
    }
  }
  return P;
}

StepParams Engine::external_params(float* qpos, float* qvel, const float* ctrl, float* qacc_warm, int n, int* work_counter, int* stats6) const {
  StepParams P;
  std::memset(&P, 0, sizeof(P));
  P.models = d_models_.p;
  P.itab = d_itab_.p;
  P.ftab = d_ftab_.p;
  P.num_envs = B_;
  P.env_model = d_model_.p;
  P.env_qadr = d_qadr_.p;
  P.env_vadr = d_vadr_.p;
  P.env_uadr = d_uadr_.p;
  P.env_badr = d_badr_.p;
  P.qpos = qpos;
  P.qvel = qvel;
  P.ctrl = ctrl;
  P.qacc_warm = qacc_warm;
  P.convex = convex_;
  P.nsub = n;
  P.work_counter = work_counter;
  P.lockstep = 0;
  P.ws_stride = ws_stride_;
  P.desc_words = desc_words_;
  P.itab_smem = itab_smem_;
  P.status = stats6;
  P.niter_sum = stats6 + B_;
  P.niter_max = stats6 + 2 * B_;
  P.ncon_out = stats6 + 3 * B_;
  P.nefc_out = stats6 + 4 * B_;
  P.warm_choice = stats6 + 5 * B_;
  if (rand_on_) {
    P.rand_mass = rand_mass_.p;
    P.rand_friction = rand_fric_.p;
    P.rand_gain = rand_gain_.p;
    if (com_on_) P.rand_com = rand_com_.p;
    if (drag_on_) {
      P.rand_drag = rand_drag_.p;
      P.env_fadr = d_fadr_.p;
    }
  }
  return P;
}

void Engine::invalidate_graphs() {
  for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
  graphs_.clear();
}

void Engine::launch_learned(int n, bool record) {
  const bool first_valid = feat_valid_;
  const Model& m = *models_[0];
  const int F = feature_count(), qskip = feature_qskip();
  const bool per_body = feature_per_body();
  // a prediction at substeps s % k == 0; each launch runs up to the next
  // prediction (the prediction is a warm-start candidate of its first
  // substep only; the kernel writes the features of every substep, so the
  // next prediction sees the latest)
  const int k = std::max(1, cfg_.predict_every);
  auto body = [&]() {
    for (int s = 0; s < n;) {
      const bool have = first_valid || s > 0;
      const int len = std::min(k, n - s);
      // per-body mode: B * (nbody - 1) rows of 6 outputs, which are the env-major [B][nv] layout
      if (have) net_->infer(feat_.p, feat_stride_, F, ctrl_.p, per_body ? 0 : m.nu, warm_.p, pred_.p, B_ * rows_per_env(), stream_);
      StepParams P = params(len, record && s + len == n);
      P.qacc_pred = have ? pred_.p : nullptr;
      P.features = feat_.p;
      P.feat_stride = feat_stride_;
      P.feat_qskip = qskip;
      P.feat_body = per_body;
      P.stats_accumulate = s > 0;
      if (persistent_ && !lockstep_) check(cudaMemsetAsync(counter_.p, 0, sizeof(int), stream_), "reset work counter");
      check(mjb_launch_step(P, grid_, warps_, smem_, stream_), "mjb_step_kernel launch");
      s += len;
    }
  };
  feat_valid_ = true;
  if (!cfg_.use_graph) {
    body();
    return;
  }
  auto key = std::make_pair(n, (record ? 1 : 0) | (first_valid ? 2 : 0) | 4);
  auto it = graphs_.find(key);
  if (it == graphs_.end()) {
    cudaGraph_t g;
    check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
    body();
    check(cudaStreamEndCapture(stream_, &g), "end capture");
    cudaGraphExec_t ge;
    check(cudaGraphInstantiate(&ge, g, 0), "graph instantiate");
    cudaGraphDestroy(g);
    it = graphs_.emplace(key, ge).first;
  }
  check(cudaGraphLaunch(it->second, stream_), "graph launch");
}

void Engine::launch(int n, bool record) {
  if (n <= 0) return;
  if (net_ && feature_per_body()) {
    launch_learned(n, record);
    return;
  }
  StepParams P = params(n, record);
  auto body = [&]() {
    if (persistent_ && !lockstep_) check(cudaMemsetAsync(counter_.p, 0, sizeof(int), stream_), "reset work counter");
    check(mjb_launch_step(P, grid_, warps_, smem_, stream_), "mjb_step_kernel launch");
  };
  if (!cfg_.use_graph) {
    body();
    return;
  }
  auto key = std::make_pair(n, record ? 1 : 0);
  auto it = graphs_.find(key);
  if (it == graphs_.end()) {
    cudaGraph_t g;
    check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
    body();
    check(cudaStreamEndCapture(stream_, &g), "end capture");
    cudaGraphExec_t ge;
    check(cudaGraphInstantiate(&ge, g, 0), "graph instantiate");
    cudaGraphDestroy(g);
    it = graphs_.emplace(key, ge).first;
  }
  check(cudaGraphLaunch(it->second, stream_), "graph launch");
}

void Engine::step(const float* ctrl_host, int n) {
  if (tot_u_ > 0) {
    if (ctrl_host) {
      cudaPointerAttributes pa{};
      const bool pinned = cudaPointerGetAttributes(&pa, ctrl_host) == cudaSuccess && pa.type == cudaMemoryTypeHost;
      if (pinned) {
        // page-locked caller buffer: DMA straight from it, and return once
        // the copy has landed so the caller may reuse the buffer
        check(cudaMemcpyAsync(ctrl_.p, ctrl_host, sizeof(float) * tot_u_, cudaMemcpyHostToDevice, stream_), "ctrl upload");
        if (!ctrl_done_) check(cudaEventCreateWithFlags(&ctrl_done_, cudaEventDisableTiming), "ctrl event");
        check(cudaEventRecord(ctrl_done_, stream_), "ctrl event record");
        launch(n, cfg_.record != 0);
        check(cudaEventSynchronize(ctrl_done_), "ctrl upload wait");
        return;
      }
      // pageable caller buffer: stage through pinned memory so the copy is
      // a true async DMA
      check(cudaStreamSynchronize(stream_), "ctrl staging sync");
      std::memcpy(h_ctrl_pinned_, ctrl_host, sizeof(float) * tot_u_);
      check(cudaMemcpyAsync(ctrl_.p, h_ctrl_pinned_, sizeof(float) * tot_u_, cudaMemcpyHostToDevice, stream_), "ctrl upload");
    } else {
      check(cudaMemsetAsync(ctrl_.p, 0, sizeof(float) * tot_u_, stream_), "ctrl zero");
    }
  }
  launch(n, cfg_.record != 0);
}

void Engine::step_device(int n) { launch(n, cfg_.record != 0); }

// d(qvel after one physics step) / d(ctrl) at the current state and the
// controls of the last step, by central differences (step eps = 1e-3 x
// max(1, |ctrl|)), one perturbed step per control and sign from the same
// saved state (position, velocity, warm start); the state is restored
// afterwards.  out[env][nv][nu], single-model batches.
void Engine::grad_step(float* out) {
  if (!uniform()) throw std::runtime_error("grad_step: needs a single-model batch");
  const Model& m = *models_[0];
  const int nv = m.nv, nu = m.nu;
  if (nu == 0 || nv == 0) return;
  sync();
  DevBuf<float> sq, sv, sw;
  sq.alloc(tot_q_);
  sv.alloc(tot_v_);
  sw.alloc(tot_v_);
  auto copy = [&](float* dst, const float* src, size_t n) { check(cudaMemcpyAsync(dst, src, sizeof(float) * n, cudaMemcpyDeviceToDevice, stream_), "grad copy"); };
  copy(sq.p, qpos_.p, tot_q_);
  copy(sv.p, qvel_.p, tot_v_);
  copy(sw.p, warm_.p, tot_v_);
  std::vector<float> c0(tot_u_), c(tot_u_), vp(tot_v_), vm(tot_v_);
  check(cudaMemcpyAsync(c0.data(), ctrl_.p, sizeof(float) * tot_u_, cudaMemcpyDeviceToHost, stream_), "grad ctrl");
  sync();
  auto probe = [&](int j, float sgn, std::vector<float>& v) {
    c = c0;
    for (int e = 0; e < B_; e++) c[(size_t)e * nu + j] += sgn * 1e-3f * std::max(1.f, std::fabs(c0[(size_t)e * nu + j]));
    check(cudaMemcpyAsync(ctrl_.p, c.data(), sizeof(float) * tot_u_, cudaMemcpyHostToDevice, stream_), "grad ctrl");
    copy(qpos_.p, sq.p, tot_q_);
    copy(qvel_.p, sv.p, tot_v_);
    copy(warm_.p, sw.p, tot_v_);
    launch(1, false);
    check(cudaMemcpyAsync(v.data(), qvel_.p, sizeof(float) * tot_v_, cudaMemcpyDeviceToHost, stream_), "grad qvel");
    sync();
  };
  for (int j = 0; j < nu; j++) {
    probe(j, 1.f, vp);
    probe(j, -1.f, vm);
    for (int e = 0; e < B_; e++) {
      const float h = 1e-3f * std::max(1.f, std::fabs(c0[(size_t)e * nu + j]));
      for (int i = 0; i < nv; i++) out[((size_t)e * nv + i) * nu + j] = (vp[(size_t)e * nv + i] - vm[(size_t)e * nv + i]) / (2.f * h);
    }
  }
  check(cudaMemcpyAsync(ctrl_.p, c0.data(), sizeof(float) * tot_u_, cudaMemcpyHostToDevice, stream_), "grad ctrl");
  copy(qpos_.p, sq.p, tot_q_);
  copy(qvel_.p, sv.p, tot_v_);
  copy(warm_.p, sw.p, tot_v_);
  feat_valid_ = false;
  sync();
}

void Engine::get_qacc_warmstart(float* out) {
  check(cudaMemcpyAsync(out, warm_.p, sizeof(float) * tot_v_, cudaMemcpyDeviceToHost, stream_), "get warm start");
  sync();
}

void Engine::set_qacc_warmstart(const float* in) {
  check(cudaMemcpyAsync(warm_.p, in, sizeof(float) * tot_v_, cudaMemcpyHostToDevice, stream_), "set warm start");
  sync();
}

void Engine::step_with_warmstart(const float* qacc, int n) {
  if (n <= 0) return;
  check(cudaMemcpyAsync(pred_.p, qacc, sizeof(float) * tot_v_, cudaMemcpyDeviceToDevice, stream_), "warm start copy");
  StepParams P = params(1, cfg_.record != 0 && n == 1);
  P.qacc_pred = pred_.p;
  P.nn_w[0] = nullptr;   // the caller's candidate, not the fused net's, for this substep
  if (persistent_ && !lockstep_) check(cudaMemsetAsync(counter_.p, 0, sizeof(int), stream_), "reset work counter");
  check(mjb_launch_step(P, grid_, warps_, smem_, stream_), "mjb_step_kernel launch");
  feat_valid_ = false;
  if (n > 1) launch(n - 1, cfg_.record != 0);
}

void Engine::step_device_ctrl(const float* dctrl, int n) {
  if (tot_u_ > 0 && dctrl) check(cudaMemcpyAsync(ctrl_.p, dctrl, sizeof(float) * tot_u_, cudaMemcpyDeviceToDevice, stream_), "ctrl device copy");
  launch(n, cfg_.record != 0);
}

void Engine::sync() { check(cudaStreamSynchronize(stream_), "stream sync"); }

void Engine::get_state(float* qpos, float* qvel) {
  if (qpos) check(cudaMemcpyAsync(qpos, qpos_.p, sizeof(float) * tot_q_, cudaMemcpyDeviceToHost, stream_), "get qpos");
  if (qvel) check(cudaMemcpyAsync(qvel, qvel_.p, sizeof(float) * tot_v_, cudaMemcpyDeviceToHost, stream_), "get qvel");
  sync();
}

// State setters copy on the sim's stream and wait: the next launch on that
// stream is ordered after the copy, and the caller's buffer is free on return.
void Engine::set_state(const float* qpos, const float* qvel) {
  feat_valid_ = false;
  if (qpos) check(cudaMemcpyAsync(qpos_.p, qpos, sizeof(float) * tot_q_, cudaMemcpyHostToDevice, stream_), "set qpos");
  if (qvel) check(cudaMemcpyAsync(qvel_.p, qvel, sizeof(float) * tot_v_, cudaMemcpyHostToDevice, stream_), "set qvel");
  sync();
}

void Engine::set_env_state(int env, const float* qpos, const float* qvel) {
  if (env < 0 || env >= B_) return;
  feat_valid_ = false;
  const Model& m = *models_[h_model_[env]];
  if (qpos) check(cudaMemcpyAsync(qpos_.p + h_qadr_[env], qpos, sizeof(float) * m.nq, cudaMemcpyHostToDevice, stream_), "set env qpos");
  if (qvel) check(cudaMemcpyAsync(qvel_.p + h_vadr_[env], qvel, sizeof(float) * m.nv, cudaMemcpyHostToDevice, stream_), "set env qvel");
  sync();
}

void Engine::reset(const int* mask) {
  if (!mask) return;
  feat_valid_ = false;
  DevBuf<int> dm;
  std::vector<int> hm(mask, mask + B_);
  dm.upload(hm, stream_);
  check(mjb_launch_reset(d_models_.p, d_model_.p, d_qadr_.p, d_vadr_.p, d_ftab_.p, dm.p, B_, qpos_.p, qvel_.p, warm_.p, sens_valid_.p, stream_), "reset kernel");
  sync();
}

const float* Engine::get_host(const char* what, int* n) {
  std::string w(what);
  float* src = nullptr;
  size_t cnt = 0;
  if (w == "qpos") { src = qpos_.p; cnt = tot_q_; }
  else if (w == "qvel") { src = qvel_.p; cnt = tot_v_; }
  else if (w == "xpos") { src = rec_xpos_.p; cnt = 3 * tot_b_; }
  else if (w == "xquat") { src = rec_xquat_.p; cnt = 4 * tot_b_; }
  else if (w == "subtree_com") { src = rec_scom_.p; cnt = 3 * tot_b_; }
  else if (w == "cinert") { src = rec_cinert_.p; cnt = 10 * tot_b_; }
  else if (w == "cvel") { src = rec_cvel_.p; cnt = 6 * tot_b_; }
  else if (w == "qfrc_actuator") { src = rec_qfa_.p; cnt = tot_v_; }
  else if (w == "cfrc_ext") { src = rec_cfrc_.p; cnt = 6 * tot_b_; }
  else if (w == "qacc") { src = rec_qacc_.p; cnt = tot_v_; }
  else if (w == "sensordata") {
    if (tot_s_ == 0) {
      if (n) *n = 0;
      return nullptr;
    }
    src = sensordata_.p;
    cnt = tot_s_;
  }
  else return nullptr;
  auto it = h_stage_.find(w);
  if (it == h_stage_.end()) {
    float* h = nullptr;
    check(cudaMallocHost(&h, sizeof(float) * std::max<size_t>(cnt, 1)), "cudaMallocHost");
    it = h_stage_.emplace(w, h).first;
    h_stage_n_[w] = cnt;
  }
  if (cnt) check(cudaMemcpyAsync(it->second, src, sizeof(float) * cnt, cudaMemcpyDeviceToHost, stream_), "getter copy");
  sync();
  if (n) *n = (int)cnt;
  return it->second;
}

void Engine::stats(int* status, int* niter_sum, int* niter_max, int* ncon, int* nefc, int* choice) {
  auto cp = [&](int* dst, DevBuf<int>& src) {
    if (dst) check(cudaMemcpyAsync(dst, src.p, sizeof(int) * B_, cudaMemcpyDeviceToHost, stream_), "stats copy");
  };
  cp(status, status_);
  cp(niter_sum, niter_sum_);
  cp(niter_max, niter_max_);
  cp(ncon, ncon_);
  cp(nefc, nefc_);
  cp(choice, choice_);
  sync();
}

void Engine::set_debug(int ncon_max, int nefc_max) {
  sync();
  dbg_ncon_ = std::max(0, ncon_max);
  dbg_nefc_ = std::max(0, nefc_max);
  if (dbg_ncon_ > 0) {
    dbg_con_.alloc((size_t)B_ * dbg_ncon_ * MJB_CONTACT_FLOATS);
    dbg_efc_.alloc((size_t)B_ * std::max(1, dbg_nefc_) * 4);
    dbg_vec_.alloc((size_t)B_ * 4 * nv_max_);
    if (uniform()) {
      dbg_feat_.alloc((size_t)B_ * warmstart_input_width());
      dbg_pred_.alloc(std::max(tot_v_, 1));
    }
  }
  invalidate_graphs();
}

int Engine::get_warmstart_debug(float* features, float* pred) {
  if (dbg_ncon_ <= 0 || !dbg_feat_.p || !fused_warmstart()) return -1;
  if (features) check(cudaMemcpyAsync(features, dbg_feat_.p, sizeof(float) * dbg_feat_.n, cudaMemcpyDeviceToHost, stream_), "dbg copy");
  if (pred) check(cudaMemcpyAsync(pred, dbg_pred_.p, sizeof(float) * tot_v_, cudaMemcpyDeviceToHost, stream_), "dbg copy");
  sync();
  return warmstart_input_width();
}

void Engine::get_debug(float* contacts, float* efc, float* vec) {
  if (dbg_ncon_ <= 0) return;
  if (contacts) check(cudaMemcpyAsync(contacts, dbg_con_.p, sizeof(float) * dbg_con_.n, cudaMemcpyDeviceToHost, stream_), "dbg copy");
  if (efc) check(cudaMemcpyAsync(efc, dbg_efc_.p, sizeof(float) * dbg_efc_.n, cudaMemcpyDeviceToHost, stream_), "dbg copy");
  if (vec) check(cudaMemcpyAsync(vec, dbg_vec_.p, sizeof(float) * dbg_vec_.n, cudaMemcpyDeviceToHost, stream_), "dbg copy");
  sync();
}

int Engine::set_env_params(const int* env_idx, int n, const float* mass_scale, const float* com_delta, const float* friction_scale, const float* gain_scale) {
  if (!rand_on_ || n < 0) return -1;
  if (!env_idx && n != B_) return -1;
  for (int i = 0; i < n; i++)
    if (env_idx && (env_idx[i] < 0 || env_idx[i] >= B_)) return -2;
  for (int i = 0; i < n; i++) {
    int e = env_idx ? env_idx[i] : i;
    const Model& m = *models_[h_model_[e]];
    if (mass_scale)
      for (int b = 0; b < m.nbody; b++) h_rand_mass_[h_badr_[e] + b] = mass_scale[(size_t)i * m.nbody + b];
    if (com_delta)
      for (int k = 0; k < 3 * m.nbody; k++) h_rand_com_[3 * h_badr_[e] + k] = com_delta[(size_t)i * 3 * m.nbody + k];
    if (friction_scale) h_rand_fric_[e] = friction_scale[i];
    if (gain_scale)
      for (int a = 0; a < m.nu; a++) h_rand_gain_[h_uadr_[e] + a] = gain_scale[(size_t)i * m.nu + a];
  }
  sync();
  rand_mass_.upload(h_rand_mass_, stream_);
  rand_fric_.upload(h_rand_fric_, stream_);
  rand_gain_.upload(h_rand_gain_, stream_);
  if (com_delta) {
    rand_com_.upload(h_rand_com_, stream_);
    if (!com_on_) invalidate_graphs();
    com_on_ = true;
  }
  sync();
  return 0;
}

int Engine::set_free_drag(const int* env_idx, int n, const float* drag_k) {
  if (!rand_on_ || n < 0 || !drag_k) return -1;
  if (tot_f_ == 0) return -3;
  if (!env_idx && n != B_) return -1;
  for (int i = 0; i < n; i++)
    if (env_idx && (env_idx[i] < 0 || env_idx[i] >= B_)) return -2;
  for (int i = 0; i < n; i++) {
    const int e = env_idx ? env_idx[i] : i;
    const int nf = layouts_[h_model_[e]].desc.nfree;
    for (int f = 0; f < nf; f++) h_rand_drag_[h_fadr_[e] + f] = drag_k[(size_t)i * nf + f];
  }
  sync();
  rand_drag_.upload(h_rand_drag_, stream_);
  if (!drag_on_) invalidate_graphs();
  drag_on_ = true;
  sync();
  return 0;
}

void Engine::stage_timing(int enable, unsigned long long* out8) {
  sync();
  if (out8) {
    if (timing_) {
      check(cudaMemcpyAsync(out8, stage_cycles_.p, 16 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_), "stage cycles");
      sync();
    } else {
      std::memset(out8, 0, 8 * sizeof(unsigned long long));
    }
  }
  if (enable >= 0) {
    bool on = enable != 0;
    if (on) {
      if (!stage_cycles_.p) stage_cycles_.alloc(16);
      check(cudaMemsetAsync(stage_cycles_.p, 0, 16 * sizeof(unsigned long long), stream_), "stage cycles reset");
      sync();
    }
    if (on != timing_) invalidate_graphs();
    timing_ = on;
  }
}

int Engine::feature_qskip() const {
  const Model& m = *models_[0];
  return (m.njnt > 0 && m.jnt_type[0] == JNT_FREE && m.jnt_bodyid[0] == 1) ? 2 : 0;
}

int Engine::feature_count() const {
  const Model& m = *models_[0];
  if (feature_per_body()) return MJB_FEAT_BODY;
  return m.nq - feature_qskip() + 2 * m.nv + 4 * MJB_FEAT_CONTACTS;
}

int Engine::warmstart_input_width() const {
  const Model& m = *models_[0];
  if (feature_per_body()) return MJB_FEAT_BODY;
  return m.nq - feature_qskip() + 3 * m.nv + m.nu + 4 * MJB_FEAT_CONTACTS;   // the step kernel's nn_feature layout
}

bool Engine::feature_per_body() const {
  const Model& m = *models_[0];
  if (m.nv <= WarmStartNet::kOutPad || m.nu != 0 || m.njnt != m.nbody - 1) return false;
  for (int j = 0; j < m.njnt; j++)
    if (m.jnt_type[j] != JNT_FREE || m.jnt_bodyid[j] != j + 1 || m.body_parentid[j + 1] != 0) return false;
  return true;
}

void Engine::ensure_features() {
  if (!uniform()) throw std::runtime_error("learned warm start: needs a single-model batch");
  const int F = feature_count();
  const int stride = (F + 3) & ~3;
  if (feat_.p && feat_stride_ == stride) return;
  sync();
  feat_stride_ = stride;
  feat_.alloc((size_t)B_ * rows_per_env() * stride);
  feat_valid_ = false;
  invalidate_graphs();
}

void Engine::set_warmstart(WarmStartNet* net) {
  sync();
  if (net) {
    if (!uniform()) throw std::runtime_error("learned warm start: needs a single-model batch");
    if (net->in_raw() != warmstart_input_width() || net->nout() != warmstart_outputs())
      throw std::runtime_error("learned warm start: the net's input / output widths do not match this model");
    if (feature_per_body()) {
      ensure_features();
      net->prepare_inference(B_ * rows_per_env());
    } else {
      if (net->in_pad() > 256) throw std::runtime_error("learned warm start: inputs past 256 do not fit the fused inference");
      net_ = net;
      if (!fused_blocker().empty() && lockstep_ && !gws_mode_) {
        // 8-warp lockstep CTAs (one per SM when the workspaces are large)
        EngineConfig c = cfg_;
        c.warps_per_block = 8;
        c.lockstep = 1;
        const EngineConfig prev = cfg_;
        cfg_ = c;
        choose_launch();
        if (!fused_blocker().empty() || smem_ > kStepSmemMax) {
          cfg_ = prev;
          choose_launch();
        }
      }
      const std::string why = fused_blocker();
      if (!why.empty()) {
        net_ = nullptr;
        throw std::runtime_error("learned warm start (fused into the step kernel): " + why);
      }
    }
  }
  net_ = net;
  invalidate_graphs();
}

int Engine::collect(const float* ctrl_seq, int nctrl, int sub_per_ctrl, float* xraw, float* traw, int max_rows) {
  if (!uniform()) throw std::runtime_error("learned warm start: needs a single-model batch");
  if (!feature_per_body()) {
    // per-env: the step kernel writes (features after the constraint build,
    // converged qacc minus the previous one) for every env and substep
    const Model& m = *models_[0];
    const int F = warmstart_input_width();
    WarmStartNet* saved = net_;
    net_ = nullptr;
    int rows = 0;
    for (int c = 0; c < nctrl; c++) {
      int n = sub_per_ctrl;
      if (rows + (long long)n * B_ > max_rows) n = (max_rows - rows) / B_;
      if (n <= 0) break;
      if (m.nu > 0) check(cudaMemcpyAsync(ctrl_.p, ctrl_seq + (size_t)c * tot_u_, sizeof(float) * tot_u_, cudaMemcpyDeviceToDevice, stream_), "collect ctrl");
      StepParams P = params(n, false);
      P.pair_x = xraw + (size_t)rows * F;
      P.pair_t = traw + (size_t)rows * m.nv;
      P.nn_in_raw = F;
      P.feat_qskip = feature_qskip();
      if (persistent_ && !lockstep_) check(cudaMemsetAsync(counter_.p, 0, sizeof(int), stream_), "reset work counter");
      check(mjb_launch_step(P, grid_, warps_, smem_, stream_), "mjb_step_kernel launch");
      rows += n * B_;
      if (n < sub_per_ctrl) break;
    }
    sync();
    net_ = saved;
    return rows;
  }
  ensure_features();
  const Model& m = *models_[0];
  const bool per_body = feature_per_body();
  const int F = feature_count(), nu = per_body ? 0 : m.nu, nv = m.nv, in_raw = F + nu;
  const int R = B_ * rows_per_env();   // training rows per substep
  tmp_prev_.alloc((size_t)B_ * nv);
  WarmStartNet* saved = net_;
  net_ = nullptr;
  bool have = false;
  int rows = 0;
  for (int c = 0; c < nctrl; c++) {
    if (nu > 0) check(cudaMemcpyAsync(ctrl_.p, ctrl_seq + (size_t)c * tot_u_, sizeof(float) * tot_u_, cudaMemcpyDeviceToDevice, stream_), "collect ctrl");
    for (int s = 0; s < sub_per_ctrl; s++) {
      const bool take = have && rows + R <= max_rows;
      if (take) {
        float* xr = xraw + (size_t)rows * in_raw;
        check(cudaMemcpy2DAsync(xr, sizeof(float) * in_raw, feat_.p, sizeof(float) * feat_stride_, sizeof(float) * F, R, cudaMemcpyDeviceToDevice,
                                stream_),
              "collect features");
        if (nu > 0)
          check(cudaMemcpy2DAsync(xr + F, sizeof(float) * in_raw, ctrl_.p, sizeof(float) * nu, sizeof(float) * nu, B_, cudaMemcpyDeviceToDevice, stream_),
                "collect ctrl rows");
        check(cudaMemcpyAsync(tmp_prev_.p, warm_.p, sizeof(float) * (size_t)B_ * nv, cudaMemcpyDeviceToDevice, stream_), "collect prev");
      }
      StepParams P = params(1, false);
      P.features = feat_.p;
      P.feat_stride = feat_stride_;
      P.feat_qskip = feature_qskip();
      P.feat_body = per_body;
      if (persistent_ && !lockstep_) check(cudaMemsetAsync(counter_.p, 0, sizeof(int), stream_), "reset work counter");
      check(mjb_launch_step(P, grid_, warps_, smem_, stream_), "mjb_step_kernel launch");
      if (take) {
        // per-body mode: R rows of 6 targets are the same B * nv floats
        check(mjb_sub(B_ * nv, warm_.p, tmp_prev_.p, traw + (size_t)rows * warmstart_outputs(), stream_), "collect target");
        rows += R;
      }
      have = true;
    }
  }
  sync();
  feat_valid_ = true;
  net_ = saved;
  return rows;
}

}  // namespace mjb

namespace mjb {

// Packed read-back row: [qpos, qvel, |F| of each selected body (force part of
// cfrc_ext), sum qfrc_actuator^2 over the dof range, sum |qfrc_actuator|]
// (reference: mjmlx_batched_set_pack_spec / get_pack, src/batched.cpp:1675-1727).
int Engine::pack_spec(const int* body_ids, int nsel, int dof_lo, int ndof) {
  if (!uniform() || nsel < 0 || ndof < 0) return -1;
  const Model& m = *models_[0];
  if (nsel > 0 && !body_ids) return -1;
  for (int i = 0; i < nsel; i++)
    if (body_ids[i] < 0 || body_ids[i] >= m.nbody) return -1;
  if (dof_lo < 0 || dof_lo + ndof > m.nv) return -1;
  pack_bodies_.assign(body_ids, body_ids + nsel);
  pack_dof_lo_ = dof_lo;
  pack_ndof_ = ndof;
  pack_stride_ = m.nq + m.nv + nsel + 2;
  return pack_stride_;
}

int Engine::pack_device(float** out_dev) {
  if (pack_stride_ < 0) return -1;
  if (!cfg_.record) throw std::runtime_error("get_pack needs the recorded cfrc_ext / qfrc_actuator (engine config record = 1)");
  const Model& m = *models_[0];
  const size_t need = (size_t)B_ * pack_stride_;
  if (d_pack_.n < need) d_pack_.alloc(need);
  std::vector<int> bodies(pack_bodies_.begin(), pack_bodies_.end());
  if (bodies.empty()) bodies.push_back(0);
  d_pack_bodies_.upload(bodies, stream_);
  check(mjb_launch_pack(B_, m.nq, m.nv, m.nbody, qpos_.p, qvel_.p, rec_cfrc_.p, rec_qfa_.p, d_pack_bodies_.p, (int)pack_bodies_.size(), pack_dof_lo_,
                        pack_ndof_, pack_stride_, d_pack_.p, stream_),
        "pack kernel");
  if (out_dev) *out_dev = d_pack_.p;
  return 0;
}

int Engine::get_pack(float* out) {
  float* dev = nullptr;
  if (pack_device(&dev) != 0) return -1;
  check(cudaMemcpyAsync(out, dev, sizeof(float) * (size_t)B_ * pack_stride_, cudaMemcpyDeviceToHost, stream_), "pack copy");
  sync();
  return 0;
}

int Engine::raycast(const float* pnt, const float* vec, int nray, int bodyexclude, const unsigned char* geomgroup, int flg_static, float* dist,
                    int* geomid) {
  if (nray <= 0 || !pnt || !vec || !dist || !geomid) return -1;
  const size_t total = (size_t)B_ * nray;
  // per-model geom table {type, size, include}; include applies the call's
  // body / group / static filters and the supported types
  std::vector<int> base(models_.size()), cnt(models_.size());
  std::vector<float> ginfo;
  int ng_max = 0;
  for (size_t mi = 0; mi < models_.size(); mi++) {
    const Model& m = *models_[mi];
    base[mi] = (int)(ginfo.size() / 5);
    cnt[mi] = m.ngeom;
    ng_max = std::max(ng_max, m.ngeom);
    for (int g = 0; g < m.ngeom; g++) {
      const int type = m.geom_type[g], body = m.geom_bodyid[g], group = m.geom_group[g];
      const bool group_ok = !geomgroup || (group >= 0 && group < 6 && geomgroup[group]);
      const bool static_ok = flg_static || m.body_weldid[body] != 0;
      const bool supported = type == GEOM_PLANE || type == GEOM_SPHERE || type == GEOM_CAPSULE || type == GEOM_ELLIPSOID || type == GEOM_CYLINDER ||
                             type == GEOM_BOX;
      const bool inc = body != bodyexclude && group_ok && static_ok && supported;
      ginfo.insert(ginfo.end(), {(float)type, (float)m.geom_size[3 * g], (float)m.geom_size[3 * g + 1], (float)m.geom_size[3 * g + 2], inc ? 1.f : 0.f});
    }
  }
  if (ng_max == 0) {
    std::fill(dist, dist + total, -1.f);
    std::fill(geomid, geomid + total, -1);
    return 0;
  }
  DevBuf<float> d_ginfo, d_rays, d_pose, d_dist;
  DevBuf<int> d_base, d_cnt, d_gid;
  d_ginfo.upload(ginfo, stream_);
  d_base.upload(base, stream_);
  d_cnt.upload(cnt, stream_);
  d_rays.alloc(total * 6);
  check(cudaMemcpyAsync(d_rays.p, pnt, sizeof(float) * total * 3, cudaMemcpyHostToDevice, stream_), "ray points");
  check(cudaMemcpyAsync(d_rays.p + total * 3, vec, sizeof(float) * total * 3, cudaMemcpyHostToDevice, stream_), "ray vectors");
  d_pose.alloc((size_t)B_ * ng_max * 12);
  d_dist.alloc(total);
  d_gid.alloc(total);
  StepParams P = params(1, false);
  check(mjb_launch_geom_pose(P, d_pose.p, ng_max, warps_, smem_, stream_), "geom pose kernel");
  check(mjb_launch_ray(B_, nray, d_model_.p, d_base.p, d_cnt.p, d_ginfo.p, d_pose.p, ng_max, d_rays.p, d_rays.p + total * 3, d_dist.p, d_gid.p, stream_),
        "ray kernel");
  check(cudaMemcpyAsync(dist, d_dist.p, sizeof(float) * total, cudaMemcpyDeviceToHost, stream_), "ray dist");
  check(cudaMemcpyAsync(geomid, d_gid.p, sizeof(int) * total, cudaMemcpyDeviceToHost, stream_), "ray geom");
  sync();
  return 0;
}

}  // namespace mjb
