// Compiled model (host, double precision) and the MJCF compiler entry points.
//
// Field names and conventions follow MuJoCo's mjModel (quaternions w,x,y,z;
// geom/joint type numbering of mjtGeom/mjtJoint), which is also what the
// reference's Model mirrors (src/internal.h:105-300).  The compiler restates
// the load-time work the reference delegates to MuJoCo (mj_loadXML/mj_compile,
// src/io.cpp:563-601) plus the reference's own collision-pair cache
// (Model::init_cache, src/io.cpp:713-1165).
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace mjb {

enum GeomType { GEOM_PLANE = 0, GEOM_HFIELD = 1, GEOM_SPHERE = 2, GEOM_CAPSULE = 3, GEOM_ELLIPSOID = 4, GEOM_CYLINDER = 5, GEOM_BOX = 6, GEOM_MESH = 7 };
enum JointType { JNT_FREE = 0, JNT_BALL = 1, JNT_SLIDE = 2, JNT_HINGE = 3 };
enum ConeType { CONE_PYRAMIDAL = 0, CONE_ELLIPTIC = 1 };
// MuJoCo 3.x mjtSensor codes of the sensor elements this compiler knows
// (ordering as in MuJoCo's mjtSensor; not checked against 3.5.0's header,
// which is absent here)
enum SensorType {
  SENS_TOUCH = 0, SENS_ACCELEROMETER, SENS_VELOCIMETER, SENS_GYRO, SENS_FORCE, SENS_TORQUE, SENS_MAGNETOMETER, SENS_RANGEFINDER,
  SENS_CAMPROJECTION, SENS_JOINTPOS, SENS_JOINTVEL, SENS_TENDONPOS, SENS_TENDONVEL, SENS_ACTUATORPOS, SENS_ACTUATORVEL, SENS_ACTUATORFRC,
  SENS_JOINTACTFRC, SENS_TENDONACTFRC, SENS_BALLQUAT, SENS_BALLANGVEL, SENS_JOINTLIMITPOS, SENS_JOINTLIMITVEL, SENS_JOINTLIMITFRC,
  SENS_TENDONLIMITPOS, SENS_TENDONLIMITVEL, SENS_TENDONLIMITFRC, SENS_FRAMEPOS, SENS_FRAMEQUAT, SENS_FRAMEXAXIS, SENS_FRAMEYAXIS,
  SENS_FRAMEZAXIS, SENS_FRAMELINVEL, SENS_FRAMEANGVEL, SENS_FRAMELINACC, SENS_FRAMEANGACC, SENS_SUBTREECOM, SENS_SUBTREELINVEL,
  SENS_SUBTREEANGMOM
};
enum ObjType { OBJ_UNKNOWN = 0, OBJ_BODY = 1, OBJ_XBODY = 2, OBJ_JOINT = 3, OBJ_GEOM = 5, OBJ_SITE = 6, OBJ_TENDON = 18, OBJ_ACTUATOR = 19 };
enum DisableBit {
  DSBL_CONSTRAINT = 1 << 0, DSBL_EQUALITY = 1 << 1, DSBL_FRICTIONLOSS = 1 << 2, DSBL_LIMIT = 1 << 3,
  DSBL_CONTACT = 1 << 4, DSBL_PASSIVE = 1 << 5, DSBL_GRAVITY = 1 << 6, DSBL_CLAMPCTRL = 1 << 7,
  DSBL_WARMSTART = 1 << 8, DSBL_FILTERPARENT = 1 << 9, DSBL_ACTUATION = 1 << 10, DSBL_REFSAFE = 1 << 11,
  DSBL_EULERDAMP = 1 << 15,
};

// One collision candidate (reference: ModelCache::CollisionPair, internal.h:284-302).
struct Pair {
  int g1 = 0, g2 = 0;        // geom ids, type(g1) <= type(g2)
  int b1 = 0, b2 = 0;        // body ids of g1, g2
  int condim = 3;
  double margin = 0, gap = 0;
  double friction[5] = {1, 1, 0.005, 0.0001, 0.0001};  // tangent1, tangent2, spin, roll1, roll2
  double solref[2] = {0.02, 1};
  double solimp[5] = {0.9, 0.95, 0.001, 0.5, 2};
  double invw_t = 0, invw_r = 0;   // body_invweight0 sums (translation, rotation)
  int is_explicit = 0;
};

struct Model {
  std::string name;
  int nq = 0, nv = 0, nu = 0, nbody = 0, njnt = 0, ngeom = 0, nmesh = 0;

  // <option>
  double timestep = 0.002;
  double gravity[3] = {0, 0, -9.81};
  double tolerance = 1e-8, ls_tolerance = 0.01, impratio = 1;
  int iterations = 100, ls_iterations = 50, cone = CONE_PYRAMIDAL, integrator = 0, disableflags = 0;
  double meaninertia = 1;   // mean diagonal of M at qpos0 (MuJoCo stat.meaninertia)
  double magnetic[3] = {0, -0.5, 0};

  std::vector<std::string> body_name, jnt_name, geom_name, actuator_name, mesh_name;

  // bodies (index 0 = world); bodies are stored in depth-first preorder
  std::vector<int> body_parentid, body_rootid, body_weldid, body_jntnum, body_jntadr, body_dofnum, body_dofadr,
      body_subtreesize, body_geomnum, body_geomadr, body_depth;
  std::vector<double> body_pos, body_quat, body_ipos, body_iquat, body_mass, body_inertia, body_invweight0, body_gravcomp;

  // joints
  std::vector<int> jnt_type, jnt_qposadr, jnt_dofadr, jnt_bodyid, jnt_limited;
  std::vector<double> jnt_pos, jnt_axis, jnt_range, jnt_margin, jnt_solref, jnt_solimp, jnt_stiffness;

  // dofs
  std::vector<int> dof_bodyid, dof_jntid, dof_parentid;
  std::vector<double> dof_armature, dof_damping, dof_frictionloss, dof_invweight0, dof_solref, dof_solimp;

  std::vector<double> qpos0, qpos_spring;

  // geoms
  std::vector<int> geom_type, geom_bodyid, geom_contype, geom_conaffinity, geom_condim, geom_priority, geom_dataid, geom_group;
  std::vector<double> geom_pos, geom_quat, geom_size, geom_friction, geom_solref, geom_solimp, geom_solmix, geom_margin, geom_gap, geom_rbound, geom_mass;

  // meshes: convex-hull vertices in the mesh frame (centred at the hull's
  // centre of mass and aligned with its principal axes, as MuJoCo does)
  std::vector<int> mesh_vertadr, mesh_vertnum;
  std::vector<double> mesh_vert;

  // actuators (joint transmission; gain = g0 + g1*len + g2*vel, bias likewise)
  std::vector<int> actuator_trntype, actuator_trnid, actuator_gaintype, actuator_biastype, actuator_ctrllimited, actuator_forcelimited;
  std::vector<double> actuator_gear, actuator_gainprm, actuator_biasprm, actuator_ctrlrange, actuator_forcerange;

  // <contact>
  std::vector<int> exclude_body1, exclude_body2;
  struct ExplicitPair {
    int g1, g2, condim;
    double friction[5], solref[2], solimp[5], margin, gap;
  };
  std::vector<ExplicitPair> explicit_pairs;

  // sites (frames fixed to bodies)
  int nsite = 0;
  std::vector<int> site_bodyid;
  std::vector<double> site_pos, site_quat;
  std::vector<std::string> site_name;

  // <sensor>: sensor_type is MuJoCo's mjtSensor code, sensor_objtype its
  // mjtObj code (1 body, 2 xbody, 3 joint, 5 geom, 6 site, 18 tendon,
  // 19 actuator); sensor_supported 0 = computed as zeros (types outside the
  // batched sensor set), as the reference does
  int nsensor = 0, nsensordata = 0;
  std::vector<int> sensor_type, sensor_objtype, sensor_objid, sensor_dim, sensor_adr, sensor_supported;
  std::vector<std::string> sensor_name;

  // <tendon>: fixed tendons (length = sum of coef * qpos over hinge / slide
  // joints) and spatial tendons (paths through sites, optionally wrapping
  // around sphere / cylinder geoms, split by pulleys).  Per wrap element:
  // wrap_type (MuJoCo mjtWrap: 1 joint, 2 pulley, 3 site, 4 sphere geom,
  // 5 cylinder geom), wrap_objid (joint / site / geom id, -1 for a pulley),
  // wrap_prm (joint coef, pulley divisor, geom side site id or -1)
  int ntendon = 0;
  std::vector<int> tendon_adr, tendon_num, tendon_limited, wrap_objid, wrap_type;
  std::vector<double> wrap_prm, tendon_range, tendon_margin, tendon_frictionloss, tendon_stiffness, tendon_damping, tendon_lengthspring,
      tendon_solref_lim, tendon_solimp_lim, tendon_solref_fri, tendon_solimp_fri, tendon_length0, tendon_invweight0;
  std::vector<std::string> tendon_name;

  // <equality>: type 0 connect, 1 weld, 2 joint, 3 tendon (this build steps
  // joint equalities: q1 - q1_0 = poly(q2 - q2_0), poly from 5 coefficients)
  std::vector<int> eq_type, eq_obj1, eq_obj2, eq_active;
  std::vector<double> eq_data, eq_solref, eq_solimp, eq_invweight;  // [5], [2], [5], [1] per equality

  // compiled collision candidates
  std::vector<Pair> pairs;

  // upper bound on contacts one env can produce (sum over pairs of the
  // per-pair contact count of its collision rule)
  int max_contacts_bound = 0;
};

struct LoadOptions {
  int self_collision = 1;
  int max_condim = 0;
};

// Compiles MJCF text into a Model; throws std::runtime_error with a message.
Model compile_mjcf(const std::string& xml, const LoadOptions& opt, const std::string& base_dir = "");

// Recomputes everything that depends on option/body parameters after edits:
// tree topology tables, inertias at qpos0, invweights, pair table.
void finalize_model(Model& m, const LoadOptions& opt);

// Number of contacts the collision rule of a (type1, type2) pair can emit.
int pair_max_contacts(int t1, int t2);

// Text dump "name kind n v0 v1 ..." (one array per line) of every field;
// used by the test-side FP64 oracle to read the compiled model.
std::string dump_model(const Model& m);

}  // namespace mjb
