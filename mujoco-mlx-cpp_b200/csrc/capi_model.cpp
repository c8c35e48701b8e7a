// C ABI: model loading and model accessors (libmjmlx part).
// Replaces the reference's model I/O bodies (src/io.cpp:1767-1860,
// mjmlx_load_model*, mjmlx_model_info, mjmlx_name2id) with the built-in MJCF
// compiler; the same entry points fail with NULL plus a stderr message.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "capi_internal.h"

namespace mjb {
thread_local std::string g_last_error;
void set_error(const std::string& msg) {
  g_last_error = msg;
  std::fprintf(stderr, "[mjb200] %s\n", msg.c_str());
}
}  // namespace mjb

using mjb::set_error;

namespace {

MjmlxModel* load_from_string(const std::string& xml, const MjmlxModelOptions* o, const std::string& dir) {
  try {
    mjb::LoadOptions lo;
    if (o) {
      lo.self_collision = o->self_collision;
      lo.max_condim = o->max_condim;
    }
    auto* h = new MjmlxModel();
    h->model = mjb::compile_mjcf(xml, lo, dir);
    h->options = lo;
    return h;
  } catch (const std::exception& e) {
    set_error(std::string("mjmlx_load_model: ") + e.what());
    return nullptr;
  }
}

MjmlxModel* load_from_file(const char* path, const MjmlxModelOptions* o) {
  if (!path) {
    set_error("mjmlx_load_model: NULL path");
    return nullptr;
  }
  std::ifstream f(path);
  if (!f) {
    set_error(std::string("mjmlx_load_model: cannot open ") + path);
    return nullptr;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  std::string p(path);
  size_t slash = p.find_last_of('/');
  return load_from_string(ss.str(), o, slash == std::string::npos ? std::string() : p.substr(0, slash));
}

}  // namespace

extern "C" {

MJMLX_API const char* mjmlx_version(void) { return "mjb200 0.1 (B200 CUDA engine)"; }

MJMLX_API const char* mjb200_last_error(void) { return mjb::g_last_error.c_str(); }

MJMLX_API MjmlxModelOptions mjmlx_default_model_options(void) {
  MjmlxModelOptions o;
  o.self_collision = 1;
  o.max_condim = 0;
  return o;
}

MJMLX_API MjmlxModel* mjmlx_load_model(const char* xml_path) { return load_from_file(xml_path, nullptr); }

MJMLX_API MjmlxModel* mjmlx_load_model_from_string(const char* xml) {
  if (!xml) {
    set_error("mjmlx_load_model_from_string: NULL string");
    return nullptr;
  }
  return load_from_string(xml, nullptr, "");
}

MJMLX_API MjmlxModel* mjmlx_load_model_ex(const char* xml_path, const MjmlxModelOptions* options) { return load_from_file(xml_path, options); }

MJMLX_API MjmlxModel* mjmlx_load_model_from_string_ex(const char* xml, const MjmlxModelOptions* options) {
  if (!xml) {
    set_error("mjmlx_load_model_from_string_ex: NULL string");
    return nullptr;
  }
  return load_from_string(xml, options, "");
}

MJMLX_API void mjmlx_free_model(MjmlxModel* model) { delete model; }

MJMLX_API MjmlxModelInfo mjmlx_model_info(const MjmlxModel* model) {
  MjmlxModelInfo i;
  std::memset(&i, 0, sizeof(i));
  if (!model) return i;
  const auto& m = model->model;
  i.nq = m.nq;
  i.nv = m.nv;
  i.nu = m.nu;
  i.na = 0;
  i.nbody = m.nbody;
  i.njnt = m.njnt;
  i.ngeom = m.ngeom;
  i.nsite = 0;
  i.ncon = (int)m.pairs.size();
  return i;
}

MJMLX_API float mjmlx_model_opt_timestep(const MjmlxModel* model) { return model ? (float)model->model.timestep : 0.0f; }

MJMLX_API void mjmlx_model_set_opt_timestep(MjmlxModel* model, float dt) {
  if (model && dt > 0) model->model.timestep = dt;
}

MJMLX_API float mjmlx_model_body_mass(const MjmlxModel* model, int body_id) {
  if (!model || body_id < 0 || body_id >= model->model.nbody) return 0.0f;
  return (float)model->model.body_mass[body_id];
}

MJMLX_API int mjmlx_name2id(const MjmlxModel* model, int obj_type, const char* name) {
  if (!model || !name) return -1;
  const auto& m = model->model;
  const std::vector<std::string>* names = nullptr;
  switch (obj_type) {
    case 1: names = &m.body_name; break;
    case 3: names = &m.jnt_name; break;
    case 5: names = &m.geom_name; break;
    case 6: names = &m.site_name; break;
    case 18: names = &m.tendon_name; break;
    case 19: names = &m.actuator_name; break;
    case 20: names = &m.sensor_name; break;
    default: return -1;
  }
  for (size_t k = 0; k < names->size(); k++)
    if ((*names)[k] == name) return (int)k;
  return -1;
}

MJMLX_API int mjmlx_model_nsensor(const MjmlxModel* model) { return model ? model->model.nsensor : 0; }
MJMLX_API int mjmlx_model_nsensordata(const MjmlxModel* model) { return model ? model->model.nsensordata : 0; }

static bool sensor_ok(const MjmlxModel* model, int id) { return model && id >= 0 && id < model->model.nsensor; }

MJMLX_API const char* mjmlx_model_sensor_name(const MjmlxModel* model, int sensor_id) {
  if (!sensor_ok(model, sensor_id) || model->model.sensor_name[sensor_id].empty()) return nullptr;
  return model->model.sensor_name[sensor_id].c_str();
}
MJMLX_API int mjmlx_model_sensor_type(const MjmlxModel* model, int sensor_id) { return sensor_ok(model, sensor_id) ? model->model.sensor_type[sensor_id] : -1; }
MJMLX_API int mjmlx_model_sensor_adr(const MjmlxModel* model, int sensor_id) { return sensor_ok(model, sensor_id) ? model->model.sensor_adr[sensor_id] : -1; }
MJMLX_API int mjmlx_model_sensor_dim(const MjmlxModel* model, int sensor_id) { return sensor_ok(model, sensor_id) ? model->model.sensor_dim[sensor_id] : -1; }

MJMLX_API int mjb200_model_dump(const MjmlxModel* model, char* buf, int bufsize) {
  if (!model) return -1;
  std::string s = mjb::dump_model(model->model);
  int need = (int)s.size() + 1;
  if (buf && bufsize >= need) std::memcpy(buf, s.c_str(), need);
  return need;
}

}  // extern "C"
