// Fluid-world checkpoints in the reference's JSON archive layout.
#include "checkpoint.h"

#include <cstdint>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <vector>

namespace phy {

namespace {

uint64_t bits_of(double v) {
  uint64_t b;
  std::memcpy(&b, &v, sizeof(b));
  return b;
}
double from_bits(uint64_t b) {
  double v;
  std::memcpy(&v, &b, sizeof(v));
  return v;
}

// ---- writer -----------------------------------------------------------------

struct Writer {
  std::ostringstream o;
  void f64(double v) { o << "{\"__f64\":" << bits_of(v) << "}"; }
  void vec3(const double* v) { o << "[" << bits_of(v[0]) << "," << bits_of(v[1]) << "," << bits_of(v[2]) << "]"; }
  void key(const char* k) { o << "\"" << k << "\":"; }
};

void write_params(Writer& w, const SphParams& p) {
  w.o << "{";
  w.key("rest_density");
  w.f64(p.rest_density);
  w.o << ",";
  w.key("stiffness");
  w.f64(p.stiffness);
  w.o << ",";
  w.key("viscosity");
  w.f64(p.viscosity);
  w.o << ",";
  w.key("visc_k");
  w.o << "[";
  for (size_t k = 0; k < p.visc_k.size(); ++k) {
    if (k) w.o << ",";
    w.f64(p.visc_k[k]);
  }
  w.o << "],";
  w.key("visc_n");
  w.o << "[";
  for (size_t k = 0; k < p.visc_n.size(); ++k) {
    if (k) w.o << ",";
    w.f64(p.visc_n[k]);
  }
  w.o << "],";
  w.key("shear_min");
  w.f64(p.shear_min);
  w.o << ",";
  w.key("mass");
  w.f64(p.mass);
  w.o << ",";
  w.key("h");
  w.f64(p.h);
  w.o << ",";
  double g[3] = {p.gravity.x, p.gravity.y, p.gravity.z};
  double lo[3] = {p.bounds_min.x, p.bounds_min.y, p.bounds_min.z};
  double hi[3] = {p.bounds_max.x, p.bounds_max.y, p.bounds_max.z};
  w.key("gravity");
  w.vec3(g);
  w.o << ",";
  w.key("bounds_min");
  w.vec3(lo);
  w.o << ",";
  w.key("bounds_max");
  w.vec3(hi);
  w.o << ",";
  w.key("boundary_damp");
  w.f64(p.boundary_damp);
  w.o << ",";
  w.key("xsph_eps");
  w.f64(p.xsph_eps);
  w.o << "}";
}

// ---- minimal JSON reader (objects, arrays, integers, strings) --------------

struct JVal {
  enum Kind { Null, Num, Str, Arr, Obj, Bool } kind = Null;
  std::string num;  // raw number text
  std::string str;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;
  const JVal* get(const char* k) const {
    for (auto& kv : obj)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
  const JVal& at(const char* k) const {
    const JVal* v = get(k);
    if (!v) throw std::runtime_error(std::string("archive: missing key ") + k);
    return *v;
  }
};

struct Parser {
  const std::string& s;
  size_t i = 0;
  explicit Parser(const std::string& t) : s(t) {}
  void ws() {
    while (i < s.size() && (s[i] == ' ' || s[i] == '\n' || s[i] == '\r' || s[i] == '\t')) ++i;
  }
  [[noreturn]] void fail(const char* what) {
    throw std::runtime_error(std::string("archive: ") + what + " at offset " + std::to_string(i));
  }
  JVal value() {
    ws();
    if (i >= s.size()) fail("unexpected end");
    char ch = s[i];
    JVal v;
    if (ch == '{') {
      v.kind = JVal::Obj;
      ++i;
      ws();
      if (i < s.size() && s[i] == '}') {
        ++i;
        return v;
      }
      for (;;) {
        ws();
        std::string k = string();
        ws();
        if (i >= s.size() || s[i] != ':') fail("expected ':'");
        ++i;
        v.obj.emplace_back(k, value());
        ws();
        if (i < s.size() && s[i] == ',') {
          ++i;
          continue;
        }
        if (i < s.size() && s[i] == '}') {
          ++i;
          break;
        }
        fail("expected ',' or '}'");
      }
    } else if (ch == '[') {
      v.kind = JVal::Arr;
      ++i;
      ws();
      if (i < s.size() && s[i] == ']') {
        ++i;
        return v;
      }
      for (;;) {
        v.arr.push_back(value());
        ws();
        if (i < s.size() && s[i] == ',') {
          ++i;
          continue;
        }
        if (i < s.size() && s[i] == ']') {
          ++i;
          break;
        }
        fail("expected ',' or ']'");
      }
    } else if (ch == '"') {
      v.kind = JVal::Str;
      v.str = string();
    } else if (s.compare(i, 4, "null") == 0) {
      i += 4;
    } else if (s.compare(i, 4, "true") == 0) {
      v.kind = JVal::Bool;
      i += 4;
    } else if (s.compare(i, 5, "false") == 0) {
      v.kind = JVal::Bool;
      i += 5;
    } else {
      v.kind = JVal::Num;
      size_t j = i;
      while (j < s.size() && (isdigit((unsigned char)s[j]) || s[j] == '-' || s[j] == '+' || s[j] == '.' ||
                              s[j] == 'e' || s[j] == 'E'))
        ++j;
      if (j == i) fail("bad value");
      v.num = s.substr(i, j - i);
      i = j;
    }
    return v;
  }
  std::string string() {
    if (i >= s.size() || s[i] != '"') fail("expected string");
    ++i;
    std::string out;
    while (i < s.size() && s[i] != '"') {
      if (s[i] == '\\' && i + 1 < s.size()) ++i;
      out.push_back(s[i++]);
    }
    if (i >= s.size()) fail("unterminated string");
    ++i;
    return out;
  }
};

uint64_t as_u64(const JVal& v) {
  if (v.kind != JVal::Num) throw std::runtime_error("archive: expected an integer");
  return std::stoull(v.num);
}
// A scalar is {"__f64": bits}; a plain JSON number is accepted too.
double as_f64(const JVal& v) {
  if (v.kind == JVal::Obj) return from_bits(as_u64(v.at("__f64")));
  if (v.kind == JVal::Num) return std::stod(v.num);
  throw std::runtime_error("archive: expected a float");
}
void as_vec3(const JVal& v, double* out) {
  if (v.kind != JVal::Arr || v.arr.size() != 3) throw std::runtime_error("archive: expected a 3-vector");
  for (int k = 0; k < 3; ++k) out[k] = from_bits(as_u64(v.arr[k]));
}

SphParams read_params(const JVal& v) {
  SphParams p;
  p.rest_density = as_f64(v.at("rest_density"));
  p.stiffness = as_f64(v.at("stiffness"));
  p.viscosity = as_f64(v.at("viscosity"));
  for (auto& e : v.at("visc_k").arr) p.visc_k.push_back(as_f64(e));
  for (auto& e : v.at("visc_n").arr) p.visc_n.push_back(as_f64(e));
  p.shear_min = as_f64(v.at("shear_min"));
  p.mass = as_f64(v.at("mass"));
  p.h = as_f64(v.at("h"));
  double t[3];
  as_vec3(v.at("gravity"), t);
  p.gravity = {t[0], t[1], t[2]};
  as_vec3(v.at("bounds_min"), t);
  p.bounds_min = {t[0], t[1], t[2]};
  as_vec3(v.at("bounds_max"), t);
  p.bounds_max = {t[0], t[1], t[2]};
  p.boundary_damp = as_f64(v.at("boundary_damp"));
  p.xsph_eps = as_f64(v.at("xsph_eps"));
  if (p.visc_k.empty() || p.visc_k.size() > (size_t)PHY_MAX_MATERIALS || p.visc_n.size() > (size_t)PHY_MAX_MATERIALS)
    throw std::runtime_error("archive: material tables must hold 1..16 entries");
  return p;
}

}  // namespace

std::string save_world_json(World& world) {
  Writer w;
  w.o << "{";
  w.key("version");
  w.o << 1 << ",";
  w.key("time");
  w.f64(world.t);
  w.o << ",";
  w.key("subsystems");
  w.o << "[";
  bool first = true;
  for (auto& s : world.subs) {
    if (!first) w.o << ",";
    first = false;
    FluidWorld& fw = *s->world;
    size_t n = fw.len();
    std::vector<double> pos(3 * n), vel(3 * n), acc(3 * n), ba(3 * n), rho(n), p(n), mass(n), mat(n);
    fw.get_field(PHY_FIELD_POS, pos.data());
    fw.get_field(PHY_FIELD_VEL, vel.data());
    fw.get_field(PHY_FIELD_ACC, acc.data());
    fw.get_field(PHY_FIELD_BODY_ACC, ba.data());
    fw.get_field(PHY_FIELD_RHO, rho.data());
    fw.get_field(PHY_FIELD_P, p.data());
    fw.get_field(PHY_FIELD_MASS, mass.data());
    fw.get_field(PHY_FIELD_MATERIAL, mat.data());
    w.o << "{\"Fluid\":{";
    w.key("world");
    w.o << "{";
    w.key("params");
    write_params(w, fw.params);
    w.o << ",";
    w.key("particles");
    w.o << "[";
    for (size_t i = 0; i < n; ++i) {
      if (i) w.o << ",";
      w.o << "{";
      w.key("pos");
      w.vec3(&pos[3 * i]);
      w.o << ",";
      w.key("vel");
      w.vec3(&vel[3 * i]);
      w.o << ",";
      w.key("acc");
      w.vec3(&acc[3 * i]);
      w.o << ",";
      w.key("body_acc");
      w.vec3(&ba[3 * i]);
      w.o << ",";
      w.key("rho");
      w.f64(rho[i]);
      w.o << ",";
      w.key("p");
      w.f64(p[i]);
      w.o << ",";
      w.key("mass");
      w.f64(mass[i]);
      w.o << ",";
      w.key("material");
      w.o << (uint64_t)mat[i];
      w.o << "}";
    }
    w.o << "]}";
    w.o << ",";
    w.key("thermal_expansion");
    w.f64(s->thermal_expansion);
    w.o << ",";
    w.key("heat_gain");
    w.f64(s->heat_gain);
    w.o << ",";
    w.key("t_ref");
    w.f64(s->t_ref);
    w.o << ",";
    w.key("drag");
    w.f64(s->drag);
    w.o << ",";
    w.key("friction");
    w.f64(s->friction);
    w.o << "}}";
  }
  w.o << "]}";
  return w.o.str();
}

std::unique_ptr<World> load_world_json(const std::string& json) {
  Parser ps(json);
  JVal root = ps.value();
  auto world = std::make_unique<World>();
  world->t = as_f64(root.at("time"));
  for (auto& sv : root.at("subsystems").arr) {
    const JVal* fl = sv.get("Fluid");
    if (!fl) {
      std::string tag = sv.obj.empty() ? std::string("?") : sv.obj[0].first;
      throw std::runtime_error("archive: subsystem '" + tag + "' is not part of this library");
    }
    const JVal& wv = fl->at("world");
    SphParams params = read_params(wv.at("params"));
    // FluidWorld::new(params).with_particles(...) (world.rs:51-58): h captured
    // from the archived params.
    auto fw = std::make_unique<FluidWorld>(params, Precision::F64Plain);
    const auto& parts = wv.at("particles").arr;
    size_t n = parts.size();
    std::vector<double> pos(3 * n), vel(3 * n), acc(3 * n), ba(3 * n), rho(n), p(n), mass(n), matd(n);
    std::vector<uint32_t> mat(n);
    bool any_ba = false;
    for (size_t i = 0; i < n; ++i) {
      const JVal& q = parts[i];
      as_vec3(q.at("pos"), &pos[3 * i]);
      as_vec3(q.at("vel"), &vel[3 * i]);
      as_vec3(q.at("acc"), &acc[3 * i]);
      as_vec3(q.at("body_acc"), &ba[3 * i]);
      rho[i] = as_f64(q.at("rho"));
      p[i] = as_f64(q.at("p"));
      mass[i] = as_f64(q.at("mass"));
      uint64_t m = as_u64(q.at("material"));
      mat[i] = m > 0xffffffffull ? 0xffffffffu : (uint32_t)m;
      matd[i] = (double)mat[i];
      any_ba = any_ba || ba[3 * i] != 0.0 || ba[3 * i + 1] != 0.0 || ba[3 * i + 2] != 0.0;
    }
    if (n) {
      fw->add_particles(n, pos.data(), vel.data(), mass.data(), mat.data());
      fw->set_field(PHY_FIELD_ACC, acc.data());
      fw->set_field(PHY_FIELD_RHO, rho.data());
      fw->set_field(PHY_FIELD_P, p.data());
      if (any_ba) fw->set_field(PHY_FIELD_BODY_ACC, ba.data());
    }
    auto sub = std::make_unique<FluidSubsystem>(std::move(fw));
    sub->thermal_expansion = as_f64(fl->at("thermal_expansion"));
    sub->heat_gain = as_f64(fl->at("heat_gain"));
    sub->t_ref = as_f64(fl->at("t_ref"));
    sub->drag = as_f64(fl->at("drag"));
    sub->friction = as_f64(fl->at("friction"));
    world->subs.push_back(std::move(sub));
  }
  return world;
}

void save_world(World& w, const char* path) {
  std::string js = save_world_json(w);
  std::ofstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error(std::string("cannot open ") + path + " for writing");
  f << js;
  if (!f) throw std::runtime_error(std::string("write failed: ") + path);
}

std::unique_ptr<World> load_world(const char* path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error(std::string("cannot open ") + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return load_world_json(ss.str());
}

}  // namespace phy
