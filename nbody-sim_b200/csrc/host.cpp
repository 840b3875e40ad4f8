// host.cpp -- host-side pieces of the nbody-b200 C ABI: JSON Config loading,
// particle radius, perturber orbit, FoF aggregate records, the frames.bin /
// stats.csv writers and the synthetic disk generator.  No CUDA here.
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nbody_b200.h"
#include "diskgen.h"

namespace nb {
void set_error(const std::string& msg);
}

namespace {

// ------------------------------------------------------------------ JSON
// A small JSON reader: enough for config files (objects, arrays, strings,
// numbers, true/false/null).  Values keep their JSON kind so that the
// accessors below can reproduce the conversion rules of nlohmann::json's
// value(key, default) that loadConfig relies on (Config.cpp:18-38).
struct JVal {
  enum Kind { Null, Bool, Int, Float, Str, Arr, Obj } kind = Null;
  bool b = false;
  long long i = 0;
  double f = 0;
  std::string s;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;
  const char* kind_name() const {
    switch (kind) {
      case Null: return "null";
      case Bool: return "boolean";
      case Int: case Float: return "number";
      case Str: return "string";
      case Arr: return "array";
      default: return "object";
    }
  }
};

struct JsonError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

class JParser {
 public:
  explicit JParser(const std::string& t) : t_(t) {}
  JVal parse() {
    JVal v = value();
    ws();
    if (p_ != t_.size()) fail("unexpected trailing characters");
    return v;
  }

 private:
  const std::string& t_;
  size_t p_ = 0;
  int line_ = 1;

  [[noreturn]] void fail(const std::string& what) {
    throw JsonError("syntax error at line " + std::to_string(line_) + ": " + what);
  }
  void ws() {
    while (p_ < t_.size() && std::isspace((unsigned char)t_[p_])) {
      if (t_[p_] == '\n') ++line_;
      ++p_;
    }
  }
  bool lit(const char* w) {
    size_t n = std::strlen(w);
    if (t_.compare(p_, n, w) == 0) { p_ += n; return true; }
    return false;
  }
  JVal value() {
    ws();
    if (p_ >= t_.size()) fail("unexpected end of input");
    char c = t_[p_];
    JVal v;
    if (c == '{') {
      ++p_;
      v.kind = JVal::Obj;
      ws();
      if (p_ < t_.size() && t_[p_] == '}') { ++p_; return v; }
      while (true) {
        ws();
        if (p_ >= t_.size() || t_[p_] != '"') fail("expected string key");
        std::string k = str();
        ws();
        if (p_ >= t_.size() || t_[p_] != ':') fail("expected ':'");
        ++p_;
        JVal child = value();
        bool replaced = false;
        for (auto& kv : v.obj)
          if (kv.first == k) { kv.second = child; replaced = true; }
        if (!replaced) v.obj.emplace_back(k, child);
        ws();
        if (p_ < t_.size() && t_[p_] == ',') { ++p_; continue; }
        if (p_ < t_.size() && t_[p_] == '}') { ++p_; break; }
        fail("expected ',' or '}'");
      }
      return v;
    }
    if (c == '[') {
      ++p_;
      v.kind = JVal::Arr;
      ws();
      if (p_ < t_.size() && t_[p_] == ']') { ++p_; return v; }
      while (true) {
        v.arr.push_back(value());
        ws();
        if (p_ < t_.size() && t_[p_] == ',') { ++p_; continue; }
        if (p_ < t_.size() && t_[p_] == ']') { ++p_; break; }
        fail("expected ',' or ']'");
      }
      return v;
    }
    if (c == '"') { v.kind = JVal::Str; v.s = str(); return v; }
    if (lit("true")) { v.kind = JVal::Bool; v.b = true; return v; }
    if (lit("false")) { v.kind = JVal::Bool; v.b = false; return v; }
    if (lit("null")) { v.kind = JVal::Null; return v; }
    if (c == '-' || (c >= '0' && c <= '9')) return number();
    fail(std::string("unexpected character '") + c + "'");
  }
  std::string str() {
    ++p_;  // opening quote
    std::string out;
    while (p_ < t_.size() && t_[p_] != '"') {
      char c = t_[p_++];
      if (c == '\\') {
        if (p_ >= t_.size()) fail("bad escape");
        char e = t_[p_++];
        switch (e) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {
            if (p_ + 4 > t_.size()) fail("bad \\u escape");
            unsigned cp = (unsigned)std::strtoul(t_.substr(p_, 4).c_str(), nullptr, 16);
            p_ += 4;
            if (cp < 0x80) out += (char)cp;
            else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
            else { out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F));
                   out += (char)(0x80 | (cp & 0x3F)); }
            break;
          }
          default: out += e;
        }
      } else {
        out += c;
      }
    }
    if (p_ >= t_.size()) fail("unterminated string");
    ++p_;
    return out;
  }
  JVal number() {
    size_t s = p_;
    if (t_[p_] == '-') ++p_;
    bool is_float = false;
    while (p_ < t_.size()) {
      char c = t_[p_];
      if (std::isdigit((unsigned char)c)) { ++p_; continue; }
      if (c == '.' || c == 'e' || c == 'E' || c == '+' || c == '-') { is_float = true; ++p_; continue; }
      break;
    }
    std::string tok = t_.substr(s, p_ - s);
    JVal v;
    char* end = nullptr;
    if (!is_float) {
      v.kind = JVal::Int;
      v.i = std::strtoll(tok.c_str(), &end, 10);
      v.f = (double)v.i;
    } else {
      v.kind = JVal::Float;
      v.f = std::strtod(tok.c_str(), &end);
    }
    if (!end || *end) fail("invalid number '" + tok + "'");
    return v;
  }
};

struct ConfigError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

const JVal* find(const JVal& o, const char* key) {
  for (const auto& kv : o.obj)
    if (kv.first == key) return &kv.second;
  return nullptr;
}

[[noreturn]] void type_error(const char* want, const JVal& v) {
  throw ConfigError(std::string("[json.exception.type_error.302] type must be ") + want +
                    ", but is " + v.kind_name());
}

void get_float(const JVal& o, const char* key, float& out) {
  const JVal* v = find(o, key);
  if (!v) return;
  if (v->kind != JVal::Int && v->kind != JVal::Float) type_error("number", *v);
  out = (float)v->f;
}
void get_int(const JVal& o, const char* key, int& out) {
  const JVal* v = find(o, key);
  if (!v) return;
  if (v->kind == JVal::Int) out = (int)v->i;
  else if (v->kind == JVal::Float) out = (int)v->f;
  else type_error("number", *v);
}
void get_bool(const JVal& o, const char* key, int& out) {
  const JVal* v = find(o, key);
  if (!v) return;
  if (v->kind != JVal::Bool) type_error("boolean", *v);
  out = v->b ? 1 : 0;
}
void get_string(const JVal& o, const char* key, char* out, size_t cap) {
  const JVal* v = find(o, key);
  if (!v) return;
  if (v->kind != JVal::Str) type_error("string", *v);
  std::snprintf(out, cap, "%s", v->s.c_str());
}

// particlePhysicalRadius constants (src/disk/DiskInit.cpp:6-8)
constexpr float kPi = 3.14159265358979f;
constexpr float kAuM = 1.496e11f;
constexpr float kMsunKg = 1.989e30f;
// Perturber.h:25
constexpr float kMjupToMsun = 9.5479e-4f;
// OutputWriter.h:10-13
constexpr float kT0ToYears = 1.0f / (2.0f * 3.14159265f);
constexpr float kMsunToMearth = 332946.0f;

template <typename T>
void write_raw(std::ofstream& f, const T& v) {
  f.write(reinterpret_cast<const char*>(&v), sizeof(T));
}

}  // namespace

struct nbody_writer {
  std::ofstream frames;
  std::ofstream stats;
  nbody_config cfg;
  std::streampos n_frames_offset;
};

extern "C" {

void nbody_config_defaults(nbody_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->n_particles = 100000;
  c->disk_r_min = 0.5f;
  c->disk_r_max = 5.0f;
  c->disk_h_factor = 0.05f;
  c->particle_mass_msun = 3.003e-7f;
  c->star_mass_msun = 1.0f;
  c->softening_AU = 0.01f;
  c->theta = 0.5f;
  c->collision_radius_factor = 100.0f;
  c->restitution = 0.3f;
  c->gas_drag_rate = 0.0f;
  c->dt = 0.01f;
  c->total_time = 2000.0f;
  c->output_every_n_steps = 200;
  std::snprintf(c->output_dir, sizeof(c->output_dir), "%s", "data");
  c->perturber_enabled = 0;
  c->perturber_mass_mjup = 1.0f;
  c->perturber_radius_AU = 20.0f;
  c->perturber_phase0 = 0.0f;
}

int nbody_config_load(const char* path, nbody_config* cfg) {
  if (!path || !cfg) {
    nb::set_error("nbody_config_load: null argument");
    return NBODY_ERR_ARG;
  }
  std::ifstream f(path);
  if (!f.is_open()) {
    nb::set_error(std::string("Cannot open config: ") + path);
    return NBODY_ERR_IO;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();
  JVal j;
  try {
    j = JParser(text).parse();
  } catch (const JsonError& e) {
    nb::set_error(std::string("JSON parse error in '") + path + "': " + e.what());
    return NBODY_ERR_CONFIG;
  }
  nbody_config c;
  nbody_config_defaults(&c);
  try {
    if (j.kind != JVal::Obj)
      throw ConfigError(std::string("[json.exception.type_error.306] cannot use value() with ") +
                        j.kind_name());
    get_int(j, "n_particles", c.n_particles);
    get_float(j, "disk_r_min", c.disk_r_min);
    get_float(j, "disk_r_max", c.disk_r_max);
    get_float(j, "disk_h_factor", c.disk_h_factor);
    get_float(j, "particle_mass_msun", c.particle_mass_msun);
    get_float(j, "star_mass_msun", c.star_mass_msun);
    get_float(j, "softening_AU", c.softening_AU);
    get_float(j, "theta", c.theta);
    get_float(j, "collision_radius_factor", c.collision_radius_factor);
    get_float(j, "restitution", c.restitution);
    get_float(j, "gas_drag_rate", c.gas_drag_rate);
    get_float(j, "dt", c.dt);
    get_float(j, "total_time", c.total_time);
    get_int(j, "output_every_n_steps", c.output_every_n_steps);
    get_string(j, "output_dir", c.output_dir, sizeof(c.output_dir));
    get_bool(j, "perturber_enabled", c.perturber_enabled);
    get_float(j, "perturber_mass_mjup", c.perturber_mass_mjup);
    get_float(j, "perturber_radius_AU", c.perturber_radius_AU);
    get_float(j, "perturber_phase0", c.perturber_phase0);
    // validation, Config.cpp:40-52 (same order and messages)
    if (c.perturber_enabled) {
      if (c.perturber_mass_mjup <= 0.0f) throw ConfigError("perturber_mass_mjup must be positive");
      if (c.perturber_radius_AU <= 0.0f) throw ConfigError("perturber_radius_AU must be positive");
    }
    if (c.n_particles <= 0)
      throw ConfigError("n_particles must be positive, got: " + std::to_string(c.n_particles));
    if (c.dt <= 0.f) throw ConfigError("dt must be positive");
    if (c.disk_r_min >= c.disk_r_max) throw ConfigError("disk_r_min must be less than disk_r_max");
  } catch (const ConfigError& e) {
    nb::set_error(e.what());
    return NBODY_ERR_CONFIG;
  }
  *cfg = c;
  return NBODY_OK;
}

float nbody_particle_radius(float particle_mass_msun) {
  // DiskInit.cpp:10-16, float arithmetic
  float mass_kg = particle_mass_msun * kMsunKg;
  float density = 3000.0f;
  float vol = mass_kg / density;
  float r_m = std::cbrt(3.0f * vol / (4.0f * kPi));
  return r_m / kAuM;
}

void nbody_perturber_make(const nbody_config* cfg, nbody_perturber* p) {
  std::memset(p, 0, sizeof(*p));
  p->enabled = cfg->perturber_enabled ? 1 : 0;
  if (!p->enabled) return;
  p->r = cfg->perturber_radius_AU;
  p->mass_msun = cfg->perturber_mass_mjup * kMjupToMsun;
  p->phase0 = cfg->perturber_phase0;
  p->omega = std::sqrt(cfg->star_mass_msun / (p->r * p->r * p->r));
  p->x = p->r * std::cos(p->phase0);
  p->z = p->r * std::sin(p->phase0);
  p->y = 0.f;
}

void nbody_perturber_update(nbody_perturber* p, float sim_time) {
  if (!p->enabled) return;
  float phi = p->phase0 + p->omega * sim_time;
  p->x = p->r * std::cos(phi);
  p->z = p->r * std::sin(phi);
  p->y = 0.f;
}

int nbody_aggregates(const float* x, const float* y, const float* z, const float* vx,
                     const float* vy, const float* vz, const int* labels, int n,
                     float particle_mass, nbody_aggregate* out, int max_aggs, int* n_aggs) {
  if (!x || !y || !z || !vx || !vy || !vz || !labels || !n_aggs || n < 0 || (max_aggs > 0 && !out)) {
    nb::set_error("nbody_aggregates: bad argument");
    return NBODY_ERR_ARG;
  }
  std::vector<int> cnt(n, 0), slot(n, -1);
  for (int i = 0; i < n; ++i) {
    if (labels[i] < 0 || labels[i] >= n) {
      nb::set_error("nbody_aggregates: label out of range");
      return NBODY_ERR_ARG;
    }
    cnt[labels[i]]++;
  }
  int g = 0;
  for (int i = 0; i < n; ++i) {
    if (labels[i] == i && cnt[i] >= 2) {
      if (g < max_aggs) {
        slot[i] = g;
        nbody_aggregate& a = out[g];
        std::memset(&a, 0, sizeof(a));
        a.id = g;
        a.n_particles = cnt[i];
        a.mass_msun = a.n_particles * particle_mass;  // Aggregate.cpp:59
        a.first_member = i;
      }
      ++g;
    }
  }
  // sums in ascending member index (Aggregate.cpp:62-66), FP32
  for (int i = 0; i < n; ++i) {
    int s = slot[labels[i]];
    if (s < 0) continue;
    nbody_aggregate& a = out[s];
    a.cx += x[i]; a.cy += y[i]; a.cz += z[i];
    a.vx += vx[i]; a.vy += vy[i]; a.vz += vz[i];
  }
  const int written = g < max_aggs ? g : max_aggs;
  for (int s = 0; s < written; ++s) {
    nbody_aggregate& a = out[s];
    float inv = 1.0f / static_cast<float>(a.n_particles);
    a.cx *= inv; a.cy *= inv; a.cz *= inv;
    a.vx *= inv; a.vy *= inv; a.vz *= inv;
    a.dist_center = std::sqrt(a.cx * a.cx + a.cy * a.cy + a.cz * a.cz);
  }
  *n_aggs = g;
  return NBODY_OK;
}

int nbody_writer_open(const char* dir, const nbody_config* cfg, nbody_writer** out) {
  if (!dir || !cfg || !out) {
    nb::set_error("nbody_writer_open: null argument");
    return NBODY_ERR_ARG;
  }
  *out = nullptr;
  nbody_writer* w = new nbody_writer();
  w->cfg = *cfg;
  std::string frames_path = std::string(dir) + "/frames.bin";
  w->frames.open(frames_path, std::ios::binary | std::ios::out | std::ios::trunc);
  if (!w->frames.is_open()) {
    nb::set_error("OutputWriter: cannot open " + frames_path);
    delete w;
    return NBODY_ERR_IO;
  }
  std::string stats_path = std::string(dir) + "/stats.csv";
  w->stats.open(stats_path, std::ios::out | std::ios::trunc);
  if (!w->stats.is_open()) {
    nb::set_error("OutputWriter: cannot open " + stats_path);
    delete w;
    return NBODY_ERR_IO;
  }
  // frames.bin v2 header (OutputWriter.cpp:56-79): "NBOD", version 2,
  // n_particles, n_frames (patched by finalize), dt, output_dt as doubles
  w->frames.write("NBOD", 4);
  write_raw(w->frames, (uint32_t)2u);
  write_raw(w->frames, (uint32_t)cfg->n_particles);
  w->n_frames_offset = w->frames.tellp();
  write_raw(w->frames, (uint32_t)0u);
  write_raw(w->frames, (double)cfg->dt);
  write_raw(w->frames, (double)cfg->dt * (double)cfg->output_every_n_steps);
  // stats.csv header (OutputWriter.cpp:84-88)
  w->stats << "frame,sim_time_T0,sim_time_years,n_aggregates,"
           << "agg_id,n_particles,mass_Msun,mass_Mearth,"
           << "cx_AU,cy_AU,cz_AU,vx,vy,vz,dist_center_AU\n";
  *out = w;
  return NBODY_OK;
}

int nbody_writer_frame(nbody_writer* w, const float* x, const float* y, const float* z, int n,
                       float sim_time, const uint16_t* agg_size) {
  if (!w || n < 0 || (n > 0 && (!x || !y || !z || !agg_size))) {
    nb::set_error("nbody_writer_frame: bad argument");
    return NBODY_ERR_ARG;
  }
  write_raw(w->frames, (double)sim_time);
  w->frames.write(reinterpret_cast<const char*>(x), (std::streamsize)n * sizeof(float));
  w->frames.write(reinterpret_cast<const char*>(y), (std::streamsize)n * sizeof(float));
  w->frames.write(reinterpret_cast<const char*>(z), (std::streamsize)n * sizeof(float));
  w->frames.write(reinterpret_cast<const char*>(agg_size), (std::streamsize)n * sizeof(uint16_t));
  if (!w->frames) {
    nb::set_error("nbody_writer_frame: write failed");
    return NBODY_ERR_IO;
  }
  return NBODY_OK;
}

int nbody_writer_stats(nbody_writer* w, const nbody_aggregate* aggs, int n_aggs, int frame_idx,
                       float sim_time) {
  if (!w || n_aggs < 0 || (n_aggs > 0 && !aggs)) {
    nb::set_error("nbody_writer_stats: bad argument");
    return NBODY_ERR_ARG;
  }
  float sim_years = sim_time * kT0ToYears;
  for (int k = 0; k < n_aggs; ++k) {
    const nbody_aggregate& a = aggs[k];
    w->stats << frame_idx << ',' << sim_time << ',' << sim_years << ',' << n_aggs << ','
             << a.id << ',' << a.n_particles << ',' << a.mass_msun << ','
             << (a.mass_msun * kMsunToMearth) << ',' << a.cx << ',' << a.cy << ',' << a.cz << ','
             << a.vx << ',' << a.vy << ',' << a.vz << ',' << a.dist_center << '\n';
  }
  return NBODY_OK;
}

int nbody_writer_perturber(nbody_writer* w, int frame_idx, float sim_time, int n_aggregates,
                           float px, float py, float pz, float mass_msun, float omega) {
  if (!w) {
    nb::set_error("nbody_writer_perturber: null writer");
    return NBODY_ERR_ARG;
  }
  // OutputWriter.cpp:161-186
  float sim_years = sim_time * kT0ToYears;
  float r = std::sqrt(px * px + pz * pz);
  float v_mag = omega * r;
  float vx = (r > 0.f) ? (-pz / r) * v_mag : 0.f;
  float vz = (r > 0.f) ? (px / r) * v_mag : 0.f;
  float vy = 0.f;
  w->stats << frame_idx << ',' << sim_time << ',' << sim_years << ',' << n_aggregates << ','
           << -1 << ',' << 0 << ',' << mass_msun << ',' << (mass_msun * kMsunToMearth) << ','
           << px << ',' << py << ',' << pz << ',' << vx << ',' << vy << ',' << vz << ',' << r
           << '\n';
  return NBODY_OK;
}

int nbody_writer_finalize(nbody_writer* w, int total_frames) {
  if (!w) {
    nb::set_error("nbody_writer_finalize: null writer");
    return NBODY_ERR_ARG;
  }
  w->frames.seekp(w->n_frames_offset);
  write_raw(w->frames, (uint32_t)total_frames);
  w->frames.flush();
  w->stats.flush();
  if (!w->frames || !w->stats) {
    nb::set_error("nbody_writer_finalize: write failed");
    return NBODY_ERR_IO;
  }
  return NBODY_OK;
}

void nbody_writer_close(nbody_writer* w) { delete w; }

int nbody_make_disk(int n, double r_min, double r_max, double sigma_e, double sigma_i,
                    double mu, uint64_t seed, double* x, double* y, double* z, double* vx,
                    double* vy, double* vz) {
  if (n < 0 || !(r_min > 0) || !(r_max > r_min) || !(mu > 0) || (n > 0 && (!x || !y || !z || !vx || !vy || !vz))) {
    nb::set_error("nbody_make_disk: bad argument");
    return NBODY_ERR_ARG;
  }
  for (int i = 0; i < n; ++i) {
    double st[6];
    nb::disk_body(seed, (uint64_t)i, r_min, r_max, sigma_e, sigma_i, mu, st);
    x[i] = st[0]; y[i] = st[1]; z[i] = st[2];
    vx[i] = st[3]; vy[i] = st[4]; vz[i] = st[5];
  }
  return NBODY_OK;
}

}  // extern "C"
