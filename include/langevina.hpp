// langevina.hpp -- C++17 host API of the B200 Model A / Model G stepper.
//
// Header-only layer over the C ABI of lgv.h that keeps the reference's host
// interface (derek-teaney/langevinA, ModelG/):
//   ModelATime / ModelACoefficients / ModelAHandlerData / ModelAData  (ModelA.h:32-269)
//     read from the same JSON keys with the same defaults;
//   NoiseGenerator (NoiseGenerator.h:62-157): the reference's serial host
//     stream (seed_seq -> per-rank xoroshiro128+ -> libstdc++ distributions),
//     used for host-side draws and written to <tag>_<rank>.rng;
//   ModelA (ModelA.h:291-526): the lattice lives on the GPU behind an lgv handle;
//   Stepper and its subclasses (Stepper.h:6-211): step(dt) / finalize();
//   Measurer (measurer.h:88-194): measure() fills the same public arrays;
//   measurer_output: one row per save() for each dataset of the reference's
//     measurement file (measurer_output.cxx:119-217), stored as raw FP64 rows.
// No computation happens here: every step and measurement runs in liblgv.so.
#pragma once

#include <array>
#include <cctype>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "lgv.h"

namespace langevina {

inline void check(int status, const char *where) {
  if (status != LGV_OK) throw std::runtime_error(std::string(where) + ": " + lgv_last_error());
}

// ---------------------------------------------------------------------------
// Minimal JSON value and reader.  Accepts what jsoncpp's default reader
// accepts in the reference's inputs, including a trailing comma before '}'
// (input.json:25).
class Json {
 public:
  enum Type { Null, Bool, Number, String, Array, Object };
  Type type = Null;
  bool b = false;
  double num = 0;
  std::string str;
  std::vector<Json> arr;
  std::map<std::string, Json> obj;

  bool has(const std::string &k) const { return type == Object && obj.count(k); }
  const Json &operator[](const std::string &k) const {
    static const Json none;
    auto it = obj.find(k);
    return it == obj.end() ? none : it->second;
  }
  double get(const std::string &k, double def) const {
    const Json &v = (*this)[k];
    if (v.type == Number) return v.num;
    if (v.type == Bool) return v.b ? 1.0 : 0.0;
    return def;
  }
  bool get(const std::string &k, bool def) const {
    const Json &v = (*this)[k];
    if (v.type == Bool) return v.b;
    if (v.type == Number) return v.num != 0;
    if (v.type == String) return v.str == "true";
    return def;
  }
  std::string get(const std::string &k, const std::string &def) const {
    const Json &v = (*this)[k];
    return v.type == String ? v.str : def;
  }

  static Json parse(const std::string &text) {
    size_t i = 0;
    Json v = parse_value(text, i);
    skip(text, i);
    if (i != text.size()) throw std::runtime_error("json: trailing characters at " + std::to_string(i));
    return v;
  }
  static Json parse_file(const std::string &path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("Unable to open input file " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return parse(ss.str());
  }

 private:
  static void skip(const std::string &s, size_t &i) {
    for (;;) {
      while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
      if (i + 1 < s.size() && s[i] == '/' && s[i + 1] == '/') {  // jsoncpp allows comments
        while (i < s.size() && s[i] != '\n') ++i;
        continue;
      }
      if (i + 1 < s.size() && s[i] == '/' && s[i + 1] == '*') {
        size_t e = s.find("*/", i + 2);
        i = (e == std::string::npos) ? s.size() : e + 2;
        continue;
      }
      return;
    }
  }
  static Json parse_value(const std::string &s, size_t &i) {
    skip(s, i);
    if (i >= s.size()) throw std::runtime_error("json: unexpected end");
    Json v;
    const char c = s[i];
    if (c == '{') {
      v.type = Object;
      ++i;
      for (;;) {
        skip(s, i);
        if (i < s.size() && s[i] == '}') { ++i; break; }
        Json key = parse_value(s, i);
        if (key.type != String) throw std::runtime_error("json: object key is not a string");
        skip(s, i);
        if (i >= s.size() || s[i] != ':') throw std::runtime_error("json: expected ':'");
        ++i;
        v.obj[key.str] = parse_value(s, i);
        skip(s, i);
        if (i < s.size() && s[i] == ',') { ++i; continue; }
        if (i < s.size() && s[i] == '}') { ++i; break; }
        throw std::runtime_error("json: expected ',' or '}'");
      }
    } else if (c == '[') {
      v.type = Array;
      ++i;
      for (;;) {
        skip(s, i);
        if (i < s.size() && s[i] == ']') { ++i; break; }
        v.arr.push_back(parse_value(s, i));
        skip(s, i);
        if (i < s.size() && s[i] == ',') { ++i; continue; }
        if (i < s.size() && s[i] == ']') { ++i; break; }
        throw std::runtime_error("json: expected ',' or ']'");
      }
    } else if (c == '"') {
      v.type = String;
      ++i;
      while (i < s.size() && s[i] != '"') {
        if (s[i] == '\\' && i + 1 < s.size()) {
          const char e = s[i + 1];
          v.str += (e == 'n') ? '\n' : (e == 't') ? '\t' : e;
          i += 2;
        } else {
          v.str += s[i++];
        }
      }
      if (i >= s.size()) throw std::runtime_error("json: unterminated string");
      ++i;
    } else if (s.compare(i, 4, "true") == 0) {
      v.type = Bool; v.b = true; i += 4;
    } else if (s.compare(i, 5, "false") == 0) {
      v.type = Bool; v.b = false; i += 5;
    } else if (s.compare(i, 4, "null") == 0) {
      i += 4;
    } else {
      size_t used = 0;
      v.type = Number;
      v.num = std::stod(s.substr(i, 64), &used);
      if (used == 0) throw std::runtime_error("json: bad value");
      i += used;
    }
    return v;
  }
};

// ---------------------------------------------------------------------------
// Run data (ModelA.h:32-269): same keys, same defaults.
struct ModelATime {
  double finaltime = 10., initialtime = 0., deltat = 0.24, time = 0.;
  double t() const { return time; }
  double dt() const { return deltat; }
  double tinitial() const { return initialtime; }
  double tfinal() const { return finaltime; }
  void operator+=(const double &d) { time += d; }
  void reset() { time = initialtime; }
  double adjust_finaltime(const int &saveFrequency) {  // ModelA.h:48-53
    finaltime = initialtime + deltat * saveFrequency *
                                  static_cast<int>((finaltime - initialtime) / (deltat * saveFrequency));
    return finaltime;
  }
  void read(const Json &p) {
    finaltime = p.get("finaltime", finaltime);
    initialtime = p.get("initialtime", initialtime);
    deltat = p.get("deltat", deltat);
    time = initialtime;
  }
};

struct ModelACoefficients {
  double mass0 = -4.70052, dmassdt = 0., lambda = 4., H = 0.003, chi = 5, gamma = 1., diffusion = 0.3333333;
  double mass(const double &t) const { return mass0 + dmassdt * t; }
  double sigma() const { return diffusion * chi; }
  double D() const { return diffusion; }
  void read(const Json &p) {
    mass0 = p.get("mass0", mass0);
    dmassdt = p.get("dmassdt", 0.);
    lambda = p.get("lambda", lambda);
    H = p.get("H", H);
    chi = p.get("chi", chi);
    gamma = p.get("gamma", gamma);
    diffusion = p.get("diffusion", 1. / 3. * gamma);
  }
};

struct ModelAHandlerData {
  std::string evolverType = "PV2HBSplit23";
  int seed = 10;
  bool restart = false;
  std::string outputfiletag = "o4output";
  int saveFrequency = 3;
  int writeFrequency = -1;
  bool eventmode = false;
  int nevents = 1;
  int current_event = 0;
  double thermalization_time = 0.;
  bool quench_mode = false;
  double quench_mode_mass0 = -4.70052;
  void read(const Json &p) {
    evolverType = p.get("evolverType", evolverType);
    seed = (int)p.get("seed", (double)seed);
    restart = p.get("restart", false);
    outputfiletag = p.get("outputfiletag", std::string("o4output"));
    saveFrequency = (int)p.get("saveFrequency", (double)saveFrequency);
    writeFrequency = (int)p.get("writeFrequency", (double)writeFrequency);
    thermalization_time = p.get("thermalization_time", thermalization_time);
    quench_mode = p.get("quench_mode", quench_mode);
    quench_mode_mass0 = p.get("quench_mode_mass0", quench_mode_mass0);
    eventmode = p.get("eventmode", eventmode);
    nevents = (int)p.get("nevents", (double)nevents);
  }
};

class ModelAData {
 public:
  int NX = 16, NY = 16, NZ = 16;
  double LX = 16., LY = 16., LZ = 16.;
  static const int Nphi = 4, NA = 3, NV = 3, Ndof = 10;
  ModelATime atime;
  ModelACoefficients acoefficients;
  ModelAHandlerData ahandler;

  explicit ModelAData(const Json &params) {
    if (!params.has("NX")) throw std::runtime_error("ModelAData: NX is required");
    NX = (int)params["NX"].num;
    NY = NZ = NX;
    LX = (double)(int)params.get("LX", (double)NX);  // read as an integer (ModelA.h:229)
    LY = LZ = LX;
    atime.read(params);
    acoefficients.read(params);
    ahandler.read(params);
    atime.adjust_finaltime(ahandler.saveFrequency);
  }
  double hX() const { return LX / NX; }
  double mass() const { return acoefficients.mass(atime.t()); }

  lgv_params params() const {
    lgv_params p{};
    p.N = NX;
    p.LX = LX;
    p.mass0 = acoefficients.mass0;
    p.dmassdt = acoefficients.dmassdt;
    p.lambda = acoefficients.lambda;
    p.H = acoefficients.H;
    p.chi = acoefficients.chi;
    p.gamma = acoefficients.gamma;
    p.diffusion = acoefficients.diffusion;
    p.seed = (uint64_t)(uint32_t)ahandler.seed;
    return p;
  }
  void print(FILE *fh = stdout) const {
    fprintf(fh, "NX = %d\nNY = %d\nNZ = %d\nLX = %e\nLY = %e\nLZ = %e\n", NX, NY, NZ, LX, LY, LZ);
    fprintf(fh, "finaltime = %e\ninitialtime = %e\ndeltat  = %e\n", atime.finaltime, atime.initialtime, atime.deltat);
    const auto &c = acoefficients;
    fprintf(fh, "mass0 = %e\ndmassdt = %e\nlambda = %e\nH = %e\nchi = %e\ngamma = %e\ndiffusion = %e\n", c.mass0,
            c.dmassdt, c.lambda, c.H, c.chi, c.gamma, c.diffusion);
    const auto &h = ahandler;
    fprintf(fh, "evolverType = %s\nseed = %d\nrestart = %s\noutputfiletag = %s\nsaveFrequency = %d\n",
            h.evolverType.c_str(), h.seed, h.restart ? "true" : "false", h.outputfiletag.c_str(), h.saveFrequency);
    fprintf(fh, "thermalization_time = %e\nquench_mode = %s\nquench_mode_mass0 = %e\neventmode = %s\nnevents = %d\n",
            h.thermalization_time, h.quench_mode ? "true" : "false", h.quench_mode_mass0,
            h.eventmode ? "true" : "false", h.nevents);
  }
};

// ---------------------------------------------------------------------------
// NoiseGenerator (NoiseGenerator.h:62-157): the reference's serial host stream.
class xoroshiro128plus {  // xoroshiro128plus.h:63-149 (engine :86-107, stream I/O :137-142)
 public:
  typedef uint64_t result_type;
  static constexpr uint64_t min() { return 0; }
  static constexpr uint64_t max() { return ~uint64_t(0); }
  void seed(uint64_t v) {
    s[0] = 0x01d353e5f3993bb0ull + v;
    s[1] = 0x7b9c0df6cb193b20ull * (v + 1);
  }
  uint64_t operator()() {
    const uint64_t s0 = s[0];
    uint64_t s1 = s[1];
    const uint64_t r = s0 + s1;
    s1 ^= s0;
    s[0] = rotl(s0, 55) ^ s1 ^ (s1 << 14);
    s[1] = rotl(s1, 36);
    return r;
  }
  friend std::ostream &operator<<(std::ostream &o, const xoroshiro128plus &x) { return o << x.s[0] << ' ' << x.s[1]; }
  friend std::istream &operator>>(std::istream &i, xoroshiro128plus &x) { return i >> x.s[0] >> x.s[1]; }

 private:
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t s[2] = {0, 0};
};

class NoiseGenerator {
 public:
  explicit NoiseGenerator(const int &baseSeed = 0, int rank = 0, int size = 1)
      : rt3(-std::sqrt(3.), std::sqrt(3.)) {
    std::seed_seq sequence = {baseSeed};
    std::vector<unsigned int> seeds(size, 0);
    sequence.generate(seeds.begin(), seeds.end());
    rng.seed(seeds[rank]);
    rank_ = rank;
  }
  double normal() { return nd(rng); }
  double uniform() { return u01(rng); }
  double uniformRt3() { return rt3(rng); }
  double variance1() { return rt3(rng); }
  xoroshiro128plus &generator() { return rng; }

  // <stub>_<rank>.rng holds "s0 s1" of the host engine (NoiseGenerator.h:112-127)
  // and, on a second line, the device counter of the counter-indexed streams.
  void write(const std::string &stub, uint64_t device_counter) const {
    std::ofstream out(stub + "_" + std::to_string(rank_) + ".rng");
    if (!out) throw std::runtime_error("NoiseGenerator::write: cannot open " + stub);
    out << rng << "\n" << device_counter << "\n";
  }
  // Returns the device counter (0 if the file has none); keeps the seed state
  // when the file is missing, like the reference (NoiseGenerator.h:131-146).
  uint64_t read(const std::string &stub) {
    std::ifstream in(stub + "_" + std::to_string(rank_) + ".rng");
    if (!in) {
      fprintf(stderr, "urng::read Unable to open file for reading in URNG. Defaulting to seed.\n");
      return 0;
    }
    in >> rng;
    uint64_t c = 0;
    if (!(in >> c)) c = 0;
    return c;
  }

 private:
  xoroshiro128plus rng;
  std::normal_distribution<double> nd;
  std::uniform_real_distribution<double> rt3;
  std::uniform_real_distribution<double> u01;
  int rank_ = 0;
};

// ---------------------------------------------------------------------------
// Raw FP64 array files: "<name>.npy" in NumPy's v1.0 format (little-endian
// '<f8', C order), so a restart state or a measurement series opens with
// numpy.load.  The reference stores the same arrays in HDF5 (o4fields of
// <tag>_save.h5, ModelA.h:384-402; ntuples of <tag>.h5).
inline void write_npy(const std::string &path, const std::vector<size_t> &shape, const double *data) {
  std::string dims;
  size_t n = 1;
  for (size_t i = 0; i < shape.size(); ++i) {
    dims += std::to_string(shape[i]) + (shape.size() == 1 ? "," : (i + 1 < shape.size() ? ", " : ""));
    n *= shape[i];
  }
  std::string header = "{'descr': '<f8', 'fortran_order': False, 'shape': (" + dims + "), }";
  const size_t total = 10 + header.size() + 1;
  header.append((64 - total % 64) % 64, ' ');
  header += '\n';
  std::ofstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot write " + path);
  const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
  f.write((const char *)magic, 8);
  const uint16_t hl = (uint16_t)header.size();
  f.write((const char *)&hl, 2);
  f.write(header.data(), header.size());
  f.write((const char *)data, n * sizeof(double));
}

inline std::vector<double> read_npy(const std::string &path, size_t expect) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::string("Unable to open file in restart mode with filename = ") + path;
  char magic[8];
  f.read(magic, 8);
  uint16_t hl = 0;
  f.read((char *)&hl, 2);
  std::string header(hl, ' ');
  f.read(&header[0], hl);
  if (header.find("'<f8'") == std::string::npos) throw std::string("restart file is not little-endian float64");
  std::vector<double> v(expect);
  f.read((char *)v.data(), expect * sizeof(double));
  if ((size_t)f.gcount() != expect * sizeof(double)) throw std::string("restart file too short: ") + path;
  return v;
}

// ---------------------------------------------------------------------------
// ModelA (ModelA.h:291-526).  The solution lives on the GPU.
class ModelA {
 public:
  ModelAData data;
  lgv_handle *handle = nullptr;
  std::unique_ptr<NoiseGenerator> rndm;  // ModelARndm for host-side draws
  int rank = 0;

  explicit ModelA(const ModelAData &in) : data(in) {
    const lgv_params p = data.params();
    check(lgv_create(&p, &handle), "lgv_create");
    rndm = std::make_unique<NoiseGenerator>(data.ahandler.seed);
    if (data.ahandler.restart && !data.ahandler.eventmode) {
      const uint64_t c = rndm->read(data.ahandler.outputfiletag);
      check(lgv_set_counter(handle, c), "lgv_set_counter");
    }
  }
  ModelA(const ModelA &) = delete;
  ModelA &operator=(const ModelA &) = delete;
  ~ModelA() {
    if (handle) lgv_destroy(handle);
  }

  size_t sites() const { return (size_t)data.NX * data.NY * data.NZ; }

  // Push the current coefficients (e.g. after a quench mass change).
  void sync_params() {
    const lgv_params p = data.params();
    check(lgv_set_params(handle, &p), "lgv_set_params");
  }

  void finalize() {  // ModelA.h:338-352
    if (!data.ahandler.eventmode) {
      uint64_t c = 0;
      check(lgv_get_counter(handle, &c), "lgv_get_counter");
      rndm->write(data.ahandler.outputfiletag, c);
      write(data.ahandler.outputfiletag);
    }
  }

  std::vector<double> get_state() const {
    std::vector<double> u(sites() * 10);
    check(lgv_get_state(handle, u.data()), "lgv_get_state");
    return u;
  }
  void set_state(const std::vector<double> &u) { check(lgv_set_state(handle, u.data()), "lgv_set_state"); }
  // Gaussian phi heat-bath proposals instead of the reference's uniform ones
  void set_hb_proposal(bool gaussian) {
    check(lgv_set_hb_proposal(handle, gaussian ? LGV_HB_PROPOSAL_GAUSSIAN : LGV_HB_PROPOSAL_UNIFORM),
          "lgv_set_hb_proposal");
  }

  // <tag>_save.npy: shape (NZ, NY, NX, 10), the o4fields layout
  void write(const std::string &tag) const {
    const auto u = get_state();
    write_npy(tag + "_save.npy", {(size_t)data.NZ, (size_t)data.NY, (size_t)data.NX, 10}, u.data());
  }
  void read(const std::string &tag) { set_state(read_npy(tag + "_save.npy", sites() * 10)); }

  // ModelA::initialize (ModelA.h:408-461): restart or zero start, or a
  // function f(x, y, z, L) evaluated on the host and uploaded.
  void initialize(double (*func)(const double &, const double &, const double &, const int &, void *) = nullptr,
                  void *params = nullptr) {
    if (data.ahandler.restart) {
      try {
        read(data.ahandler.outputfiletag);
        return;
      } catch (const std::string &error) {
        fprintf(stderr, "Error in restart -- aborting!\n%s\n", error.c_str());
        std::abort();
      }
    }
    if (!func) {
      check(lgv_initialize(handle, LGV_INIT_ZERO, 0.0), "lgv_initialize");
      return;
    }
    std::vector<double> u(sites() * 10);
    const double hx = data.hX();
    for (int k = 0; k < data.NZ; ++k)
      for (int j = 0; j < data.NY; ++j)
        for (int i = 0; i < data.NX; ++i)
          for (int L = 0; L < 10; ++L)
            u[(((size_t)k * data.NY + j) * data.NX + i) * 10 + L] = func(i * hx, j * hx, k * hx, L, params);
    set_state(u);
  }

  // ModelA::initialize_gaussian_charges (ModelA.h:463-525).  By default the
  // charges come from the device counter streams; with reference_stream the
  // host NoiseGenerator draws them in the reference's order (k, j, i, L).
  void initialize_gaussian_charges(bool reference_stream = false) {
    if (!reference_stream) {
      check(lgv_initialize(handle, LGV_INIT_CHARGES_GAUSSIAN, 0.0), "lgv_initialize");
      return;
    }
    auto u = get_state();
    std::vector<double> sum(10, 0.);
    const double sc = std::sqrt(data.acoefficients.chi);
    const size_t V = sites();
    for (size_t n = 0; n < V; ++n)
      for (int L = 4; L < 10; ++L) {
        u[n * 10 + L] = sc * rndm->normal();
        sum[L] += u[n * 10 + L];
      }
    for (size_t n = 0; n < V; ++n)
      for (int L = 4; L < 10; ++L) u[n * 10 + L] -= sum[L] / (double)V;
    set_state(u);
  }
};

// ---------------------------------------------------------------------------
// Steppers (Stepper.h).
class Stepper {
 public:
  virtual bool step(const double &dt) = 0;
  virtual void finalize() = 0;
  virtual ~Stepper() = default;
};

class LgvStepper : public Stepper {
 public:
  LgvStepper(ModelA &in, int evolver, unsigned inner = 1, unsigned outer = 1)
      : model(&in), ev(evolver), in_(inner), out_(outer) {}
  bool step(const double &dt) override {
    check(lgv_step(model->handle, ev, (int)in_, (int)out_, dt, model->data.atime.t(), 1), "lgv_step");
    return true;
  }
  void finalize() override {
    if (!print_monitors) return;
    const char *names[3] = {"Statistics of IdealPV2", "Phi HB Steps", "Charge HB Steps"};
    for (int w = 0; w < 3; ++w) {
      lgv_monitor m{};
      if (lgv_get_monitor(model->handle, w, &m) != LGV_OK) continue;
      const double tot = (double)(m.down_counts + m.up_counts);
      if (tot <= 0) continue;
      printf("==== Statistics for %s ====\n", names[w]);
      printf("Probability of up acceptance = %f\n", (m.up_yes + m.down_counts) / tot);
      printf("dS >0: accepts = %lld; probability of up accept = %f; mean dS=%f\n", (long long)m.up_yes,
             m.up_yes / tot, m.up_yes ? m.up_dS / m.up_yes : 0.);
      printf("dS <0: counts  = %lld; probability of down steps= %f; mean dS=%f\n", (long long)m.down_counts,
             m.down_counts / tot, m.down_counts ? m.down_dS / m.down_counts : 0.);
      printf("============================================\n");
    }
  }
  bool print_monitors = false;

 protected:
  ModelA *model;
  int ev;
  unsigned in_, out_;
};

class IdealPV2 : public LgvStepper {
 public:
  explicit IdealPV2(ModelA &in) : LgvStepper(in, LGV_IDEAL_PV2) {}
};
class EulerLangevinHB : public LgvStepper {
 public:
  explicit EulerLangevinHB(ModelA &in) : LgvStepper(in, LGV_EULER_LANGEVIN_HB) {}
};
class ModelGChargeHB : public LgvStepper {
 public:
  explicit ModelGChargeHB(ModelA &in) : LgvStepper(in, LGV_CHARGE_HB) {}
};
class ModelAEulerMaruyama : public LgvStepper {
 public:
  explicit ModelAEulerMaruyama(ModelA &in) : LgvStepper(in, LGV_MODELA_EM) {}
};
// Ideal step then Euler-Maruyama relaxation of phi (no counterpart in the reference).
class IdealEulerMaruyama : public LgvStepper {
 public:
  explicit IdealEulerMaruyama(ModelA &in) : LgvStepper(in, LGV_IDEAL_EM) {}
};
class PV2HBSplit : public LgvStepper {  // Stepper.h:176-211
 public:
  PV2HBSplit(ModelA &in, const std::array<unsigned int, 2> &scounts = {1, 1}, const bool &nodiffuse = false,
             const bool &onlydiffuse = false)
      : LgvStepper(in, onlydiffuse ? LGV_PV2HBSPLIT_ONLYDIFFUSE : nodiffuse ? LGV_PV2HBSPLIT_NODIFFUSE : LGV_PV2HBSPLIT,
                   scounts[0], scounts[1]) {}
};

// The evolverType switch of SuperPions.cxx:209-225 (plus the Model A steppers).
inline std::unique_ptr<Stepper> make_stepper(ModelA &model, const std::string &etype) {
  if (etype == "PV2HBSplit23") return std::make_unique<PV2HBSplit>(model, std::array<unsigned, 2>{2, 3});
  if (etype == "PV2HBSplit23NoDiffuse")
    return std::make_unique<PV2HBSplit>(model, std::array<unsigned, 2>{2, 3}, true);
  if (etype == "PV2HBSplit23OnlyDiffuse")
    return std::make_unique<PV2HBSplit>(model, std::array<unsigned, 2>{2, 3}, false, true);
  if (etype == "PV2HBSplit11") return std::make_unique<PV2HBSplit>(model, std::array<unsigned, 2>{1, 1});
  if (etype == "EulerLangevinHB") return std::make_unique<EulerLangevinHB>(model);
  if (etype == "ModelAEulerMaruyama") return std::make_unique<ModelAEulerMaruyama>(model);
  if (etype == "IdealEulerMaruyama") return std::make_unique<IdealEulerMaruyama>(model);
  return nullptr;
}

// ---------------------------------------------------------------------------
// Measurer (measurer.h:88-194): the same public arrays, filled on the GPU.
template <typename T>
struct nvector2 {  // row-major [N0][N1] (nvector.h)
  std::array<size_t, 2> N{{0, 0}};
  std::vector<T> v;
  void resize(size_t a, size_t b) {
    N = {a, b};
    v.assign(a * b, T());
  }
  T &operator()(size_t i, size_t j) { return v[i * N[1] + j]; }
  const T &operator()(size_t i, size_t j) const { return v[i * N[1] + j]; }
};

class Measurer {
 public:
  static const int NObs = 11, NScalars = 11, NObsRotated = 14, NObsPhase = 14;
  std::vector<double> OAverage;
  nvector2<double> wallX, wallY, wallZ;
  nvector2<std::complex<double>> wallX_k, wallY_k, wallZ_k;
  nvector2<std::complex<double>> wallX_k_rotated, wallY_k_rotated, wallZ_k_rotated;
  nvector2<double> wallXPhase, wallYPhase, wallZPhase;
  nvector2<std::complex<double>> wallXPhase_k, wallYPhase_k, wallZPhase_k;

  explicit Measurer(ModelA *ptr) : model(ptr), N(ptr->data.NX) {
    if (ptr->data.NX != ptr->data.NY || ptr->data.NX != ptr->data.NZ)
      throw std::runtime_error("Nx, Ny, and Nz must be equal for the correlation analysis to work");
    const size_t NK = N / 2 + 1;
    OAverage.assign(NScalars, 0.);
    for (auto *w : {&wallX, &wallY, &wallZ}) w->resize(NObs, N);
    for (auto *w : {&wallX_k, &wallY_k, &wallZ_k}) w->resize(NObs, NK);
    for (auto *w : {&wallX_k_rotated, &wallY_k_rotated, &wallZ_k_rotated}) w->resize(NObsRotated, NK);
    for (auto *w : {&wallXPhase, &wallYPhase, &wallZPhase}) w->resize(NObsPhase, N);
    for (auto *w : {&wallXPhase_k, &wallYPhase_k, &wallZPhase_k}) w->resize(NObsPhase, NK);
  }

  void measure() {
    lgv_measurement m{};
    m.OAverage = OAverage.data();
    nvector2<double> *W[3] = {&wallX, &wallY, &wallZ};
    nvector2<double> *P[3] = {&wallXPhase, &wallYPhase, &wallZPhase};
    nvector2<std::complex<double>> *K[3] = {&wallX_k, &wallY_k, &wallZ_k};
    nvector2<std::complex<double>> *R[3] = {&wallX_k_rotated, &wallY_k_rotated, &wallZ_k_rotated};
    nvector2<std::complex<double>> *PK[3] = {&wallXPhase_k, &wallYPhase_k, &wallZPhase_k};
    for (int a = 0; a < 3; ++a) {
      m.wall[a] = W[a]->v.data();
      m.wall_phase[a] = P[a]->v.data();
      // std::complex<double> is laid out as (re, im)
      m.wall_k[a] = reinterpret_cast<double *>(K[a]->v.data());
      m.wall_k_rotated[a] = reinterpret_cast<double *>(R[a]->v.data());
      m.wall_phase_k[a] = reinterpret_cast<double *>(PK[a]->v.data());
    }
    check(lgv_measure(model->handle, &m), "lgv_measure");
  }
  ModelA *getModel() { return model; }
  int getN() const { return N; }

 private:
  ModelA *model;
  int N;
};

// ---------------------------------------------------------------------------
// Measurement output (measurer_output.cxx:97-217): the datasets of the
// reference's measurement file, one row per save(), each written as
// <tag>.<dataset>.f64 (raw little-endian FP64 rows) with a JSON index
// <tag>.datasets.json giving every dataset's row shape.
class measurer_output {
 public:
  measurer_output(Measurer *in, const std::string &tag, bool append) : m(in), tag(tag) {
    const size_t N = in->getN(), NK = N / 2 + 1;
    shapes = {{"phi", {11}},
              {"timeout", {2}},
              {"wallx_k", {11, NK, 2}},
              {"wally_k", {11, NK, 2}},
              {"wallz_k", {11, NK, 2}},
              {"wallx_k_rotated", {14, NK, 2}},
              {"wally_k_rotated", {14, NK, 2}},
              {"wallz_k_rotated", {14, NK, 2}},
              {"wallx_phase_k", {14, NK, 2}},
              {"wally_phase_k", {14, NK, 2}},
              {"wallz_phase_k", {14, NK, 2}}};
    for (auto &s : shapes) {
      FILE *f = fopen((tag + "." + s.first + ".f64").c_str(), append ? "ab" : "wb");
      if (!f) throw std::runtime_error("measurer_output: cannot open " + tag + "." + s.first);
      files[s.first] = f;
    }
    std::ofstream idx(tag + ".datasets.json");
    idx << "{";
    bool first = true;
    for (auto &s : shapes) {
      idx << (first ? "" : ", ") << "\"" << s.first << "\": [";
      for (size_t i = 0; i < s.second.size(); ++i) idx << (i ? ", " : "") << s.second[i];
      idx << "]";
      first = false;
    }
    idx << "}\n";
  }
  ~measurer_output() {
    for (auto &f : files) fclose(f.second);
  }
  void save() {
    const double tm[2] = {m->getModel()->data.atime.t(), m->getModel()->data.mass()};
    put("timeout", tm, 2);
    put("phi", m->OAverage.data(), 11);
    put("wallx_k", (const double *)m->wallX_k.v.data(), m->wallX_k.v.size() * 2);
    put("wally_k", (const double *)m->wallY_k.v.data(), m->wallY_k.v.size() * 2);
    put("wallz_k", (const double *)m->wallZ_k.v.data(), m->wallZ_k.v.size() * 2);
    put("wallx_k_rotated", (const double *)m->wallX_k_rotated.v.data(), m->wallX_k_rotated.v.size() * 2);
    put("wally_k_rotated", (const double *)m->wallY_k_rotated.v.data(), m->wallY_k_rotated.v.size() * 2);
    put("wallz_k_rotated", (const double *)m->wallZ_k_rotated.v.data(), m->wallZ_k_rotated.v.size() * 2);
    put("wallx_phase_k", (const double *)m->wallXPhase_k.v.data(), m->wallXPhase_k.v.size() * 2);
    put("wally_phase_k", (const double *)m->wallYPhase_k.v.data(), m->wallYPhase_k.v.size() * 2);
    put("wallz_phase_k", (const double *)m->wallZPhase_k.v.data(), m->wallZPhase_k.v.size() * 2);
    for (auto &f : files) fflush(f.second);
  }

 private:
  void put(const std::string &name, const double *p, size_t n) {
    if (fwrite(p, sizeof(double), n, files[name]) != n) throw std::runtime_error("measurer_output: write failed");
  }
  Measurer *m;
  std::string tag;
  std::vector<std::pair<std::string, std::vector<size_t>>> shapes;
  std::map<std::string, FILE *> files;
};

}  // namespace langevina
