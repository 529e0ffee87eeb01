// ref_stepper_main.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Driver for the oracle's reference build: the reference's own ModelA,
// NoiseGenerator, Stepper (IdealPV2, EulerLangevinHB, ModelGChargeHB,
// PV2HBSplit) and Measurer, compiled unmodified against the single-node
// PETSc/MPI/FFTW stand-ins of oracle/shim/ (built by `make -C oracle ref`).
// It replaces SuperPions.cxx, whose measurement writer needs HDF5: the loop
// below is run_event's (SuperPions.cxx:76-161): step(atime.dt()), then
// atime += dt.
//
//   ref_stepper [--ranks R] params.json out.bin op [op ...]
//
// params.json is the reference's input file (ModelAData(Json::Value&),
// ModelA.h:222-248).  Operations, in order:
//   load=FILE             state from FILE: N^3 * 10 doubles, u[k][j][i][L]
//   phi=SCALE             ModelA::initialize with phi_a = SCALE * normal() from
//                         the reference's stream, charges 0 (ModelA.h:408-461)
//   charges               ModelA::initialize_gaussian_charges (ModelA.h:463-525)
//   step=NAME,n           n x { NAME.step(atime.dt()); atime += atime.dt() }
//   sub=NAME,n,d          n x NAME.step(atime.dt() / d), clock unchanged (the
//                         thermalisation loop, SuperPions.cxx:47-53)
//   measure               Measurer::measure; appends the packed measurement
//   sample=NAME,n,every   n x { every x NAME.step(atime.dt()); Measurer::measure },
//                         appending OAverage (11 doubles) of each measurement
//   save                  appends the state
//   energy                appends IdealPV2::computeEnergy of the state
//   finalize              finalize() of every stepper built so far (the
//                         reference prints its accept statistics)
// NAME: PV2HBSplit<inner><outer>[NoDiffuse|OnlyDiffuse], IdealPV2,
// EulerLangevinHB, ModelGChargeHB.  Steppers are built on first use and kept.
//
// out.bin is a sequence of records {u32 tag, u64 count, count doubles}; tags:
// 1 state, 2 measurement (OAverage, wall[3], wall_k[3], wall_k_rotated[3],
// wall_phase[3], wall_phase_k[3], each row-major, complex as re, im), 3
// energy, 4 OAverage of a sample.  Rank 0 writes it.  For every operation rank 0 prints
// "REFTIME <op> <seconds>" (wall clock between barriers), and at the end one
// "REFEVENT <name> <seconds> <count>" line per PetscLogEvent of the stepper.
//
// --ranks R forks R processes that share the global vectors and split the
// lattice into z-slabs, each rank with its own NoiseGenerator stream seeded as
// the reference seeds rank r of R (NoiseGenerator.h:68-81).

#include <sys/wait.h>
#include <unistd.h>

#include <array>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "ModelA.h"
#include "Stepper.h"
#include "measurer.h"

namespace {

struct Out {
  FILE *f = nullptr;
  void rec(uint32_t tag, const double *p, uint64_t n) {
    if (!f) return;
    std::fwrite(&tag, 4, 1, f);
    std::fwrite(&n, 8, 1, f);
    std::fwrite(p, 8, n, f);
  }
};

void append(std::vector<double> &v, const std::vector<double> &a) { v.insert(v.end(), a.begin(), a.end()); }
void append(std::vector<double> &v, const std::vector<std::complex<double>> &a) {
  for (const auto &c : a) {
    v.push_back(c.real());
    v.push_back(c.imag());
  }
}

// Initial condition for ModelA::initialize: phi_a ~ scale * N(0, 1) drawn
// from the reference's global stream, charges zero.
double gaussian_phi(const double &, const double &, const double &, const int &L, void *params) {
  return L < ModelAData::Nphi ? *(const double *)params * ModelARndm->normal() : 0.0;
}

std::unique_ptr<Stepper> make_stepper(const std::string &name, ModelA &model) {
  if (name == "IdealPV2") return std::make_unique<IdealPV2>(model);
  if (name == "EulerLangevinHB") return std::make_unique<EulerLangevinHB>(model);
  if (name == "ModelGChargeHB") return std::make_unique<ModelGChargeHB>(model);
  const std::string pre = "PV2HBSplit";
  if (name.compare(0, pre.size(), pre) == 0 && name.size() >= pre.size() + 2) {
    const unsigned inner = name[pre.size()] - '0', outer = name[pre.size() + 1] - '0';
    const std::string tail = name.substr(pre.size() + 2);
    if (inner >= 1 && inner <= 9 && outer >= 1 && outer <= 9 && (tail.empty() || tail == "NoDiffuse" || tail == "OnlyDiffuse")) {
      std::array<unsigned int, 2> s = {inner, outer};
      return std::make_unique<PV2HBSplit>(model, s, tail == "NoDiffuse", tail == "OnlyDiffuse");
    }
  }
  lgvshim::fail(("unknown stepper " + name).c_str());
}

int run(const std::string &params_path, const std::string &out_path, const std::vector<std::string> &ops) {
  const int rank = lgvshim::g_rank;
  Json::Value inputs;
  {
    std::ifstream ifs(params_path);
    if (!ifs) lgvshim::fail("cannot open the parameter file");
    ifs >> inputs;
  }
  ModelAData data(inputs);
  ModelA model(data);
  model.initialize();
  auto &atime = model.data.atime;
  atime.reset();

  Out out;
  if (rank == 0) {
    out.f = std::fopen(out_path.c_str(), "wb");
    if (!out.f) lgvshim::fail("cannot open the output file");
  }
  const int N = model.data.NX;
  const size_t V = (size_t)N * N * N;
  std::map<std::string, std::unique_ptr<Stepper>> steppers;
  std::vector<std::string> built;
  std::unique_ptr<Measurer> measurer;
  std::unique_ptr<IdealPV2> energy_probe;

  for (const std::string &op : ops) {
    lgvshim::barrier();
    const auto t0 = std::chrono::steady_clock::now();
    const size_t eq = op.find('=');
    const std::string verb = op.substr(0, eq);
    const std::string arg = eq == std::string::npos ? "" : op.substr(eq + 1);
    if (verb == "load") {
      Vec u = model.solution;
      FILE *f = std::fopen(arg.c_str(), "rb");
      if (!f) lgvshim::fail("cannot open the state file");
      if (std::fseek(f, (long)(u->lo * sizeof(double)), SEEK_SET) != 0) lgvshim::fail("seek in the state file");
      const size_t n = u->hi - u->lo;
      if (std::fread(u->a + u->lo, sizeof(double), n, f) != n) lgvshim::fail("short state file");
      std::fclose(f);
    } else if (verb == "phi") {
      double scale = std::stod(arg);
      model.initialize(gaussian_phi, &scale);
    } else if (verb == "charges") {
      model.initialize_gaussian_charges();
    } else if (verb == "step" || verb == "sub") {
      std::vector<std::string> f;
      size_t a = 0;
      for (;;) {
        const size_t c = arg.find(',', a);
        f.push_back(arg.substr(a, c == std::string::npos ? std::string::npos : c - a));
        if (c == std::string::npos) break;
        a = c + 1;
      }
      if ((verb == "step" && f.size() != 2) || (verb == "sub" && f.size() != 3)) lgvshim::fail("bad step operation");
      auto it = steppers.find(f[0]);
      if (it == steppers.end()) {
        it = steppers.emplace(f[0], make_stepper(f[0], model)).first;
        built.push_back(f[0]);
      }
      const int n = std::stoi(f[1]);
      if (verb == "step") {
        for (int s = 0; s < n; ++s) {
          it->second->step(atime.dt());
          atime += atime.dt();
        }
      } else {
        const double d = std::stod(f[2]);
        for (int s = 0; s < n; ++s) it->second->step(atime.dt() / d);
      }
    } else if (verb == "sample") {
      const size_t c1 = arg.find(','), c2 = arg.find(',', c1 + 1);
      if (c1 == std::string::npos || c2 == std::string::npos) lgvshim::fail("bad sample operation");
      const std::string name = arg.substr(0, c1);
      const int n = std::stoi(arg.substr(c1 + 1, c2 - c1 - 1)), every = std::stoi(arg.substr(c2 + 1));
      auto it = steppers.find(name);
      if (it == steppers.end()) {
        it = steppers.emplace(name, make_stepper(name, model)).first;
        built.push_back(name);
      }
      if (!measurer) measurer = std::make_unique<Measurer>(&model);
      for (int c = 0; c < n; ++c) {
        for (int s = 0; s < every; ++s) {
          it->second->step(atime.dt());
          atime += atime.dt();
        }
        measurer->measure(&model.solution);
        if (rank == 0) out.rec(4, measurer->OAverage.data(), measurer->OAverage.size());
      }
    } else if (verb == "measure") {
      if (!measurer) measurer = std::make_unique<Measurer>(&model);
      measurer->measure(&model.solution);
      if (rank == 0) {
        Measurer &m = *measurer;
        std::vector<double> v;
        append(v, m.OAverage);
        append(v, m.wallX.v), append(v, m.wallY.v), append(v, m.wallZ.v);
        append(v, m.wallX_k.v), append(v, m.wallY_k.v), append(v, m.wallZ_k.v);
        append(v, m.wallX_k_rotated.v), append(v, m.wallY_k_rotated.v), append(v, m.wallZ_k_rotated.v);
        append(v, m.wallXPhase.v), append(v, m.wallYPhase.v), append(v, m.wallZPhase.v);
        append(v, m.wallXPhase_k.v), append(v, m.wallYPhase_k.v), append(v, m.wallZPhase_k.v);
        out.rec(2, v.data(), v.size());
      }
    } else if (verb == "save") {
      lgvshim::barrier();
      if (rank == 0) out.rec(1, model.solution->a, V * ModelAData::Ndof);
    } else if (verb == "energy") {
      if (!energy_probe) energy_probe = std::make_unique<IdealPV2>(model);
      const double e = energy_probe->computeEnergy(atime.dt());
      if (rank == 0) out.rec(3, &e, 1);
    } else if (verb == "finalize") {
      std::fflush(stdout);
      for (const std::string &name : built) steppers[name]->finalize();
      steppers.clear();
      built.clear();
      std::fflush(stdout);
    } else {
      lgvshim::fail(("unknown operation " + op).c_str());
    }
    lgvshim::barrier();
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rank == 0) {
      std::printf("REFTIME %s %.9f\n", op.c_str(), sec);
      std::fflush(stdout);
    }
  }
  if (rank == 0) {
    for (const auto &e : lgvshim::g_events) std::printf("REFEVENT %s %.9f %ld\n", e.name.c_str(), e.seconds, e.count);
    std::fflush(stdout);
    std::fclose(out.f);
  }
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  int R = 1, a = 1;
  if (argc > 2 && std::string(argv[1]) == "--ranks") {
    R = std::atoi(argv[2]);
    a = 3;
  }
  if (argc - a < 2 || R < 1) {
    std::fprintf(stderr, "usage: %s [--ranks R] params.json out.bin op [op ...]\n", argv[0]);
    return 2;
  }
  const std::string params = argv[a], outp = argv[a + 1];
  std::vector<std::string> ops(argv + a + 2, argv + argc);

  // The arena holds the global vectors ModelA creates (solution and
  // previoussolution), with room to spare.
  size_t N = 0;
  {
    Json::Value in;
    std::ifstream ifs(params);
    if (!ifs) {
      std::fprintf(stderr, "cannot open %s\n", params.c_str());
      return 2;
    }
    ifs >> in;
    N = (size_t)in["NX"].asInt();
  }
  const size_t vec_bytes = (N * N * N * ModelAData::Ndof * sizeof(double) + 255) / 256 * 256;
  lgvshim::setup_shared(R, 3 * vec_bytes, (N + 64) * sizeof(double) * 2);

  std::vector<pid_t> kids;
  for (int r = 1; r < R; ++r) {
    const pid_t p = fork();
    if (p < 0) lgvshim::fail("fork failed");
    if (p == 0) {
      lgvshim::g_rank = r;
      std::_Exit(run(params, outp, ops));
    }
    kids.push_back(p);
  }
  int rc = run(params, outp, ops);
  for (pid_t p : kids) {
    int st = 0;
    waitpid(p, &st, 0);
    if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) rc = 3;
  }
  return rc;
}
