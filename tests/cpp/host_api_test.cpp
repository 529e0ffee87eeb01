// Host-side checks of include/langevina.hpp that need no GPU: the JSON reader
// on a reference-style input (trailing comma, comments), ModelAData keys and
// defaults (ModelA.h:32-269), adjust_finaltime (ModelA.h:48-53), the host
// NoiseGenerator stream against the reference engine's golden draws, and the
// .npy writer.  Prints "ok" and exits 0 on success.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>

#include "langevina.hpp"

using namespace langevina;

#define REQUIRE(c)                                                   \
  do {                                                               \
    if (!(c)) {                                                      \
      fprintf(stderr, "FAILED %s at %s:%d\n", #c, __FILE__, __LINE__); \
      return 1;                                                      \
    }                                                                \
  } while (0)

int main(int argc, char **argv) {
  const std::string golden = argc > 1 ? argv[1] : "tests/golden/ref_xoro.txt";
  const Json j = Json::parse(R"({
      "NX": 32,            // lattice
      "finaltime": 3.0, "initialtime": 0, "deltat": 0.6,
      "mass0": -4.813, "lambda": 10, "H": 0.01, "chi": 5.0,
      /* no gamma, no diffusion: defaults */
      "evolverType" : "PV2HBSplit23", "seed": 122335456, "restart": false,
      "outputfiletag": "run1", "saveFrequency": 3, "eventmode": true, "nevents": 4,
  })");
  ModelAData d(j);
  REQUIRE(d.NX == 32 && d.NY == 32 && d.NZ == 32);
  REQUIRE(d.LX == 32.0);
  REQUIRE(std::fabs(d.atime.tfinal() - 1.8) < 1e-12);  // 3.0 -> whole saveFrequency*dt units
  REQUIRE(d.acoefficients.gamma == 1.0);
  REQUIRE(std::fabs(d.acoefficients.diffusion - 1.0 / 3.0) < 1e-15);  // default 1/3 * gamma
  REQUIRE(d.acoefficients.lambda == 10.0 && d.acoefficients.H == 0.01);
  REQUIRE(d.ahandler.evolverType == "PV2HBSplit23" && d.ahandler.eventmode && d.ahandler.nevents == 4);
  REQUIRE(d.ahandler.outputfiletag == "run1" && d.ahandler.writeFrequency == -1);
  REQUIRE(std::fabs(d.mass() + 4.813) < 1e-15);
  const lgv_params p = d.params();
  REQUIRE(p.N == 32 && p.reserved0 == 0 && p.seed == 122335456u);

  // host stream vs the reference engine (tests/golden/ref_xoro.txt "var1"/"norm" records)
  std::ifstream g(golden);
  REQUIRE(g.good());
  std::string line;
  int checked = 0;
  while (std::getline(g, line)) {
    std::istringstream ss(line);
    std::string kind;
    int base, rank, size, n;
    ss >> kind;
    if (kind != "var1" && kind != "norm" && kind != "unif") continue;
    ss >> base >> rank >> size >> n;
    NoiseGenerator ng(base, rank, size);
    for (int i = 0; i < n; ++i) {
      double want;
      ss >> want;
      const double got = kind == "var1" ? ng.variance1() : kind == "norm" ? ng.normal() : ng.uniform();
      REQUIRE(got == want);
    }
    ++checked;
  }
  REQUIRE(checked >= 18);

  // .npy round trip
  std::vector<double> a = {1.5, -2.0, 3.25, 4.0, 5.0, 6.0};
  write_npy("host_api_test.npy", {2, 3}, a.data());
  auto b = read_npy("host_api_test.npy", 6);
  REQUIRE(b == a);
  printf("ok\n");
  return 0;
}
