// superpions.cpp -- run driver on the B200 stepper, the counterpart of the
// reference's ModelG/SuperPions.cxx:
//
//   superpions -input run.json [-quit]
//
// Reads the reference's JSON input keys (ModelA.h:55-159), thermalises with
// the phi heat bath (6 sub-steps per dt, optional quench mass), runs the
// configured evolverType, measures every saveFrequency steps into
// <tag>.<dataset>.f64 series, dumps <tag>_t_<t>_save.npy every writeFrequency
// steps, and at the end writes <tag>_0.rng and <tag>_save.npy for a restart.
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>

#include "langevina.hpp"

using namespace langevina;

// thermalize_event (SuperPions.cxx:21-76)
static void thermalize_event(ModelA &model) {
  auto &ah = model.data.ahandler;
  auto &atime = model.data.atime;
  auto &ac = model.data.acoefficients;
  const double mass0 = ac.mass0, dmassdt = ac.dmassdt;
  if (ah.quench_mode) {
    ac.mass0 = ah.quench_mode_mass0;
    ac.dmassdt = 0.;
    printf("Settinng up a quench initial condition with initial mass %e\n", ac.mass0);
  }
  model.sync_params();
  const int nsteps = static_cast<int>(ah.thermalization_time / atime.dt());
  printf("Thermalizing event %d\n", ah.current_event);
  model.initialize_gaussian_charges();
  const int substeps = 6;
  // the clock does not advance while thermalising: every sub-step uses m^2(t0)
  for (int i = 0; i < nsteps * substeps; ++i)
    check(lgv_step(model.handle, LGV_EULER_LANGEVIN_HB, 1, 1, atime.dt() / substeps, atime.t(), 1), "thermalize");
  if (ah.quench_mode) {
    ac.mass0 = mass0;
    ac.dmassdt = dmassdt;
    printf("Finalizing  quench initial condition with initial mass %e\n", ac.mass0);
  }
  model.sync_params();
}

// run_event (SuperPions.cxx:78-161)
static void run_event(ModelA &model, Stepper &step) {
  auto &ah = model.data.ahandler;
  auto &atime = model.data.atime;
  atime.reset();
  if (!ah.restart) thermalize_event(model);
  std::string tag = ah.outputfiletag;
  if (ah.eventmode) {
    std::ostringstream ns;
    ns << ah.outputfiletag << "_" << std::setw(4) << std::setfill('0') << ah.current_event;
    tag = ns.str();
  }
  Measurer measurer(&model);
  measurer_output out(&measurer, tag, ah.restart);
  int steps = 0;
  const double tiny = 1.e-10;
  while (atime.t() < atime.tfinal() - tiny) {
    if (steps % ah.saveFrequency == 0) {
      measurer.measure();
      out.save();
      printf("Event/Timestep %d/%d: step size = %g, time = %g, final = %g, mass = %e\n", ah.current_event, steps,
             atime.dt(), atime.t(), atime.tfinal(), model.data.mass());
    }
    if (ah.writeFrequency > 0 && steps % ah.writeFrequency == 0) {
      std::ostringstream ts;
      ts << std::setprecision(4) << "_t_" << atime.t();
      model.write(ah.outputfiletag + ts.str());
    }
    step.step(atime.dt());
    steps++;
    atime += atime.dt();
  }
}

int main(int argc, char **argv) {
  std::string input;
  bool quit = false;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "-input" && i + 1 < argc) input = argv[++i];
    else if (a == "-quit") quit = true;
  }
  if (input.empty()) {
    printf("Usage: \n\n\t ./superpions -input input.json [options]\n\n");
    return 1;
  }
  try {
    const Json inputs = Json::parse_file(input);
    ModelAData data(inputs);
    data.print();
    if (quit) return 0;
    ModelA model(data);
    model.initialize();
    auto step = make_stepper(model, data.ahandler.evolverType);
    if (!step) {
      printf("Unrecognized stepper type %s. Aborting...\n", data.ahandler.evolverType.c_str());
      return 1;
    }
    auto &ah = model.data.ahandler;
    if (ah.eventmode) {
      for (int i = 0; i < ah.nevents; ++i) {
        run_event(model, *step);
        ah.current_event++;
      }
    } else {
      run_event(model, *step);
    }
    step->finalize();
    model.finalize();
  } catch (const std::exception &e) {
    fprintf(stderr, "superpions: %s\n", e.what());
    return 2;
  }
  return 0;
}
