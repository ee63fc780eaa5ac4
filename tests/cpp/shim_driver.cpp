// A driver written against the reference's call surface (src/dqmc_handle.cpp:56-162),
// compiled against the header-only facade include/hubbard_b200.hpp.
#include <cstdio>
#include <cstdlib>
#include "hubbard_b200.hpp"

using namespace hq_b200;

int main(int argc, char** argv) {
  DQMC::Params p;
  p.nl = 4; p.ns = p.ng = 16; p.beta = 4.0; p.nt = 40; p.dt = p.beta / p.nt; p.u = 4.0; p.mu = 0.0;
  p.stabilization_pace = 10; p.is_fft = false;
  const long long seed = argc > 1 ? std::atoll(argv[1]) : 42;
  Model::HubbardAttractiveU model;
  model.initialize(p, seed);
  model.set_ising_fields_to_random();
  DQMC::Core core;
  core.initialize(p, true, true);
  core.initialize_svdstacks(model);
  core.initialize_green_functions();
  core.set_thermalization(true);
  for (int s = 0; s < 2; ++s) {
    core.sweep_from_0_to_beta(model);
    core.sweep_from_beta_to_0(model);
  }
  const auto g = core.current_gftt();
  std::printf("%.17g %.17g %.17g\n", g[0], g[17], core.equaltimeWrapError());
  const auto f = model.ising_fields();
  long s = 0;
  for (int v : f) s += v;
  std::printf("%ld\n", s);
  // the stacks after an up + down pair: left empty, right holding every interval
  Utils::SvdStack left(model, 0), right(model, 1);
  const auto d = right.SingularValues();
  std::printf("%d %d %d %.17g\n", left.StackLength(), right.StackLength(), right.MatDim(), d[0]);
  return 0;
}
