// A C++ host program on the native C ABI alone (no Python): the call
// sequence a driver keeps when it moves to the device-resident step
// (step.cpp:13-147 -> cudasph_step).  Reads n and the ten input fields
// (x, y, z, range, vx, vy, vz, m, u, mu; doubles, caller's order) from
// argv[1], runs argv[3] steps with the reference's constants except the
// ones set below, prints the energy of every step, and writes all
// SPH_NFIELDS fields to argv[2].  Exit status 0 on success.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "cudasph_b200.h"

int main(int argc, char **argv) {
  if (argc < 4) return 2;
  FILE *f = std::fopen(argv[1], "rb");
  if (!f) return 3;
  int n = 0;
  if (std::fread(&n, sizeof(int), 1, f) != 1 || n <= 0) return 3;
  const int in_ids[10] = {SPH_X, SPH_Y, SPH_Z, SPH_RANGE, SPH_VX, SPH_VY, SPH_VZ, SPH_M, SPH_U, SPH_MU};
  std::vector<std::vector<double>> in(10, std::vector<double>(n));
  for (auto &a : in)
    if (std::fread(a.data(), sizeof(double), n, f) != (size_t)n) return 3;
  std::fclose(f);

  sph_params p = cudasph_default_params();
  p.n_target = 50.0;
  p.eos_mode = SPH_EOS_IDEAL;
  p.soft_mode = SPH_SOFT_PLUMMER;
  p.eps = 0.01;
  p.precision = SPH_PREC_FP64;
  sph_ctx *ctx = nullptr;
  if (cudasph_create(&p, n, 0, &ctx) != SPH_OK) {
    std::fprintf(stderr, "create: %s\n", cudasph_last_error());
    return 4;
  }
  const double *fields[SPH_NFIELDS] = {};
  for (int k = 0; k < 10; k++) fields[in_ids[k]] = in[k].data();
  if (cudasph_set_state(ctx, fields, 0) != SPH_OK || cudasph_set_time(ctx, 0.0, 0.0) != SPH_OK) return 5;
  const int steps = std::atoi(argv[3]);
  double st[SPH_NSTATS];
  for (int s = 0; s < steps; s++) {
    if (cudasph_step(ctx) != SPH_OK) {
      std::fprintf(stderr, "step: %s\n", cudasph_last_error());
      return 6;
    }
    if (cudasph_statistics(ctx, st) != SPH_OK) return 7;
    std::printf("step %d E %.17g dt %.17g\n", s + 1, st[SPH_ST_E], st[SPH_ST_DT]);
  }
  unsigned flags = 0;
  if (cudasph_device_status(ctx, &flags) != SPH_OK || (flags & ~SPH_FLAG_H_NOT_CONVERGED)) return 8;
  std::vector<std::vector<double>> out(SPH_NFIELDS, std::vector<double>(n));
  double *outp[SPH_NFIELDS];
  for (int k = 0; k < SPH_NFIELDS; k++) outp[k] = out[k].data();
  if (cudasph_get_state(ctx, outp, 0) != SPH_OK) return 9;
  cudasph_destroy(ctx);
  FILE *g = std::fopen(argv[2], "wb");
  if (!g) return 10;
  for (auto &a : out) std::fwrite(a.data(), sizeof(double), n, g);
  std::fclose(g);
  return 0;
}
