// main.cpp -- `mcb200_main input.txt`: the engine's drop-in for the
// reference's `main input.txt` (src/main.cpp): reads the deck and runs the
// self-consistent simulation on GPU 0, writing ./data like the reference.
// Band tables: $MCB200_TABLES, else ../input next to the executable's
// directory (the reference's bs_path, src/mcmodel.cpp:3986), else the
// package's tables directory.  Options: --fp32 (FP32 flight), --steps N,
// --heat-steps N, --poisson-every N, --seed S, --device D, --quiet.
#include <unistd.h>

#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "mcb200.h"

static std::string exe_dir() {
  char buf[PATH_MAX] = {0};
  const ssize_t n = readlink("/proc/self/exe", buf, sizeof(buf) - 1);
  if (n <= 0) return ".";
  std::string p(buf, (size_t)n);
  const size_t s = p.find_last_of('/');
  return s == std::string::npos ? "." : p.substr(0, s);
}

static bool has_tables(const std::string &dir) { return access((dir + "/bs.si.asc").c_str(), R_OK) == 0; }

int main(int argc, char **argv) {
  const char *input = nullptr;
  mcb200_run_options o;
  std::memset(&o, 0, sizeof(o));
  o.max_heat_steps = -1;
  o.write_outputs = 1;
  o.verbose = 1;
  int device = 0;
  for (int a = 1; a < argc; ++a) {
    const std::string s(argv[a]);
    auto next = [&]() { return a + 1 < argc ? argv[++a] : (char *)"0"; };
    if (s == "--fp32") o.flight_precision = MCB200_FLIGHT_FP32;
    else if (s == "--steps") o.max_steps = std::atoi(next());
    else if (s == "--heat-steps") o.max_heat_steps = std::atoi(next());
    else if (s == "--poisson-every") o.poisson_every = std::atoi(next());
    else if (s == "--seed") o.seed = std::strtoull(next(), nullptr, 10);
    else if (s == "--device") device = std::atoi(next());
    else if (s == "--quiet") o.verbose = 0;
    else input = argv[a];
  }
  if (!input) {
    std::fprintf(stderr, "input file missing, Usage: %s input_file [--fp32] [--steps N] ...\n", argv[0]);
    return 1;
  }
  std::string tables;
  if (const char *env = std::getenv("MCB200_TABLES")) tables = env;
  else if (has_tables(exe_dir() + "/../input")) tables = exe_dir() + "/../input";
  else tables = exe_dir() + "/tables";
  o.table_dir = tables.c_str();
  mcb200_run_report r;
  char err[1024] = {0};
  const int rc = mcb200_run_deck(input, device, &o, &r, err, sizeof(err));
  if (rc != MCB200_OK) {
    std::fprintf(stderr, "run failed (%d): %s\n", rc, err);
    return 1;
  }
  std::printf("done: %d steps + %d heat steps, %zu -> %zu particles, %.3g particle-steps in %.2f s "
              "(%.3g particle-steps/s), flight %.1f ms, Poisson %d solves (max residual %.2e), drain current %.4g A/cm\n",
              r.steps_done, r.heat_steps_done, r.initial_particles, r.final_particles, (double)r.particle_steps,
              r.wall_s, r.particle_steps / (r.wall_s > 0 ? r.wall_s : 1), r.flight_ms, r.poisson_solves,
              r.poisson_max_residual, r.last_current[0]);
  return 0;
}
