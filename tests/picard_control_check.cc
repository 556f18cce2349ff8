// Host driver for the Picard-loop decisions of ssa_state.h (the functions the whole-solve
// graph's control kernels run on the device).  Reads commands from stdin, one per line,
// and prints the state after each "print" as one JSON object:
//   const <adaptive> <ksp_rtol> <ksp_rtol_max> <factor> <picard_rtol> <max_iterations> <mg_rebuild_rtol>
//   start | begin | print
//   ksp_end <iter> <status> <rnorm2> <bnorm2> <body_iters>
//   refine_end <iter> <status> <outer_r2> <outer_b2> <max_refine>
//   after <zero_diag_cell (-1 = none)>
//   test <norm> <change>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>

#include "ssa_state.h"

using namespace pism_gpu;

// a double as a JSON token Python reads back (NaN / Infinity for the non-finite)
static std::string js(double v) {
  if (std::isnan(v)) return "NaN";
  if (std::isinf(v)) return v > 0 ? "Infinity" : "-Infinity";
  char b[64];
  snprintf(b, sizeof(b), "%.17g", v);
  return b;
}

// a number token, "nan" and "inf" included
static double num(std::istringstream &in) {
  std::string t;
  in >> t;
  return strtod(t.c_str(), nullptr);
}

int main() {
  PState P{};
  PicardConst c{};
  std::string line;
  while (std::getline(std::cin, line)) {
    std::istringstream in(line);
    std::string cmd;
    in >> cmd;
    if (cmd == "const") {
      c.adaptive = (int)num(in);
      c.ksp_rtol = num(in);
      c.ksp_rtol_max = num(in);
      c.ksp_rtol_factor = num(in);
      c.picard_rtol = num(in);
      c.max_iterations = (int)num(in);
      c.mg_rebuild_rtol = num(in);
    } else if (cmd == "start") {
      picard_start(P);
    } else if (cmd == "begin") {
      picard_begin(P, c);
    } else if (cmd == "ksp_end") {
      KState st{};
      int body = 1;
      st.iter = (int)num(in);
      st.status = (int)num(in);
      st.rnorm2 = num(in);
      st.bnorm2 = num(in);
      body = (int)num(in);
      ksp_end(P, st, body);
    } else if (cmd == "refine_end") {
      KState st{};
      int max_refine = 60;
      st.iter = (int)num(in);
      st.status = (int)num(in);
      st.outer_r2 = num(in);
      st.outer_b2 = num(in);
      max_refine = (int)num(in);
      refine_end(P, st, max_refine);
    } else if (cmd == "after") {
      const int zd = (int)num(in);
      picard_after_solve(P, zd < 0 ? INT_MAX : zd);
    } else if (cmd == "test") {
      const double norm = num(in), change = num(in);
      picard_test(P, norm, change, c);
    } else if (cmd == "print") {
      printf("{\"rtol\": %s, \"last_change\": %s, \"final_res\": %s, \"k\": %d, \"passes\": %d, "
             "\"done\": %d, \"status\": %d, \"zd_cell\": %d, \"ksp_its\": %d, \"ksp_status\": %d, "
             "\"ksp_total\": %d, \"refine\": %d, \"refine_done\": %d, \"go\": %d, \"go_count\": %d, "
             "\"refine_steps\": %d, \"refine_passes\": %d, \"inner_passes\": %lld, \"rebuild\": %d, "
             "\"rebuilds\": %d, \"coarse_change\": %s}\n",
             js(P.rtol).c_str(), js(P.last_change).c_str(), js(P.final_res).c_str(), P.k, P.passes, P.done, P.status, P.zd_cell, P.ksp_its,
             P.ksp_status, P.ksp_total, P.refine, P.refine_done, P.go, P.go_count, P.refine_steps,
             P.refine_passes, P.inner_passes, P.rebuild, P.rebuilds, js(P.coarse_change).c_str());
    }
  }
  return 0;
}
