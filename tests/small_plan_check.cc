// Host driver for the split of the small multigrid levels over the cluster's CTAs
// (pismv0.7.3_b200/csrc/ssa_small_plan.h).  Reads lines "nlev max_smem Mx My ax ay ..." (fine
// to coarse) and prints the plan as one JSON object per line ({"ok": false} when it does not
// fit), with the owner lookup of every row and column of every level.
#include <cstdio>
#include <iostream>
#include <sstream>
#include <string>

#include "ssa_small_plan.h"

using namespace pism_gpu;

int main() {
  std::string line;
  while (std::getline(std::cin, line)) {
    std::istringstream in(line);
    int nlev = 0, max_smem = 0;
    in >> nlev >> max_smem;
    int Mx[SC_MAX_LEV + 4], My[SC_MAX_LEV + 4], ax[SC_MAX_LEV + 4], ay[SC_MAX_LEV + 4];
    for (int l = 0; l < nlev && l < SC_MAX_LEV + 4; ++l) in >> Mx[l] >> My[l] >> ax[l] >> ay[l];
    SmallPlan P;
    const bool ok = small_plan(nlev, Mx, My, ax, ay, max_smem, P);
    if (!ok) {
      printf("{\"ok\": false}\n");
      continue;
    }
    printf("{\"ok\": true, \"Pr\": %d, \"Pc\": %d, \"smem\": %d, \"levels\": [", P.Pr, P.Pc, P.smem);
    for (int l = 0; l < P.nlev; ++l) {
      printf("%s{\"mi\": %d, \"mj\": %d, \"off4\": %d, \"off2\": %d, \"offp\": %d, \"rb\": [", l ? ", " : "",
             P.mi[l], P.mj[l], P.off4[l], P.off2[l], P.offp[l]);
      for (int p = 0; p <= P.Pr; ++p) printf("%s%d", p ? ", " : "", P.rb[l][p]);
      printf("], \"cb\": [");
      for (int q = 0; q <= P.Pc; ++q) printf("%s%d", q ? ", " : "", P.cb[l][q]);
      printf("], \"row_owner\": [");
      for (int i = 0; i < P.Mx[l]; ++i) printf("%s%d", i ? ", " : "", small_owner(P.rb[l], P.Pr, i));
      printf("], \"col_owner\": [");
      for (int j = 0; j < P.My[l]; ++j) printf("%s%d", j ? ", " : "", small_owner(P.cb[l], P.Pc, j));
      printf("]}");
    }
    printf("]}\n");
  }
  return 0;
}
