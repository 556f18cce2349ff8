// Checks the work split of the L2-staged small-level cycle (csrc/ssa_small_plan.h
// small_span / small_chunk / small_down_rows / small_window) on the level chains given on
// stdin, one "Mx My ax ay Mxc Myc parts local_items" line per down step.  For every CTA's
// chunk of restriction items and of post-smoothing items it checks that the chunks cover the
// items once, start on whole warps, and that every row a chunk's stencils read (the rows of
// the aggregates' fine cells and one neighbour row each side, wrapped periodically) lies in
// its staged window, whose rows are distinct modulo Mx.  Prints one line per step:
// "ok <largest window cells>" or "bad <reason>".
#include <cstdio>
#include <set>
#include <vector>

#include "ssa_small_plan.h"

using namespace pism_gpu;

static int pmod(int a, int n) { return ((a % n) + n) % n; }

static bool in_window(int Mx, int w0, int nrows, int row) {
  for (int r = 0; r < nrows; ++r)
    if (pmod(w0 + r, Mx) == pmod(row, Mx)) return true;
  return false;
}

static bool distinct(int Mx, int w0, int nrows) {
  std::set<int> rows;
  for (int r = 0; r < nrows; ++r) rows.insert(pmod(w0 + r, Mx));
  return (int)rows.size() == nrows;
}

int main() {
  int Mx, My, ax, ay, Mxc, Myc, parts, local_items;
  while (std::scanf("%d %d %d %d %d %d %d %d", &Mx, &My, &ax, &ay, &Mxc, &Myc, &parts, &local_items) == 8) {
    const int Nc = Mxc * Myc, N = Mx * My;
    const char *bad = nullptr;
    int most = 0;
    // down step
    const int span = small_span(Nc), pd = span <= local_items ? 1 : parts;
    std::vector<int> seen(span, 0);
    for (int c = 0; c < pd && !bad; ++c) {
      int b0, b1;
      small_chunk(span, pd, c, 32, b0, b1);
      if (b0 % 32 != 0 || b1 % 32 != 0) bad = "restriction chunk not on whole warps";
      if (b1 <= b0) continue;
      for (int b = b0; b < b1; ++b) seen[b] += 1;
      int r0, r1, w0, nrows;
      small_down_rows(ax, Myc, Nc, b0, b1, r0, r1);
      small_window(Mx, r0, r1, w0, nrows);
      if (nrows > Mx || !distinct(Mx, w0, nrows)) bad = "down window rows repeat";
      most = nrows * My > most ? nrows * My : most;
      for (int b = b0; b < b1 && !bad; ++b) {
        const int kc = b >> 2, pi = (b >> 1) & 1, pj = b & 1;
        if (kc >= Nc || pi >= ax || pj >= ay) continue;
        const int i = (kc / Myc) * ax + pi, j = (kc % Myc) * ay + pj;
        if (i >= Mx || j >= My) continue;
        for (int di = -1; di <= 1; ++di)
          if (!in_window(Mx, w0, nrows, i + di)) bad = "a restriction stencil row is outside its window";
      }
    }
    for (int b = 0; b < span && !bad; ++b)
      if (seen[b] != 1) bad = "restriction items not covered once";
    // up step on the fine level
    const int pu = N <= local_items ? 1 : parts;
    std::vector<int> seen_up(N, 0);
    for (int c = 0; c < pu && !bad; ++c) {
      int k0, k1, w0, nrows;
      small_chunk(N, pu, c, 32, k0, k1);
      if (k1 <= k0) continue;
      for (int k = k0; k < k1; ++k) seen_up[k] += 1;
      small_window(Mx, k0 / My, (k1 - 1) / My, w0, nrows);
      if (nrows > Mx || !distinct(Mx, w0, nrows)) bad = "up window rows repeat";
      most = nrows * My > most ? nrows * My : most;
      for (int k = k0; k < k1 && !bad; ++k)
        for (int di = -1; di <= 1; ++di)
          if (!in_window(Mx, w0, nrows, k / My + di)) bad = "a post-smoothing stencil row is outside its window";
    }
    for (int k = 0; k < N && !bad; ++k)
      if (seen_up[k] != 1) bad = "post-smoothing items not covered once";
    if (bad) std::printf("bad %s\n", bad);
    else std::printf("ok %d\n", most);
  }
  return 0;
}
