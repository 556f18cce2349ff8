// ssa_small_plan.h — how the small multigrid levels are split over the CTAs of one
// thread-block cluster (the shared-memory cycle of ssa_mg.cu, and the work split of the
// L2-staged cycle), as plain C++ so that the host compiler can check the split too.
//
// The coarsest level's rows and columns are cut into a Pr x Pc grid of blocks, one block per
// CTA (Pr * Pc <= cluster size); every finer small level takes the blocks of the level below
// it expanded by the aggregation factors, so the fine cells of a coarse cell's aggregate
// always live on the coarse cell's CTA.  Each CTA keeps its block of every level in its own
// shared memory, in arrays shaped by the largest block of that level (the same offsets on
// every CTA, so a neighbour's value is read from the same offset in the neighbour's shared
// memory); the smoothed iterates x0 and x also carry a one-cell halo ring, filled from the
// neighbours once per step.
#pragma once

#if defined(__CUDACC__)
#define SMALL_HD __host__ __device__ inline
#else
#define SMALL_HD inline
#endif

namespace pism_gpu {

constexpr int SC_CTAS = 8;       // CTAs of the cluster
constexpr int SC_MAX_LEV = 12;   // small levels handled by the shared-memory cycle

// (plain members only: the cycle kernel copies the plan into a __shared__ variable)
struct SmallPlan {
  int nlev;                            // small levels first .. first + nlev - 1
  int Pr, Pc;                          // CTA grid
  int Mx[SC_MAX_LEV], My[SC_MAX_LEV];  // level sizes
  int ax[SC_MAX_LEV], ay[SC_MAX_LEV];  // aggregation towards the next (coarser) level
  int rb[SC_MAX_LEV][SC_CTAS + 1];     // row boundaries: CTA row p owns rows [rb[p], rb[p+1])
  int cb[SC_MAX_LEV][SC_CTAS + 1];     // column boundaries
  int mi[SC_MAX_LEV], mj[SC_MAX_LEV];  // largest block: the shape of every CTA's arrays
  int off4[SC_MAX_LEV];                // byte offset of the level's float4 arrays (9 blocks of A, D^-1)
  int off2[SC_MAX_LEV];                // byte offset of the level's float2 arrays (b, z)
  int offp[SC_MAX_LEV];                // byte offset of the padded float2 arrays (x0, x) with a halo ring
  int smem;                            // bytes of dynamic shared memory per CTA
};


// Plan the split of levels (Mx[l], My[l], ax[l], ay[l]), l = 0 .. nlev-1 from fine to
// coarse (level l+1 has ceil(Mx[l] / ax[l]) x ceil(My[l] / ay[l]) cells).  Returns false
// when the levels do not fit (too many, or more shared memory than max_smem per CTA).
inline bool small_plan(int nlev, const int *Mx, const int *My, const int *ax, const int *ay, int max_smem,
                       SmallPlan &P) {
  if (nlev < 1 || nlev > SC_MAX_LEV) return false;
  P = SmallPlan{};
  P.nlev = nlev;
  for (int l = 0; l < nlev; ++l) {
    P.Mx[l] = Mx[l];
    P.My[l] = My[l];
    P.ax[l] = ax[l];
    P.ay[l] = ay[l];
    if (Mx[l] < 1 || My[l] < 1) return false;
    if (l + 1 < nlev &&
        (Mx[l + 1] != (Mx[l] + ax[l] - 1) / ax[l] || My[l + 1] != (My[l] + ay[l] - 1) / ay[l]))
      return false;
  }
  const int c = nlev - 1;
  // the CTA grid over the coarsest level: as many rows as allowed, then columns
  P.Pr = Mx[c] < SC_CTAS ? Mx[c] : SC_CTAS;
  P.Pc = SC_CTAS / P.Pr;
  if (P.Pc > My[c]) P.Pc = My[c];
  for (int p = 0; p <= P.Pr; ++p) P.rb[c][p] = (int)((long long)p * Mx[c] / P.Pr);
  for (int q = 0; q <= P.Pc; ++q) P.cb[c][q] = (int)((long long)q * My[c] / P.Pc);
  for (int l = c - 1; l >= 0; --l) {
    for (int p = 0; p <= P.Pr; ++p) {
      const int r = P.rb[l + 1][p] * ax[l];
      P.rb[l][p] = r < Mx[l] ? r : Mx[l];
    }
    for (int q = 0; q <= P.Pc; ++q) {
      const int r = P.cb[l + 1][q] * ay[l];
      P.cb[l][q] = r < My[l] ? r : My[l];
    }
  }
  int bytes = 0;
  for (int l = 0; l < nlev; ++l) {
    int mi = 0, mj = 0;
    for (int p = 0; p < P.Pr; ++p) mi = P.rb[l][p + 1] - P.rb[l][p] > mi ? P.rb[l][p + 1] - P.rb[l][p] : mi;
    for (int q = 0; q < P.Pc; ++q) mj = P.cb[l][q + 1] - P.cb[l][q] > mj ? P.cb[l][q + 1] - P.cb[l][q] : mj;
    P.mi[l] = mi;
    P.mj[l] = mj;
    const int cells = mi * mj;
    P.off4[l] = bytes;
    bytes += 10 * 16 * cells;   // the nine 2 x 2 blocks and D^-1
    P.off2[l] = bytes;
    bytes += 2 * 8 * cells;     // b, z
    P.offp[l] = bytes;
    bytes += 2 * 8 * (mi + 2) * (mj + 2);   // x0, x with their halo rings
    bytes = (bytes + 127) / 128 * 128;
  }
  P.smem = bytes;
  return bytes <= max_smem;
}

// the CTA row / column block that holds row i (column j) of level l
inline
#if defined(__CUDACC__)
    __host__ __device__
#endif
    int small_owner(const int *bounds, int parts, int i) {
  int p = parts - 1;
  while (p > 0 && bounds[p] > i) --p;
  return p;
}

// Work split of the small-level cycle, shared by the kernel and the host's sizing of its
// staging buffer.  A down step from a level to the next coarser one (Nc cells) has
// span(Nc) restriction items, four per coarse cell (one per fine cell of a 2 x 2 aggregate);
// an up step has one post-smoothing item per cell.  Each of `parts` CTAs takes a contiguous
// chunk of items (whole warps for the restriction's shuffles) and stages the fine rows those
// items read: a window of rows, wrapped periodically, or the whole level once the window would
// reach every row.
SMALL_HD int small_span(int Nc) { return (4 * Nc + 31) & ~31; }

SMALL_HD void small_chunk(int items, int parts, int c, int align, int &b0, int &b1) {
  const int chunk = ((items + parts - 1) / parts + align - 1) / align * align;
  b0 = c * chunk < items ? c * chunk : items;
  b1 = b0 + chunk < items ? b0 + chunk : items;
}

// the fine rows [w0, w0 + nrows) read by the cells of rows r0 .. r1 of a level with Mx rows
// (one halo row each side)
SMALL_HD void small_window(int Mx, int r0, int r1, int &w0, int &nrows) {
  w0 = r0 - 1;
  nrows = r1 - r0 + 3;
  if (nrows >= Mx) {
    w0 = 0;
    nrows = Mx;
  }
}

// the rows of a down step's restriction items b0 .. b1 - 1 (b1 > b0): the fine rows of the
// aggregates of coarse rows I0 .. I1
SMALL_HD void small_down_rows(int ax, int Myc, int Nc, int b0, int b1, int &r0, int &r1) {
  const int k0 = (b0 >> 2) < Nc ? (b0 >> 2) : Nc - 1, k1 = ((b1 - 1) >> 2) < Nc ? ((b1 - 1) >> 2) : Nc - 1;
  r0 = (k0 / Myc) * ax;
  r1 = (k1 / Myc) * ax + ax - 1;
}

}  // namespace pism_gpu
