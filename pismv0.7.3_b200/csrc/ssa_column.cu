// ssa_column.cu — the consumers of the SSA velocity in StressBalance::update with a full
// update (PISMStressBalance.cc:79-116), on the device, from the handle's velocity, mask,
// thickness and enthalpy columns:
//
//   u3, v3  ConstantInColumn::update (SSB_Modifier.cc:126-152): every level of the 3-D
//           horizontal velocity is the column's SSA velocity
//   sigma   StressBalance::compute_volumetric_strain_heating (PISMStressBalance.cc:369-499)
//   w3      StressBalance::compute_vertical_velocity (PISMStressBalance.cc:192-287)
//
// The 3-D fields are [i][j][k] (a column's Mz levels contiguous).  One thread per column:
// the horizontal velocity is constant in each column, so u_z = v_z = 0 exactly and the
// horizontal derivatives, D^2 and its power are the column's, computed once; the thread then
// walks up its column, summing w by the trapezoid rule in the reference's order of operations
// and scaling the strain heating by each level's hardness.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>

#include "ssa_internal.h"

namespace pism_gpu {

namespace {

constexpr int NTC = 256;

__device__ __forceinline__ bool icy(int m) { return m == 2 || m == 3; }   // Mask.hh:46-48

// the margin-aware difference weights of one column (PISMStressBalance.cc:229-257): (west,
// east, D_x), (south, north, D_y)
struct ColumnDiff {
  double west, east, D_x, south, north, D_y;
};

__device__ __forceinline__ ColumnDiff column_diff(const GridDev &g, const int8_t *__restrict__ mask, int i, int j) {
  const int m = mask[cell(g, i, j)];
  auto cut = [&](int di, int dj) {
    const int n = mask[nbr(g, i, j, di, dj)];
    return ((icy(m) && !icy(n)) || (!icy(m) && icy(n))) ? 0.0 : 1.0;
  };
  ColumnDiff d;
  d.east = cut(1, 0);
  d.west = cut(-1, 0);
  d.north = cut(0, 1);
  d.south = cut(0, -1);
  d.D_x = d.east + d.west > 0 ? 1.0 / (g.dx * (d.east + d.west)) : 0.0;
  d.D_y = d.north + d.south > 0 ? 1.0 / (g.dy * (d.north + d.south)) : 0.0;
  return d;
}

// IceGrid::kBelowHeight through gsl_interp_accel_find: the largest k in [0, Mz - 2] with
// z[k] <= height (GSL's bisection, lo = 0, hi = Mz - 1)
__device__ __forceinline__ int k_below_height(const double *__restrict__ z, int Mz, double height) {
  int lo = 0, hi = Mz - 1;
  while (hi > lo + 1) {
    const int mid = (lo + hi) / 2;
    if (z[mid] > height) hi = mid;
    else lo = mid;
  }
  return lo;
}

// One warp per 32 consecutive columns (whose [i][j][k] data are 32 Mz consecutive doubles):
// lane r computes column c0 + r level by level into a shared-memory tile (rows padded to an
// odd length, so the lanes' writes at one level fall in different banks), then the warp
// copies the tile out with consecutive lanes on consecutive addresses.  One field at a time.
__global__ void __launch_bounds__(NTC) k_stress_balance_3d(GridDev g, pism_gpu_ssa_config c, int Mz, int S,
                                                           double e_to_a_power, double exponent, double B_iso,
                                                           const double2 *__restrict__ vel,
                                                           const int8_t *__restrict__ mask,
                                                           const double *__restrict__ H,
                                                           const double *__restrict__ E,
                                                           const double *__restrict__ z,
                                                           const double *__restrict__ bmr, double *__restrict__ u3,
                                                           double *__restrict__ v3, double *__restrict__ w3,
                                                           double *__restrict__ sigma) {
  extern __shared__ double tiles[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  double *const tile = tiles + (size_t)warp * 32 * S;
  const int N = g.Mx * g.My;
  for (int c0 = (blockIdx.x * wpb + warp) * 32; c0 < N; c0 += gridDim.x * wpb * 32) {
    const int col = c0 + lane, ncol = min(32, N - c0);
    const bool mine = col < N;
    const int i = mine ? col / g.My : 0, j = mine ? col - i * g.My : 0;
    const double2 U = mine ? vel[col] : make_double2(0.0, 0.0);
    // the tile of field q out to dst: columns c0 .. c0 + ncol - 1, all Mz levels
    auto flush = [&](double *dst) {
      __syncwarp();
      const int n = ncol * Mz;
      double *const out = dst + (size_t)c0 * Mz;
      int r = lane / Mz, k = lane - r * Mz;   // (column, level) of element e, advanced by 32
      for (int e = lane; e < n; e += 32) {
        out[e] = tile[r * S + k];
        k += 32;
        while (k >= Mz) {
          k -= Mz;
          ++r;
        }
      }
      __syncwarp();
    };
    if (u3) {
      if (mine)
        for (int k = 0; k < Mz; ++k) tile[lane * S + k] = U.x;
      flush(u3);
    }
    if (v3) {
      if (mine)
        for (int k = 0; k < Mz; ++k) tile[lane * S + k] = U.y;
      flush(v3);
    }
    if (!w3 && !sigma) continue;
    double u_x = 0.0, v_y = 0.0, u_y = 0.0, v_x = 0.0;
    if (mine) {
      const ColumnDiff d = column_diff(g, mask, i, j);
      const double2 Uw = vel[nbr(g, i, j, -1, 0)], Ue = vel[nbr(g, i, j, 1, 0)], Us = vel[nbr(g, i, j, 0, -1)],
                    Un = vel[nbr(g, i, j, 0, 1)];
      u_x = d.D_x * (d.west * (U.x - Uw.x) + d.east * (Ue.x - U.x));
      v_y = d.D_y * (d.south * (U.y - Us.y) + d.north * (Un.y - U.y));
      u_y = d.D_y * (d.south * (U.x - Us.x) + d.north * (Un.x - U.x));
      v_x = d.D_x * (d.west * (U.y - Uw.y) + d.east * (Ue.y - U.y));
    }
    if (w3) {
      // w(0) = -bmr (or 0); w(k) = w(k-1) - (integrand(k) + integrand(k-1)) / 2 dz, the
      // integrand u_x + v_y the same at every level; the products and sums in that order
      if (mine) {
        const double integrand = __dadd_rn(u_x, v_y);
        const double half_sum = __dmul_rn(0.5, __dadd_rn(integrand, integrand));
        double w = bmr ? -bmr[col] : 0.0;
        tile[lane * S] = w;
        for (int k = 1; k < Mz; ++k) {
          w = __dsub_rn(w, __dmul_rn(half_sum, __dsub_rn(z[k], z[k - 1])));
          tile[lane * S + k] = w;
        }
      }
      flush(w3);
    }
    if (sigma) {
      if (mine) {
        const double Hc = H[col];
        const int ks = k_below_height(z, Mz, Hc);
        const double a = u_x + v_y, b = u_y + v_x;   // u_z = v_z = 0
        // D2(), PISMStressBalance.cc:309-311
        const double D2 = 0.5 * (a * a + u_x * u_x + v_y * v_y + 0.5 * (b * b));
        const double two_e = 2.0 * e_to_a_power, D2e = pow(D2, exponent);
        const double *const Ec = E ? E + (size_t)col * Mz : nullptr;
        for (int k = 0; k < Mz; ++k) {
          double s = 0.0;
          if (k <= ks) {
            const double B = Ec ? hardness_parameter(c, Ec[k], ec_pressure(c, Hc - z[k])) : B_iso;
            s = two_e * B * D2e;   // the reference's order: (2 e^(-1/n) B) D^(1/n + 1)
          }
          tile[lane * S + k] = s;
        }
      }
      flush(sigma);
    }
  }
}

}  // namespace

int stress_balance_3d_smem(int Mz, int *warps) {
  const int S = Mz | 1;
  const int per_warp = 32 * S * (int)sizeof(double);
  *warps = std::max(1, std::min(NTC / 32, (200 * 1024) / per_warp));
  return *warps * per_warp;
}

void launch_stress_balance_3d(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, int Mz,
                              const Fields &f, const double *z, const double *bmr, double *u3, double *v3,
                              double *w3, double *sigma) {
  const int N = g.Mx * g.My;
  int warps = 0;
  const int smem = stress_balance_3d_smem(Mz, &warps);
  const int blocks = std::max(1, std::min((N + 32 * warps - 1) / (32 * warps), 4 * L.max_blocks));
  // PISMStressBalance.cc:384-387: the flow law's exponent and enhancement factor; an
  // isothermal flow law's hardness A^(-1/n) is the same at every level
  const double n = c.ssa_Glen_exponent, exponent = 0.5 * (1.0 / n + 1.0);
  const double e_to_a_power = std::pow(c.ssa_enhancement_factor, -1.0 / n);
  const bool iso = c.flow_law == PISM_FLOW_LAW_ISOTHERMAL_GLEN;
  const double B_iso = iso ? std::pow(c.ice_softness, -1.0 / n) : 0.0;
  L.tick();
  k_stress_balance_3d<<<blocks, 32 * warps, smem, L.stream>>>(g, c, Mz, Mz | 1, e_to_a_power, exponent, B_iso, f.vel,
                                                               f.mask, f.H, iso ? nullptr : f.enthalpy, z, bmr, u3,
                                                               v3, w3, sigma);
}

// the kernel's dynamic shared-memory limit for Mz levels on the current device: a function
// attribute shared by every handle on that device, so it is only ever raised, under a lock
int stress_balance_3d_prepare(int Mz) {
  static std::mutex lock;
  static std::map<int, int> raised;   // device -> bytes granted
  int warps = 0, dev = 0;
  const int smem = stress_balance_3d_smem(Mz, &warps);
  if (smem <= 48 * 1024) return 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  std::lock_guard<std::mutex> guard(lock);
  auto it = raised.find(dev);
  if (it != raised.end() && smem <= it->second) return 0;
  if (cudaFuncSetAttribute((const void *)k_stress_balance_3d, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
      cudaSuccess)
    return 1;
  raised[dev] = smem;
  return 0;
}

}  // namespace pism_gpu
