// ssa_calving.cu — what the calving front takes from the SSA velocity: the principal strain
// rates and 2-D deviatoric stresses of ShallowStressBalance (ShallowStressBalance.cc:224-386)
// and the eigen-calving step that uses them (EigenCalving::update / max_timestep,
// PISMEigenCalving.cc:77-341, with remove_narrow_tongues, :420-493).
//
// Strain rates and stresses: one thread per cell, grid-stride.  Eigen-calving: the front
// cells (ice-free ocean next to floating ice) are few, so the first pass evaluates the
// strain rates of the four cells two away from a front cell on the spot instead of storing
// a strain-rate field; the cut of the floating neighbours is a second pass over the
// per-cell losses.  remove_narrow_tongues runs in the reference as one in-place sweep in
// (i, j) order, so a cell sees the new mask of its neighbours earlier in that order; here
// that recurrence is solved by repeated parallel sweeps over (original mask, live mask) until
// none changes a cell — the unique fixed point of the recurrence, which is the sequential
// answer.  Arithmetic follows the reference's order with no contraction where a rounding
// could differ.
#include <algorithm>

#include "ssa_reduce.cuh"

namespace pism_gpu {

namespace {

constexpr int NTC = RED_THREADS;
constexpr int8_t MASK_GROUNDED_ = 2, MASK_FLOATING_ = 3, MASK_OCEAN_ = 4;

// Mask.hh:28-65
__device__ __forceinline__ bool icy(int m) { return m == MASK_GROUNDED_ || m == MASK_FLOATING_; }
__device__ __forceinline__ bool floating_ice(int m) { return m == MASK_FLOATING_; }
__device__ __forceinline__ bool ice_free_ocean(int m) { return m >= MASK_FLOATING_ && !icy(m); }

struct Gradient {
  double u_x, u_y, v_x, v_y;
};

// ShallowStressBalance.cc:249-293: centred differences as weighted one-sided ones, a side
// dropped where that neighbour is ice-free.  The weights are 0 or 1, so the products in
// the weighted sums are exact and a fused multiply-add rounds like the reference; the
// scaling by 1 / (dx (west + east)) is rounded on its own (__dmul_rn), so that no later sum
// of two derivatives is contracted into a fused multiply-add where the function is inlined.
__device__ __forceinline__ Gradient velocity_gradient(const GridDev &g, const double2 *vel, const int8_t *mask,
                                                      int i, int j) {
  const int ke = nbr(g, i, j, 1, 0), kw = nbr(g, i, j, -1, 0), kn = nbr(g, i, j, 0, 1), ks = nbr(g, i, j, 0, -1);
  const double east = icy(mask[ke]) ? 1.0 : 0.0, west = icy(mask[kw]) ? 1.0 : 0.0;
  const double north = icy(mask[kn]) ? 1.0 : 0.0, south = icy(mask[ks]) ? 1.0 : 0.0;
  const double2 U = vel[i * g.My + j];
  Gradient d{0.0, 0.0, 0.0, 0.0};
  if (west + east > 0) {
    const double2 Ue = vel[ke], Uw = vel[kw];
    const double r = 1.0 / (g.dx * (west + east));
    d.u_x = __dmul_rn(r, west * (U.x - Uw.x) + east * (Ue.x - U.x));
    d.v_x = __dmul_rn(r, west * (U.y - Uw.y) + east * (Ue.y - U.y));
  }
  if (south + north > 0) {
    const double2 Un = vel[kn], Us = vel[ks];
    const double r = 1.0 / (g.dy * (south + north));
    d.u_y = __dmul_rn(r, south * (U.x - Us.x) + north * (Un.x - U.x));
    d.v_y = __dmul_rn(r, south * (U.y - Us.y) + north * (Un.y - U.y));
  }
  return d;
}

// ShallowStressBalance.cc:295-302: eigenvalues (max, min) of the strain rate tensor
__device__ __forceinline__ double2 principal(const Gradient &d) {
  const double A = 0.5 * (d.u_x + d.v_y), B = 0.5 * (d.u_x - d.v_y), Dxy = 0.5 * (d.v_x + d.u_y);
  const double q = sqrt(__dadd_rn(__dmul_rn(B, B), __dmul_rn(Dxy, Dxy)));
  return make_double2(A + q, A - q);
}

__global__ void __launch_bounds__(NTC) k_strain_rates(GridDev g, const double2 *vel, const int8_t *mask,
                                                      double *edot, double *stress, double hardness,
                                                      double schoof_reg, double viscosity_power) {
  const int N = g.Mx * g.My;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const int i = k / g.My, j = k - i * g.My;
    if (!icy(mask[k])) {
      if (edot) edot[2 * k] = edot[2 * k + 1] = 0.0;
      if (stress) stress[3 * k] = stress[3 * k + 1] = stress[3 * k + 2] = 0.0;
      continue;
    }
    const Gradient d = velocity_gradient(g, vel, mask, i, j);
    if (edot) {   // plain doubles: a caller's array need only be 8-byte aligned
      const double2 e = principal(d);
      edot[2 * k] = e.x;
      edot[2 * k + 1] = e.y;
    }
    if (stress) {
      // secondInvariant_2D (flowlaws.hh:36-39) and FlowLaw::effective_viscosity (:100-112)
      const double s = __dadd_rn(__dmul_rn(d.u_x, d.u_x), __dmul_rn(d.v_y, d.v_y));
      const double xy = d.u_x + d.v_y, sh = d.u_y + d.v_x;
      const double gamma = 0.5 * __dadd_rn(__dadd_rn(s, __dmul_rn(xy, xy)), 0.5 * __dmul_rn(sh, sh));
      const double nu = 0.5 * hardness * pow(schoof_reg + gamma, viscosity_power);
      stress[3 * k] = nu * d.u_x;
      stress[3 * k + 1] = nu * d.v_y;
      stress[3 * k + 2] = 0.5 * nu * sh;   // (0.5 nu) (u_y + v_x)
    }
  }
}

__global__ void k_mask_from_doubles(int N, const double *in, int8_t *a, int8_t *b) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const int8_t m = (int8_t)floor(in[k] + 0.5);   // IceModelVec2Int::as_int
    a[k] = m;
    if (b) b[k] = m;
  }
}

struct Front {
  bool front, law;
  double rate;   // K eigen1 eigen2 where the calving law applies, else 0
};

// PISMEigenCalving.cc:115-176 (and :283-322): a front cell and its horizontal calving rate
__device__ Front calving_front(const GridDev &g, const double2 *vel, const int8_t *mask, double K, int i, int j) {
  Front f{false, false, 0.0};
  const int k = i * g.My + j;
  if (!ice_free_ocean(mask[k])) return f;
  const int kn[4] = {nbr(g, i, j, 1, 0), nbr(g, i, j, -1, 0), nbr(g, i, j, 0, 1), nbr(g, i, j, 0, -1)};
  if (!(floating_ice(mask[kn[0]]) || floating_ice(mask[kn[1]]) || floating_ice(mask[kn[2]]) ||
        floating_ice(mask[kn[3]])))
    return f;
  f.front = true;
  constexpr int o = 2;   // EigenCalving::m_stencil_width
  const int di[4] = {-o, o, 0, 0}, dj[4] = {0, 0, -o, o};
  double e1 = 0.0, e2 = 0.0;
  int M = 0;
  for (int q = 0; q < 4; ++q) {
    const int ii = i + di[q], jj = j + dj[q];
    const int io = wrap(ii, g.Mx), jo = wrap(jj, g.My);
    const int ko = io * g.My + jo;
    if (!floating_ice(mask[ko])) continue;
    // ice_margin (Mask.hh:177-181): icy with an ice-free neighbour
    if (!icy(mask[nbr(g, io, jo, 1, 0)]) || !icy(mask[nbr(g, io, jo, -1, 0)]) || !icy(mask[nbr(g, io, jo, 0, 1)]) ||
        !icy(mask[nbr(g, io, jo, 0, -1)]))
      continue;
    // inside the grid: the strain rate there; across its edge: the ghost value, which
    // EigenCalving::init set to 0 and nothing refreshes (it still counts in M)
    if (ii == io && jj == jo) {
      const double2 e = principal(velocity_gradient(g, vel, mask, io, jo));
      e1 += e.x;
      e2 += e.y;
    }
    M += 1;
  }
  if (M > 0) {
    e1 /= M;
    e2 /= M;
  }
  if (e2 > 0.0 && e1 > 0.0) {   // spreading in all directions; eigenCalvOffset = 0
    f.law = true;
    f.rate = K * e1 * (e2 - 0.0);
  }
  return f;
}

// pass 1, PISMEigenCalving.cc:107-200: lower Href at the front, record the thickness loss
// to be shared by the floating neighbours
__global__ void __launch_bounds__(NTC) k_ec_front(GridDev g, const double2 *vel, const int8_t *mask, double K,
                                                  double dt, const double *H, double *Href, double *loss) {
  const int N = g.Mx * g.My;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const int i = k / g.My, j = k - i * g.My;
    double lost = 0.0;
    const Front f = calving_front(g, vel, mask, K, i, j);
    if (f.front) {
      const int kn[4] = {nbr(g, i, j, 1, 0), nbr(g, i, j, -1, 0), nbr(g, i, j, 0, 1), nbr(g, i, j, 0, -1)};
      int nfl = 0;
      double H_average = 0.0;
      for (int q = 0; q < 4; ++q)
        if (floating_ice(mask[kn[q]])) {
          nfl += 1;
          H_average += H[kn[q]];
        }
      if (nfl > 0) H_average /= nfl;
      const double calving_rate = f.rate * H_average / g.dx;
      if (calving_rate > 0.0) {
        double h = Href[k] - __dmul_rn(calving_rate, dt);   // no fused multiply-add
        if (h < 0.0) {
          lost = -h;
          h = 0.0;
          if (nfl > 0) lost /= nfl;
        }
        Href[k] = h;
      }
    }
    loss[k] = lost;
  }
}

// pass 2, PISMEigenCalving.cc:204-226: floating cells next to a loss are cut
__global__ void __launch_bounds__(NTC) k_ec_cut(GridDev g, const double *loss, double *H, double *Href, int8_t *m0,
                                                int8_t *live) {
  const int N = g.Mx * g.My;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const int i = k / g.My, j = k - i * g.My;
    if (!floating_ice(m0[k])) continue;
    const double le = loss[nbr(g, i, j, 1, 0)], lw = loss[nbr(g, i, j, -1, 0)];
    const double ln = loss[nbr(g, i, j, 0, 1)], ls = loss[nbr(g, i, j, 0, -1)];
    if (le > 0.0 || lw > 0.0 || ln > 0.0 || ls > 0.0) {
      const double total = le + lw + ln + ls;
      const double rest = H[k] - total;
      Href[k] = rest < 0.0 ? 0.0 : rest;   // std::max(rest, 0.0)
      H[k] = 0.0;
      m0[k] = MASK_OCEAN_;
      live[k] = MASK_OCEAN_;
    }
  }
}

// one sweep of remove_narrow_tongues (PISMEigenCalving.cc:420-493).  A neighbour earlier in
// the reference's (i outer, j inner) order and inside the grid is read from the live mask,
// every other one (later, or across the periodic edge: a ghost) from the mask before the loop.
__global__ void __launch_bounds__(NTC) k_ec_tongues(GridDev g, const int8_t *m0, int8_t *live, int *changed) {
  const int N = g.Mx * g.My;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const int i = k / g.My, j = k - i * g.My;
    const int m = m0[k];
    if (!icy(m)) continue;
    auto at = [&](int di, int dj) -> int {
      const int ii = i + di, jj = j + dj;
      const bool inside = ii >= 0 && ii < g.Mx && jj >= 0 && jj < g.My;
      const bool earlier = di < 0 || (di == 0 && dj < 0);
      const int kk = wrap(ii, g.Mx) * g.My + wrap(jj, g.My);
      return (inside && earlier) ? (int)live[kk] : (int)m0[kk];
    };
    // grounded ice: ice-free ocean neighbours; floating ice: any ice-free neighbour
    auto free_ = [&](int a) { return m == MASK_GROUNDED_ ? ice_free_ocean(a) : !icy(a); };
    const bool N_ = free_(at(0, 1)), E = free_(at(1, 0)), S = free_(at(0, -1)), W = free_(at(-1, 0));
    const bool NE = free_(at(1, 1)), NW = free_(at(-1, 1)), SE = free_(at(1, -1)), SW = free_(at(-1, -1));
    const bool cut = (!W && NW && SW && N_ && S && E) || (!N_ && NW && NE && W && E && S) ||
                     (!E && NE && SE && W && S && N_) || (!S && SW && SE && W && E && N_);
    const int8_t want = cut ? MASK_OCEAN_ : (int8_t)m;
    if (live[k] != want) {
      live[k] = want;
      *changed = 1;
    }
  }
}

__global__ void k_ec_finish(int N, const int8_t *m0, const int8_t *live, double *H, double *mask_out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    if (icy(m0[k]) && live[k] == MASK_OCEAN_) H[k] = 0.0;
    mask_out[k] = (double)live[k];
  }
}

// EigenCalving::max_timestep's statistics (PISMEigenCalving.cc:283-330): the number of cells
// where the calving law applies and the sum of their rates, in block order; the maximum
// rate by an integer maximum over the bits of the non-negative rates (K >= 0)
__global__ void __launch_bounds__(NTC) k_ec_rates(GridDev g, const double2 *vel, const int8_t *mask, double K,
                                                  double *out, unsigned long long *rmax, double *partials,
                                                  unsigned *ticket) {
  const int N = g.Mx * g.My;
  double acc[2] = {0.0, 0.0};
  double mine = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const int i = k / g.My, j = k - i * g.My;
    const Front f = calving_front(g, vel, mask, K, i, j);
    if (f.law) {
      acc[0] += 1.0;
      acc[1] += f.rate;
      mine = mine < f.rate ? f.rate : mine;
    }
  }
  if (mine > 0.0) atomicMax(rmax, (unsigned long long)__double_as_longlong(mine));
  double tot[2];
  if (grid_reduce<2>(acc, partials, ticket, tot)) {
    out[0] = tot[0];
    out[1] = tot[1];
  }
}

int blocks_for(const Launch &L, int N) { return std::max(1, std::min((N + NTC - 1) / NTC, L.max_blocks)); }

}  // namespace

void launch_strain_rates(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, const double2 *vel,
                         const int8_t *mask, double *edot, double *stress) {
  const double n = c.ssa_Glen_exponent;
  const double hardness = pow(c.ice_softness, -1.0 / n);   // ShallowStressBalance.cc:318
  const double reg = (c.Schoof_regularizing_velocity / c.Schoof_regularizing_length) *
                     (c.Schoof_regularizing_velocity / c.Schoof_regularizing_length);   // flowlaws.cc:83-85
  L.tick();
  k_strain_rates<<<blocks_for(L, g.Mx * g.My), NTC, 0, L.stream>>>(g, vel, mask, edot, stress, hardness, reg,
                                                                   (1.0 - n) / (2.0 * n));
}

void launch_mask_from_doubles(const Launch &L, int N, const double *in, int8_t *a, int8_t *b) {
  L.tick();
  k_mask_from_doubles<<<blocks_for(L, N), NTC, 0, L.stream>>>(N, in, a, b);
}

void launch_eigen_calving_passes(const Launch &L, const GridDev &g, const double2 *vel, double K, double dt,
                                 double *H, double *Href, double *loss, int8_t *m0, int8_t *live) {
  const int blocks = blocks_for(L, g.Mx * g.My);
  L.tick(2);
  k_ec_front<<<blocks, NTC, 0, L.stream>>>(g, vel, m0, K, dt, H, Href, loss);
  k_ec_cut<<<blocks, NTC, 0, L.stream>>>(g, loss, H, Href, m0, live);
}

void launch_tongue_sweep(const Launch &L, const GridDev &g, const int8_t *m0, int8_t *live, int *changed) {
  L.tick();
  k_ec_tongues<<<blocks_for(L, g.Mx * g.My), NTC, 0, L.stream>>>(g, m0, live, changed);
}

void launch_eigen_calving_finish(const Launch &L, int N, const int8_t *m0, const int8_t *live, double *H,
                                 double *mask_out) {
  L.tick();
  k_ec_finish<<<blocks_for(L, N), NTC, 0, L.stream>>>(N, m0, live, H, mask_out);
}

void launch_eigen_calving_rates(const Launch &L, const GridDev &g, const double2 *vel, const int8_t *mask, double K,
                                double *out, unsigned long long *rmax) {
  L.tick();
  k_ec_rates<<<blocks_for(L, g.Mx * g.My), NTC, 0, L.stream>>>(g, vel, mask, K, out, rmax, L.partials, L.ticket);
}

}  // namespace pism_gpu
