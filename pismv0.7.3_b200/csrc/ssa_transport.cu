// ssa_transport.cu — the explicit mass-continuity step that consumes the SSA velocity
// (IceModel::massContExplicitStep, iMgeometry.cc:497-819, with the ConstantInColumn
// modifier: no diffusive flux), then the mask and surface of the new thickness
// (IceModel::updateSurfaceElevationAndMask, iMgeometry.cc:56-68, GeometryCalculator,
// Mask.hh:66-120).  part_grid and the residual redistribution are not restated (off by
// default, pism_config.cdl:77-79).
//
// One thread per cell, grid-stride: the four face velocities of cell_interface_fluxes
// (iMgeometry.cc:309-410), the upwinded flux divergence, the source terms, the
// non-negativity rule, the new mask and surface; the eight flux totals of the step are
// summed per thread in FP64 and over the grid in block order (ssa_reduce.cuh).
#include <algorithm>

#include "ssa_reduce.cuh"

namespace pism_gpu {

namespace {

constexpr int NTT = RED_THREADS;

__device__ __forceinline__ bool icy(int m) { return m == 2 || m == 3; }   // Mask.hh:46-48

// the face velocity between cell (m, a, bm, bv) and its neighbour (mn, an, bmn, bvn), one
// component (a: the cell's SSA velocity component, bv: its Dirichlet value)
__device__ __forceinline__ double face_velocity(bool dirichlet, int m, int mn, double a, double an, int bm, int bmn,
                                                double bv, double bvn) {
  double out;
  if (icy(m) && icy(mn)) out = 0.5 * (a + an);   // both sides icy
  else if (icy(m)) out = a;                        // icy next to ice-free
  else if (icy(mn)) out = an;                      // ice-free next to icy
  else out = 0.0;                                  // both ice-free
  if (dirichlet) {
    if (bm == 1 && bmn == 1) out = 0.5 * (bv + bvn);
    else if (bm == 1 && bmn == 0) out = bv;
    else if (bm == 0 && bmn == 1) out = bvn;
  }
  return out;
}

struct MassStep {
  double dt, rho, icefree_thickness, is_floating_thickness;
  int dirichlet;
  const double2 *vel, *bcv;
  const int8_t *mask;
  const uint8_t *bc;
  const double *H, *bed, *cmb, *bmr, *area;
  double *Hnew, *fdiv, *mask_new, *surface_new, *totals;
};

__global__ void __launch_bounds__(NTT) k_mass_continuity(GridDev g, pism_gpu_ssa_config c, MassStep a,
                                                         double *partials, unsigned *ticket) {
  const int N = g.Mx * g.My;
  const double alpha = 1.0 - c.ice_density / c.sea_water_density;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const int i = k / g.My, j = k - i * g.My;
    const int ke = nbr(g, i, j, 1, 0), kw = nbr(g, i, j, -1, 0), kn = nbr(g, i, j, 0, 1), ks = nbr(g, i, j, 0, -1);
    const int m = a.mask[k];
    const double2 U = a.vel[k];
    const double2 B = a.dirichlet ? a.bcv[k] : make_double2(0.0, 0.0);
    const int bm = a.dirichlet ? a.bc[k] : 0;
    auto face = [&](int kk, bool x) {
      const double2 Un = a.vel[kk];
      const double2 Bn = a.dirichlet ? a.bcv[kk] : make_double2(0.0, 0.0);
      return face_velocity(a.dirichlet, m, a.mask[kk], x ? U.x : U.y, x ? Un.x : Un.y, bm,
                           a.dirichlet ? a.bc[kk] : 0, x ? B.x : B.y, x ? Bn.x : Bn.y);
    };
    const double ve = face(ke, true), vw = face(kw, true), vn = face(kn, false), vs = face(ks, false);
    const double Hc = a.H[k];
    const double meter_to_kg = (a.area ? a.area[k] : g.dx * g.dy) * a.rho, meter_per_s_to_kg = meter_to_kg * a.dt;
    double divQ_SIA = 0.0, divQ_SSA = 0.0;   // no diffusive flux: (Q.e - Q.w) / dx + (Q.n - Q.s) / dy = 0
    // upwinded SSA flux divergence, iMgeometry.cc:641-644
    divQ_SSA += (ve * (ve > 0 ? Hc : a.H[ke]) - vw * (vw > 0 ? a.H[kw] : Hc)) / g.dx;
    divQ_SSA += (vn * (vn > 0 ? Hc : a.H[kn]) - vs * (vs > 0 ? a.H[ks] : Hc)) / g.dy;
    double smb = a.cmb[k] / a.rho, melt = a.bmr ? a.bmr[k] : 0.0, href_to_h = 0.0;
    if (m >= 3 && !icy(m)) {   // ice-free ocean (Mask.hh:59-61): neither mass balance applies
      smb = 0.0;
      melt = 0.0;
    }
    if (a.dirichlet && bm == 1) {   // iMgeometry.cc:714-721
      smb = 0.0;
      melt = 0.0;
      href_to_h = 0.0;
      divQ_SIA = 0.0;
      divQ_SSA = 0.0;
    }
    if (a.fdiv) a.fdiv[k] = divQ_SIA + divQ_SSA;
    double Hn = Hc + (a.dt * (smb - melt - (divQ_SIA + divQ_SSA)) + href_to_h);
    double nonneg = 0.0;
    if (Hn < 0.0) {
      nonneg += -Hn;
      Hn = 0.0;
    }
    a.Hnew[k] = Hn;
    // GeometryCalculator::compute on the new thickness (dry simulation off)
    const double hgrounded = a.bed[k] + Hn, hfloating = c.sea_level + alpha * Hn;
    const bool floating = hfloating > hgrounded + a.is_floating_thickness, ice_free = Hn < a.icefree_thickness;
    if (a.mask_new) a.mask_new[k] = floating ? (ice_free ? 4.0 : 3.0) : (ice_free ? 0.0 : 2.0);
    if (a.surface_new) a.surface_new[k] = floating ? hfloating : hgrounded;
    // the step's flux totals in kg, iMgeometry.cc:755-770 (grounded: Mask.hh:42-44)
    if (m < 3) acc[0] += -melt * meter_per_s_to_kg;
    else acc[2] += -melt * meter_per_s_to_kg;
    acc[1] += nonneg * meter_to_kg;
    acc[3] += smb * meter_per_s_to_kg;
    acc[4] += -divQ_SIA * meter_per_s_to_kg;
    acc[5] += -divQ_SSA * meter_per_s_to_kg;
    acc[6] += href_to_h * meter_to_kg;   // acc[7], H_to_Href_flux: part_grid only
  }
  double tot[8];
  if (grid_reduce<8>(acc, partials, ticket, tot))
    for (int v = 0; v < 8; ++v) a.totals[v] = tot[v];
}

}  // namespace

void launch_mass_continuity(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, const Fields &f,
                            double dt, double icefree_thickness, double is_floating_thickness, const double *cmb,
                            const double *bmr, const double *area, double *Hnew, double *fdiv, double *mask_new,
                            double *surface_new, double *totals) {
  const int N = g.Mx * g.My;
  const int blocks = std::max(1, std::min((N + NTT - 1) / NTT, L.max_blocks));
  MassStep a;
  a.dt = dt;
  a.rho = c.ice_density;
  a.icefree_thickness = icefree_thickness;
  a.is_floating_thickness = is_floating_thickness;
  a.dirichlet = c.ssa_dirichlet_bc ? 1 : 0;
  a.vel = f.vel;
  a.bcv = f.bcv;
  a.mask = f.mask;
  a.bc = f.bc;
  a.H = f.H;
  a.bed = f.bed;
  a.cmb = cmb;
  a.bmr = bmr;
  a.area = area;
  a.Hnew = Hnew;
  a.fdiv = fdiv;
  a.mask_new = mask_new;
  a.surface_new = surface_new;
  a.totals = totals;
  L.tick();
  k_mass_continuity<<<blocks, NTT, 0, L.stream>>>(g, c, a, L.partials, L.ticket);
}

}  // namespace pism_gpu
