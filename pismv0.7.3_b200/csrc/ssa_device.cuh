// ssa_device.cuh — device-side helpers of the B200 SSAFD solver.
//
// Layout: cell (i, j) is element k = i*My + j (j, the y index, contiguous); vector
// fields are double2 (u, v) per cell; staggered fields are double2 (east face,
// north face) per cell.  Every neighbour access wraps periodically, as the
// reference's DMDA does (src/base/util/IceGrid.cc:807-819).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pism_ssa_gpu.h"

namespace pism_gpu {

// mask values (src/base/util/Mask.hh:28-34)
enum : int { MASK_ICE_FREE_BEDROCK = 0, MASK_GROUNDED = 2, MASK_FLOATING = 3, MASK_ICE_FREE_OCEAN = 4 };

// mask predicates (Mask.hh:37-65)
__host__ __device__ __forceinline__ bool m_ocean(int M) { return M >= MASK_FLOATING; }
__host__ __device__ __forceinline__ bool m_grounded(int M) { return !m_ocean(M); }
__host__ __device__ __forceinline__ bool m_icy(int M) { return M == MASK_GROUNDED || M == MASK_FLOATING; }
__host__ __device__ __forceinline__ bool m_grounded_ice(int M) { return m_icy(M) && m_grounded(M); }
__host__ __device__ __forceinline__ bool m_floating_ice(int M) { return m_icy(M) && m_ocean(M); }
__host__ __device__ __forceinline__ bool m_ice_free(int M) { return !m_icy(M); }
__host__ __device__ __forceinline__ bool m_ice_free_ocean(int M) { return m_ocean(M) && m_ice_free(M); }
__host__ __device__ __forceinline__ bool m_ice_free_land(int M) { return m_grounded(M) && m_ice_free(M); }

// Per-cell flag word built once per solve.  Bits 0-11 are the CFBC stencil weights
// aMn..bMe of SSAFD::assemble_matrix (SSAFD.cc:594-684), set = weight 1.
enum : uint32_t {
  F_aMn = 1u << 0, F_aPn = 1u << 1, F_aMM = 1u << 2, F_aPP = 1u << 3, F_aMs = 1u << 4, F_aPs = 1u << 5,
  F_bPw = 1u << 6, F_bPP = 1u << 7, F_bPe = 1u << 8, F_bMw = 1u << 9, F_bMM = 1u << 10, F_bMe = 1u << 11,
  F_WEIGHTS = 0xFFFu,
  F_DIAG_ONLY = 1u << 12,   // Dirichlet or CFBC ice-free row: m_scaling on the diagonal only
  F_BC = 1u << 13,          // Dirichlet location (bc_mask == 1)
  F_MASK_SHIFT = 16,        // bits 16-18: the integer mask value
  // nu_bedrock_set overrides of c_w, c_e, c_n, c_s (SSAFD.cc:561-585)
  F_NB_W = 1u << 20, F_NB_E = 1u << 21, F_NB_N = 1u << 22, F_NB_S = 1u << 23,
  F_NB_ANY = F_NB_W | F_NB_E | F_NB_N | F_NB_S
};
__host__ __device__ __forceinline__ int flag_mask(uint32_t f) { return (int)((f >> F_MASK_SHIFT) & 7u); }

struct GridDev {
  int Mx, My;
  double dx, dy;
};

__device__ __forceinline__ int wrap(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }
__device__ __forceinline__ int cell(const GridDev &g, int i, int j) { return i * g.My + j; }
__device__ __forceinline__ int nbr(const GridDev &g, int i, int j, int di, int dj) {
  return wrap(i + di, g.Mx) * g.My + wrap(j + dj, g.My);
}

// ---- enthalpy converter (src/base/enthalpyConverter.cc) --------------------
__device__ __forceinline__ double ec_pressure(const pism_gpu_ssa_config &c, double depth) {
  // enthalpyConverter.cc:92-98
  return depth > 0.0 ? c.surface_pressure + c.ice_density * c.standard_gravity * depth : c.surface_pressure;
}
__device__ __forceinline__ double ec_melting_temperature(const pism_gpu_ssa_config &c, double P) {
  return c.water_melting_point_temperature - c.beta_CC * P;
}
__device__ __forceinline__ double ec_enthalpy_cts(const pism_gpu_ssa_config &c, double P) {
  return c.ice_specific_heat_capacity * (ec_melting_temperature(c, P) - c.enthalpy_converter_reference_temperature);
}
__device__ __forceinline__ double ec_temperature(const pism_gpu_ssa_config &c, double E, double P) {
  return E < ec_enthalpy_cts(c, P) ? E / c.ice_specific_heat_capacity + c.enthalpy_converter_reference_temperature
                                   : ec_melting_temperature(c, P);
}
__device__ __forceinline__ double ec_pressure_adjusted_temperature(const pism_gpu_ssa_config &c, double E,
                                                                   double P) {
  return ec_temperature(c, E, P) - ec_melting_temperature(c, P) + c.water_melting_point_temperature;
}
__device__ __forceinline__ double ec_water_fraction(const pism_gpu_ssa_config &c, double E, double P) {
  double Es = ec_enthalpy_cts(c, P);
  return E <= Es ? 0.0 : (E - Es) / c.water_latent_heat_fusion;
}

// ---- flow laws (src/base/rheology/flowlaws.{hh,cc}) ------------------------
__device__ __forceinline__ double softness_pb(const pism_gpu_ssa_config &c, double T_pa) {
  // FlowLaw::softness_parameter_paterson_budd, flowlaws.cc:90-95
  return T_pa < c.Paterson_Budd_critical_temperature
             ? c.Paterson_Budd_A_cold * exp(-c.Paterson_Budd_Q_cold / (c.ideal_gas_constant * T_pa))
             : c.Paterson_Budd_A_warm * exp(-c.Paterson_Budd_Q_warm / (c.ideal_gas_constant * T_pa));
}

__device__ __forceinline__ double softness(const pism_gpu_ssa_config &c, double E, double P) {
  switch (c.flow_law) {
    case PISM_FLOW_LAW_GPBLD: {  // GPBLD::softness_parameter, flowlaws.cc:209-221
      double Es = ec_enthalpy_cts(c, P);
      if (E < Es) return softness_pb(c, ec_pressure_adjusted_temperature(c, E, P));
      double omega = fmin(ec_water_fraction(c, E, P), c.gpbld_water_frac_observed_limit);
      return softness_pb(c, c.water_melting_point_temperature) * (1.0 + c.gpbld_water_frac_coeff * omega);
    }
    case PISM_FLOW_LAW_PB:
      return softness_pb(c, ec_pressure_adjusted_temperature(c, E, P));
    case PISM_FLOW_LAW_ARR:
      return c.Paterson_Budd_A_cold *
             exp(-c.Paterson_Budd_Q_cold / (c.ideal_gas_constant * ec_pressure_adjusted_temperature(c, E, P)));
    case PISM_FLOW_LAW_ARRWARM:
      return c.Paterson_Budd_A_warm *
             exp(-c.Paterson_Budd_Q_warm / (c.ideal_gas_constant * ec_pressure_adjusted_temperature(c, E, P)));
    case PISM_FLOW_LAW_HOOKE: {  // Hooke::softness_parameter_from_temp, flowlaws.cc:267-270
      double T_pa = ec_pressure_adjusted_temperature(c, E, P);
      return c.Hooke_A * exp(-c.Hooke_Q / (c.ideal_gas_constant * T_pa) +
                             3.0 * c.Hooke_C * pow(c.Hooke_Tr - T_pa, -c.Hooke_k));
    }
    default:
      return c.ice_softness;
  }
}

__device__ __forceinline__ double hardness_parameter(const pism_gpu_ssa_config &c, double E, double P) {
  return pow(softness(c, E, P), -1.0 / c.ssa_Glen_exponent);   // flowlaws.cc:104-106
}

// second invariant, flowlaws.hh:36-39
__device__ __forceinline__ double second_invariant_2d(double u_x, double u_y, double v_x, double v_y) {
  double a = u_x + v_y, b = u_y + v_x;
  return 0.5 * (u_x * u_x + v_y * v_y + a * a + 0.5 * (b * b));
}

// basal drag, basal_resistance.cc:46-50 (plastic) and 154-163 (pseudo-plastic)
__device__ __forceinline__ double basal_drag(const pism_gpu_ssa_config &c, double tauc, double u, double v) {
  double magreg2 = c.plastic_regularization * c.plastic_regularization + u * u + v * v;
  if (!c.do_pseudo_plastic_till) return tauc / sqrt(magreg2);
  double q = c.pseudo_plastic_q;
  double t = tauc;
  if (c.sliding_scale_factor_reduces_tauc > 0.0) t = tauc / pow(c.sliding_scale_factor_reduces_tauc, q);
  return t * pow(magreg2, 0.5 * (q - 1)) * pow(c.pseudo_plastic_uthreshold, -q);
}

}  // namespace pism_gpu
