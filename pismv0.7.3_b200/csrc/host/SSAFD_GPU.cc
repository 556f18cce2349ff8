// SSAFD_GPU.cc — the C++ SSA class over the C-ABI of include/pism_ssa_gpu.h.
#include "SSAFD_GPU.hh"

#include <cstdio>

namespace pism_b200 {

// IceGrid::compute_horizontal_coordinates, IceGrid.cc:550-610
static double coord(int idx, int M, double L, double c0, bool periodic) {
  const double d = periodic ? 2.0 * L / M : 2.0 * L / (M - 1);
  const double vmin = c0 - L, vmax = c0 + L;
  if (periodic) return idx == M - 1 ? vmax - 0.5 * d : vmin + (idx + 0.5) * d;
  return idx == M - 1 ? vmax : vmin + idx * d;
}

double Grid::x(int i) const { return coord(i, Mx, Lx, x0, periodicity & PISM_X_PERIODIC); }
double Grid::y(int j) const { return coord(j, My, Ly, y0, periodicity & PISM_Y_PERIODIC); }

Grid Grid::Shallow(double Lx, double Ly, int Mx, int My, int periodicity) {
  Grid g;
  g.Lx = Lx;
  g.Ly = Ly;
  g.Mx = Mx;
  g.My = My;
  g.periodicity = periodicity;
  return g;
}

SSAFD_GPU::SSAFD_GPU(const Grid &g, const pism_gpu_ssa_config &c, int device) : SSA(g, c) {
  pism_gpu_grid gd{g.Mx, g.My, g.dx(), g.dy(), g.periodicity, (int)g.z.size(), g.z.data()};
  int rc = pism_gpu_ssa_create(&gd, &c, device, &m_gpu);
  if (rc != PISM_GPU_SSA_OK) throw RuntimeError("pism_gpu_ssa_create failed with status " + std::to_string(rc));
}

SSAFD_GPU::~SSAFD_GPU() { pism_gpu_ssa_destroy(m_gpu); }

void SSAFD_GPU::check(int rc, const char *what) const {
  if (rc == PISM_GPU_SSA_OK) return;
  const std::string msg = std::string(what) + ": " + pism_gpu_ssa_last_error(m_gpu);
  if (rc == PISM_GPU_SSA_EKSP) throw KSPFailure(msg);
  if (rc == PISM_GPU_SSA_EPICARD) throw PicardFailure(msg);
  throw RuntimeError(msg);
}

void SSAFD_GPU::init_impl() {
  // SSAFD::init_impl (SSAFD.cc:221-258): the FD solver needs a surface elevation
  if (!m_vars.surface)
    throw RuntimeError("The finite difference SSA solver requires a surface elevation.");
  m_velocity = Field2V(m_grid.Mx, m_grid.My);   // default initial guess, SSA.cc:178
}

void SSAFD_GPU::solve() {
  if (!m_vars.mask || !m_vars.thickness || !m_vars.tauc || !m_vars.surface || !m_vars.bed)
    throw RuntimeError("SSA inputs are missing (mask, thickness, tauc, surface, bed)");
  check(pism_gpu_ssa_set_config(m_gpu, &m_config), "set_config");
  pism_gpu_ssa_inputs in{};
  in.where = PISM_MEM_HOST;
  in.thickness = m_vars.thickness->a.data();
  in.surface = m_vars.surface->a.data();
  in.bed = m_vars.bed->a.data();
  in.mask = m_vars.mask->a.data();
  in.tauc = m_vars.tauc->a.data();
  if (m_bc_mask && m_bc_values) {
    in.bc_mask = m_bc_mask->a.data();
    in.bc_values = m_bc_values->a.data();
  }
  in.melange = m_melange ? m_melange->a.data() : nullptr;
  in.gl_mask = m_vars.gl_mask ? m_vars.gl_mask->a.data() : nullptr;
  in.enthalpy = m_vars.enthalpy ? m_vars.enthalpy->data() : nullptr;
  in.fracture_density = m_vars.fracture_density ? m_vars.fracture_density->a.data() : nullptr;
  check(pism_gpu_ssa_set_inputs(m_gpu, &in), "set_inputs");
  if (m_net)
    check(pism_gpu_ssa_learned_guess(m_gpu, m_net, m_stride), "learned initial guess");
  else
    check(pism_gpu_ssa_set_initial_guess(m_gpu, m_velocity.a.data(), PISM_MEM_HOST), "set_initial_guess");
  check(pism_gpu_ssa_solve(m_gpu, m_velocity.a.data(), PISM_MEM_HOST, &m_stats), "SSAFD solve");
  check(pism_gpu_ssa_get_field(m_gpu, PISM_FIELD_BFRICT, m_bfrict.a.data(), PISM_MEM_HOST), "bfrict");
  char buf[128];
  snprintf(buf, sizeof(buf), "%5d outer iterations, ~%3.1f KSP iterations each\n", m_stats.picard_iterations,
           (double)m_stats.ksp_iterations / (m_stats.picard_iterations > 0 ? m_stats.picard_iterations : 1));
  m_stdout = buf;
}

std::vector<double> SSAFD_GPU::nuH() const {
  std::vector<double> out(2 * (size_t)m_grid.Mx * m_grid.My);
  check(pism_gpu_ssa_get_field(m_gpu, PISM_FIELD_NUH, out.data(), PISM_MEM_HOST), "nuH");
  return out;
}

SSA *SSAFD_GPUFactory(const Grid &g, const pism_gpu_ssa_config &c) { return new SSAFD_GPU(g, c); }

}  // namespace pism_b200
