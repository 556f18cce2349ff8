// SSAFD_GPU.hh — C++ host side of the B200 SSA solver, with the interface of PISM's
// stress-balance classes:
//   ShallowStressBalance  src/base/stressbalance/ShallowStressBalance.hh:39-99
//   SSA                   src/base/stressbalance/ssa/SSA.hh:110-156
//   SSAFD (KSPFailure, PicardFailure)  src/base/stressbalance/ssa/SSAFD.hh:30-123
//   SSAFactory            SSA.hh:77
// It stands alone (no PETSc): fields are plain arrays in the reference's DMDA layout,
// [i][j] with j contiguous, vectors interleaved (u, v).  Inside pismr the same class
// derives from pism::stressbalance::SSA and reads IceModelVec arrays.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "pism_unet_gpu.h"

namespace pism_b200 {

// IceGrid subset: sizes, spacing (IceGrid.cc:540-610), vertical levels
struct Grid {
  int Mx = 0, My = 0;
  double Lx = 0, Ly = 0, x0 = 0, y0 = 0;
  int periodicity = PISM_NOT_PERIODIC;
  std::vector<double> z{0.0, 500.0, 1000.0};
  double dx() const { return 2.0 * Lx / ((periodicity & PISM_X_PERIODIC) ? Mx : Mx - 1); }
  double dy() const { return 2.0 * Ly / ((periodicity & PISM_Y_PERIODIC) ? My : My - 1); }
  double x(int i) const;
  double y(int j) const;
  static Grid Shallow(double Lx, double Ly, int Mx, int My, int periodicity);
};

// IceModelVec2S / IceModelVec2V stand-ins
struct Field2 {
  int Mx = 0, My = 0;
  std::vector<double> a;
  Field2() = default;
  Field2(int mx, int my, double v = 0.0) : Mx(mx), My(my), a((size_t)mx * my, v) {}
  double &operator()(int i, int j) { return a[(size_t)i * My + j]; }
  double operator()(int i, int j) const { return a[(size_t)i * My + j]; }
  void set(double v) { a.assign(a.size(), v); }
};

struct Field2V {
  int Mx = 0, My = 0;
  std::vector<double> a;
  Field2V() = default;
  Field2V(int mx, int my) : Mx(mx), My(my), a(2 * (size_t)mx * my, 0.0) {}
  double &u(int i, int j) { return a[2 * ((size_t)i * My + j)]; }
  double &v(int i, int j) { return a[2 * ((size_t)i * My + j) + 1]; }
  double u(int i, int j) const { return a[2 * ((size_t)i * My + j)]; }
  double v(int i, int j) const { return a[2 * ((size_t)i * My + j) + 1]; }
};

// pism::RuntimeError and the SSAFD failure classes
struct RuntimeError : std::runtime_error {
  explicit RuntimeError(const std::string &m) : std::runtime_error(m) {}
};
struct KSPFailure : RuntimeError {
  explicit KSPFailure(const std::string &m) : RuntimeError("SSAFD KSP (linear solver) failed: " + m) {}
};
struct PicardFailure : RuntimeError {
  explicit PicardFailure(const std::string &m) : RuntimeError("SSAFD Picard iterations failed: " + m) {}
};

// the fields SSA::init_impl fetches from m_grid->variables() (SSA.cc:134-184)
struct Vars {
  const Field2 *mask = nullptr, *thickness = nullptr, *tauc = nullptr, *surface = nullptr, *bed = nullptr;
  const Field2 *gl_mask = nullptr, *fracture_density = nullptr;
  const std::vector<double> *enthalpy = nullptr;   // Mx*My*Mz, [i][j][k]
};

class ShallowStressBalance {
 public:
  virtual ~ShallowStressBalance() = default;
  void init() { init_impl(); }
  void set_boundary_conditions(const Field2 &locations, const Field2V &velocities) {
    m_bc_mask = &locations;
    m_bc_values = &velocities;
  }
  void set_sea_level_elevation(double sea_level) { m_config.sea_level = sea_level; }
  virtual void update(bool fast, const Field2 &melange_back_pressure) = 0;
  const Field2V &velocity() const { return m_velocity; }
  const Field2 &basal_frictional_heating() const { return m_bfrict; }
  virtual std::string stdout_report() const { return m_stdout; }

 protected:
  ShallowStressBalance(const Grid &g, const pism_gpu_ssa_config &c)
      : m_grid(g), m_config(c), m_velocity(g.Mx, g.My), m_bfrict(g.Mx, g.My) {}
  virtual void init_impl() {}
  Grid m_grid;
  pism_gpu_ssa_config m_config;
  Field2V m_velocity;
  Field2 m_bfrict;
  const Field2 *m_bc_mask = nullptr;
  const Field2V *m_bc_values = nullptr;
  std::string m_stdout;
};

class SSA : public ShallowStressBalance {
 public:
  void update(bool fast, const Field2 &melange_back_pressure) override {   // SSA.cc:188-196
    m_melange = &melange_back_pressure;
    if (!fast) solve();
  }
  void set_initial_guess(const Field2V &guess) { m_velocity = guess; }      // SSA.cc:361-363
  void set_variables(const Vars &v) { m_vars = v; }

 protected:
  SSA(const Grid &g, const pism_gpu_ssa_config &c) : ShallowStressBalance(g, c) {}
  virtual void solve() = 0;
  Vars m_vars;
  const Field2 *m_melange = nullptr;
};

// The B200 solver behind the SSA interface; solve() replaces SSAFD::solve().
class SSAFD_GPU : public SSA {
 public:
  SSAFD_GPU(const Grid &g, const pism_gpu_ssa_config &c, int device = 0);
  ~SSAFD_GPU() override;
  SSAFD_GPU(const SSAFD_GPU &) = delete;
  SSAFD_GPU &operator=(const SSAFD_GPU &) = delete;
  const pism_gpu_ssa_stats &stats() const { return m_stats; }
  // the SSAFD_nuH diagnostic (SSAFD.cc:1790-1823): staggered nu*H, interleaved
  std::vector<double> nuH() const;
  // Start the solves from the learned initial guess (include/pism_unet_gpu.h) instead of the
  // previous velocity; nullptr restores the reference's start.  The network is borrowed.
  void set_warm_start(pism_gpu_unet *net, int stride = 1) {
    m_net = net;
    m_stride = stride;
  }

 protected:
  void init_impl() override;
  void solve() override;

 private:
  void check(int rc, const char *what) const;
  pism_gpu_ssa *m_gpu = nullptr;
  pism_gpu_ssa_stats m_stats{};
  pism_gpu_unet *m_net = nullptr;
  int m_stride = 1;
};

typedef SSA *(*SSAFactory)(const Grid &, const pism_gpu_ssa_config &);
SSA *SSAFD_GPUFactory(const Grid &g, const pism_gpu_ssa_config &c);

}  // namespace pism_b200
