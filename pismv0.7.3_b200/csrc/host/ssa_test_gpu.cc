// ssa_test_gpu — the verification driver of the B200 SSA solver: the counterpart of the
// reference's ssa_testi / ssa_testj / ssa_test_cfbc executables
// (src/base/stressbalance/ssa/tests/, SSATestCase.cc) on top of SSAFD_GPU.
//
//   ssa_test_gpu -test I|J|V [-Mx N] [-My N] [-ssa_rtol R] [-ssafd_ksp_rtol R] [-pc mg|bjacobi|line]
//                [-learned params.f32]   (start from the learned guess; raw FP32 parameters)
//
// It prints the error table of SSATestCase::report (SSATestCase.cc:231-244) in the same
// format, so its output can be compared with test/regression/ssa/*.sh line by line.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "SSAFD_GPU.hh"

using namespace pism_b200;

namespace {

const double kSecPerYear = 31556925.9747;   // UDUNITS-2 year

// Schoof's plastic-till stream (exactTestsIJ.c:29-77)
void exact_i(double m, double x, double y, double *bed, double *tauc, double *u, double *v) {
  const double L = 40e3, h0 = 0.05 * L, theta = atan(0.001), rho = 910, g = 9.81;
  const double f = rho * g * h0 * tan(theta), W = pow(m + 1.0, 1.0 / m) * L, B = 3.7e8;
  const double s = fabs(y / L);
  *tauc = f * pow(s, m);
  *bed = -x * tan(theta);
  *v = 0.0;
  if (fabs(y) < W) {
    const double C0 = 2.0 * pow(f / (B * h0), 3.0) * pow(L, 4.0), C1 = pow(m + 1.0, 4.0 / m);
    const double C2 = (m + 1.0) * C1, C3 = (m + 1.0) * C2, C4 = (m + 1.0) * C3;
    const double z1 = (pow(s, 4.0) - C1) / 4.0;
    const double z2 = (pow(s, m + 4.0) - C2) / ((m + 1.0) * (m + 4.0));
    const double z3 = (pow(s, 2.0 * m + 4.0) - C3) / ((m + 1.0) * (m + 1.0) * (2.0 * m + 4.0));
    const double z4 = (pow(s, 3.0 * m + 4.0) - C4) / (pow(m + 1.0, 3.0) * (3.0 * m + 4.0));
    *u = -C0 * (z1 - 3.0 * z2 + 3.0 * z3 - z4);
  } else {
    *u = 0.0;
  }
}

// periodic linearised shelf (exactTestsIJ.c:80-120)
void exact_j(double x, double y, double *H, double *u, double *v) {
  const double pi = 3.14159265358979, L = 300.0e3, H0 = 500.0, nu0 = 30.0 * 1.0e6 * 31556926.0;
  const double rho_ice = 910.0, rho_sw = 1028.0, g = 9.81;
  const double C = rho_ice * g * (1.0 - rho_ice / rho_sw) * H0 / (2.0 * nu0), A = L / (4.0 * pi);
  const double gam[3][3] = {{1.0854, 0.108, 0.0027}, {0.402, 0.04, 0.001}, {0.0402, 0.004, 0.0001}};
  *H = H0 * (1.0 + 0.4 * cos(pi * x / L)) * (1.0 + 0.1 * cos(pi * y / L));
  double uu = 0, vv = 0;
  for (int k = -2; k <= 2; ++k)
    for (int l = -2; l <= 2; ++l) {
      if (k == 0 && l == 0) continue;
      const double kx = k * pi * x / L, ly = l * pi * y / L;
      const double B = (A / (double)(k * k + l * l)) * (C * gam[abs(k)][abs(l)]) * (cos(kx) * sin(ly) + sin(kx) * cos(ly));
      uu += B * k;
      vv += B * l;
    }
  *u = uu;
  *v = vv;
}

// van der Veen shelf (ssa_test_cfbc.cc:44-54)
double vdv_thickness(double V0, double H0, double C, double x) { return pow(4 * C / (V0 * H0) * x + 1 / pow(H0, 4), -0.25); }

struct Case {
  Grid grid;
  pism_gpu_ssa_config cfg;
  Field2 mask, thickness, surface, bed, tauc, bc_mask, melange;
  Field2V bc_values, exact;
};

void init_fields(Case &c) {
  const int Mx = c.grid.Mx, My = c.grid.My;
  c.mask = Field2(Mx, My, 2.0);   // SSATestCase.cc:110
  c.thickness = Field2(Mx, My);
  c.surface = Field2(Mx, My);
  c.bed = Field2(Mx, My);
  c.tauc = Field2(Mx, My);
  c.bc_mask = Field2(Mx, My);
  c.melange = Field2(Mx, My);
  c.bc_values = Field2V(Mx, My);
  c.exact = Field2V(Mx, My);
}

// SSATestCaseI (ssa_testi.cc:71-145)
void build_i(Case &c, int Mx, int My) {
  const double L = 40e3, H0 = 0.05 * L, B = 3.7e8, Ly = 3 * L;
  const double Lx = std::max(60.0e3, ((Mx - 1) / 2) * (2.0 * Ly / (My - 1)));
  c.grid = Grid::Shallow(Lx, Ly, Mx, My, PISM_NOT_PERIODIC);
  c.cfg.do_pseudo_plastic_till = 0;
  c.cfg.flow_law = PISM_FLOW_LAW_ISOTHERMAL_GLEN;
  c.cfg.ice_softness = pow(B, -c.cfg.ssa_Glen_exponent);
  c.cfg.compute_surf_grad_inward_ssa = 1;
  c.cfg.epsilon_ssa = 0.0;
  init_fields(c);
  const double f = c.cfg.ice_density * c.cfg.standard_gravity * H0 * tan(atan(0.001));
  for (int i = 0; i < Mx; ++i)
    for (int j = 0; j < My; ++j) {
      const double x = c.grid.x(i), y = c.grid.y(j);
      double bed, tc, u, v;
      exact_i(10.0, x, y, &bed, &tc, &u, &v);
      c.thickness(i, j) = H0;
      c.tauc(i, j) = f * pow(fabs(y / L), 10.0);
      c.bed(i, j) = bed;
      c.surface(i, j) = bed + H0;
      c.exact.u(i, j) = u;
      c.exact.v(i, j) = v;
      if (j == 0 || j == My - 1 || i == 0 || i == Mx - 1) {
        c.bc_mask(i, j) = 1;
        c.bc_values.u(i, j) = u;
        c.bc_values.v(i, j) = v;
      }
    }
}

// SSATestCaseJ (ssa_testj.cc:64-134)
void build_j(Case &c, int Mx, int My) {
  c.grid = Grid::Shallow(300.0e3, 300.0e3, Mx, My, PISM_XY_PERIODIC);
  c.cfg.do_pseudo_plastic_till = 0;
  c.cfg.flow_law = PISM_FLOW_LAW_ISOTHERMAL_GLEN;
  const double nu0 = 30.0 * 1.0e6 * kSecPerYear, H0 = 500.0;
  const double nu_c = (nu0 * H0) / c.cfg.min_thickness_strength_extension_ssa;   // SSA.cc:41-58
  const double nuH_c = nu_c * c.cfg.min_thickness_strength_extension_ssa;
  c.cfg.min_thickness_strength_extension_ssa = 800.0;
  c.cfg.constant_nu_strength_extension_ssa = nuH_c / 800.0;
  init_fields(c);
  c.mask.set(3.0);
  for (int i = 0; i < Mx; ++i)
    for (int j = 0; j < My; ++j) {
      double H, u, v;
      exact_j(c.grid.x(i), c.grid.y(j), &H, &u, &v);
      c.thickness(i, j) = H;
      c.surface(i, j) = (1.0 - c.cfg.ice_density / c.cfg.sea_water_density) * H;
      c.exact.u(i, j) = u;
      c.exact.v(i, j) = v;
      if (i == Mx / 2 && j == My / 2) {
        c.bc_mask(i, j) = 1;
        c.bc_values.u(i, j) = u;
        c.bc_values.v(i, j) = v;
      }
    }
}

// SSATestCaseCFBC (ssa_test_cfbc.cc:92-170)
void build_v(Case &c, int Mx, int My) {
  c.grid = Grid::Shallow(250.0e3, 250.0e3, Mx, My, PISM_Y_PERIODIC);
  c.cfg.ice_softness = pow(1.9e8, -c.cfg.ssa_Glen_exponent);
  c.cfg.compute_surf_grad_inward_ssa = 0;
  c.cfg.calving_front_stress_boundary_condition = 1;
  c.cfg.flow_law = PISM_FLOW_LAW_ISOTHERMAL_GLEN;
  init_fields(c);
  c.bed.set(-1000.0);
  const double V0 = 300.0 / kSecPerYear, H0 = 600.0, C = 2.45e-18;
  for (int i = 0; i < Mx; ++i)
    for (int j = 0; j < My; ++j) {
      const double x = c.grid.x(i) + c.grid.Lx;
      if (i != Mx - 1) {
        c.thickness(i, j) = vdv_thickness(V0, H0, C, x);
        c.mask(i, j) = 3.0;
        c.exact.u(i, j) = V0 * H0 / vdv_thickness(V0, H0, C, x);
      } else {
        c.thickness(i, j) = 0.0;
        c.mask(i, j) = 4.0;
      }
      c.surface(i, j) = (1.0 - c.cfg.ice_density / c.cfg.sea_water_density) * c.thickness(i, j);
      if (i == 0) {
        c.bc_mask(i, j) = 1;
        c.bc_values.u(i, j) = V0;
      }
    }
}

// SSATestCase::report, SSATestCase.cc:173-253
void report(const Field2V &vel, const Field2V &exact) {
  const int Mx = vel.Mx, My = vel.My;
  double maxvec = 0, avvec = 0, avu = 0, avv = 0, maxu = 0, maxv = 0, exactmax = 0;
  for (int i = 0; i < Mx; ++i)
    for (int j = 0; j < My; ++j) {
      exactmax = std::max(exactmax, sqrt(exact.u(i, j) * exact.u(i, j) + exact.v(i, j) * exact.v(i, j)));
      const double ue = fabs(vel.u(i, j) - exact.u(i, j)), ve = fabs(vel.v(i, j) - exact.v(i, j));
      avu += ue;
      avv += ve;
      maxu = std::max(maxu, ue);
      maxv = std::max(maxv, ve);
      const double vec = sqrt(ue * ue + ve * ve);
      maxvec = std::max(maxvec, vec);
      avvec += vec;
    }
  const double N = (double)Mx * My;
  printf("NUMERICAL ERRORS in velocity relative to exact solution:\n");
  printf("velocity  :  maxvector   prcntavvec      maxu      maxv       avu       avv\n");
  printf("           %11.4f%13.5f%10.4f%10.4f%10.4f%10.4f\n", maxvec * kSecPerYear, (avvec / N / exactmax) * 100.0,
         maxu * kSecPerYear, maxv * kSecPerYear, avu / N * kSecPerYear, avv / N * kSecPerYear);
  printf("NUM ERRORS DONE\n");
}

}  // namespace

int main(int argc, char **argv) {
  std::string test = "I", pc = "mg", learned;
  int Mx = -1, My = -1;
  double ssa_rtol = -1, ksp_rtol = -1;
  for (int a = 1; a + 1 < argc; a += 2) {
    const std::string k = argv[a];
    if (k == "-test") test = argv[a + 1];
    else if (k == "-Mx") Mx = atoi(argv[a + 1]);
    else if (k == "-My") My = atoi(argv[a + 1]);
    else if (k == "-ssa_rtol") ssa_rtol = atof(argv[a + 1]);
    else if (k == "-ssafd_ksp_rtol") ksp_rtol = atof(argv[a + 1]);
    else if (k == "-pc") pc = argv[a + 1];
    else if (k == "-learned") learned = argv[a + 1];
    else {
      fprintf(stderr, "unknown option %s\n", k.c_str());
      return 2;
    }
  }
  Case c;
  pism_gpu_ssa_config_defaults(&c.cfg);
  if (test == "I") build_i(c, Mx > 0 ? Mx : 5, My > 0 ? My : 61);
  else if (test == "J") build_j(c, Mx > 0 ? Mx : 61, My > 0 ? My : 61);
  else if (test == "V") build_v(c, Mx > 0 ? Mx : 201, My > 0 ? My : 3);
  else {
    fprintf(stderr, "unknown test %s\n", test.c_str());
    return 2;
  }
  if (ssa_rtol > 0) c.cfg.ssafd_relative_convergence = ssa_rtol;
  if (ksp_rtol > 0) c.cfg.ksp_rtol = ksp_rtol;
  c.cfg.pc_type = pc == "bjacobi" ? PISM_PC_BLOCK_JACOBI : pc == "line" ? PISM_PC_LINE : PISM_PC_MULTIGRID;
  pism_gpu_unet *net = nullptr;
  if (!learned.empty()) {   // the warm-start network, parameters as raw FP32
    std::vector<float> params((size_t)pism_gpu_unet_param_count());
    FILE *fp = fopen(learned.c_str(), "rb");
    const size_t got = fp ? fread(params.data(), sizeof(float), params.size(), fp) : 0;
    if (fp) fclose(fp);
    const int hh = (c.grid.Mx + 7) / 8 * 8, ww = (c.grid.My + 7) / 8 * 8;
    if (got != params.size() || pism_gpu_unet_create(0, 1, hh, ww, &net) != PISM_GPU_SSA_OK ||
        pism_gpu_unet_set_params(net, params.data(), PISM_MEM_HOST) != PISM_GPU_SSA_OK) {
      fprintf(stderr, "cannot load the network parameters from %s\n", learned.c_str());
      return 2;
    }
  }
  try {
    SSA *ssa = SSAFD_GPUFactory(c.grid, c.cfg);   // testcase.init(Mx, My, ssafactory)
    if (net) static_cast<SSAFD_GPU *>(ssa)->set_warm_start(net, 1);
    Vars v;
    v.mask = &c.mask;
    v.thickness = &c.thickness;
    v.tauc = &c.tauc;
    v.surface = &c.surface;
    v.bed = &c.bed;
    ssa->set_variables(v);
    ssa->init();
    ssa->set_boundary_conditions(c.bc_mask, c.bc_values);
    ssa->update(false, c.melange);                  // testcase.run()
    fprintf(stderr, "  SSA: %s", ssa->stdout_report().c_str());
    report(ssa->velocity(), c.exact);               // testcase.report()
    delete ssa;
  } catch (const std::exception &e) {
    fprintf(stderr, "PISM ERROR: %s\n", e.what());
    pism_gpu_unet_destroy(net);
    return 1;
  }
  pism_gpu_unet_destroy(net);
  return 0;
}
