// ssa_fem.h — device state and launchers of the Q1 finite-element SSA (ssa_fem.cu); not
// part of the C-ABI.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ssa_internal.h"

namespace pism_gpu {

// Quadrature (FETools.cc:300-316): test-function values and derivatives at the four Gauss
// points [q][k] and the weighted Jacobian, for one grid spacing
struct FemGerms {
  double val[4][4], gx[4][4], gy[4][4], JxW[4];
};
FemGerms fem_germs(double dx, double dy);

// the coefficients at the quadrature points, [q * Ne + e]
struct FemCoef {
  double *H, *tauc, *tdu, *tdv, *B;
  int8_t *mask;
};

// the state of the conjugate-gradient solve of one Newton step
struct FemCG {
  double rz, pq, rr, bb, alpha, beta, rtol;
  int its, maxit, done;   // done: 1 converged, 2 breakdown (p.Ap <= 0), 3 iteration limit
};

// the scalars of a Newton step: ||F||^2, then ||lambda du||^2 and ||u + lambda du||^2
struct FemScalars {
  double f2, step2, x2;
};

struct FemState {
  int nex = 0, ney = 0, Ne = 0, N = 0;
  FemCoef C{};
  double *J = nullptr;                 // [36][N]: neighbour block (di+1)*3+(dj+1), row c, column d
  double4 *dinv = nullptr;             // inverse diagonal blocks
  double2 *F = nullptr, *Ft = nullptr, *du = nullptr, *trial = nullptr;
  double2 *vel0 = nullptr;             // the velocity before the solve, put back if it fails
  double2 *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;
  FemCG *cg = nullptr;
  FemScalars *sc = nullptr;
  int *zero_pivot = nullptr;
  cudaGraphExec_t cg_batch = nullptr;  // FEM_CG_BATCH CG iterations captured once (all buffers fixed)
  bool cg_batch_failed = false;
};
constexpr int FEM_CG_BATCH = 16;

struct FemProblem {
  int Mx, My, periodicity;
  pism_gpu_ssa_config c;
  FemGerms W;
  double scale;                        // Dirichlet scaling (-ssa_fe_dirichlet_scale)
  double notional_strength;            // the strength extension's nu H
};

int fem_allocate(FemState &S, int Mx, int My, int periodicity);
void fem_free(FemState &S);
void launch_fem_coefficients(const Launch &L, const FemProblem &P, const FemState &S, const double *H,
                             const double *bed, const double *tauc, const double *srf, const double *enthalpy,
                             const double *z, int Mz, double icefree_thickness, double is_floating_thickness);
// F(vel) into F (and, with the Jacobian, J and its inverse diagonal blocks); ||F||^2 into sc->f2
void launch_fem_residual(const Launch &L, const FemProblem &P, const FemState &S, const double2 *vel, double2 *F,
                         bool jacobian, const uint8_t *bc, const double2 *bcv);
// CG on J du = -F: init, then `n` iterations (each skipped once cg->done)
void launch_fem_cg_init(const Launch &L, const FemProblem &P, const FemState &S, double rtol, int maxit);
void launch_fem_cg_iterations(const Launch &L, const FemProblem &P, const FemState &S, int n);
// trial = vel + lambda du with ||lambda du||^2 and ||trial||^2 into sc
void launch_fem_trial(const Launch &L, const FemState &S, const double2 *vel, double lambda);

}  // namespace pism_gpu
