// ssa_stencil.cuh — the SSAFD stencil, matrix-free (shared by the Krylov and multigrid kernels).
#pragma once

#include "ssa_internal.h"

namespace pism_gpu {

// ---------------------------------------------------------------------------
// the SSAFD stencil (SSAFD::assemble_matrix, SSAFD.cc:540-796), matrix-free
// ---------------------------------------------------------------------------
struct StencilConst {
  double rdx2, rdy2, r2, r4, scaling;   // 1/dx^2, 1/dy^2, 1/(2 dx dy), 1/(4 dx dy), m_scaling
  double nu_bedrock;                    // nu_bedrock (used where F_NB_* flags are set)
  const double *H;                      // thickness, read only where F_NB_* flags are set
};

// staggered coefficients of row (i, j): c_w, c_e, c_s, c_n (SSAFD.cc:556-585)
__device__ __forceinline__ void row_coefficients(const GridDev &g, const StencilConst &s, int i, int j, uint32_t f,
                                                 const double2 *__restrict__ nuH, double &c_w, double &c_e,
                                                 double &c_s, double &c_n) {
  const int k = cell(g, i, j);
  const double2 nC = nuH[k];
  c_w = nuH[nbr(g, i, j, -1, 0)].x;
  c_e = nC.x;
  c_s = nuH[nbr(g, i, j, 0, -1)].y;
  c_n = nC.y;
  if (f & F_NB_ANY) {
    const double Hc = s.H[k], HE = s.H[nbr(g, i, j, 1, 0)];
    if (f & F_NB_W) c_w = s.nu_bedrock * 0.5 * (Hc + s.H[nbr(g, i, j, -1, 0)]);
    if (f & F_NB_E) c_e = s.nu_bedrock * 0.5 * (Hc + HE);
    if (f & F_NB_N) c_n = s.nu_bedrock * 0.5 * (Hc + s.H[nbr(g, i, j, 0, 1)]);
    if (f & F_NB_S) c_s = s.nu_bedrock * 0.5 * (Hc + HE);   // thickness(i+1, j), as SSAFD.cc:582
  }
}

// the 36 row coefficients of one cell; eq1 = u-row, eq2 = v-row; positions
// NW N NE / W C E / SW S SE
template <class T>
struct Row2T {
  T uNW, uN, uNE, uW, uC, uE, uSW, uS, uSE;
  T vNW, vN, vNE, vW, vC, vE, vSW, vS, vSE;
};
using Row2 = Row2T<double>;

// The two rows of one cell: T = double for the operator itself, T = float inside the
// multigrid preconditioner.  rdx2, rdy2, r2, r4 = 1/dx^2, 1/dy^2, 1/(2 dx dy), 1/(4 dx dy).
template <class T>
__device__ __forceinline__ void stencil_rows_t(T rdx2, T rdy2, T r2, T r4, uint32_t f, T c_w, T c_e, T c_s, T c_n,
                                               T bta, Row2T<T> &e1, Row2T<T> &e2) {
  const T one = T(1), zero = T(0);
  const T aMn = (f & F_aMn) ? one : zero, aPn = (f & F_aPn) ? one : zero, aMM = (f & F_aMM) ? one : zero,
          aPP = (f & F_aPP) ? one : zero, aMs = (f & F_aMs) ? one : zero, aPs = (f & F_aPs) ? one : zero;
  const T bPw = (f & F_bPw) ? one : zero, bPP = (f & F_bPP) ? one : zero, bPe = (f & F_bPe) ? one : zero,
          bMw = (f & F_bMw) ? one : zero, bMM = (f & F_bMM) ? one : zero, bMe = (f & F_bMe) ? one : zero;
  // products of a staggered coefficient with its weights (exact: weights are 0 or 1)
  const T w = c_w * aMM, e = c_e * aPP, sS = c_s * bMM, n = c_n * bPP;
  const T wPw = w * bPw, wMw = w * bMw, wPP = w * bPP, wMM = w * bMM;
  const T ePe = e * bPe, eMe = e * bMe, ePP = e * bPP, eMM = e * bMM;
  const T nMn = n * aMn, nPn = n * aPn, nPP = n * aPP, nMM = n * aMM;
  const T sMs = sS * aMs, sPs = sS * aPs, sPP = sS * aPP, sMM = sS * aMM;
  // first equation, u part
  e1.uNW = zero; e1.uN = -n * rdy2; e1.uNE = zero;
  e1.uW = -4 * w * rdx2;
  e1.uC = (n + sS) * rdy2 + (4 * e + 4 * w) * rdx2 + bta;
  e1.uE = -4 * e * rdx2;
  e1.uSW = zero; e1.uS = -sS * rdy2; e1.uSE = zero;
  // first equation, v part
  e1.vNW = wPw * r2 + nMn * r4;
  e1.vN = (nPn - nMn) * r4 + (wPP - ePP) * r2;
  e1.vNE = -ePe * r2 - nPn * r4;
  e1.vW = (wMw - wPw) * r2 + (nMM - sMM) * r4;
  e1.vC = (nPP - nMM - sPP + sMM) * r4 + (ePP - wPP - eMM + wMM) * r2;
  e1.vE = (ePe - eMe) * r2 + (sPP - nPP) * r4;
  e1.vSW = -wMw * r2 - sMs * r4;
  e1.vS = (sMs - sPs) * r4 + (eMM - wMM) * r2;
  e1.vSE = eMe * r2 + sPs * r4;
  // second equation, u part (cross terms with 1/d2 and 1/d4 swapped)
  e2.uNW = wPw * r4 + nMn * r2;
  e2.uN = (nPn - nMn) * r2 + (wPP - ePP) * r4;
  e2.uNE = -ePe * r4 - nPn * r2;
  e2.uW = (wMw - wPw) * r4 + (nMM - sMM) * r2;
  e2.uC = (nPP - nMM - sPP + sMM) * r2 + (ePP - wPP - eMM + wMM) * r4;
  e2.uE = (ePe - eMe) * r4 + (sPP - nPP) * r2;
  e2.uSW = -wMw * r4 - sMs * r2;
  e2.uS = (sMs - sPs) * r2 + (eMM - wMM) * r4;
  e2.uSE = eMe * r4 + sPs * r2;
  // second equation, v part
  e2.vNW = zero; e2.vN = -4 * n * rdy2; e2.vNE = zero;
  e2.vW = -w * rdx2;
  e2.vC = (4 * n + 4 * sS) * rdy2 + (e + w) * rdx2 + bta;
  e2.vE = -e * rdx2;
  e2.vSW = zero; e2.vS = -4 * sS * rdy2; e2.vSE = zero;
}

__device__ __forceinline__ void stencil_rows(const StencilConst &s, uint32_t f, double c_w, double c_e, double c_s,
                                             double c_n, double bta, Row2 &e1, Row2 &e2) {
  stencil_rows_t<double>(s.rdx2, s.rdy2, s.r2, s.r4, f, c_w, c_e, c_s, c_n, bta, e1, e2);
}

// y = the two rows applied to x, with x at the offset (di, dj) read through xr(di, dj)
template <class T, class V, class XR>
__device__ __forceinline__ V apply_rows_rel(const Row2T<T> &e1, const Row2T<T> &e2, const XR &xr) {
  const V xNW = xr(-1, 1), xN = xr(0, 1), xNE = xr(1, 1);
  const V xW = xr(-1, 0), xC = xr(0, 0), xE = xr(1, 0);
  const V xSW = xr(-1, -1), xS = xr(0, -1), xSE = xr(1, -1);
  T y1 = e1.uN * xN.x + e1.uW * xW.x + e1.uC * xC.x + e1.uE * xE.x + e1.uS * xS.x;
  y1 += e1.vNW * xNW.y + e1.vN * xN.y + e1.vNE * xNE.y + e1.vW * xW.y + e1.vC * xC.y + e1.vE * xE.y +
        e1.vSW * xSW.y + e1.vS * xS.y + e1.vSE * xSE.y;
  T y2 = e2.uNW * xNW.x + e2.uN * xN.x + e2.uNE * xNE.x + e2.uW * xW.x + e2.uC * xC.x + e2.uE * xE.x +
         e2.uSW * xSW.x + e2.uS * xS.x + e2.uSE * xSE.x;
  y2 += e2.vN * xN.y + e2.vW * xW.y + e2.vC * xC.y + e2.vE * xE.y + e2.vS * xS.y;
  V y;
  y.x = y1;
  y.y = y2;
  return y;
}

// y = A x for a regular row whose CFBC weights are all 1 (every cell without -cfbc): the
// rows of stencil_rows_t with the weights substituted, written in difference form
// (about 40 flops instead of forming 36 coefficients); xr(di, dj) reads x at the offset.
template <class T, class V, class XR>
__device__ __forceinline__ V apply_regular(T rdx2, T rdy2, T r2, T r4, T c_w, T c_e, T c_s, T c_n, T bta,
                                           const XR &xr) {
  const V xNW = xr(-1, 1), xN = xr(0, 1), xNE = xr(1, 1);
  const V xW = xr(-1, 0), xC = xr(0, 0), xE = xr(1, 0);
  const V xSW = xr(-1, -1), xS = xr(0, -1), xSE = xr(1, -1);
  // d/dy (c du/dy), d/dx (4 c du/dx) and the mixed terms of the first equation
  const T uy = c_n * (xC.x - xN.x) + c_s * (xC.x - xS.x);
  const T ux = c_e * (xC.x - xE.x) + c_w * (xC.x - xW.x);
  const T vA = c_w * (xNW.y + xN.y - xSW.y - xS.y) + c_e * (xSE.y + xS.y - xNE.y - xN.y);
  const T vB = c_n * (xNW.y - xNE.y + xW.y - xE.y) + c_s * (xSE.y - xSW.y - xW.y + xE.y);
  // and of the second equation
  const T vy = c_n * (xC.y - xN.y) + c_s * (xC.y - xS.y);
  const T vx = c_e * (xC.y - xE.y) + c_w * (xC.y - xW.y);
  const T uA = c_w * (xNW.x + xN.x - xSW.x - xS.x) + c_e * (xSE.x + xS.x - xNE.x - xN.x);
  const T uB = c_n * (xNW.x - xNE.x + xW.x - xE.x) + c_s * (xSE.x - xSW.x - xW.x + xE.x);
  V y;
  y.x = rdy2 * uy + 4 * rdx2 * ux + r2 * vA + r4 * vB + bta * xC.x;
  y.y = 4 * rdy2 * vy + rdx2 * vx + r4 * uA + r2 * uB + bta * xC.y;
  return y;
}

// Tiles of 32 (j) x 8 (i) cells with a one-cell halo, staged in shared memory.  Element
// [a][b] holds the value at (i0 - 1 + a, j0 - 1 + b), indices wrapped periodically (a true
// modulo: grids may be narrower than a tile).
constexpr int TILE_J = 32, TILE_I = 8, TILE_THREADS = TILE_J * TILE_I;
template <class T>
using HaloTile = T[TILE_I + 2][TILE_J + 2];

__device__ __forceinline__ int pmod(int a, int n) {
  // the halo indices of a tile are at most one period out of range except on grids narrower
  // than a tile: those take the integer remainder, the rest a compare and an add
  if (a >= 0 && a < n) return a;
  if (a < 0 && a >= -n) return a + n;
  if (a >= n && a < 2 * n) return a - n;
  a %= n;
  return a < 0 ? a + n : a;
}

// One load round: thread (ti, tj) loads its own cell; threads of rows 0-5 also load one
// halo element each (top / bottom rows, the two corner pairs, left / right columns).
template <class T, class LOAD>
__device__ __forceinline__ void load_halo_tile(HaloTile<T> &tile, int i0, int j0, int Mx, int My, const LOAD &load) {
  const int ti = threadIdx.x >> 5, tj = threadIdx.x & 31;
  const int i = i0 + ti, j = j0 + tj;
  const T own = load(i < Mx ? i : pmod(i, Mx), j < My ? j : pmod(j, My));
  T halo;
  int ha = -1, hb = 0;
  if (ti < 2) {                       // top (a = 0) / bottom (a = 9) row, b = 0..31
    ha = ti == 0 ? 0 : TILE_I + 1;
    hb = tj;
  } else if (ti < 4 && tj < 2) {      // the same rows, b = 32, 33
    ha = ti == 2 ? 0 : TILE_I + 1;
    hb = 32 + tj;
  } else if (ti < 6 && tj < TILE_I) { // left (b = 0) / right (b = 33) column, a = 1..8
    ha = tj + 1;
    hb = ti == 4 ? 0 : TILE_J + 1;
  }
  if (ha >= 0) halo = load(pmod(i0 - 1 + ha, Mx), pmod(j0 - 1 + hb, My));
  tile[ti + 1][tj + 1] = own;
  if (ha >= 0) tile[ha][hb] = halo;
}

// y(i, j) = sum over the 9 neighbours of the two rows applied to x, read through an
// accessor xa(i', j') (i', j' already wrapped)
template <class XA>
__device__ __forceinline__ double2 apply_rows(const GridDev &g, int i, int j, const Row2 &e1, const Row2 &e2,
                                              const XA &xa) {
  const int ip = wrap(i + 1, g.Mx), im = wrap(i - 1, g.Mx), jp = wrap(j + 1, g.My), jm = wrap(j - 1, g.My);
  const double2 xNW = xa(im, jp), xN = xa(i, jp), xNE = xa(ip, jp);
  const double2 xW = xa(im, j), xC = xa(i, j), xE = xa(ip, j);
  const double2 xSW = xa(im, jm), xS = xa(i, jm), xSE = xa(ip, jm);
  double y1 = e1.uN * xN.x + e1.uW * xW.x + e1.uC * xC.x + e1.uE * xE.x + e1.uS * xS.x;
  y1 += e1.vNW * xNW.y + e1.vN * xN.y + e1.vNE * xNE.y + e1.vW * xW.y + e1.vC * xC.y + e1.vE * xE.y +
        e1.vSW * xSW.y + e1.vS * xS.y + e1.vSE * xSE.y;
  double y2 = e2.uNW * xNW.x + e2.uN * xN.x + e2.uNE * xNE.x + e2.uW * xW.x + e2.uC * xC.x + e2.uE * xE.x +
              e2.uSW * xSW.x + e2.uS * xS.x + e2.uSE * xSE.x;
  y2 += e2.vN * xN.y + e2.vW * xW.y + e2.vC * xC.y + e2.vE * xE.y + e2.vS * xS.y;
  return make_double2(y1, y2);
}

// the rows of cell (i, j); false for a diagonal-only (Dirichlet / CFBC ice-free) row
__device__ __forceinline__ bool cell_rows(const GridDev &g, const StencilConst &s, int i, int j, uint32_t f,
                                          const double2 *__restrict__ nuH, const double *__restrict__ beta,
                                          Row2 &e1, Row2 &e2) {
  if (f & F_DIAG_ONLY) return false;
  double c_w, c_e, c_s, c_n;
  row_coefficients(g, s, i, j, f, nuH, c_w, c_e, c_s, c_n);
  stencil_rows(s, f, c_w, c_e, c_s, c_n, beta[cell(g, i, j)], e1, e2);
  return true;
}

// y(i, j) = (A x)(i, j)
__device__ __forceinline__ double2 apply_cell(const GridDev &g, const StencilConst &s, int i, int j, uint32_t f,
                                              const double2 *__restrict__ nuH, const double *__restrict__ beta,
                                              const double2 *__restrict__ x) {
  const int k = cell(g, i, j);
  if (f & F_DIAG_ONLY) {
    const double2 xc = x[k];
    return make_double2(s.scaling * xc.x, s.scaling * xc.y);
  }
  const int ip = wrap(i + 1, g.Mx), im = wrap(i - 1, g.Mx), jp = wrap(j + 1, g.My), jm = wrap(j - 1, g.My);
  const int rC = i * g.My, rE = ip * g.My, rW = im * g.My;
  double c_w, c_e, c_s, c_n;
  row_coefficients(g, s, i, j, f, nuH, c_w, c_e, c_s, c_n);
  Row2 e1, e2;
  stencil_rows(s, f, c_w, c_e, c_s, c_n, beta[k], e1, e2);
  const double2 xNW = x[rW + jp], xN = x[rC + jp], xNE = x[rE + jp];
  const double2 xW = x[rW + j], xC = x[k], xE = x[rE + j];
  const double2 xSW = x[rW + jm], xS = x[rC + jm], xSE = x[rE + jm];
  double y1 = e1.uN * xN.x + e1.uW * xW.x + e1.uC * xC.x + e1.uE * xE.x + e1.uS * xS.x;
  y1 += e1.vNW * xNW.y + e1.vN * xN.y + e1.vNE * xNE.y + e1.vW * xW.y + e1.vC * xC.y + e1.vE * xE.y +
        e1.vSW * xSW.y + e1.vS * xS.y + e1.vSE * xSE.y;
  double y2 = e2.uNW * xNW.x + e2.uN * xN.x + e2.uNE * xNE.x + e2.uW * xW.x + e2.uC * xC.x + e2.uE * xE.x +
              e2.uSW * xSW.x + e2.uS * xS.x + e2.uSE * xSE.x;
  y2 += e2.vN * xN.y + e2.vW * xW.y + e2.vC * xC.y + e2.vE * xE.y + e2.vS * xS.y;
  return make_double2(y1, y2);
}

__device__ __forceinline__ double2 dmul(const double4 &m, const double2 &v) {
  return make_double2(m.x * v.x + m.y * v.y, m.z * v.x + m.w * v.y);
}
__device__ __forceinline__ double dot2(const double2 &a, const double2 &b) { return a.x * b.x + a.y * b.y; }

inline StencilConst stencil_const(const GridDev &g, const Fields &f) {
  StencilConst s;
  s.nu_bedrock = f.nu_bedrock;
  s.H = f.H;
  s.rdx2 = 1.0 / (g.dx * g.dx);
  s.rdy2 = 1.0 / (g.dy * g.dy);
  s.r2 = 1.0 / (2 * g.dx * g.dy);
  s.r4 = 1.0 / (4 * g.dx * g.dy);
  s.scaling = 1.0e9;
  return s;
}

}  // namespace pism_gpu
