// ssa_capi.cu — the C-ABI of the B200 SSAFD solver (include/pism_ssa_gpu.h) and its
// host-side driver: the Picard loop and the strategy ladder of SSAFD::solve
// (src/base/stressbalance/ssa/SSAFD.cc:869-1155), driving the kernels of
// ssa_kernels.cu on one CUDA stream.  Host <-> device traffic per Picard
// iteration is one small read-back (the Krylov state and the two nu*H norms).
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pism_unet_gpu.h"
#include "ssa_internal.h"
#include "ssa_fem.h"
#include "unet_internal.h"

using namespace pism_gpu;

struct pism_gpu_ssa {
  pism_gpu_grid grid{};
  std::vector<double> z_host;
  pism_gpu_ssa_config cfg{};
  int device = 0;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  GridDev g{};
  int N = 0;
  Launch L{};
  // inputs
  double *H = nullptr, *srf = nullptr, *bed = nullptr, *tauc = nullptr, *melange = nullptr, *gl_mask = nullptr;
  double *enthalpy = nullptr, *fracture = nullptr, *z_dev = nullptr, *stage = nullptr, *stage2 = nullptr;
  int8_t *mask = nullptr;
  uint8_t *bc = nullptr;
  double2 *bcv = nullptr;
  // derived / state
  double2 *taud = nullptr, *rhs = nullptr, *hardness = nullptr, *nuH = nullptr, *vel = nullptr, *vel_old = nullptr;
  double *beta = nullptr, *bfrict = nullptr;
  double *sb3d = nullptr;   // host-destination staging of pism_gpu_ssa_stress_balance_3d
  double *mc = nullptr;     // staging of pism_gpu_ssa_mass_continuity_step: 7 fields and 8 totals
  double *ec = nullptr;     // staging of the strain rates and eigen-calving: 5 fields and 8 scalars
  int8_t *ec_mask = nullptr;   // eigen-calving's mask before and during remove_narrow_tongues
  FemState fem{};              // the finite-element solve's state, allocated by its first call
  uint32_t *flags = nullptr;
  Krylov K{};
  Krylov32 K32{};
  Gmres G{};   // allocated by the first GMRES solve
  LinePC line{};   // allocated by the first set-up of the line preconditioner
  // captured Krylov iterations (GRAPH_ITERS per graph), one per kind of iteration
  struct IterGraph {
    cudaGraphExec_t exec = nullptr;
    const void *x = nullptr;   // the solution vector the iterations update
    long long kernels = 0;
    bool failed = false;
  } graphs[4];
  // graph-resident Krylov loops (a conditional WHILE node around one iteration)
  struct LoopGraph {
    cudaGraphExec_t exec = nullptr;
    const void *x = nullptr;
    long long per_iteration = 0;   // kernels of one iteration
    int body_iters = 1;            // iterations per pass of the loop body
    bool failed = false;
  } loops[4];
  // the whole Picard loop as one graph (graphs = 3), with the kernels per pass of each of its
  // loops (for the launch count)
  struct SolveGraph {
    cudaGraphExec_t exec = nullptr;
    double reg = 0.0, underrelax = 0.0;
    Fields key{};
    bool mixed = false;
    long long pre = 0, per_picard = 0, per_refine = 0, per_inner = 0, per_go = 0, per_test = 0, per_rebuild = 0;
    bool failed = false;
  } sgraph;
  PState *pstate = nullptr;
  PState *pstate_host = nullptr;
  double *res_dev = nullptr;   // {||r||^2, ||b||^2} of the refinement
  double *res_host = nullptr;
  MGHierarchy mg{};
  double *partials = nullptr;
  unsigned *ticket = nullptr;
  double *norm_dev = nullptr;
  int *zd_dev = nullptr;
  // pinned host mirrors
  KState *st_host = nullptr;
  double *norm_host = nullptr;
  int *zd_host = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool inputs_set = false, have_melange = false, have_gl = false, have_enthalpy = false, have_hardness = false,
       have_fracture = false, prepared = false;
  int default_pc_failure_count = 0;   // SSAFD.cc:252-253 (m_default_pc_failure_*)
  int use_fallback = 0;
  int last_ksp_its = 0;
  // the learned initial guess: feature image and network output
  float *lfeat = nullptr, *lout = nullptr;
  size_t lcap = 0;   // pixels allocated
  // the learned preconditioner correction inside FGMRES (pism_gpu_ssa_set_learned_pc)
  struct LearnedPC {
    pism_gpu_unet *net = nullptr;
    int stride = 1, height = 0, width = 0;
    float *img = nullptr, *out = nullptr;
    double2 *r = nullptr, *d = nullptr, *ad = nullptr;
    double *part = nullptr, *rho = nullptr, *gamma = nullptr;
  } lpc;
  std::string err;
  pism_gpu_ssa_stats stats{};
};

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

int fail(pism_gpu_ssa *h, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (h) h->err = buf;
  return code;
}

#define CK(h, call)                                                                                  \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return fail((h), e_ == cudaErrorMemoryAllocation ? PISM_GPU_SSA_ENOMEM : PISM_GPU_SSA_ECUDA,   \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);       \
  } while (0)

#define RET(x)                      \
  do {                              \
    int r_ = (x);                   \
    if (r_ != PISM_GPU_SSA_OK) return r_; \
  } while (0)

template <class T>
int dalloc(pism_gpu_ssa *h, T **p, size_t count) {
  CK(h, cudaMalloc((void **)p, std::max<size_t>(count, 1) * sizeof(T)));
  return PISM_GPU_SSA_OK;
}

Fields fields_of(pism_gpu_ssa *h) {
  Fields f;
  f.H = h->H; f.srf = h->srf; f.bed = h->bed; f.tauc = h->tauc;
  f.melange = h->have_melange ? h->melange : nullptr;
  f.gl_mask = h->gl_mask;
  f.enthalpy = h->have_enthalpy ? h->enthalpy : nullptr;
  f.fracture = h->have_fracture ? h->fracture : nullptr;
  f.bcv = h->bcv; f.mask = h->mask; f.bc = h->bc;
  f.taud = h->taud; f.rhs = h->rhs; f.hardness = h->hardness; f.nuH = h->nuH; f.vel = h->vel;
  f.beta = h->beta; f.flags = h->flags;
  f.nu_bedrock = h->cfg.nu_bedrock;
  return f;
}

// The preconditioner in use.  A KSP failure switches multigrid to block Jacobi and block
// Jacobi or the line solve to multigrid (the reference switches BJacobi -> ASM,
// SSAFD.cc:929-958); grids too small for a coarse level use block Jacobi.
int active_pc(pism_gpu_ssa *h) {
  int pc = h->cfg.pc_type;
  if (h->use_fallback) pc = pc == PISM_PC_MULTIGRID ? PISM_PC_BLOCK_JACOBI : PISM_PC_MULTIGRID;
  if (pc == PISM_PC_MULTIGRID && h->mg.nlev == 0) pc = PISM_PC_BLOCK_JACOBI;
  return pc;
}
const MGHierarchy *active_mg(pism_gpu_ssa *h) { return active_pc(h) == PISM_PC_MULTIGRID ? &h->mg : nullptr; }
const LinePC *active_line(pism_gpu_ssa *h) { return active_pc(h) == PISM_PC_LINE ? &h->line : nullptr; }

// preconditioner set-up after nu*H / beta changed (replaces PCSetUp); the multigrid coarse
// levels only when rebuild_coarse (lagged coarse levels, mg_rebuild_rtol)
int pc_setup(pism_gpu_ssa *h, bool rebuild_coarse = true) {
  Fields f = fields_of(h);
  *h->zd_host = INT_MAX;
  CK(h, cudaMemcpyAsync(h->zd_dev, h->zd_host, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  launch_diag_setup(h->L, h->g, f, h->K.dinv, h->zd_dev);
  h->mg.omega = (float)h->cfg.mg_omega;
  h->mg.correction = (float)h->cfg.mg_correction;
  h->mg.post_blocks = h->cfg.mg_post_blocks_per_sm > 0 ? h->L.max_blocks / 4 * h->cfg.mg_post_blocks_per_sm : 0;
  h->mg.small_kernel = h->cfg.mg_small_kernel;
  h->mg.apply_kernel = h->cfg.mixed_apply_kernel;
  if (active_mg(h)) {
    mg_setup_fine(h->L, h->g, f, h->K.dinv, h->mg);
    if (rebuild_coarse) {
      mg_setup_coarse(h->L, h->g, f, h->mg);
      h->stats.mg_rebuilds += 1;
    }
  }
  if (active_line(h)) {
    if (!h->line.P) {
      RET(dalloc(h, &h->line.P, h->N));
      RET(dalloc(h, &h->line.F, h->N));
      RET(dalloc(h, &h->line.G, h->N));
    }
    line_setup(h->L, h->g, f, h->K.dinv, h->line);
  }
  CK(h, cudaGetLastError());
  return PISM_GPU_SSA_OK;
}

int check_config(pism_gpu_ssa *h, const pism_gpu_ssa_config *c) {
  if (!c) return fail(h, PISM_GPU_SSA_EINVAL, "config is NULL");
  if (c->flow_law < PISM_FLOW_LAW_ISOTHERMAL_GLEN || c->flow_law > PISM_FLOW_LAW_HOOKE)
    return fail(h, PISM_GPU_SSA_EINVAL, "unknown flow law %d", c->flow_law);
  if (c->ksp_type != PISM_KSP_BICGSTAB && c->ksp_type != PISM_KSP_GMRES)
    return fail(h, PISM_GPU_SSA_EINVAL, "unknown ksp_type %d", c->ksp_type);
  if (c->precision != PISM_PRECISION_FP64 && c->precision != PISM_PRECISION_MIXED)
    return fail(h, PISM_GPU_SSA_EINVAL, "unknown precision %d", c->precision);
  if (c->precision == PISM_PRECISION_MIXED && !(c->mixed_inner_rtol > 0.0 && c->mixed_inner_rtol < 1.0))
    return fail(h, PISM_GPU_SSA_EINVAL, "mixed_inner_rtol must be in (0, 1)");
  if (c->ksp_type == PISM_KSP_GMRES && (c->gmres_restart < 1 || c->gmres_restart > GM_MAXM))
    return fail(h, PISM_GPU_SSA_EINVAL, "gmres_restart must be in [1, %d]", GM_MAXM);
  if (c->ksp_type == PISM_KSP_GMRES && c->precision == PISM_PRECISION_MIXED)
    return fail(h, PISM_GPU_SSA_EINVAL, "the mixed-precision inner solve is BiCGStab; use ksp_type GMRES with fp64");
  if (c->pc_type != PISM_PC_BLOCK_JACOBI && c->pc_type != PISM_PC_MULTIGRID && c->pc_type != PISM_PC_LINE)
    return fail(h, PISM_GPU_SSA_EINVAL, "unknown pc_type %d", c->pc_type);
  if (c->ksp_rtol_adaptive && !(c->ksp_rtol_max >= c->ksp_rtol && c->ksp_rtol_max < 1.0 && c->ksp_rtol_factor > 0.0))
    return fail(h, PISM_GPU_SSA_EINVAL, "adaptive KSP tolerance needs ksp_rtol <= ksp_rtol_max < 1, ksp_rtol_factor > 0");
  if (c->graphs < 0 || c->graphs > 3) return fail(h, PISM_GPU_SSA_EINVAL, "graphs must be 0, 1, 2 or 3");
  if (c->mg_post_blocks_per_sm < 0 || c->mg_post_blocks_per_sm > 4)
    return fail(h, PISM_GPU_SSA_EINVAL, "mg_post_blocks_per_sm must be in [0, 4]");
  if (c->mg_small_kernel < 0 || c->mg_small_kernel > 2)
    return fail(h, PISM_GPU_SSA_EINVAL, "mg_small_kernel must be 0, 1 or 2");
  if (c->mixed_apply_kernel < 0 || c->mixed_apply_kernel > 2)
    return fail(h, PISM_GPU_SSA_EINVAL, "mixed_apply_kernel must be 0, 1 or 2");
  if (!(c->mg_rebuild_rtol >= 0.0)) return fail(h, PISM_GPU_SSA_EINVAL, "mg_rebuild_rtol must be >= 0");
  if (!(c->ksp_rtol > 0.0) || c->ksp_max_it < 1 || c->max_iterations_ssafd < 1)
    return fail(h, PISM_GPU_SSA_EINVAL, "ksp_rtol, ksp_max_it and max_iterations_ssafd must be positive");
  if (!(c->ssa_Glen_exponent > 0.0) || !(c->min_thickness_strength_extension_ssa > 0.0))
    return fail(h, PISM_GPU_SSA_EINVAL, "Glen exponent and strength-extension thickness must be positive");
  return PISM_GPU_SSA_OK;
}

// Launch `count` Krylov iterations.  Every iteration is the same fixed sequence of kernels
// whose scalars live on the device, so GRAPH_ITERS of them are captured once into a CUDA
// graph and replayed (fewer launches, shorter gaps between dependent kernels); a stream
// that cannot be captured (the legacy default stream) keeps the direct launches.
constexpr int GRAPH_ITERS = 4;
enum { GRAPH_BICG_MG = 0, GRAPH_BICG_JACOBI = 1, GRAPH_MIXED = 2, GRAPH_BICG_LINE = 3 };

template <class ONE>
int run_iterations(pism_gpu_ssa *h, int kind, const void *x, int count, const ONE &one) {
  auto &G = h->graphs[kind];
  if (G.exec && G.x != x) {
    cudaGraphExecDestroy(G.exec);
    G = {};
  }
  if (h->cfg.graphs >= 1 && !G.exec && !G.failed) {
    const long long before = h->stats.kernel_launches;
    cudaGraph_t graph = nullptr;
    bool ok = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      for (int q = 0; q < GRAPH_ITERS; ++q) one();
      ok = cudaStreamEndCapture(h->stream, &graph) == cudaSuccess && graph != nullptr;
    }
    if (ok) ok = cudaGraphInstantiate(&G.exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (ok) {
      G.x = x;
      G.kernels = h->stats.kernel_launches - before;
    } else {
      G.exec = nullptr;
      G.failed = true;
      cudaGetLastError();   // clear the capture's error; the direct launches follow
    }
    h->stats.kernel_launches = before;   // nothing ran during the capture
  }
  int q = 0;
  if (G.exec && h->cfg.graphs >= 1)
    for (; q + GRAPH_ITERS <= count; q += GRAPH_ITERS) {
      CK(h, cudaGraphLaunch(G.exec, h->stream));
      h->stats.kernel_launches += G.kernels;
    }
  for (; q < count; ++q) one();
  return PISM_GPU_SSA_OK;
}

// A Krylov solve as one graph: a kernel sets a conditional handle from st->done, and a
// WHILE node runs the loop body (one or a few iterations) plus that kernel again until the
// solve is done, so the whole solve is one graph launch and one read-back.  Iterations of a
// pass that start after convergence return at once.  Built once per handle and kind.
template <class ONE>
bool build_loop(pism_gpu_ssa *h, pism_gpu_ssa::LoopGraph &G, const KState *st, const ONE &one) {
  const cudaStream_t s = h->stream;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  bool ok = true;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaGraph_t cg = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  cudaGraphConditionalHandle cond{};
  ok = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd) == cudaSuccess && cs == cudaStreamCaptureStatusActive;
  if (ok) ok = cudaGraphConditionalHandleCreate(&cond, cg, 0, 0) == cudaSuccess;
  if (ok) {
    launch_loop_condition(h->L, cond, st);
    ok = cudaGetLastError() == cudaSuccess;
  }
  if (ok) ok = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd) == cudaSuccess;
  cudaGraphNode_t node{};
  cudaGraphNodeParams p{};
  if (ok) {
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = cond;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    ok = cudaGraphAddNode(&node, cg, deps, nd, &p) == cudaSuccess;
  }
  cudaStream_t bs = nullptr;
  if (ok) ok = cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking) == cudaSuccess;
  if (ok) ok = cudaStreamBeginCaptureToGraph(bs, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    h->L.stream = bs;
    one();
    launch_loop_condition(h->L, cond, st);
    h->L.stream = s;
    const bool launched = cudaGetLastError() == cudaSuccess;
    ok = cudaStreamEndCapture(bs, nullptr) == cudaSuccess && launched;
  }
  if (ok) ok = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies) == cudaSuccess;
  cudaGraph_t out = nullptr;
  const bool ended = cudaStreamEndCapture(s, &out) == cudaSuccess;
  ok = ok && ended && out != nullptr;
  if (ok) ok = cudaGraphInstantiate(&G.exec, out, 0) == cudaSuccess;
  if (out) cudaGraphDestroy(out);
  if (bs) cudaStreamDestroy(bs);
  if (!ok) {
    G.exec = nullptr;
    cudaGetLastError();
  }
  return ok;
}

// Run Krylov iterations until st->done: the graph-resident loop, or (where the loop graph
// cannot be built) chunks of iterations with a read-back before each chunk.  Leaves the
// final state in h->st_host.
template <class ONE>
int run_until_done(pism_gpu_ssa *h, int kind, const void *x, KState *st, int chunk0, int body_iters,
                   const ONE &one) {
  auto &G = h->loops[kind];
  if (G.exec && G.x != x) {
    cudaGraphExecDestroy(G.exec);
    G = {};
  }
  if (h->cfg.graphs >= 2 && !G.exec && !G.failed) {
    const long long before = h->stats.kernel_launches;
    long long per = 0;
    G.failed = !build_loop(h, G, st, [&] {
      const long long b0 = h->stats.kernel_launches;
      for (int q = 0; q < body_iters; ++q) one();
      per = (h->stats.kernel_launches - b0) / body_iters;
    });
    G.x = x;
    G.per_iteration = per;
    G.body_iters = body_iters;
    h->stats.kernel_launches = before;   // nothing ran during the capture
  }
  if (G.exec && h->cfg.graphs >= 2) {
    CK(h, cudaGraphLaunch(G.exec, h->stream));
    CK(h, cudaMemcpyAsync(h->st_host, st, sizeof(KState), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    const long long passes = (h->st_host->iter + G.body_iters - 1) / G.body_iters;
    h->stats.kernel_launches += 1 + passes * (G.body_iters * G.per_iteration + 1);
    return PISM_GPU_SSA_OK;
  }
  // graphs == 0 (kernel profiling): one read-back per iteration, so that no iteration is
  // launched after convergence; otherwise growing chunks
  int launched = 0, chunk = h->cfg.graphs == 0 ? 1 : chunk0;
  while (true) {
    CK(h, cudaMemcpyAsync(h->st_host, st, sizeof(KState), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    if (h->st_host->done) break;
    RET(run_iterations(h, kind, x, chunk, one));
    CK(h, cudaGetLastError());
    launched += chunk;
    if (h->cfg.graphs != 0) chunk = std::max(4, std::min(64, launched / 8));
  }
  return PISM_GPU_SSA_OK;
}

// Inside an active capture on h->L.stream: add a conditional node (WHILE or IF) after the
// capture's current dependencies.  `set(cond)` launches the kernel that gives the node its
// value, once before the node and, for a WHILE node, again at the end of each pass of the
// body; `body()` launches the body on h->L.stream (itself capturing into the node's body
// graph, so bodies nest).  *body_kernels gets the kernels of one pass, nested bodies
// included.  The capture continues after the node.
template <class SET, class BODY>
bool add_conditional(pism_gpu_ssa *h, cudaGraphConditionalNodeType type, const SET &set, const BODY &body,
                     long long *body_kernels) {
  const cudaStream_t s = h->L.stream;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaGraph_t cg = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  if (cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd) != cudaSuccess || cs != cudaStreamCaptureStatusActive)
    return false;
  cudaGraphConditionalHandle cond{};
  if (cudaGraphConditionalHandleCreate(&cond, cg, 0, 0) != cudaSuccess) return false;
  set(cond);
  if (cudaGetLastError() != cudaSuccess) return false;
  if (cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd) != cudaSuccess) return false;
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = cond;
  p.conditional.type = type;
  p.conditional.size = 1;
  cudaGraphNode_t node{};
  if (cudaGraphAddNode(&node, cg, deps, nd, &p) != cudaSuccess) return false;
  cudaStream_t bs = nullptr;
  if (cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking) != cudaSuccess) return false;
  bool ok = cudaStreamBeginCaptureToGraph(bs, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    const long long b0 = h->stats.kernel_launches;
    h->L.stream = bs;
    ok = body();
    if (type == cudaGraphCondTypeWhile) set(cond);
    h->L.stream = s;
    *body_kernels = h->stats.kernel_launches - b0;
    ok = cudaGetLastError() == cudaSuccess && ok;
    ok = cudaStreamEndCapture(bs, nullptr) == cudaSuccess && ok;
  }
  cudaStreamDestroy(bs);
  return ok && cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies) == cudaSuccess;
}

// ---- the whole Picard loop as one CUDA graph (graphs = 3) ----
// SSAFD::picard_manager with its linear solves, nu*H updates and stopping test in one graph
// launch and one read-back: a WHILE node over Picard iterations (its decisions taken on the
// device by ssa_control.cu), inside it the linear solve — FP64 BiCGStab as a WHILE node of
// four iterations per pass, or the mixed-precision refinement as a WHILE node over
// refinement steps around the inner FP32 BiCGStab's WHILE node and an IF node for the
// correction — and an IF node for the nu*H update and Picard test after a successful solve.
// Used for BiCGStab without a fallback preconditioner and verbosity <= 2; everything else
// (and a stream that cannot be captured) takes the host loop.
bool solve_graph_eligible(const pism_gpu_ssa *h) {
  return h->cfg.graphs >= 3 && !h->use_fallback && h->cfg.verbosity <= 2 && h->cfg.ksp_type == PISM_KSP_BICGSTAB;
}

int build_solve_graph(pism_gpu_ssa *h, double reg, double underrelax, bool *built) {
  auto &S = h->sgraph;
  *built = false;
  if (S.exec) cudaGraphExecDestroy(S.exec);
  S = {};
  const pism_gpu_ssa_config &c = h->cfg;
  const GridDev &g = h->g;
  const Fields f = fields_of(h);
  const MGHierarchy *mg = active_mg(h);
  const LinePC *line = active_line(h);
  const bool mixed = c.precision == PISM_PRECISION_MIXED && mg;
  const int N = g.Mx * g.My;
  if (!h->pstate) RET(dalloc(h, &h->pstate, 1));
  if (!h->pstate_host) CK(h, cudaMallocHost((void **)&h->pstate_host, sizeof(PState)));
  if (line && !h->line.P) {
    RET(dalloc(h, &h->line.P, h->N));
    RET(dalloc(h, &h->line.F, h->N));
    RET(dalloc(h, &h->line.G, h->N));
  }
  h->mg.omega = (float)c.mg_omega;   // captured by value, as pc_setup sets them
  h->mg.correction = (float)c.mg_correction;
  h->mg.post_blocks = c.mg_post_blocks_per_sm > 0 ? h->L.max_blocks / 4 * c.mg_post_blocks_per_sm : 0;
  h->mg.small_kernel = c.mg_small_kernel;
  h->mg.apply_kernel = c.mixed_apply_kernel;
  PicardConst pc{c.ksp_rtol, c.ksp_rtol_max, c.ksp_rtol_factor, c.ssafd_relative_convergence,
                 c.ksp_rtol_adaptive ? 1 : 0, c.max_iterations_ssafd, c.mg_rebuild_rtol};
  PState *P = h->pstate;
  const long long t0 = h->stats.kernel_launches;
  long long inc_picard = 0, inc_refine = 0, inc_inner = 0, inc_go = 0, inc_test = 0, inc_rebuild = 0, pre = 0;
  const bool lagged = mg && c.mg_rebuild_rtol > 0.0;
  // a second capture stream for the per-Picard set-up that the coarse-level builds do not read
  struct SideBranch {
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    ~SideBranch() {
      if (fork) cudaEventDestroy(fork);
      if (join) cudaEventDestroy(join);
      if (stream) cudaStreamDestroy(stream);
    }
  } side;
  bool split = mixed && !lagged && !line;
  if (split && (cudaStreamCreateWithFlags(&side.stream, cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&side.fork, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&side.join, cudaEventDisableTiming) != cudaSuccess)) {
    cudaGetLastError();
    split = false;
  }
  if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    S.failed = true;
    return PISM_GPU_SSA_OK;
  }
  launch_nuH(h->L, g, c, f, reg, 1.0, false, h->norm_dev);
  launch_picard_start(h->L, P);
  auto not_done = [&](const int *flag) {
    return [&h, flag](cudaGraphConditionalHandle cond) { launch_flag_condition(h->L, cond, flag, true); };
  };
  const long long before_loop = h->stats.kernel_launches;
  bool ok = add_conditional(h, cudaGraphCondTypeWhile, not_done(&P->done), [&] {
    bool inner_ok = true, rebuild_ok = true;
    launch_picard_begin(h->L, P, pc, h->zd_dev);
    bool residual_queued = false;
    if (split) {
      // The set-up in two branches of the graph. On the loop's stream: the coarse-level
      // Galerkin builds and the coarsest inverse, which read nu*H, beta and the masks only.
      // Beside them: the FP64 diagonal blocks, the FP32 fine-level copies and the first
      // refinement residual. The small levels' builds run on one cluster and the inverse on
      // one block, so most SMs are free for the second branch. Same kernels, same inputs:
      // the results are those of the serial order.
      cudaEventRecord(side.fork, h->L.stream);
      cudaStreamWaitEvent(side.stream, side.fork, 0);
      Launch Ls = h->L;
      Ls.stream = side.stream;
      launch_diag_setup(Ls, g, f, h->K.dinv, h->zd_dev);
      mg_setup_fine(Ls, g, f, h->K.dinv, h->mg);
      launch_residual32(Ls, g, f, h->rhs, h->vel, h->K32.rhs, h->res_dev);
      cudaEventRecord(side.join, side.stream);
      mg_setup_coarse(h->L, g, f, h->mg);
      cudaStreamWaitEvent(h->L.stream, side.join, 0);
      residual_queued = true;
    } else if (lagged) {
      launch_diag_setup(h->L, g, f, h->K.dinv, h->zd_dev);
      mg_setup_fine(h->L, g, f, h->K.dinv, h->mg);
      rebuild_ok = add_conditional(
          h, cudaGraphCondTypeIf,
          [&](cudaGraphConditionalHandle cond) { launch_flag_condition(h->L, cond, &P->rebuild, false); },
          [&] {
            mg_setup_coarse(h->L, g, f, h->mg);
            return true;
          },
          &inc_rebuild);
    } else {
      launch_diag_setup(h->L, g, f, h->K.dinv, h->zd_dev);
      if (mg) mg_setup(h->L, g, f, h->K.dinv, h->mg);
    }
    if (line) line_setup(h->L, g, f, h->K.dinv, h->line);
    if (mixed) {
      if (!residual_queued) launch_residual32(h->L, g, f, h->rhs, h->vel, h->K32.rhs, h->res_dev);
      inner_ok = add_conditional(h, cudaGraphCondTypeWhile, not_done(&P->refine_done), [&] {
        launch_mixed_init_dev(h->L, N, h->K32, h->res_dev, &P->rtol, c.mixed_inner_rtol, c.ksp_max_it);
        bool ok2 = add_conditional(
            h, cudaGraphCondTypeWhile,
            [&](cudaGraphConditionalHandle cond) { launch_loop_condition(h->L, cond, h->K32.st); },
            [&] {
              launch_mixed_iteration(h->L, g, f, *mg, h->K32);
              return true;
            },
            &inc_inner);
        launch_refine_end(h->L, P, h->K32.st, 60);
        ok2 = ok2 && add_conditional(
                         h, cudaGraphCondTypeIf,
                         [&](cudaGraphConditionalHandle cond) { launch_flag_condition(h->L, cond, &P->go, false); },
                         [&] {
                           launch_axpy32(h->L, N, h->K32.d, h->vel);
                           launch_residual32(h->L, g, f, h->rhs, h->vel, h->K32.rhs, h->res_dev);
                           return true;
                         },
                         &inc_go);
        return ok2;
      }, &inc_refine);
    } else {
      launch_ksp_begin(h->L, h->K.st, P, c.ksp_max_it);
      launch_bicg_init(h->L, g, f, h->K, h->rhs, h->vel);
      inner_ok = add_conditional(
          h, cudaGraphCondTypeWhile,
          [&](cudaGraphConditionalHandle cond) { launch_loop_condition(h->L, cond, h->K.st); },
          [&] {
            for (int q = 0; q < 4; ++q) launch_bicg_iteration(h->L, g, f, h->K, h->vel, mg, line);
            return true;
          },
          &inc_inner);
      launch_ksp_end(h->L, P, h->K.st, 4);
    }
    launch_picard_after_solve(h->L, P, h->zd_dev);
    inner_ok = inner_ok && add_conditional(h, cudaGraphCondTypeIf, not_done(&P->done), [&] {
      launch_nuH(h->L, g, c, f, reg, underrelax, true, h->norm_dev);
      launch_picard_test(h->L, P, h->norm_dev, pc);
      return true;
    }, &inc_test);
    return inner_ok && rebuild_ok;
  }, &inc_picard);
  pre = before_loop - t0 + 1;   // + the WHILE node's first condition kernel
  cudaGraph_t out = nullptr;
  const bool ended = cudaStreamEndCapture(h->stream, &out) == cudaSuccess;
  ok = ok && ended && out != nullptr;
  if (ok) ok = cudaGraphInstantiate(&S.exec, out, 0) == cudaSuccess;
  if (out) cudaGraphDestroy(out);
  h->stats.kernel_launches = t0;   // nothing ran during the capture
  if (!ok) {
    S.exec = nullptr;
    S.failed = true;
    cudaGetLastError();
    return PISM_GPU_SSA_OK;
  }
  S.reg = reg;
  S.underrelax = underrelax;
  S.key = f;
  S.mixed = mixed;
  S.pre = pre;
  S.per_inner = inc_inner;
  S.per_go = inc_go;
  S.per_test = inc_test;
  S.per_rebuild = inc_rebuild;
  S.per_refine = mixed ? inc_refine - inc_inner - inc_go : 0;
  S.per_picard = inc_picard - (mixed ? inc_refine : inc_inner) - inc_test - inc_rebuild;
  *built = true;
  return PISM_GPU_SSA_OK;
}

// Launch the whole-solve graph (built on first use) and queue the read-back of its state,
// without waiting; *launched is false where the graph does not apply or cannot be built.
int solve_graph_launch(pism_gpu_ssa *h, double reg, double underrelax, bool *launched) {
  *launched = false;
  if (!solve_graph_eligible(h)) return PISM_GPU_SSA_OK;
  auto &S = h->sgraph;
  const Fields f = fields_of(h);
  if (!S.exec || S.reg != reg || S.underrelax != underrelax || memcmp(&S.key, &f, sizeof(Fields)) != 0) {
    if (S.failed && S.reg == reg && S.underrelax == underrelax) return PISM_GPU_SSA_OK;
    bool built = false;
    RET(build_solve_graph(h, reg, underrelax, &built));
    if (!built) {
      S.reg = reg;
      S.underrelax = underrelax;
      return PISM_GPU_SSA_OK;
    }
  }
  CK(h, cudaGraphLaunch(S.exec, h->stream));
  CK(h, cudaMemcpyAsync(h->pstate_host, h->pstate, sizeof(PState), cudaMemcpyDeviceToHost, h->stream));
  *launched = true;
  return PISM_GPU_SSA_OK;
}

// Wait for a launched whole-solve graph; the host loop's return codes, messages and
// statistics.
int solve_graph_collect(pism_gpu_ssa *h, double reg) {
  CK(h, cudaStreamSynchronize(h->stream));
  const auto &S = h->sgraph;
  const PState &P = *h->pstate_host;
  h->stats.kernel_launches += S.pre + P.passes * S.per_picard + P.refine_passes * S.per_refine +
                              P.inner_passes * S.per_inner + P.go_count * S.per_go + P.k * S.per_test +
                              P.rebuilds * S.per_rebuild;
  if (active_mg(h)) h->stats.mg_rebuilds += P.rebuilds;
  h->stats.ksp_iterations += P.ksp_total;
  h->stats.refinement_steps += P.refine_steps;
  h->stats.final_linear_residual = P.final_res;
  h->last_ksp_its = P.ksp_its;
  if (P.k > 0) {
    h->stats.picard_iterations = P.k;
    h->stats.nuH_norm = P.norm;
    h->stats.nuH_norm_change = P.change;
  }
  switch (P.status) {
    case PISM_GPU_SSA_OK:
      return PISM_GPU_SSA_OK;
    case PISM_GPU_SSA_EZERODIAG:
      return fail(h, PISM_GPU_SSA_EZERODIAG,
                  "SSAFD system: zero diagonal entry at a regular (not Dirichlet B.C.) location: i = %d, j = %d",
                  P.zd_cell / h->g.My, P.zd_cell % h->g.My);
    case PISM_GPU_SSA_EKSP:
      return fail(h, PISM_GPU_SSA_EKSP, "SSAFD KSP (linear solver) failed: reason %d after %d iterations",
                  P.ksp_status, P.ksp_its);
    case PISM_GPU_SSA_ENAN:
      return fail(h, PISM_GPU_SSA_ENAN, "non-finite nu*H norm at Picard iteration %d", P.k - 1);
    default:
      return fail(h, PISM_GPU_SSA_EPICARD,
                  "SSAFD Picard iterations failed: effective viscosity not converged after %d iterations with "
                  "nuH_regularization=%8.2e.",
                  h->cfg.max_iterations_ssafd, reg);
  }
}

// The Picard loop through the whole-solve graph when it applies (*used).
int picard_manager_graph(pism_gpu_ssa *h, double reg, double underrelax, bool *used) {
  *used = false;
  bool launched = false;
  RET(solve_graph_launch(h, reg, underrelax, &launched));
  if (!launched) return PISM_GPU_SSA_OK;
  *used = true;
  return solve_graph_collect(h, reg);
}

// ---- one linear solve: BiCGStab on the device, host reads the state per chunk ----
int linear_solve(pism_gpu_ssa *h, double2 *x, double rtol, int *its_out, int *status_out) {
  const GridDev &g = h->g;
  Fields f = fields_of(h);
  KState init{};
  init.rtol = rtol;
  init.maxit = h->use_fallback ? 4 * h->cfg.ksp_max_it : h->cfg.ksp_max_it;
  *h->st_host = init;
  CK(h, cudaMemcpyAsync(h->K.st, h->st_host, sizeof(KState), cudaMemcpyHostToDevice, h->stream));
  launch_bicg_init(h->L, g, f, h->K, h->rhs, x);
  const MGHierarchy *mg = active_mg(h);
  const LinePC *line = active_line(h);
  const int kind = mg ? GRAPH_BICG_MG : line ? GRAPH_BICG_LINE : GRAPH_BICG_JACOBI;
  // long FP64 solves: four iterations per pass of the loop body
  RET(run_until_done(h, kind, x, h->K.st, std::max(8, (int)(0.8 * h->last_ksp_its)), 4,
                     [&] { launch_bicg_iteration(h->L, g, f, h->K, x, mg, line); }));
  h->last_ksp_its = h->st_host->iter;
  *its_out = h->st_host->iter;
  *status_out = h->st_host->status;
  h->stats.final_linear_residual =
      h->st_host->bnorm2 > 0 ? sqrt(h->st_host->rnorm2 / h->st_host->bnorm2) : sqrt(h->st_host->rnorm2);
  return PISM_GPU_SSA_OK;
}

// ---- the learned preconditioner correction ----
// After z = M^-1 v: r = v - A z, the network's input from the solve's features and the
// block-Jacobi-scaled residual D^-1 r (normalised by its RMS rho), d = rho * its output
// interpolated to the grid, and z += gamma d with gamma = (r, A d) / (A d, A d), the step that
// minimises ||v - A (z + gamma d)||: the corrected step never leaves a larger residual than
// the preconditioner alone, whatever the network returns.  Right preconditioning in FGMRES
// allows a preconditioner that changes from one step to the next; the FP64 residual test of
// the Krylov solve decides every accepted answer as without it.
int learned_correction(pism_gpu_ssa *h, const double2 *v, double2 *z, const int *done) {
  auto &P = h->lpc;
  const Fields f = fields_of(h);
  launch_pc_residual(h->L, h->g, f, v, z, P.r, h->G.st);
  pism_unet::launch_features(h->stream, h->g.Mx, h->g.My, P.stride, h->H, h->bed, h->tauc, h->hardness, h->mask,
                             h->taud, P.img, P.height, P.width);
  pism_unet::launch_pc_input(h->stream, h->g.Mx, h->g.My, P.stride, P.r, h->K.dinv, P.img, P.height, P.width, P.part,
                             P.rho, done);
  cudaStream_t ns = pism_unet::stream_of(P.net);
  pism_gpu_unet_set_stream(P.net, h->stream);
  const int rc = pism_gpu_unet_forward(P.net, P.img, 1, P.height, P.width, P.out);
  pism_gpu_unet_set_stream(P.net, ns);
  if (rc != PISM_GPU_SSA_OK)
    return fail(h, rc, "learned preconditioner: network forward failed: %s", pism_gpu_unet_last_error(P.net));
  pism_unet::launch_pc_expand(h->stream, P.out, P.height, P.width, P.stride, h->g.Mx, h->g.My, P.rho, P.d, done);
  h->L.tick(22);   // features, input (2), network (18), expansion; the residual and line search tick their own
  launch_pc_line_search(h->L, h->g, f, P.r, P.d, P.ad, P.gamma, z, h->G.st);
  CK(h, cudaGetLastError());
  return PISM_GPU_SSA_OK;
}

// ---- one linear solve: restarted flexible GMRES(m) on the device (PETSc's default KSP
// type, restart gmres_restart), right-preconditioned by the active preconditioner ----
int linear_solve_gmres(pism_gpu_ssa *h, double2 *x, double rtol, int *its_out, int *status_out) {
  const GridDev &g = h->g;
  const int m = h->cfg.gmres_restart;
  if (h->G.m != m) {
    for (void *p : {(void *)h->G.V, (void *)h->G.Z, (void *)h->G.partials, (void *)h->G.gs, (void *)h->G.st})
      if (p) cudaFree(p);
    h->G = Gmres{};
    RET(dalloc(h, &h->G.V, (size_t)(m + 1) * h->N));
    RET(dalloc(h, &h->G.Z, (size_t)m * h->N));
    RET(dalloc(h, &h->G.partials, (size_t)h->L.max_blocks * (GM_MAXM + 2)));
    RET(dalloc(h, &h->G.gs, 1));
    RET(dalloc(h, &h->G.st, 1));
    h->G.m = m;
  }
  Fields f = fields_of(h);
  KState init{};
  init.rtol = rtol;
  init.maxit = h->use_fallback ? 4 * h->cfg.ksp_max_it : h->cfg.ksp_max_it;
  *h->st_host = init;
  CK(h, cudaMemcpyAsync(h->G.st, h->st_host, sizeof(KState), cudaMemcpyHostToDevice, h->stream));
  launch_gmres_residual(h->L, g, f, h->G, h->rhs, x, 1);
  int j = 0, launched = 0;
  int chunk = std::max(8, (int)(0.8 * h->last_ksp_its));
  while (true) {
    const MGHierarchy *mg = active_mg(h);
    const LinePC *line = active_line(h);
    for (int q = 0; q < chunk; ++q) {
      if (h->lpc.net) {
        launch_gmres_precondition(h->L, g, f, h->G, h->K.dinv, mg, line, j);
        RET(learned_correction(h, h->G.V + (size_t)j * h->N, h->G.Z + (size_t)j * h->N, &h->G.st->done));
        launch_gmres_orthogonalize(h->L, g, f, h->G, j);
      } else {
        launch_gmres_step(h->L, g, f, h->G, h->K.dinv, mg, line, j);
      }
      if (j == m - 1) {   // end of a cycle: x += Z y, then a restart unless converged
        launch_gmres_update(h->L, g, h->G, x);
        launch_gmres_residual(h->L, g, f, h->G, h->rhs, x, 0);
        j = 0;
      } else {
        ++j;
      }
    }
    launched += chunk;
    CK(h, cudaGetLastError());
    CK(h, cudaMemcpyAsync(h->st_host, h->G.st, sizeof(KState), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    if (h->st_host->done) break;
    chunk = std::max(4, std::min(64, launched / 8));
  }
  launch_gmres_update(h->L, g, h->G, x);   // a cycle that converged part-way
  CK(h, cudaGetLastError());
  CK(h, cudaStreamSynchronize(h->stream));
  h->last_ksp_its = h->st_host->iter;
  *its_out = h->st_host->iter;
  *status_out = h->st_host->status;
  h->stats.final_linear_residual =
      h->st_host->bnorm2 > 0 ? sqrt(h->st_host->rnorm2 / h->st_host->bnorm2) : sqrt(h->st_host->rnorm2);
  return PISM_GPU_SSA_OK;
}

// Mixed precision: FP64 iterative refinement around FP32 BiCGStab + FP32 multigrid.  The
// convergence test ||b - A x|| <= ksp_rtol ||b|| is evaluated in FP64 each refinement step.
int linear_solve_mixed(pism_gpu_ssa *h, double2 *x, double rtol, int *its_out, int *status_out) {
  const GridDev &g = h->g;
  Fields f = fields_of(h);
  const MGHierarchy *mg = active_mg(h);
  const int max_refine = 60;
  int inner_total = 0, status = KSP_OK;
  // One host read-back per chunk of inner iterations: the outer test (FP64 residual of the
  // step) and the inner tolerance are taken on the device by the inner solve's start.
  launch_residual32(h->L, g, f, h->rhs, x, h->K32.rhs, h->res_dev);
  for (int refine = 0;; ++refine) {
    launch_mixed_init(h->L, g.Mx * g.My, h->K32, h->res_dev, rtol, h->cfg.mixed_inner_rtol, h->cfg.ksp_max_it);
    // short inner solves (a few iterations each): one iteration per pass
    RET(run_until_done(h, GRAPH_MIXED, nullptr, h->K32.st, 8, 1,
                       [&] { launch_mixed_iteration(h->L, g, f, *mg, h->K32); }));
    const double rn = sqrt(h->st_host->outer_r2), bn = sqrt(h->st_host->outer_b2);
    h->stats.final_linear_residual = bn > 0 ? rn / bn : rn;
    if (!std::isfinite(rn)) { status = KSP_NAN; break; }
    if (h->st_host->status == KSP_OUTER_DONE) break;
    if (refine >= max_refine) { status = KSP_MAXIT; break; }
    inner_total += h->st_host->iter;
    h->stats.refinement_steps += 1;
    if (h->st_host->status == KSP_NAN || h->st_host->status == KSP_STALLED) {
      status = h->st_host->status;
      break;
    }
    if (h->st_host->iter == 0) { status = KSP_BREAKDOWN; break; }   // no progress possible
    launch_axpy32(h->L, g.Mx * g.My, h->K32.d, x);
    launch_residual32(h->L, g, f, h->rhs, x, h->K32.rhs, h->res_dev);
  }
  *its_out = inner_total;
  *status_out = status;
  return PISM_GPU_SSA_OK;
}

// SSAFD::picard_manager, SSAFD.cc:962-1119
int picard_manager(pism_gpu_ssa *h, double reg, double underrelax) {
  bool used = false;
  const int rc = picard_manager_graph(h, reg, underrelax, &used);
  if (used || rc != PISM_GPU_SSA_OK) return rc;
  const pism_gpu_ssa_config &c = h->cfg;
  Fields f = fields_of(h);
  launch_nuH(h->L, h->g, c, f, reg, 1.0, false, h->norm_dev);
  double last_change = 1.0;   // relative nu*H change of the previous iteration
  double coarse_change = 0.0;   // relative nu*H changes summed since the coarse levels were built
  for (int k = 0; k < c.max_iterations_ssafd; ++k) {
    RET(pc_setup(h, mg_rebuild_due(coarse_change, k == 0, c.mg_rebuild_rtol)));
    // inexact Picard: the linear solve of an iterate that is still far from the fixed point
    // only needs to be as accurate as the nonlinear iteration it feeds
    double rtol = c.ksp_rtol;
    if (c.ksp_rtol_adaptive && last_change >= 2.0 * c.ssafd_relative_convergence)
      rtol = std::min(c.ksp_rtol_max, std::max(c.ksp_rtol, c.ksp_rtol_factor * last_change));
    int its = 0, status = 0;
    if (h->cfg.precision == PISM_PRECISION_MIXED && active_mg(h))
      RET(linear_solve_mixed(h, h->vel, rtol, &its, &status));
    else if (h->cfg.ksp_type == PISM_KSP_GMRES)
      RET(linear_solve_gmres(h, h->vel, rtol, &its, &status));
    else
      RET(linear_solve(h, h->vel, rtol, &its, &status));
    CK(h, cudaMemcpyAsync(h->zd_host, h->zd_dev, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    h->stats.ksp_iterations += its;
    if (*h->zd_host != INT_MAX) {
      const int cidx = *h->zd_host;
      return fail(h, PISM_GPU_SSA_EZERODIAG,
                  "SSAFD system: zero diagonal entry at a regular (not Dirichlet B.C.) location: i = %d, j = %d",
                  cidx / h->g.My, cidx % h->g.My);
    }
    if (status != KSP_OK)
      return fail(h, PISM_GPU_SSA_EKSP, "SSAFD KSP (linear solver) failed: reason %d after %d iterations",
                  status, its);
    launch_nuH(h->L, h->g, c, f, reg, underrelax, true, h->norm_dev);
    CK(h, cudaMemcpyAsync(h->norm_host, h->norm_dev, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    const double norm = h->norm_host[0], change = h->norm_host[1];
    mg_change_add(coarse_change, norm, change);
    h->stats.picard_iterations = k + 1;
    h->stats.nuH_norm = norm;
    h->stats.nuH_norm_change = change;
    if (c.verbosity > 2)
      fprintf(stderr, "  %2d: S:%d,%d (rtol %.1e): |nu|_2, |Delta nu|_2/|nu|_2 = %10.3e %10.3e\n", k, its, status,
              rtol, norm, change / norm);
    if (!std::isfinite(norm) || !std::isfinite(change))
      return fail(h, PISM_GPU_SSA_ENAN, "non-finite nu*H norm at Picard iteration %d", k);
    if (norm == 0 || (change / norm < c.ssafd_relative_convergence && rtol <= c.ksp_rtol)) return PISM_GPU_SSA_OK;
    last_change = norm > 0 ? change / norm : 0.0;
  }
  return fail(h, PISM_GPU_SSA_EPICARD,
              "SSAFD Picard iterations failed: effective viscosity not converged after %d iterations with "
              "nuH_regularization=%8.2e.",
              c.max_iterations_ssafd, reg);
}

// SSAFD::picard_iteration, SSAFD.cc:926-959: a KSP failure switches to the fallback
// solver (the reference's ASM + LU) and restarts from the previous velocity.
int picard_iteration(pism_gpu_ssa *h, double reg, double underrelax) {
  if (h->default_pc_failure_count < 5) {
    h->use_fallback = 0;
    int rc = picard_manager(h, reg, underrelax);
    if (rc != PISM_GPU_SSA_EKSP) return rc;
    h->default_pc_failure_count += 1;
    h->stats.ksp_failures += 1;
    if (h->cfg.verbosity > 0) fprintf(stderr, "  re-trying using the fallback linear solver...\n");
    h->use_fallback = 1;
    CK(h, cudaMemcpyAsync(h->vel, h->vel_old, sizeof(double2) * h->N, cudaMemcpyDeviceToDevice, h->stream));
    return picard_manager(h, reg, underrelax);
  }
  h->use_fallback = 1;
  return picard_manager(h, reg, underrelax);
}

// SSAFD::picard_strategy_regularization, SSAFD.cc:1122-1155
int picard_strategy_regularization(pism_gpu_ssa *h) {
  double reg = h->cfg.epsilon_ssa;
  if (reg <= 0.0)
    return fail(h, PISM_GPU_SSA_EPICARD,
                "SSAFD Picard iterations failed: will not attempt over-regularization of nuH because "
                "nuH_regularization == 0.0.");
  for (int k = 0; k < 5; ++k) {
    CK(h, cudaMemcpyAsync(h->vel, h->vel_old, sizeof(double2) * h->N, cudaMemcpyDeviceToDevice, h->stream));
    if (h->cfg.verbosity > 0) fprintf(stderr, "  re-trying with nuH_regularization multiplied by %8.2f...\n", 4.0);
    reg *= 4.0;
    int rc = picard_iteration(h, reg, 1.0);
    if (rc == PISM_GPU_SSA_OK) return rc;
    if (rc != PISM_GPU_SSA_EPICARD) return rc;
  }
  return fail(h, PISM_GPU_SSA_EPICARD,
              "SSAFD Picard iterations failed: exceeded the max. number of nuH over-regularization attempts");
}

int prepare(pism_gpu_ssa *h) {
  if (!h->inputs_set) return fail(h, PISM_GPU_SSA_ESTATE, "pism_gpu_ssa_set_inputs was not called");
  Fields f = fields_of(h);
  launch_prepare(h->L, h->g, h->cfg, h->grid.periodicity, f);
  if (!h->have_hardness) {
    if (h->cfg.flow_law != PISM_FLOW_LAW_ISOTHERMAL_GLEN && !h->have_enthalpy)
      return fail(h, PISM_GPU_SSA_EINVAL, "the flow law needs enthalpy (or a precomputed hardness)");
    launch_hardness(h->L, h->g, h->cfg, f, (int)h->z_host.size(), h->z_dev);
  }
  CK(h, cudaGetLastError());
  h->prepared = true;
  return PISM_GPU_SSA_OK;
}

// staging of the strain rates and eigen-calving, in doubles from h->ec: strain rates 2 N at
// EC_EDOT, stresses 3 N at EC_STRESS, the caller's mask N at EC_MASK; eigen-calving's Href,
// thickness and per-cell loss N each at EC_HREF, EC_H, EC_LOSS (over the strain-rate slots,
// which it does not use); 8 scalars at EC_SCALARS.  Plus 2 N bytes of masks in h->ec_mask.
enum : size_t { EC_EDOT = 0, EC_STRESS = 2, EC_MASK = 5, EC_HREF = 0, EC_H = 1, EC_LOSS = 2, EC_SCALARS = 6 };

int ec_buffers(pism_gpu_ssa *h) {
  if (!h->ec) RET(dalloc(h, &h->ec, EC_SCALARS * (size_t)h->N + 8));
  if (!h->ec_mask) RET(dalloc(h, &h->ec_mask, 2 * (size_t)h->N));
  return PISM_GPU_SSA_OK;
}

int copy_in(pism_gpu_ssa *h, void *dst, const void *src, size_t bytes, int where) {
  CK(h, cudaMemcpyAsync(dst, src, bytes, where == PISM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                        h->stream));
  return PISM_GPU_SSA_OK;
}

int copy_out(pism_gpu_ssa *h, void *dst, const void *src, size_t bytes, int where) {
  CK(h, cudaMemcpyAsync(dst, src, bytes, where == PISM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return PISM_GPU_SSA_OK;
}

}  // namespace

extern "C" {

int pism_gpu_ssa_config_defaults(pism_gpu_ssa_config *c) {
  if (!c) return PISM_GPU_SSA_EINVAL;
  const double secpera = 31556925.9747;   // UDUNITS-2 year
  memset(c, 0, sizeof(*c));
  // src/pism_config.cdl
  c->ice_density = 910.0;
  c->sea_water_density = 1028.0;
  c->standard_gravity = 9.81;
  c->sea_level = 0.0;
  c->epsilon_ssa = 1.0e13;
  c->ssafd_relative_convergence = 1.0e-4;
  c->max_iterations_ssafd = 300;
  c->ssafd_nuH_iter_failure_underrelaxation = 0.8;
  c->min_thickness_strength_extension_ssa = 50.0;
  c->constant_nu_strength_extension_ssa = 9.48680701906572e14;
  c->plastic_regularization = 0.01 / secpera;
  c->do_pseudo_plastic_till = 0;
  c->pseudo_plastic_q = 0.25;
  c->pseudo_plastic_uthreshold = 100.0 / secpera;
  c->sliding_scale_factor_reduces_tauc = -1.0;
  c->beta_ice_free_bedrock = 1.8e9;
  c->nu_bedrock = 5.0e15;
  c->flow_law = PISM_FLOW_LAW_GPBLD;
  c->ssa_Glen_exponent = 3.0;
  c->ssa_enhancement_factor = 1.0;
  c->ice_softness = 3.1689e-24;
  c->Schoof_regularizing_length = 1000.0e3;
  c->Schoof_regularizing_velocity = 1.0 / secpera;
  c->Paterson_Budd_A_cold = 3.61e-13;
  c->Paterson_Budd_A_warm = 1.73e3;
  c->Paterson_Budd_Q_cold = 6.0e4;
  c->Paterson_Budd_Q_warm = 13.9e4;
  c->Paterson_Budd_critical_temperature = 263.15;
  c->ideal_gas_constant = 8.31441;
  c->gpbld_water_frac_coeff = 181.25;
  c->gpbld_water_frac_observed_limit = 0.01;
  c->Hooke_A = 4.42165e-9;
  c->Hooke_Q = 7.88e4;
  c->Hooke_C = 0.16612;
  c->Hooke_k = 1.17;
  c->Hooke_Tr = 273.39;
  c->beta_CC = 7.9e-8;
  c->ice_specific_heat_capacity = 2009.0;
  c->water_latent_heat_fusion = 3.34e5;
  c->surface_pressure = 0.0;
  c->water_melting_point_temperature = 273.15;
  c->enthalpy_converter_reference_temperature = 223.15;
  c->fracture_density_softening_lower_limit = 1.0;
  c->brutal_sliding_scale = 1.0;
  // PETSc KSP defaults
  c->ksp_type = PISM_KSP_BICGSTAB;
  c->pc_type = PISM_PC_BLOCK_JACOBI;
  c->ksp_rtol = 1.0e-5;
  c->ksp_max_it = 10000;
  c->gmres_restart = 30;
  c->precision = PISM_PRECISION_FP64;
  c->mixed_inner_rtol = 1.0e-3;
  c->mg_omega = 0.9;
  c->mg_correction = 1.2;
  c->ksp_rtol_adaptive = 0;
  c->ksp_rtol_max = 1.0e-2;
  c->ksp_rtol_factor = 1.0e-2;
  c->graphs = 2;
  c->verbosity = 0;
  c->mixed_apply_kernel = 2;
  return PISM_GPU_SSA_OK;
}

const char *pism_gpu_ssa_last_error(const pism_gpu_ssa *h) { return h ? h->err.c_str() : "null handle"; }

int pism_gpu_ssa_create(const pism_gpu_grid *grid, const pism_gpu_ssa_config *cfg, int device, pism_gpu_ssa **out) {
  if (!grid || !cfg || !out) return PISM_GPU_SSA_EINVAL;
  *out = nullptr;
  if (grid->Mx < 3 || grid->My < 3 || !(grid->dx > 0) || !(grid->dy > 0) || grid->Mz < 0 ||
      (grid->Mz > 0 && !grid->z) || (long long)grid->Mx * grid->My > (1LL << 30))
    return PISM_GPU_SSA_EINVAL;
  pism_gpu_ssa *h = new pism_gpu_ssa();
  if (check_config(h, cfg) != PISM_GPU_SSA_OK) {
    delete h;
    return PISM_GPU_SSA_EINVAL;
  }
  h->grid = *grid;
  if (grid->Mz > 0) h->z_host.assign(grid->z, grid->z + grid->Mz);
  h->grid.z = nullptr;
  h->cfg = *cfg;
  h->device = device;
  h->g.Mx = grid->Mx;
  h->g.My = grid->My;
  h->g.dx = grid->dx;
  h->g.dy = grid->dy;
  h->N = grid->Mx * grid->My;
  DeviceGuard dg(device);
  auto bail = [&](int rc) {
    pism_gpu_ssa_destroy(h);
    return rc;
  };
  if (cudaSetDevice(device) != cudaSuccess) return bail(PISM_GPU_SSA_ECUDA);
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return bail(PISM_GPU_SSA_ECUDA);
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) return bail(PISM_GPU_SSA_ECUDA);
  h->stream = h->own_stream;
  const size_t N = h->N;
  int rc = PISM_GPU_SSA_OK;
#define AL(p, n) \
  if ((rc = dalloc(h, &p, n)) != PISM_GPU_SSA_OK) return bail(rc)
  AL(h->H, N); AL(h->srf, N); AL(h->bed, N); AL(h->tauc, N); AL(h->melange, N); AL(h->gl_mask, N);
  AL(h->fracture, N); AL(h->stage, N); AL(h->stage2, N);
  AL(h->enthalpy, N * std::max(1, grid->Mz)); AL(h->z_dev, std::max(1, grid->Mz));
  AL(h->mask, N); AL(h->bc, N); AL(h->bcv, N);
  AL(h->taud, N); AL(h->rhs, N); AL(h->hardness, N); AL(h->nuH, N); AL(h->vel, N); AL(h->vel_old, N);
  AL(h->beta, N); AL(h->bfrict, N); AL(h->flags, N);
  AL(h->K.r, N); AL(h->K.rhat, N); AL(h->K.p, N); AL(h->K.v, N); AL(h->K.s, N); AL(h->K.t, N);
  AL(h->K.phat, N); AL(h->K.shat, N); AL(h->K.dinv, N); AL(h->K.st, 1);
  AL(h->K32.rhs, N); AL(h->K32.r, N); AL(h->K32.rhat, N); AL(h->K32.p, N); AL(h->K32.v, N);
  AL(h->K32.t, N); AL(h->K32.phat, N); AL(h->K32.shat, N); AL(h->K32.d, N); AL(h->K32.st, 1);
  AL(h->res_dev, 2);
  h->L.max_blocks = sms * 4;   // persistent grids: one wave at the tile kernels' 4 blocks per SM
  if (mg_plan(grid->Mx, grid->My, h->mg) > 0) {
    if (mg_allocate(h->mg, h->N) != 0) return bail(PISM_GPU_SSA_ENOMEM);
    if (cudaMemsetAsync(h->mg.singular, 0, sizeof(int), h->stream) != cudaSuccess) return bail(PISM_GPU_SSA_ECUDA);
  }
  AL(h->partials, (size_t)h->L.max_blocks * 8); AL(h->ticket, 1); AL(h->norm_dev, 2); AL(h->zd_dev, 1);
#undef AL
  if (cudaMallocHost((void **)&h->st_host, sizeof(KState)) != cudaSuccess ||
      cudaMallocHost((void **)&h->norm_host, 2 * sizeof(double)) != cudaSuccess ||
      cudaMallocHost((void **)&h->zd_host, sizeof(int)) != cudaSuccess ||
      cudaMallocHost((void **)&h->res_host, 2 * sizeof(double)) != cudaSuccess)
    return bail(PISM_GPU_SSA_ENOMEM);
  if (cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess)
    return bail(PISM_GPU_SSA_ECUDA);
  if (cudaMemsetAsync(h->ticket, 0, sizeof(unsigned), h->stream) != cudaSuccess ||
      cudaMemsetAsync(h->vel, 0, sizeof(double2) * N, h->stream) != cudaSuccess ||     // SSA.cc:178
      cudaMemsetAsync(h->nuH, 0, sizeof(double2) * N, h->stream) != cudaSuccess)
    return bail(PISM_GPU_SSA_ECUDA);
  if (grid->Mz > 0 &&
      cudaMemcpyAsync(h->z_dev, h->z_host.data(), sizeof(double) * grid->Mz, cudaMemcpyHostToDevice, h->stream) !=
          cudaSuccess)
    return bail(PISM_GPU_SSA_ECUDA);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bail(PISM_GPU_SSA_ECUDA);
  h->L.stream = h->stream;
  h->L.partials = h->partials;
  h->L.ticket = h->ticket;
  h->L.count = &h->stats.kernel_launches;
  *out = h;
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_destroy(pism_gpu_ssa *h) {
  if (!h) return PISM_GPU_SSA_OK;
  DeviceGuard dg(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  void *dev[] = {h->H, h->srf, h->bed, h->tauc, h->melange, h->gl_mask, h->fracture, h->stage, h->stage2,
                 h->enthalpy, h->z_dev, h->mask, h->bc, h->bcv, h->taud, h->rhs, h->hardness, h->nuH, h->vel,
                 h->vel_old, h->beta, h->bfrict, h->flags, h->K.r, h->K.rhat, h->K.p, h->K.v, h->K.s, h->K.t,
                 h->K.phat, h->K.shat, h->K.dinv, h->K.st, h->partials, h->ticket, h->norm_dev, h->zd_dev,
                 h->K32.rhs, h->K32.r, h->K32.rhat, h->K32.p, h->K32.v, h->K32.t, h->K32.phat,
                 h->K32.shat, h->K32.d, h->K32.st, h->res_dev, h->lfeat, h->lout, h->G.V, h->G.Z,
                 h->G.partials, h->G.gs, h->G.st, h->line.P, h->line.F, h->line.G, h->lpc.img, h->lpc.out,
                 h->lpc.r, h->lpc.d, h->lpc.ad, h->lpc.part, h->lpc.rho, h->lpc.gamma, h->sb3d, h->mc,
                 h->ec, h->ec_mask};
  for (void *p : dev)
    if (p) cudaFree(p);
  fem_free(h->fem);
  if (h->st_host) cudaFreeHost(h->st_host);
  if (h->norm_host) cudaFreeHost(h->norm_host);
  if (h->zd_host) cudaFreeHost(h->zd_host);
  if (h->res_host) cudaFreeHost(h->res_host);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  for (auto &gr : h->graphs)
    if (gr.exec) cudaGraphExecDestroy(gr.exec);
  for (auto &lp : h->loops)
    if (lp.exec) cudaGraphExecDestroy(lp.exec);
  if (h->sgraph.exec) cudaGraphExecDestroy(h->sgraph.exec);
  if (h->pstate) cudaFree(h->pstate);
  if (h->pstate_host) cudaFreeHost(h->pstate_host);
  mg_free(h->mg);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_set_stream(pism_gpu_ssa *h, void *s) {
  if (!h) return PISM_GPU_SSA_EINVAL;
  h->stream = s ? (cudaStream_t)s : h->own_stream;
  h->L.stream = h->stream;
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_set_config(pism_gpu_ssa *h, const pism_gpu_ssa_config *cfg) {
  if (!h) return PISM_GPU_SSA_EINVAL;
  RET(check_config(h, cfg));
  h->cfg = *cfg;
  h->prepared = false;
  for (auto &gr : h->graphs) {   // the multigrid damping is captured by value
    if (gr.exec) cudaGraphExecDestroy(gr.exec);
    gr = {};
  }
  for (auto &lp : h->loops) {
    if (lp.exec) cudaGraphExecDestroy(lp.exec);
    lp = {};
  }
  if (h->sgraph.exec) cudaGraphExecDestroy(h->sgraph.exec);
  h->sgraph = {};
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_set_inputs(pism_gpu_ssa *h, const pism_gpu_ssa_inputs *in) {
  if (!h) return PISM_GPU_SSA_EINVAL;
  if (!in || !in->thickness || !in->surface || !in->bed || !in->mask || !in->tauc)
    return fail(h, PISM_GPU_SSA_EINVAL, "thickness, surface, bed, mask and tauc are required");
  if ((in->bc_mask == nullptr) != (in->bc_values == nullptr))
    return fail(h, PISM_GPU_SSA_EINVAL, "bc_mask and bc_values must be given together");
  if (h->cfg.sub_groundingline && !in->gl_mask)
    return fail(h, PISM_GPU_SSA_EINVAL, "sub_groundingline needs gl_mask");
  if (h->cfg.do_fracture_density && !in->fracture_density)
    return fail(h, PISM_GPU_SSA_EINVAL, "do_fracture_density needs fracture_density");
  if (in->enthalpy && h->z_host.empty())
    return fail(h, PISM_GPU_SSA_EINVAL, "enthalpy given but the grid has no vertical levels (Mz = 0)");
  DeviceGuard dg(h->device);
  const size_t N = h->N, B = N * sizeof(double);
  const int w = in->where;
  RET(copy_in(h, h->H, in->thickness, B, w));
  RET(copy_in(h, h->srf, in->surface, B, w));
  RET(copy_in(h, h->bed, in->bed, B, w));
  RET(copy_in(h, h->tauc, in->tauc, B, w));
  RET(copy_in(h, h->stage, in->mask, B, w));
  if (in->bc_mask) {
    RET(copy_in(h, h->stage2, in->bc_mask, B, w));
    RET(copy_in(h, h->bcv, in->bc_values, 2 * B, w));
  }
  h->have_melange = in->melange != nullptr;
  if (in->melange) RET(copy_in(h, h->melange, in->melange, B, w));
  h->have_gl = in->gl_mask != nullptr;
  if (in->gl_mask) RET(copy_in(h, h->gl_mask, in->gl_mask, B, w));
  h->have_enthalpy = in->enthalpy != nullptr;
  if (in->enthalpy) RET(copy_in(h, h->enthalpy, in->enthalpy, B * h->z_host.size(), w));
  h->have_hardness = in->hardness_stag != nullptr;
  if (in->hardness_stag) RET(copy_in(h, h->hardness, in->hardness_stag, 2 * B, w));
  h->have_fracture = in->fracture_density != nullptr;
  if (in->fracture_density) RET(copy_in(h, h->fracture, in->fracture_density, B, w));
  launch_convert_masks(h->L, h->N, h->stage, in->bc_mask ? h->stage2 : nullptr, h->mask, h->bc);
  CK(h, cudaGetLastError());
  CK(h, cudaStreamSynchronize(h->stream));
  h->inputs_set = true;
  h->prepared = false;
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_set_initial_guess(pism_gpu_ssa *h, const double *velocity, int where) {
  if (!h || !velocity) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  RET(copy_in(h, h->vel, velocity, sizeof(double2) * h->N, where));
  CK(h, cudaStreamSynchronize(h->stream));
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_solve(pism_gpu_ssa *h, double *velocity_out, int where, pism_gpu_ssa_stats *stats) {
  if (!h) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  auto t0 = std::chrono::steady_clock::now();
  h->stats = pism_gpu_ssa_stats{};
  h->err.clear();
  h->L.count = &h->stats.kernel_launches;
  CK(h, cudaEventRecord(h->ev0, h->stream));
  // SSAFD::solve, SSAFD.cc:869-924
  CK(h, cudaMemcpyAsync(h->vel_old, h->vel, sizeof(double2) * h->N, cudaMemcpyDeviceToDevice, h->stream));
  int rc = prepare(h);
  if (rc == PISM_GPU_SSA_OK) {
    for (int k = 0; k < 3; ++k) {
      h->stats.strategy = k;
      if (k == 0)
        rc = picard_iteration(h, h->cfg.epsilon_ssa, 1.0);
      else if (k == 1) {
        if (h->cfg.verbosity > 0)
          fprintf(stderr, "  re-trying with effective viscosity under-relaxation (parameter = %.2f) ...\n",
                  h->cfg.ssafd_nuH_iter_failure_underrelaxation);
        rc = picard_iteration(h, h->cfg.epsilon_ssa, h->cfg.ssafd_nuH_iter_failure_underrelaxation);
      } else {
        rc = picard_strategy_regularization(h);
      }
      if (rc == PISM_GPU_SSA_OK) {
        h->stats.converged = 1;
        break;
      }
      if (rc != PISM_GPU_SSA_EPICARD) break;
    }
    // the reference's strategy loop ends silently when every strategy failed
    // (SSAFD.cc:882-911: the k == 3 branch is unreachable); stats.converged = 0 says so
    if (rc == PISM_GPU_SSA_EPICARD) rc = PISM_GPU_SSA_OK;
  }
  if (rc == PISM_GPU_SSA_OK) {
    if (h->cfg.brutal_sliding) launch_scale(h->L, 2 * h->N, h->cfg.brutal_sliding_scale, (double *)h->vel);
    Fields f = fields_of(h);
    launch_bfrict(h->L, h->N, h->cfg, f, h->bfrict);   // SSA::update, SSA.cc:193-194
    CK(h, cudaGetLastError());
  }
  CK(h, cudaEventRecord(h->ev1, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  h->stats.kernel_ms = ms;
  h->stats.status = rc;
  h->stats.solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (stats) *stats = h->stats;
  if (rc != PISM_GPU_SSA_OK) return rc;
  if (velocity_out) RET(copy_out(h, velocity_out, h->vel, sizeof(double2) * h->N, where));
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_get_field(pism_gpu_ssa *h, int field, double *out, int where) {
  if (!h || !out) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  const size_t N = h->N;
  switch (field) {
    case PISM_FIELD_VELOCITY: return copy_out(h, out, h->vel, 16 * N, where);
    case PISM_FIELD_TAUD: return copy_out(h, out, h->taud, 16 * N, where);
    case PISM_FIELD_RHS: return copy_out(h, out, h->rhs, 16 * N, where);
    case PISM_FIELD_HARDNESS: return copy_out(h, out, h->hardness, 16 * N, where);
    case PISM_FIELD_NUH: return copy_out(h, out, h->nuH, 16 * N, where);
    case PISM_FIELD_BETA: return copy_out(h, out, h->beta, 8 * N, where);
    case PISM_FIELD_BFRICT: return copy_out(h, out, h->bfrict, 8 * N, where);
    default: return fail(h, PISM_GPU_SSA_EINVAL, "unknown field %d", field);
  }
}

int pism_gpu_ssa_stress_balance_3d(pism_gpu_ssa *h, const double *basal_melt_rate, double *u3, double *v3,
                                   double *w3, double *strain_heating, int where) {
  if (!h) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  if (where != PISM_MEM_HOST && where != PISM_MEM_DEVICE) return fail(h, PISM_GPU_SSA_EINVAL, "bad memory kind");
  if (!h->inputs_set) return fail(h, PISM_GPU_SSA_ESTATE, "pism_gpu_ssa_set_inputs was not called");
  const int Mz = (int)h->z_host.size();
  if (Mz < 2 || Mz > SB3D_MAX_LEVELS)
    return fail(h, PISM_GPU_SSA_EINVAL, "the 3-D fields need a grid with 2 <= Mz <= %d levels", SB3D_MAX_LEVELS);
  if (stress_balance_3d_prepare(Mz) != 0) return fail(h, PISM_GPU_SSA_ECUDA, "shared memory for the 3-D fields");
  if (strain_heating && h->cfg.flow_law != PISM_FLOW_LAW_ISOTHERMAL_GLEN && !h->have_enthalpy)
    return fail(h, PISM_GPU_SSA_EINVAL, "the strain heating's flow law needs enthalpy");
  const size_t N3 = (size_t)h->N * Mz;
  double *out[4] = {u3, v3, w3, strain_heating};
  double *dev[4] = {u3, v3, w3, strain_heating};
  const double *bmr = basal_melt_rate;
  if (where == PISM_MEM_HOST) {   // device staging: the four fields and the melt rate
    if (!h->sb3d) RET(dalloc(h, &h->sb3d, 4 * N3 + h->N));
    for (int q = 0; q < 4; ++q) dev[q] = out[q] ? h->sb3d + q * N3 : nullptr;
    if (basal_melt_rate) {
      RET(copy_in(h, h->sb3d + 4 * N3, basal_melt_rate, sizeof(double) * h->N, PISM_MEM_HOST));
      bmr = h->sb3d + 4 * N3;
    }
  }
  launch_stress_balance_3d(h->L, h->g, h->cfg, Mz, fields_of(h), h->z_dev, bmr, dev[0], dev[1], dev[2], dev[3]);
  CK(h, cudaGetLastError());
  if (where == PISM_MEM_HOST)
    for (int q = 0; q < 4; ++q)
      if (out[q]) RET(copy_out(h, out[q], dev[q], sizeof(double) * N3, PISM_MEM_HOST));
  CK(h, cudaStreamSynchronize(h->stream));
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_mass_continuity_step(pism_gpu_ssa *h, double dt, const double *climatic_mass_balance,
                                      const double *basal_melt_rate, const double *cell_area,
                                      double icefree_thickness, double is_floating_thickness, double *thickness_out,
                                      double *mask_out, double *surface_out, double *flux_divergence,
                                      double *totals, int where) {
  if (!h || !climatic_mass_balance || !thickness_out) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  if (where != PISM_MEM_HOST && where != PISM_MEM_DEVICE) return fail(h, PISM_GPU_SSA_EINVAL, "bad memory kind");
  if (!h->inputs_set) return fail(h, PISM_GPU_SSA_ESTATE, "pism_gpu_ssa_set_inputs was not called");
  if (!(dt >= 0.0)) return fail(h, PISM_GPU_SSA_EINVAL, "dt must be >= 0");
  const size_t N = h->N;
  if (!h->mc) RET(dalloc(h, &h->mc, 7 * N + 8));
  const double *in[3] = {climatic_mass_balance, basal_melt_rate, cell_area};
  double *out[4] = {thickness_out, mask_out, surface_out, flux_divergence};
  const double *din[3];
  double *dout[4];
  for (int q = 0; q < 3; ++q) {
    din[q] = in[q];
    if (in[q] && where == PISM_MEM_HOST) {
      RET(copy_in(h, h->mc + q * N, in[q], sizeof(double) * N, PISM_MEM_HOST));
      din[q] = h->mc + q * N;
    }
  }
  for (int q = 0; q < 4; ++q) dout[q] = (out[q] && where == PISM_MEM_HOST) ? h->mc + (3 + q) * N : out[q];
  double *dtot = h->mc + 7 * N;
  launch_mass_continuity(h->L, h->g, h->cfg, fields_of(h), dt, icefree_thickness, is_floating_thickness, din[0],
                         din[1], din[2], dout[0], dout[3], dout[1], dout[2], dtot);
  CK(h, cudaGetLastError());
  for (int q = 0; q < 4; ++q)
    if (out[q] && where == PISM_MEM_HOST) RET(copy_out(h, out[q], dout[q], sizeof(double) * N, PISM_MEM_HOST));
  if (totals) RET(copy_out(h, totals, dtot, sizeof(double) * 8, PISM_MEM_HOST));
  CK(h, cudaStreamSynchronize(h->stream));
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_strain_rates(pism_gpu_ssa *h, const double *mask, double *edot, double *stresses, int where) {
  if (!h) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  if (where != PISM_MEM_HOST && where != PISM_MEM_DEVICE) return fail(h, PISM_GPU_SSA_EINVAL, "bad memory kind");
  if (!h->inputs_set) return fail(h, PISM_GPU_SSA_ESTATE, "pism_gpu_ssa_set_inputs was not called");
  const size_t N = h->N;
  RET(ec_buffers(h));
  const int8_t *m = h->mask;
  if (mask) {
    const double *dm = mask;
    if (where == PISM_MEM_HOST) {
      RET(copy_in(h, h->ec + EC_MASK * N, mask, sizeof(double) * N, PISM_MEM_HOST));
      dm = h->ec + EC_MASK * N;
    }
    launch_mask_from_doubles(h->L, h->N, dm, h->ec_mask, nullptr);
    m = h->ec_mask;
  }
  double *de = (edot && where == PISM_MEM_HOST) ? h->ec + EC_EDOT * N : edot;
  double *ds = (stresses && where == PISM_MEM_HOST) ? h->ec + EC_STRESS * N : stresses;
  launch_strain_rates(h->L, h->g, h->cfg, h->vel, m, de, ds);
  CK(h, cudaGetLastError());
  if (edot && where == PISM_MEM_HOST) RET(copy_out(h, edot, de, sizeof(double) * 2 * N, PISM_MEM_HOST));
  if (stresses && where == PISM_MEM_HOST) RET(copy_out(h, stresses, ds, sizeof(double) * 3 * N, PISM_MEM_HOST));
  CK(h, cudaStreamSynchronize(h->stream));
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_eigen_calving(pism_gpu_ssa *h, double dt, double K, double *mask, double *Href, double *thickness,
                               int where) {
  if (!h || !mask || !Href || !thickness) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  if (where != PISM_MEM_HOST && where != PISM_MEM_DEVICE) return fail(h, PISM_GPU_SSA_EINVAL, "bad memory kind");
  if (!h->inputs_set) return fail(h, PISM_GPU_SSA_ESTATE, "pism_gpu_ssa_set_inputs was not called");
  if (!(dt >= 0.0) || !(K >= 0.0)) return fail(h, PISM_GPU_SSA_EINVAL, "dt and eigen_calving_K must be >= 0");
  RET(ec_buffers(h));
  const size_t N = h->N;
  double *dm = mask, *dHref = Href, *dH = thickness;
  if (where == PISM_MEM_HOST) {
    dm = h->ec + EC_MASK * N;
    dHref = h->ec + EC_HREF * N;
    dH = h->ec + EC_H * N;
    RET(copy_in(h, dm, mask, sizeof(double) * N, PISM_MEM_HOST));
    RET(copy_in(h, dHref, Href, sizeof(double) * N, PISM_MEM_HOST));
    RET(copy_in(h, dH, thickness, sizeof(double) * N, PISM_MEM_HOST));
  }
  int8_t *m0 = h->ec_mask, *live = h->ec_mask + N;
  int *changed = reinterpret_cast<int *>(h->ec + EC_SCALARS * N + 3);
  launch_mask_from_doubles(h->L, h->N, dm, m0, live);
  launch_eigen_calving_passes(h->L, h->g, h->vel, K, dt, dH, dHref, h->ec + EC_LOSS * N, m0, live);
  // remove_narrow_tongues: sweep until no cell changes; a chain of dependent cells is at
  // most N long, so N + 1 sweeps always reach the fixed point
  for (size_t sweep = 0;; ++sweep) {
    if (sweep > N) return fail(h, PISM_GPU_SSA_ECUDA, "remove_narrow_tongues did not settle");
    CK(h, cudaMemsetAsync(changed, 0, sizeof(int), h->stream));
    launch_tongue_sweep(h->L, h->g, m0, live, changed);
    CK(h, cudaGetLastError());
    int flag = 0;
    RET(copy_out(h, &flag, changed, sizeof(int), PISM_MEM_HOST));
    if (!flag) break;
  }
  launch_eigen_calving_finish(h->L, h->N, m0, live, dH, dm);
  CK(h, cudaGetLastError());
  if (where == PISM_MEM_HOST) {
    RET(copy_out(h, mask, dm, sizeof(double) * N, PISM_MEM_HOST));
    RET(copy_out(h, Href, dHref, sizeof(double) * N, PISM_MEM_HOST));
    RET(copy_out(h, thickness, dH, sizeof(double) * N, PISM_MEM_HOST));
  }
  CK(h, cudaStreamSynchronize(h->stream));
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_eigen_calving_max_timestep(pism_gpu_ssa *h, double K, const double *mask, double *result,
                                            int where) {
  if (!h || !mask || !result) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  if (where != PISM_MEM_HOST && where != PISM_MEM_DEVICE) return fail(h, PISM_GPU_SSA_EINVAL, "bad memory kind");
  if (!h->inputs_set) return fail(h, PISM_GPU_SSA_ESTATE, "pism_gpu_ssa_set_inputs was not called");
  if (!(K >= 0.0)) return fail(h, PISM_GPU_SSA_EINVAL, "eigen_calving_K must be >= 0");
  RET(ec_buffers(h));
  const size_t N = h->N;
  const double *dm = mask;
  if (where == PISM_MEM_HOST) {
    RET(copy_in(h, h->ec + EC_MASK * N, mask, sizeof(double) * N, PISM_MEM_HOST));
    dm = h->ec + EC_MASK * N;
  }
  double *stats = h->ec + EC_SCALARS * N;   // count, sum of rates, maximum rate (bits)
  CK(h, cudaMemsetAsync(stats, 0, 3 * sizeof(double), h->stream));
  launch_mask_from_doubles(h->L, h->N, dm, h->ec_mask, nullptr);
  launch_eigen_calving_rates(h->L, h->g, h->vel, h->ec_mask, K, stats,
                             reinterpret_cast<unsigned long long *>(stats + 2));
  CK(h, cudaGetLastError());
  double s[3];
  RET(copy_out(h, s, stats, sizeof(s), PISM_MEM_HOST));
  // PISMEigenCalving.cc:324-340, with units::convert's year of 31556925.9747 s
  const double secpera = 31556925.9747, dx = h->grid.dx, dy = h->grid.dy;
  const double count = s[0], rmax = s[2], mean = count > 0.0 ? s[1] / count : 0.0;
  const double epsilon = 0.001 / (dx + dy) / secpera, dt_min = 0.001 * secpera;
  const double dt = 1.0 / (rmax / dx + epsilon);
  result[0] = std::max(dt, dt_min);
  result[1] = rmax;
  result[2] = mean;
  result[3] = count;
  return PISM_GPU_SSA_OK;
}

void pism_gpu_ssafem_options_defaults(pism_gpu_ssafem_options *o) {
  if (!o) return;
  o->snes_rtol = 1e-8;
  o->snes_stol = 1e-8;
  o->snes_max_it = 200;
  o->ksp_rtol = 1e-5;
  o->ksp_max_it = 10000;
  o->dirichlet_scale = 1.0e9;
  o->icefree_thickness = 0.01;       // pism_config.cdl mask_icefree_thickness_standard
  o->is_floating_thickness = 1.0;    // pism_config.cdl mask_is_floating_thickness_standard
}

int pism_gpu_ssafem_solve(pism_gpu_ssa *h, const pism_gpu_ssafem_options *o, pism_gpu_ssafem_stats *stats) {
  if (!h || !o) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  if (!h->inputs_set) return fail(h, PISM_GPU_SSA_ESTATE, "pism_gpu_ssa_set_inputs was not called");
  if (h->cfg.flow_law != PISM_FLOW_LAW_ISOTHERMAL_GLEN && !h->have_enthalpy)
    return fail(h, PISM_GPU_SSA_EINVAL, "the flow law needs enthalpy");
  if (h->grid.Mx < 2 || h->grid.My < 2) return fail(h, PISM_GPU_SSA_EINVAL, "SSAFEM needs Mx, My >= 2");
  if (!(o->snes_rtol >= 0.0) || !(o->snes_stol >= 0.0) || o->snes_max_it < 0 || !(o->ksp_rtol > 0.0) ||
      o->ksp_max_it < 1 || !(o->dirichlet_scale > 0.0))
    return fail(h, PISM_GPU_SSA_EINVAL, "bad SSAFEM options");
  FemState &S = h->fem;
  if (fem_allocate(S, h->grid.Mx, h->grid.My, h->grid.periodicity) != 0)
    return fail(h, PISM_GPU_SSA_ENOMEM, "SSAFEM buffers");
  FemProblem P;
  P.Mx = h->grid.Mx;
  P.My = h->grid.My;
  P.periodicity = h->grid.periodicity;
  P.c = h->cfg;
  P.W = fem_germs(h->grid.dx, h->grid.dy);
  P.scale = o->dirichlet_scale;
  P.notional_strength = h->cfg.constant_nu_strength_extension_ssa * h->cfg.min_thickness_strength_extension_ssa;
  const Launch &L = h->L;
  const int Mz = (int)h->z_host.size();
  if (h->cfg.flow_law != PISM_FLOW_LAW_ISOTHERMAL_GLEN && Mz < 2)
    return fail(h, PISM_GPU_SSA_EINVAL, "the column-averaged hardness needs a grid with Mz >= 2 levels");
  launch_fem_coefficients(L, P, S, h->H, h->bed, h->tauc, h->srf, h->have_enthalpy ? h->enthalpy : nullptr,
                          h->z_dev, Mz, o->icefree_thickness, o->is_floating_thickness);
  CK(h, cudaMemsetAsync(S.zero_pivot, 0, sizeof(int), h->stream));
  FemScalars sc{};
  FemCG cg{};
  pism_gpu_ssafem_stats st{};
  double2 *vel = h->vel;
  // SSAFEM::solve_nocache keeps the velocity of a failed solve (SSAFEM.cc:215-228)
  CK(h, cudaMemcpyAsync(S.vel0, vel, sizeof(double2) * h->N, cudaMemcpyDeviceToDevice, h->stream));
  launch_fem_residual(L, P, S, vel, S.F, false, h->bc, h->bcv);
  CK(h, cudaGetLastError());
  RET(copy_out(h, &sc, S.sc, sizeof(sc), PISM_MEM_HOST));
  double fn = sqrt(sc.f2);
  st.fnorm0 = fn;
  const double f0 = fn;
  int rc = PISM_GPU_SSA_OK;
  // SNES Newton (SNESNEWTONLS): the convergence tests of SNESConvergedDefault with atol 0
  while (true) {
    if (!std::isfinite(fn)) {
      rc = fail(h, PISM_GPU_SSA_ENAN, "SSAFEM: non-finite residual");
      break;
    }
    if (fn <= o->snes_rtol * f0 || fn == 0.0) {
      st.converged = 1;
      break;
    }
    if (st.newton_iterations >= o->snes_max_it) {
      rc = fail(h, PISM_GPU_SSA_EPICARD, "SSAFEM solve failed to converge (%d Newton steps, ||F|| %g of %g)",
                st.newton_iterations, fn, f0);
      break;
    }
    // the Jacobian at the current iterate (its residual is the one already held)
    launch_fem_residual(L, P, S, vel, S.F, true, h->bc, h->bcv);
    launch_fem_cg_init(L, P, S, o->ksp_rtol, o->ksp_max_it);
    CK(h, cudaGetLastError());
    int zp = 0;
    RET(copy_out(h, &zp, S.zero_pivot, sizeof(int), PISM_MEM_HOST));
    if (zp) {
      rc = fail(h, PISM_GPU_SSA_EZERODIAG, "SSAFEM: singular diagonal block at node %d", zp - 1);
      break;
    }
    // conjugate gradients in batches of FEM_CG_BATCH iterations, each skipped on the device once
    // done; the batch is captured into a CUDA graph on first use (its buffers never move) and
    // replayed, with direct launches if the capture fails
    if (!S.cg_batch && !S.cg_batch_failed && h->cfg.graphs >= 1) {
      cudaGraph_t graph = nullptr;
      const long long before = h->stats.kernel_launches;
      bool ok = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (ok) {
        launch_fem_cg_iterations(L, P, S, FEM_CG_BATCH);
        ok = cudaStreamEndCapture(h->stream, &graph) == cudaSuccess && graph != nullptr;
      }
      if (ok) ok = cudaGraphInstantiate(&S.cg_batch, graph, 0) == cudaSuccess;
      if (graph) cudaGraphDestroy(graph);
      if (!ok) {
        S.cg_batch = nullptr;
        S.cg_batch_failed = true;
        cudaGetLastError();   // clear the capture's error; the direct launches follow
      }
      h->stats.kernel_launches = before;   // nothing ran during the capture
    }
    for (;;) {
      if (S.cg_batch) {
        CK(h, cudaGraphLaunch(S.cg_batch, h->stream));
        L.tick(3 * FEM_CG_BATCH);
      } else {
        launch_fem_cg_iterations(L, P, S, FEM_CG_BATCH);
      }
      CK(h, cudaGetLastError());
      RET(copy_out(h, &cg, S.cg, sizeof(cg), PISM_MEM_HOST));
      if (cg.done) break;
    }
    st.ksp_iterations += cg.its;
    if (cg.done != 1) {
      rc = fail(h, PISM_GPU_SSA_EKSP, "SSAFEM: the linear solve %s after %d iterations",
                cg.done == 2 ? "broke down (J not positive definite)" : "reached ksp_max_it", cg.its);
      break;
    }
    // backtracking line search on ||F||
    double lambda = 1.0, ft = 0.0;
    for (;;) {
      launch_fem_trial(L, S, vel, lambda);
      launch_fem_residual(L, P, S, S.trial, S.Ft, false, h->bc, h->bcv);
      CK(h, cudaGetLastError());
      RET(copy_out(h, &sc, S.sc, sizeof(sc), PISM_MEM_HOST));
      ft = sqrt(sc.f2);
      if (ft < (1.0 - 1e-4 * lambda) * fn || lambda < 1e-6) break;
      lambda *= 0.5;
    }
    // accept the step: the trial point becomes the iterate
    CK(h, cudaMemcpyAsync(vel, S.trial, sizeof(double2) * h->N, cudaMemcpyDeviceToDevice, h->stream));
    CK(h, cudaMemcpyAsync(S.F, S.Ft, sizeof(double2) * h->N, cudaMemcpyDeviceToDevice, h->stream));
    st.newton_iterations += 1;
    const double prev = fn;
    fn = ft;
    if (sqrt(sc.step2) <= o->snes_stol * sqrt(sc.x2) && fn <= prev) {
      st.converged = 2;
      break;
    }
  }
  st.fnorm = fn;
  if (stats) *stats = st;
  if (rc != PISM_GPU_SSA_OK)
    CK(h, cudaMemcpyAsync(vel, S.vel0, sizeof(double2) * h->N, cudaMemcpyDeviceToDevice, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return rc;
}

int pism_gpu_ssa_assemble_rhs(pism_gpu_ssa *h) {
  if (!h) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  if (!h->inputs_set) return fail(h, PISM_GPU_SSA_ESTATE, "pism_gpu_ssa_set_inputs was not called");
  launch_prepare(h->L, h->g, h->cfg, h->grid.periodicity, fields_of(h));
  CK(h, cudaGetLastError());
  CK(h, cudaStreamSynchronize(h->stream));
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_compute_hardness(pism_gpu_ssa *h) {
  if (!h) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  if (!h->inputs_set) return fail(h, PISM_GPU_SSA_ESTATE, "pism_gpu_ssa_set_inputs was not called");
  if (h->have_hardness) return PISM_GPU_SSA_OK;
  if (h->cfg.flow_law != PISM_FLOW_LAW_ISOTHERMAL_GLEN && !h->have_enthalpy)
    return fail(h, PISM_GPU_SSA_EINVAL, "the flow law needs enthalpy (or a precomputed hardness)");
  launch_hardness(h->L, h->g, h->cfg, fields_of(h), (int)h->z_host.size(), h->z_dev);
  CK(h, cudaGetLastError());
  CK(h, cudaStreamSynchronize(h->stream));
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_compute_nuH(pism_gpu_ssa *h, double reg) {
  if (!h) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  if (!h->inputs_set) return fail(h, PISM_GPU_SSA_ESTATE, "pism_gpu_ssa_set_inputs was not called");
  launch_nuH(h->L, h->g, h->cfg, fields_of(h), reg, 1.0, false, h->norm_dev);
  CK(h, cudaGetLastError());
  CK(h, cudaStreamSynchronize(h->stream));
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_apply(pism_gpu_ssa *h, const double *x_dev, double *y_dev) {
  if (!h || !x_dev || !y_dev) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  launch_apply(h->L, h->g, fields_of(h), (const double2 *)x_dev, (double2 *)y_dev);
  CK(h, cudaGetLastError());
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_apply_preconditioner(pism_gpu_ssa *h, const double *r_dev, double *z_dev) {
  if (!h || !r_dev || !z_dev) return PISM_GPU_SSA_EINVAL;
  if (r_dev == z_dev) return fail(h, PISM_GPU_SSA_EINVAL, "apply_preconditioner: r and z must be different vectors");
  DeviceGuard dg(h->device);
  RET(pc_setup(h));
  launch_pc_apply(h->L, h->g, fields_of(h), h->K.dinv, active_mg(h), active_line(h), (const double2 *)r_dev,
                  (double2 *)z_dev);
  CK(h, cudaGetLastError());
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_linear_solve_rhs(pism_gpu_ssa *h, const double *b_dev, double *x_dev, int *iterations,
                                  double *rel_residual) {
  if (!h || !b_dev || !x_dev) return PISM_GPU_SSA_EINVAL;
  if (b_dev == x_dev) return fail(h, PISM_GPU_SSA_EINVAL, "linear_solve_rhs: b and x must be different vectors");
  // the solve reads its right-hand side through h->rhs (outside any captured graph)
  double2 *keep = h->rhs;
  h->rhs = const_cast<double2 *>(reinterpret_cast<const double2 *>(b_dev));
  const int rc = pism_gpu_ssa_linear_solve(h, x_dev, iterations, rel_residual);
  h->rhs = keep;
  return rc;
}

int pism_gpu_ssa_linear_solve(pism_gpu_ssa *h, double *x_dev, int *iterations, double *rel_residual) {
  if (!h || !x_dev) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  RET(pc_setup(h));
  int its = 0, status = 0;
  if (h->cfg.precision == PISM_PRECISION_MIXED && active_mg(h))
    RET(linear_solve_mixed(h, (double2 *)x_dev, h->cfg.ksp_rtol, &its, &status));
  else
    if (h->cfg.ksp_type == PISM_KSP_GMRES)
      RET(linear_solve_gmres(h, (double2 *)x_dev, h->cfg.ksp_rtol, &its, &status));
    else
      RET(linear_solve(h, (double2 *)x_dev, h->cfg.ksp_rtol, &its, &status));
  if (iterations) *iterations = its;
  if (rel_residual) *rel_residual = h->stats.final_linear_residual;
  if (status != KSP_OK)
    return fail(h, PISM_GPU_SSA_EKSP, "SSAFD KSP (linear solver) failed: reason %d after %d iterations", status, its);
  return PISM_GPU_SSA_OK;
}

// ---- the learned initial guess (include/pism_unet_gpu.h) ----
namespace {

int learned_image(pism_gpu_ssa *h, int stride, int *height, int *width) {
  if (stride < 1 || stride > 2) return fail(h, PISM_GPU_SSA_EINVAL, "stride must be 1 or 2");
  *height = ((h->g.Mx + stride - 1) / stride + 7) / 8 * 8;
  *width = ((h->g.My + stride - 1) / stride + 7) / 8 * 8;
  if (!h->prepared) RET(prepare(h));
  return PISM_GPU_SSA_OK;
}

}  // namespace

int pism_gpu_ssa_learned_features(pism_gpu_ssa *h, int stride, float *features_dev, int height, int width) {
  if (!h || !features_dev) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  int hh = 0, ww = 0;
  RET(learned_image(h, stride, &hh, &ww));
  if (height < (h->g.Mx + stride - 1) / stride || width < (h->g.My + stride - 1) / stride)
    return fail(h, PISM_GPU_SSA_EINVAL, "feature image %d x %d is smaller than the grid at stride %d", height, width,
                stride);
  pism_unet::launch_features(h->stream, h->g.Mx, h->g.My, stride, h->H, h->bed, h->tauc, h->hardness, h->mask,
                             h->taud, features_dev, height, width);
  CK(h, cudaGetLastError());
  CK(h, cudaStreamSynchronize(h->stream));
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_learned_guess(pism_gpu_ssa *h, pism_gpu_unet *net, int stride) {
  if (!h || !net) return PISM_GPU_SSA_EINVAL;
  if (pism_unet::device_of(net) != h->device)
    return fail(h, PISM_GPU_SSA_EINVAL, "network and solver on different devices");
  DeviceGuard dg(h->device);
  int hh = 0, ww = 0;
  RET(learned_image(h, stride, &hh, &ww));
  const size_t pix = (size_t)hh * ww;
  if (pix > h->lcap) {
    if (h->lfeat) cudaFree(h->lfeat);
    if (h->lout) cudaFree(h->lout);
    h->lfeat = h->lout = nullptr;
    h->lcap = 0;
    CK(h, cudaMalloc((void **)&h->lfeat, pix * 8 * sizeof(float)));
    CK(h, cudaMalloc((void **)&h->lout, pix * 2 * sizeof(float)));
    h->lcap = pix;
  }
  pism_unet::launch_features(h->stream, h->g.Mx, h->g.My, stride, h->H, h->bed, h->tauc, h->hardness, h->mask,
                             h->taud, h->lfeat, hh, ww);
  CK(h, cudaGetLastError());
  // the network runs on the solver's stream for this call
  cudaStream_t ns = pism_unet::stream_of(net);
  pism_gpu_unet_set_stream(net, h->stream);
  const int rc = pism_gpu_unet_forward(net, h->lfeat, 1, hh, ww, h->lout);
  pism_gpu_unet_set_stream(net, ns);
  if (rc != PISM_GPU_SSA_OK)
    return fail(h, rc, "learned guess: network forward failed: %s", pism_gpu_unet_last_error(net));
  pism_unet::launch_velocity(h->stream, h->lout, hh, ww, stride, h->g.Mx, h->g.My, 31556925.9747, h->vel);
  CK(h, cudaGetLastError());
  CK(h, cudaStreamSynchronize(h->stream));
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_set_learned_pc(pism_gpu_ssa *h, pism_gpu_unet *net, int stride) {
  if (!h) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  auto &P = h->lpc;
  if (!net) {
    P.net = nullptr;
    return PISM_GPU_SSA_OK;
  }
  if (pism_unet::device_of(net) != h->device)
    return fail(h, PISM_GPU_SSA_EINVAL, "network and solver on different devices");
  if (stride < 1 || stride > 2) return fail(h, PISM_GPU_SSA_EINVAL, "stride must be 1 or 2");
  const int hh = ((h->g.Mx + stride - 1) / stride + 7) / 8 * 8, ww = ((h->g.My + stride - 1) / stride + 7) / 8 * 8;
  if (!P.r || hh != P.height || ww != P.width) {
    for (void *q : {(void *)P.img, (void *)P.out, (void *)P.r, (void *)P.d, (void *)P.ad, (void *)P.part,
                     (void *)P.rho, (void *)P.gamma})
      if (q) cudaFree(q);
    P = {};
    CK(h, cudaMalloc((void **)&P.img, (size_t)hh * ww * 8 * sizeof(float)));
    CK(h, cudaMemset(P.img, 0, (size_t)hh * ww * 8 * sizeof(float)));
    CK(h, cudaMalloc((void **)&P.out, (size_t)hh * ww * 2 * sizeof(float)));
    CK(h, cudaMalloc((void **)&P.r, sizeof(double2) * h->N));
    CK(h, cudaMalloc((void **)&P.d, sizeof(double2) * h->N));
    CK(h, cudaMalloc((void **)&P.ad, sizeof(double2) * h->N));
    CK(h, cudaMalloc((void **)&P.gamma, sizeof(double)));
    CK(h, cudaMalloc((void **)&P.part, sizeof(double) * pism_unet::pc_parts(hh, ww)));
    CK(h, cudaMalloc((void **)&P.rho, sizeof(double)));
  }
  P.net = net;
  P.stride = stride;
  P.height = hh;
  P.width = ww;
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_learned_pc_input(pism_gpu_ssa *h, int stride, const double *r_dev, float *image_dev, int height,
                                  int width, double *rho_dev) {
  if (!h || !r_dev || !image_dev || !rho_dev) return PISM_GPU_SSA_EINVAL;
  DeviceGuard dg(h->device);
  int hh = 0, ww = 0;
  RET(learned_image(h, stride, &hh, &ww));
  if (height < (h->g.Mx + stride - 1) / stride || width < (h->g.My + stride - 1) / stride)
    return fail(h, PISM_GPU_SSA_EINVAL, "image %d x %d is smaller than the grid at stride %d", height, width, stride);
  RET(pc_setup(h));   // D^-1 at the current nu*H and beta
  double *part = nullptr;
  CK(h, cudaMalloc((void **)&part, sizeof(double) * pism_unet::pc_parts(height, width)));
  pism_unet::launch_features(h->stream, h->g.Mx, h->g.My, stride, h->H, h->bed, h->tauc, h->hardness, h->mask,
                             h->taud, image_dev, height, width);
  pism_unet::launch_pc_input(h->stream, h->g.Mx, h->g.My, stride, (const double2 *)r_dev, h->K.dinv, image_dev,
                             height, width, part, rho_dev, nullptr);
  const cudaError_t e = cudaGetLastError();
  cudaStreamSynchronize(h->stream);
  cudaFree(part);
  CK(h, e);
  return PISM_GPU_SSA_OK;
}

int pism_gpu_ssa_solve_batch(pism_gpu_ssa *h, pism_gpu_unet *net, int stride, int n, pism_gpu_ssa_member *members,
                             pism_gpu_ssa_stats *stats) {
  if (!h || n < 0 || (n > 0 && !members)) return PISM_GPU_SSA_EINVAL;
  const double A0 = h->cfg.ice_softness;
  int first = PISM_GPU_SSA_OK;
  for (int q = 0; q < n; ++q) {
    pism_gpu_ssa_member &m = members[q];
    if (!m.velocity) {
      h->cfg.ice_softness = A0;
      return fail(h, PISM_GPU_SSA_EINVAL, "member %d: velocity is NULL", q);
    }
    h->cfg.ice_softness = m.ice_softness > 0.0 ? m.ice_softness : A0;
    int rc = pism_gpu_ssa_set_inputs(h, &m.inputs);
    if (rc == PISM_GPU_SSA_OK)
      rc = net ? pism_gpu_ssa_learned_guess(h, net, stride)
               : pism_gpu_ssa_set_initial_guess(h, m.velocity, m.inputs.where);
    if (rc == PISM_GPU_SSA_OK) rc = pism_gpu_ssa_solve(h, m.velocity, m.inputs.where, stats ? &stats[q] : nullptr);
    else if (stats) {
      stats[q] = pism_gpu_ssa_stats{};
      stats[q].status = rc;
    }
    if (rc == PISM_GPU_SSA_EINVAL || rc == PISM_GPU_SSA_ECUDA || rc == PISM_GPU_SSA_ENOMEM ||
        rc == PISM_GPU_SSA_ESTATE || rc == PISM_GPU_SSA_ETOOLARGE) {
      h->cfg.ice_softness = A0;
      return rc;
    }
    if (rc != PISM_GPU_SSA_OK && first == PISM_GPU_SSA_OK) first = rc;
  }
  h->cfg.ice_softness = A0;
  h->prepared = false;
  return first;
}

}  // extern "C"
