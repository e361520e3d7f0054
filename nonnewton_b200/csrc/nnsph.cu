// nnsph.cu — libnnsph.so: context, C ABI (include/nnsph.h) and step orchestration.
//
// One step (SPHBase.step, SPH/main.py:915-940) is a fixed sequence of kernels; the
// three data-dependent solver loops (divergence, implicit-viscosity CG, pressure)
// become CUDA-graph while-nodes whose condition is set on the device by the loop's
// check kernel, so a step runs without a host round-trip. A host-driven mode (one
// stream sync per iteration, like the reference's Python loops) is kept for the
// per-pass API and as a fallback.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstddef>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "ns.cuh"
#include "sph.cuh"

namespace {

constexpr double kPi = 3.14159265358979323846;

enum SyncMask : uint32_t {
  SM_X = 1, SM_V = 2, SM_A = 4, SM_VOL = 8, SM_DENS = 16, SM_ALPHA = 32, SM_RHOADV = 64, SM_NNV = 128, SM_MASS = 256,
  SM_ALL = 511
};

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) return cudaSuccess;
  return cudaMalloc((void**)p, count * sizeof(T));
}

}  // namespace

// Default launch shape of the neighbour passes: the autotuner's pick for the
// 2.4M-particle dam break on B200 (128 threads was the fastest of {128, 256, 512};
// cell factor 1 of {1, 2}). Neighbour chains in flight per thread (`unroll`): 0 gives
// each pass its own depth (U_* below); 1, 2 or 4 sets all of them.
#define NN_DEFAULT_BLOCK 128
#define NN_DEFAULT_UNROLL 0
#define NN_DEFAULT_XSPLIT 2  // 2.4M scene: list build 0.66 -> 0.60 ms, step -0.7 % (x split 3 and 4: slower steps)

struct nn_ctx {
  int cap = 0, max_scenes = 0, max_nb = 0;
  int64_t max_cells = 0;
  int dev_id = 0, sms = 148;
  cudaStream_t stream = nullptr;      // caller stream (0 = legacy default)
  cudaStream_t side = nullptr;        // capture stream for loop bodies
  cudaStream_t own = nullptr;         // execution stream when the caller sets none
  std::string err;
  int64_t launches = 0;
  int block = NN_DEFAULT_BLOCK;
  int unroll = NN_DEFAULT_UNROLL;      // neighbour chains in flight per thread (1, 2, 4; 0: per pass)
  int cell_factor = 1;                 // cells of edge h / cell_factor
  int x_split = NN_DEFAULT_XSPLIT;     // x cells per cell edge
  // state binding and scenes
  nn_state state{};
  bool bound = false;
  std::vector<nn_scene_desc> scenes;
  std::vector<SceneDev> sdev;
  int n = 0, ncells = 0, ne = 0;
  bool any_fluid = false, any_div = false, any_nonnewton = false, any_implicit = false, any_cfl = false;
  int forces_feat = 0;                 // FF_* terms of the force pass any scene needs
  bool fold_np = false;                // the step takes the fluid's non-pressure terms from the
                                       // divergence loop's last density change (no force pass)
  int el_mult_max = 0;
  // device buffers
  WorkSet set[2]{};
  int cur = 0;                         // set holding the current slots
  bool searched = false;
  bool resident_ok = false;            // the slots hold the state the last nn_step left
  int32_t* d_n = nullptr;
  SceneDev* d_sc = nullptr;
  SceneDyn* d_dyn = nullptr;
  double* d_acc = nullptr;
  int32_t* d_scene_of_id = nullptr;
  int32_t* d_src_flag = nullptr;
  real4* acc4 = nullptr;
  real *alpha = nullptr, *rho_adv = nullptr, *kappa = nullptr, *srn = nullptr, *mu = nullptr;
  int32_t* slot_of_id = nullptr;
  uint32_t *key = nullptr, *rank = nullptr, *cell_count = nullptr, *tile_sums = nullptr;
  int32_t *src = nullptr, *nbr = nullptr, *nbr_cnt = nullptr;
  real4 *cg_x = nullptr, *cg_r = nullptr, *cg_z = nullptr, *cg_p = nullptr, *cg_Ap = nullptr, *cg_pos = nullptr;
  real2* cg_aux = nullptr;
  real* cg_pinv = nullptr;
  int el_cap = 64, el_stride = 0;
  bool el_stale = false;               // rest lists re-sized since the last nn_initialize
  int32_t *el_id = nullptr, *el_slot = nullptr, *e_of_id = nullptr, *el_nb = nullptr, *el_cnt = nullptr;
  real4* el_x0 = nullptr;
  real *el_R = nullptr, *el_S = nullptr;
  int n_rb = 0, rb_rounds = 0, coupling_max = 1;
  int32_t *rb_of_id = nullptr, *rb_round = nullptr;
  double *rb_acc = nullptr, *rb_rest = nullptr, *rb_cm = nullptr, *rb_R = nullptr;
  int32_t* d_any = nullptr;
  int32_t* h_any = nullptr;            // pinned
  cudaEvent_t status_ev = nullptr;     // recorded after nn_status_async's copy
  int32_t* d_body = nullptr;
  int64_t fixed_nodes_per_step = 0;    // kernel nodes outside loop bodies (graph mode)
  int64_t graph_replays = 0;
  int64_t body_nodes[3] = {3, 3, 5};   // kernels per loop body: divergence, pressure, CG
  // graphs: [parity]
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  bool in_capture = false;
  unsigned long long cur_handle = 0;
  int64_t capture_nodes = 0;
  std::map<const void*, int> occ;      // blocks per SM per kernel
  uint64_t graph_sig = 0;              // features the captured graphs were built for
};

// The kernels and loops a captured step contains depend only on these features.
static uint64_t feature_sig(const nn_ctx* c) {
  return (uint64_t)c->any_fluid | ((uint64_t)c->any_div << 1) | ((uint64_t)c->any_nonnewton << 2) |
         ((uint64_t)c->any_implicit << 3) | ((uint64_t)std::min(c->el_mult_max, 255) << 8) |
         ((uint64_t)(c->ne > 0) << 16) | ((uint64_t)c->block << 20) |
         ((uint64_t)c->forces_feat << 40) | ((uint64_t)c->fold_np << 48);
}

static thread_local char g_err[512];

static int fail(nn_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  snprintf(g_err, sizeof(g_err), "%s", buf);
  return code;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t _e = (call);                                                                  \
    if (_e != cudaSuccess) return fail(c, NN_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, __LINE__); \
  } while (0)

static Dev make_dev(nn_ctx* c, int cur) {
  Dev d{};
  d.d_n = c->d_n;
  d.sc = c->d_sc;
  d.dyn = c->d_dyn;
  d.acc = c->d_acc;
  d.scene_of_id = c->d_scene_of_id;
  const nn_state& s = c->state;
  d.t = Truth{s.x, s.x_0, s.v, s.acceleration, s.volume, s.m, s.density, s.dfsph_factor, s.density_adv,
              s.material, s.is_dynamic, s.phase_id, s.strain_rate_norm, s.nonnewton_viscosity, s.stress, s.rotations};
  d.w = c->set[cur];
  d.wo = c->set[1 - cur];
  d.src_from_truth = c->d_src_flag;
  d.acc4 = c->acc4;
  d.alpha = c->alpha;
  d.rho_adv = c->rho_adv;
  d.kappa = c->kappa;
  d.slot_of_id = c->slot_of_id;
  d.key = c->key;
  d.rank = c->rank;
  d.src = c->src;
  d.cell_count = c->cell_count;
  d.tile_sums = c->tile_sums;
  d.nbr = c->nbr;
  d.nbr_cnt = c->nbr_cnt;
  d.cap = c->cap;
  d.max_nb = c->max_nb;
  d.srn = c->srn;
  d.mu = c->mu;
  d.cg_x = c->cg_x; d.cg_r = c->cg_r; d.cg_z = c->cg_z; d.cg_p = c->cg_p; d.cg_Ap = c->cg_Ap; d.cg_pos = c->cg_pos;
  d.cg_aux = c->cg_aux;
  d.cg_pinv = c->cg_pinv;
  d.el_id = c->el_id; d.el_slot = c->el_slot; d.e_of_id = c->e_of_id; d.el_x0 = c->el_x0;
  d.el_nb = c->el_nb; d.el_cnt = c->el_cnt; d.el_cap = c->el_cap; d.el_stride = c->el_stride;
  d.el_R = c->el_R; d.el_S = c->el_S;
  d.n_rb = c->n_rb; d.rb_of_id = c->rb_of_id; d.rb_round = c->rb_round; d.rb_acc = c->rb_acc;
  d.rb_rest = c->rb_rest; d.rb_cm = c->rb_cm; d.rb_R = c->rb_R;
  d.any_active = c->d_any;
  d.loop_handle = c->cur_handle;
  d.body_count = c->d_body;
  return d;
}

// Launch helpers: grids are a multiple of the SM count (resident blocks per SM from
// the occupancy calculator), capped by the work; kernels grid-stride over device sizes.
template <typename... KArgs, typename... Args>
static int launch(nn_ctx* c, cudaStream_t s, void (*k)(KArgs...), int block, int work, Args... args) {
  auto it = c->occ.find((const void*)k);
  int per_sm;
  if (it == c->occ.end()) {
    per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block, 0);
    per_sm = std::max(per_sm, 1);
    c->occ[(const void*)k] = per_sm;
  } else {
    per_sm = it->second;
  }
  // A captured graph must serve any batch composition up to the capacity, so its
  // grids are sized by the capacity (kernels grid-stride over the device sizes).
  if (c->in_capture) work = std::max(work, c->cap);
  int64_t want = ((int64_t)std::max(work, 1) + block - 1) / block;
  int grid = (int)std::min<int64_t>(want, (int64_t)c->sms * per_sm);
  grid = std::max(grid, 1);
  k<<<grid, block, 0, s>>>(args...);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(c, NN_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
  if (c->in_capture) c->capture_nodes++;
  else c->launches++;
  return NN_OK;
}
template <typename... KArgs, typename... Args>
static int launch1(nn_ctx* c, cudaStream_t s, void (*k)(KArgs...), Args... args) {
  k<<<1, 256, 0, s>>>(args...);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(c, NN_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
  if (c->in_capture) c->capture_nodes++;
  else c->launches++;
  return NN_OK;
}

// Each pass's neighbour-batch depth at unroll 0, measured against the other depth on
// the 2.4M-particle dam break (early and settled states): the update passes, with
// little arithmetic per pair, keep 2 neighbours in flight (at 1: k_pressure_update
// +17-31 %, k_density_adv +3 %); the passes with more arithmetic per pair gather one
// at a time, with 8 list entries loaded ahead (k_density_change_np -9 %, k_cg_setup
// -7 %, k_density_factor -6 %, k_cg_matvec -4 %, k_density_change -2 %). The force
// pass keeps 2 (the 23k-particle dam break: 29.0 against 31.0 us at 1).
enum : int {
  U_PRESSURE_UPDATE = 2, U_DENSITY_ADV = 2, U_DIVERGENCE_UPDATE = 2, U_BOUNDARY_VOLUME = 2, U_FORCES = 2,
  U_DENSITY_FACTOR = 1, U_DENSITY_CHANGE = 1, U_DENSITY_CHANGE_NP = 1, U_CG_SETUP = 1, U_CG_MATVEC = 1
};
static inline int ku(const nn_ctx* c, int pass_default) { return c->unroll ? c->unroll : pass_default; }
// The instantiation of a neighbour kernel for the context's (or the pass's) batch depth.
#define KU(k, def) (ku(c, def) == 4 ? &k<4> : ku(c, def) == 2 ? &k<2> : &k<1>)
#define KU2(k, B, def) (ku(c, def) == 4 ? &k<4, B> : ku(c, def) == 2 ? &k<2, B> : &k<1, B>)

// The force pass instance for the batch's terms (c->forces_feat) and batch depth.
template <int U, int... F>
static void (*forces_pick(int feat, std::integer_sequence<int, F...>))(Dev, int) {
  static void (*const tbl[])(Dev, int) = {forces_kernel_of<U, F>()...};
  return tbl[feat];
}
static void (*forces_kernel(const nn_ctx* c))(Dev, int) {
  using All = std::make_integer_sequence<int, 16>;
  const int f = c->forces_feat & 15;
  const int u = ku(c, U_FORCES);
  return u == 4 ? forces_pick<4>(f, All{}) : u == 2 ? forces_pick<2>(f, All{}) : forces_pick<1>(f, All{});
}

#define RC(x)                 \
  do {                        \
    int _r = (x);             \
    if (_r != NN_OK) return _r; \
  } while (0)

template <typename... KArgs, typename... Args>
static int launch_g(nn_ctx* c, cudaStream_t s, void (*k)(KArgs...), int grid, int block, Args... args) {
  k<<<std::max(grid, 1), block, 0, s>>>(args...);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(c, NN_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
  if (c->in_capture) c->capture_nodes++;
  else c->launches++;
  return NN_OK;
}

// Data-dependent solver loop. In a capture, `pre` runs in the parent graph (it may
// set the loop condition) and `body` becomes the body of a CUDA-graph while-node;
// otherwise both run from the host with one synchronisation per iteration.
// A loop without check_first always runs its body once (the DFSPH solves count from
// zero and test after the body, SPH/main.py:1695-1703, 1778-1784): that first body is
// captured straight into the parent graph, where its closing check sets the condition
// of the while-node that runs the further bodies, so a solve that stops after one body
// launches no body graph.
// Body launches are counted per execution on the device (body_count).
template <typename Pre, typename Body>
static int solver_loop(nn_ctx* c, cudaStream_t s, bool check_first, Pre pre, Body body) {
  if (c->in_capture) {
    cudaStreamCaptureStatus st;
    cudaGraph_t g;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    CK(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    c->cur_handle = (unsigned long long)h;
    int rc = pre(s);
    if (rc != NN_OK) { c->cur_handle = 0; return rc; }
    if (!check_first) {
      const int64_t first = c->capture_nodes;
      rc = body(s);
      c->capture_nodes = first;
      if (rc != NN_OK) { c->cur_handle = 0; return rc; }
    }
    CK(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, nd, &p));
    cudaGraph_t bodyg = p.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(c->side, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    int64_t before = c->capture_nodes;
    rc = body(c->side);
    c->capture_nodes = before;
    c->cur_handle = 0;
    cudaGraph_t out;
    cudaError_t e = cudaStreamEndCapture(c->side, &out);
    if (rc != NN_OK) return rc;
    if (e != cudaSuccess) return fail(c, NN_ERR_CUDA, "loop body capture: %s", cudaGetErrorString(e));
    CK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    return NN_OK;
  }
  RC(pre(s));
  if (check_first) {
    CK(cudaMemcpyAsync(c->h_any, c->d_any, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (!*c->h_any) return NN_OK;
  }
  for (int it = 0; it < 1000000; ++it) {
    int64_t before = c->launches;
    RC(body(s));
    c->launches = before;
    CK(cudaMemcpyAsync(c->h_any, c->d_any, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (!*c->h_any) break;
  }
  return NN_OK;
}

// ---- pass sequences ---------------------------------------------------------------
// NeighborhoodSearchSparse.run_search (SPH/main.py:822-829): the new slots go into the
// other working set; the source (caller state or previous slots) is a device flag.
// `reset_step`: the step's first launch (k_zero_cells) also resets its per-scene counters.
static int enq_search(nn_ctx* c, cudaStream_t s, bool reset_step = false) {
  c->cur = 1 - c->cur;
  Dev d = make_dev(c, c->cur);
  const int B = 256;
  const int64_t cells = c->in_capture ? c->max_cells : c->ncells;
  const int tiles = (int)((cells + 1 + SCAN_TILE - 1) / SCAN_TILE);
  RC(launch(c, s, k_zero_cells, B, (int)std::min<int64_t>(cells + 1, INT32_MAX), d, reset_step ? 1 : 0));
  RC(launch(c, s, k_keys, B, c->n, d));
  RC(launch_g(c, s, k_scan_tiles, std::min(tiles, c->sms * 2), SCAN_THREADS, d));
  RC(launch_g(c, s, k_scan_apply, std::min(tiles, c->sms * 2), SCAN_THREADS, d));
  RC(launch(c, s, k_scatter, B, c->n, d));
  RC(launch(c, s, k_cell_sort, B, (int)std::min<int64_t>(cells, INT32_MAX), d));
  RC(launch(c, s, k_gather, B, c->n, d));
  RC(launch(c, s, k_build_lists, NS_WARPS * 32, c->n, d));
  c->searched = true;
  return NN_OK;
}

// DFSPHSolver.divergence_solve (SPH/main.py:1683-1713). In the fused step the first
// density change and alpha *= 1/dt were done by k_density_factor<CHANGE> and the
// closing alpha *= dt is folded into the pressure solve's first pass (fused = true);
// with c->fold_np the loop's density change also computes the fluid's non-pressure terms.
static int enq_divergence(nn_ctx* c, cudaStream_t s, bool fused) {
  Dev d = make_dev(c, c->cur);
  const int B = c->block;
  const bool np = fused && c->fold_np;
  if (!fused) RC(launch1(c, s, k_solver_begin, d, 0));
  RC(solver_loop(c, s, false,
                 [&](cudaStream_t q) {
                   return fused ? NN_OK : launch(c, q, KU(k_density_change, U_DENSITY_CHANGE), B, c->n, make_dev(c, c->cur), 0, 0);
                 },
                 [&](cudaStream_t q) {
                   Dev e = make_dev(c, c->cur);
                   RC(launch(c, q, KU(k_divergence_update, U_DIVERGENCE_UPDATE), B, c->n, e));
                   RC(launch(c, q, KU(k_density_change, U_DENSITY_CHANGE), B, c->n, e, 1, np ? 1 : 0));
                   if (np) RC(launch(c, q, KU(k_density_change_np, U_DENSITY_CHANGE_NP), B, c->n, e, 1, 1));
                   return launch1(c, q, k_solver_check, e, 0, np ? 1 : 0);
                 }));
  return fused ? NN_OK : launch(c, s, k_alpha_times_dt, 256, c->n, d);
}

// DFSPHSolver.pressure_solve (SPH/main.py:1762-1791); init_mode 2 also folds the
// divergence solve's alpha *= dt.
// `begun`: the loop start is done (k_clear_acc at the start of the step).
static int enq_pressure(nn_ctx* c, cudaStream_t s, int init_mode, bool begun = false) {
  Dev d = make_dev(c, c->cur);
  const int B = c->block;
  if (!begun) RC(launch1(c, s, k_solver_begin, d, 1));
  return solver_loop(c, s, false,
                     [&](cudaStream_t q) {
                       return launch(c, q, KU(k_density_adv, U_DENSITY_ADV), B, c->n, make_dev(c, c->cur), init_mode);
                     },
                     [&](cudaStream_t q) {
                       Dev e = make_dev(c, c->cur);
                       RC(launch(c, q, KU(k_pressure_update, U_PRESSURE_UPDATE), B, c->n, e));
                       RC(launch(c, q, KU(k_density_adv, U_DENSITY_ADV), B, c->n, e, 1));
                       return launch1(c, q, k_solver_check, e, 1, 0);
                     });
}

// compute_non_pressure_forces (SPH/main.py:1557-1567), with the substep's
// clear_accelerations when `clear`, then the implicit viscosity and, when `advect`,
// non_pressure_advect. The force pass skips the scenes whose terms the divergence loop
// already computed (SceneDyn::np_fresh).
static int enq_nonpressure(nn_ctx* c, cudaStream_t s, int advect, int clear) {
  Dev d = make_dev(c, c->cur);
  const int B = c->block;
  RC(launch(c, s, forces_kernel(c), B, c->n, d, clear));
  if (c->any_implicit) {
    RC(launch(c, s, KU(k_cg_setup, U_CG_SETUP), B, c->n, d));
    RC(solver_loop(c, s, true, [&](cudaStream_t q) { return launch1(c, q, k_cg_check0, make_dev(c, c->cur)); },
                   [&](cudaStream_t q) {
                     Dev e = make_dev(c, c->cur);
                     RC(launch(c, q, KU(k_cg_matvec, U_CG_MATVEC), B, c->n, e));
                     RC(launch1(c, q, k_cg_alpha, e));
                     RC(launch(c, q, k_cg_update, 256, c->n, e));
                     RC(launch1(c, q, k_cg_check, e));
                     return launch(c, q, k_cg_pupdate, 256, c->n, e);
                   }));
  }
  if (c->any_implicit || advect) RC(launch(c, s, k_cg_finish, 256, c->n, d, advect));
  return NN_OK;
}

static int enq_elastic(nn_ctx* c, cudaStream_t s) {
  if (c->el_mult_max <= 0 || c->ne == 0) return NN_OK;
  Dev d = make_dev(c, c->cur);
  RC(launch(c, s, k_el_slots, 256, c->ne, d));
  for (int rep = 0; rep < c->el_mult_max; ++rep) {
    RC(launch(c, s, k_el_rotations, 128, c->ne, d, rep));
    RC(launch(c, s, k_el_stress, 128, c->ne, d, rep));
    RC(launch(c, s, k_el_forces, 128, c->ne, d, rep));
  }
  return NN_OK;
}

// for rb in meta.rbs: coupling_interval x RigidBodySolver.substep (SPH/main.py:929-931)
static int enq_rigid(nn_ctx* c, cudaStream_t s) {
  if (c->n_rb == 0) return NN_OK;
  Dev d = make_dev(c, c->cur);
  for (int rep = 0; rep < c->coupling_max; ++rep)
    for (int r = 0; r < c->rb_rounds; ++r) {
      RC(launch(c, s, k_rigid_ground, 256, c->n, d, r, rep));
      RC(launch(c, s, k_rigid_com, 256, c->n, d, r, 0));
      RC(launch1(c, s, k_rigid_cm, d, r, 0));
      RC(launch(c, s, k_rigid_A, 256, c->n, d, r));
      RC(launch1(c, s, k_rigid_R, d, r));
      RC(launch(c, s, k_rigid_apply, 256, c->n, d, r));
    }
  return NN_OK;
}

// DFSPHSolver.substep (SPH/main.py:1546-1555) with the fused passes.
// `begun`: the loops' start is done (k_clear_acc at the start of the step).
static int enq_substep(nn_ctx* c, cudaStream_t s, bool begun = false) {
  if (!c->any_fluid) return NN_OK;
  Dev d = make_dev(c, c->cur);
  if (c->any_div) {
    if (!begun) RC(launch1(c, s, k_solver_begin, d, 0));
    RC(launch(c, s, KU2(k_density_factor, true, U_DENSITY_FACTOR), c->block, c->n, d, 1, 1));
    RC(enq_divergence(c, s, true));
  } else {
    RC(launch(c, s, KU2(k_density_factor, false, U_DENSITY_FACTOR), c->block, c->n, d, 1, 1));
  }
  RC(enq_nonpressure(c, s, 1, 1));
  return enq_pressure(c, s, 2, begun);
}

// SPHBase.step (SPH/main.py:915-937)
static int enq_step(nn_ctx* c, cudaStream_t s) {
  // k_step_reset rides in the search's first launch, k_step_dt and the solves' loop
  // start in k_clear_acc's first block: one-block kernels cost a graph node each
  RC(enq_search(c, s, true));
  Dev d = make_dev(c, c->cur);
  RC(launch(c, s, KU(k_boundary_volume, U_BOUNDARY_VOLUME), c->block, c->n, d, 1));
  RC(launch(c, s, k_clear_acc, 256, c->n, d, c->fold_np ? 1 : 0, 1));
  RC(enq_substep(c, s, true));
  RC(enq_elastic(c, s));
  RC(enq_rigid(c, s));
  RC(launch(c, s, k_advect_boundary, 256, c->n, d, 1, 1, 1));
  return launch1(c, s, k_step_end, d);
}

static int enq_sync_out(nn_ctx* c, cudaStream_t s, uint32_t mask) {
  Dev d = make_dev(c, c->cur);
  RC(launch(c, s, k_sync_out, 256, c->n, d, mask));
  if (c->ne > 0 && (c->state.stress || c->state.rotations)) RC(launch(c, s, k_sync_out_elastic, 256, c->ne, d));
  return NN_OK;
}

static cudaStream_t run_stream(nn_ctx* c) { return c->stream ? c->stream : c->own; }

static void drop_graphs(nn_ctx* c) {
  for (int p = 0; p < 2; ++p)
    if (c->exec[p]) { cudaGraphExecDestroy(c->exec[p]); c->exec[p] = nullptr; }
}

static int capture_step(nn_ctx* c, cudaStream_t s, int parity) {
  const int saved = c->cur;
  c->cur = parity;
  c->in_capture = true;
  c->capture_nodes = 0;
  CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int rc = enq_step(c, s);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &g);
  c->in_capture = false;
  c->cur = saved;
  if (rc != NN_OK) { if (g) cudaGraphDestroy(g); return rc; }
  if (e != cudaSuccess) return fail(c, NN_ERR_CUDA, "step capture: %s", cudaGetErrorString(e));
  c->graph_sig = feature_sig(c);
  e = cudaGraphInstantiate(&c->exec[parity], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(c, NN_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  c->fixed_nodes_per_step = c->capture_nodes;
  return NN_OK;
}

// ---- scene setup ----------------------------------------------------------------------
// cubic_kernel (SPH/main.py:859-880) on the host, in the arithmetic type of the build
static real host_kernel_w(real rn, real h, real k_w, real k2_w) {
  real q = rn / h;
  real res = 0;
  if (q <= 1) {
    if (q <= real(0.5)) {
      real q2 = q * q;
      real q3 = q2 * q;
      res = k_w * (6 * q3 - 6 * q2 + 1);
    } else {
      real t = 1 - q;
      res = k2_w * (t * t * t);
    }
  }
  return res;
}

static SceneDev make_scene(const nn_scene_desc& sd, int64_t cell_base, int el_mult, int cell_factor = 1,
                           int x_split = 1) {
  const nn_scene_params& p = sd.params;
  SceneDev s{};
  s.flags = p.flags;
  s.start = sd.start;
  s.n = sd.n;
  s.n_fluid = sd.n_fluid;
  s.cell_base = cell_base;
  const double h = p.support_radius;
  int g[3];
  // Cells are 0.1 % longer than h / cell_factor: the cell of a position is computed in
  // the arithmetic type, floor((x - origin) / cell), whose rounding can move a particle
  // across a cell boundary by a few ulp of the quotient (up to about 1e-4 of a cell on
  // grids of hundreds of cells); with cells of exactly h / cell_factor a neighbour just
  // under h away could then fall outside the stencil. The margin covers that rounding.
  const double cell = h / cell_factor * (1.0 + 1e-3);
  const double cellx = cell / x_split;  // x cells may be shorter: rows stay contiguous in x
  for (int k = 0; k < 3; ++k) {
    s.origin[k] = (real)(p.domain_start[k] - 2.0 * h);
    double ext = (p.domain_end[k] - p.domain_start[k]) + 4.0 * h;
    g[k] = (int)std::min(65535.0, std::max(1.0, std::ceil(ext / (k == 0 ? cellx : cell)) + 1.0));
  }
  s.gx = g[0]; s.gy = g[1]; s.gz = g[2];
  int mb = 0;
  while ((1 << mb) < std::max(g[1], g[2])) ++mb;
  s.mbits = mb;
  s.cell = (real)cell;
  s.nf = cell_factor;
  s.cellx = (real)cellx;
  s.nfx = cell_factor * x_split;
  s.h = (real)h;
  s.inv_h = (real)(1.0 / h);
#ifdef NN_FP64
  s.h2_thr = s.h * s.h;  // the search tests r2 < h^2 in double
#else
  {  // exact squared cut-off: sqrt_rn(r2) < h  <=>  r2 < h2_thr
    float t = s.h * s.h;
    while (t > 0.f && std::sqrt(t) >= s.h) t = std::nextafter(t, 0.f);
    while (std::sqrt(t) < s.h) t = std::nextafter(t, INFINITY);
    s.h2_thr = t;
  }
#endif
  const double k = 8.0 / kPi / (h * h * h);
  s.k_w = (real)k;
  s.k2_w = (real)(k * 2.0);
  s.k_grad = (real)(6.0 * (8.0 / kPi) / (h * h * h));
  s.W0 = host_kernel_w(0.f, s.h, s.k_w, s.k2_w);
  s.rho0 = (real)p.density0;
  s.inv_rho0 = (real)(1.0 / p.density0);
  for (int q = 0; q < 3; ++q) s.g[q] = (real)p.gravity[q];
  s.eps = (real)p.eps;
  s.sigma = (real)p.surface_tension;
  const double dia = 2.0 * p.particle_radius;
  s.dia2 = (real)(dia * dia);
  s.w_dia = host_kernel_w(std::sqrt((real)dia * (real)dia), s.h, s.k_w, s.k2_w);
  s.visc = (real)p.viscosity;
  s.visc_b = (real)p.boundary_viscosity;
  s.c01h2 = (real)(0.01 * h * h);
  for (int q = 0; q < 3; ++q) {
    s.xmin[q] = (real)(p.domain_start[q] + p.padding);
    s.xmax[q] = (real)(p.domain_end[q] - p.padding);
  }
  s.cf = (real)p.collision_coeff;
  s.sticky = (real)p.sticky_coeff;
  s.eta_v_fac = p.max_error_v * 0.01 * p.density0;
  s.eta_p = p.max_error * 0.01 * p.density0;
  s.max_iter_v = std::min(std::max(p.max_iterations_v, 0), 100000);
  s.max_iter = std::min(std::max(p.max_iterations, 0), 100000);
  s.visco_max_iter = std::min(std::max(p.visco_max_iter, 0), 100000);
  s.nn_method = p.nonnewton_method;
  s.visco_tol = p.visco_max_error;
  s.nn_n = (real)p.power_index;
  s.nn_K = (real)p.consistency_index;
  s.nn_mu0 = (real)p.viscosity0;
  s.nn_muinf = (real)p.viscosity_inf;
  s.nn_gc = (real)p.critical_strain_rate;
  s.nn_muc = (real)p.mu_c;
  s.nn_tauy = (real)p.yield_stress;
  s.mu_newton = (real)(p.viscosity * p.density0);
  s.mu_b = (real)(p.visco_boundary * p.density0);
  double E = p.youngs_modulus, nu = p.poisson_ratio;
  if (p.flags & NN_F_QUIRKS) { E = 25e4; nu = 0.33; }  // SPH/main.py:1188-1189
  const double f = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
  s.el_cd = (real)(f * (1.0 - nu));
  s.el_co = (real)(f * nu);
  s.el_cs = (real)(f * 0.5 * (1.0 - 2.0 * nu));
  s.el_mult = el_mult;
  s.cfl_factor = (real)p.cfl_factor;
  s.cfl_min_dt = (real)p.cfl_min_dt;
  s.cfl_max_dt = (real)p.cfl_max_dt;
  s.diameter = (real)dia;
  s.V0 = (real)p.volume0;
  s.padding = (real)p.padding;
  s.coupling = std::max(p.coupling_interval, 1);
  return s;
}

static int ensure_cells(nn_ctx* c, int64_t cells) {
  if (cells <= c->max_cells && c->cell_count) return NN_OK;
  cudaFree(c->cell_count);
  cudaFree(c->tile_sums);
  c->cell_count = nullptr;
  c->tile_sums = nullptr;
  c->max_cells = std::max<int64_t>(cells, c->max_cells);
  CK(dalloc(&c->cell_count, (size_t)c->max_cells + 1));
  CK(dalloc(&c->tile_sums, (size_t)(c->max_cells + 1) / SCAN_TILE + 2));
  return NN_OK;
}

static void free_elastic(nn_ctx* c) {
  cudaFree(c->el_id); cudaFree(c->el_slot); cudaFree(c->el_nb); cudaFree(c->el_cnt);
  cudaFree(c->el_x0); cudaFree(c->el_R); cudaFree(c->el_S);
  c->el_id = c->el_slot = c->el_nb = c->el_cnt = nullptr;
  c->el_x0 = nullptr;
  c->el_R = c->el_S = nullptr;
  c->el_stride = 0;
}

extern "C" {

int nn_abi_version(void) { return NNSPH_ABI_VERSION; }

int nn_real_bytes(void) { return (int)sizeof(real); }

const char* nn_last_error(const nn_ctx* c) { return c ? c->err.c_str() : g_err; }

int nn_ctx_create(int32_t max_particles, int32_t max_scenes, int32_t max_neighbors, int64_t max_cells, nn_ctx** out) {
  nn_ctx* c = nullptr;
  if (!out || max_particles <= 0 || max_scenes <= 0 || max_neighbors <= 0 || max_neighbors > 1024 || max_cells < 0)
    return fail(nullptr, NN_ERR_INVALID_ARG, "nn_ctx_create: invalid capacities");
  *out = nullptr;
  c = new nn_ctx();
  c->cap = max_particles;
  c->max_scenes = max_scenes;
  c->max_nb = max_neighbors;
  c->el_cap = max_neighbors;
  auto bail = [&](int code) { nn_ctx_destroy(c); return code; };
  cudaError_t e = cudaGetDevice(&c->dev_id);
  if (e != cudaSuccess) return bail(fail(nullptr, NN_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e)));
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->dev_id);
  const size_t N = (size_t)max_particles;
#define AL(p, cnt)                                                                                   \
  do {                                                                                               \
    cudaError_t _e = dalloc(&(p), (cnt));                                                            \
    if (_e != cudaSuccess) return bail(fail(nullptr, NN_ERR_OOM, "cudaMalloc %s: %s", #p, cudaGetErrorString(_e))); \
  } while (0)
  for (int k = 0; k < 2; ++k) {
    AL(c->set[k].pos, N); AL(c->set[k].vel, N); AL(c->set[k].mass, N); AL(c->set[k].dens, N);
    AL(c->set[k].flags, N); AL(c->set[k].id, N);
  }
  AL(c->d_n, 4); AL(c->d_sc, (size_t)max_scenes); AL(c->d_dyn, (size_t)max_scenes);
  AL(c->d_acc, (size_t)max_scenes * ACC_COUNT * NN_STRIPES);
  AL(c->d_scene_of_id, N); AL(c->d_src_flag, 1); AL(c->acc4, N);
  AL(c->alpha, N); AL(c->rho_adv, N); AL(c->kappa, N); AL(c->srn, N); AL(c->mu, N);
  AL(c->slot_of_id, N); AL(c->key, N); AL(c->rank, N); AL(c->src, N);
  AL(c->nbr, N * (size_t)max_neighbors); AL(c->nbr_cnt, N);
  AL(c->cg_x, N); AL(c->cg_r, N); AL(c->cg_z, N); AL(c->cg_p, N); AL(c->cg_Ap, N); AL(c->cg_pos, N); AL(c->cg_aux, N);
  AL(c->cg_pinv, 6 * N);
  AL(c->e_of_id, N);
  AL(c->d_any, 1); AL(c->d_body, 4);
#undef AL
  if (cudaMallocHost((void**)&c->h_any, sizeof(int32_t)) != cudaSuccess)
    return bail(fail(nullptr, NN_ERR_OOM, "cudaMallocHost failed"));
  cudaMemset(c->d_acc, 0, (size_t)max_scenes * ACC_COUNT * NN_STRIPES * sizeof(double));
  cudaMemset(c->d_body, 0, 4 * sizeof(int32_t));
  cudaMemset(c->d_n, 0, 4 * sizeof(int32_t));
  cudaMemset(c->nbr_cnt, 0, N * sizeof(int32_t));
  if (cudaStreamCreateWithFlags(&c->side, cudaStreamDefault) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->own, cudaStreamDefault) != cudaSuccess)
    return bail(fail(nullptr, NN_ERR_CUDA, "cudaStreamCreate failed"));
  if (cudaEventCreateWithFlags(&c->status_ev, cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(nullptr, NN_ERR_CUDA, "cudaEventCreate failed"));
  if (max_cells > 0) {
    int rc = ensure_cells(c, max_cells);
    if (rc != NN_OK) return bail(rc);
  }
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return bail(fail(nullptr, NN_ERR_CUDA, "setup: %s", cudaGetErrorString(e)));
  *out = c;
  return NN_OK;
}

int nn_ctx_destroy(nn_ctx* c) {
  if (!c) return NN_OK;
  drop_graphs(c);
  for (int k = 0; k < 2; ++k) {
    cudaFree(c->set[k].pos); cudaFree(c->set[k].vel); cudaFree(c->set[k].mass); cudaFree(c->set[k].dens);
    cudaFree(c->set[k].flags); cudaFree(c->set[k].id);
  }
  void* bufs[] = {c->d_n, c->d_sc, c->d_dyn, c->d_acc, c->d_scene_of_id, c->d_src_flag, c->acc4, c->alpha,
                  c->rho_adv, c->kappa, c->srn, c->mu, c->slot_of_id, c->key, c->rank, c->src, c->nbr,
                  c->nbr_cnt, c->cg_x, c->cg_r, c->cg_z, c->cg_p, c->cg_Ap, c->cg_pos, c->cg_aux, c->cg_pinv,
                  c->e_of_id, c->d_any, c->d_body, c->cell_count, c->tile_sums};
  for (void* b : bufs) cudaFree(b);
  free_elastic(c);
  cudaFree(c->rb_of_id); cudaFree(c->rb_round); cudaFree(c->rb_acc); cudaFree(c->rb_rest); cudaFree(c->rb_cm);
  cudaFree(c->rb_R);
  if (c->h_any) cudaFreeHost(c->h_any);
  if (c->status_ev) cudaEventDestroy(c->status_ev);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
  return NN_OK;
}

int nn_ctx_set_stream(nn_ctx* c, void* stream) {
  if (!c) return fail(nullptr, NN_ERR_INVALID_ARG, "null context");
  if ((cudaStream_t)stream != c->stream) drop_graphs(c);
  c->stream = (cudaStream_t)stream;
  return NN_OK;
}

int nn_set_block_size(nn_ctx* c, int32_t threads) {
  if (!c) return fail(nullptr, NN_ERR_INVALID_ARG, "null context");
  if (threads == 0) threads = NN_DEFAULT_BLOCK;
  if (threads < 32 || threads > 1024 || (threads % 32)) return fail(c, NN_ERR_INVALID_ARG, "block size %d", threads);
  if (threads != c->block) drop_graphs(c);
  c->block = threads;
  c->occ.clear();
  return NN_OK;
}

int nn_set_tuning(nn_ctx* c, int32_t block, int32_t unroll, int32_t cell_factor) {
  if (!c) return fail(nullptr, NN_ERR_INVALID_ARG, "null context");
  if (block == 0) block = NN_DEFAULT_BLOCK;
  if (cell_factor == 0) cell_factor = 1;
  if (block < 32 || block > 1024 || (block % 32) || (unroll != 0 && unroll != 1 && unroll != 2 && unroll != 4) ||
      (cell_factor != 1 && cell_factor != 2))
    return fail(c, NN_ERR_INVALID_ARG, "tuning: block %d, unroll %d, cell factor %d", block, unroll, cell_factor);
  if (block != c->block || unroll != c->unroll || cell_factor != c->cell_factor) drop_graphs(c);
  if (cell_factor != c->cell_factor) c->scenes.clear();  // cell layout changes: set the scenes again
  c->block = block;
  c->unroll = unroll;
  c->cell_factor = cell_factor;
  c->occ.clear();
  return NN_OK;
}

int nn_set_x_split(nn_ctx* c, int32_t x_split) {
  if (!c) return fail(nullptr, NN_ERR_INVALID_ARG, "null context");
  if (x_split == 0) x_split = NN_DEFAULT_XSPLIT;
  if (x_split < 1 || x_split > 4) return fail(c, NN_ERR_INVALID_ARG, "x split %d (1..4)", x_split);
  if (x_split != c->x_split) {
    drop_graphs(c);
    c->scenes.clear();  // the cell layout changes: set the scenes again
  }
  c->x_split = x_split;
  return NN_OK;
}

int64_t nn_launch_count(const nn_ctx* cc) {
  nn_ctx* c = const_cast<nn_ctx*>(cc);
  if (!c) return -1;
  int32_t body[4] = {0, 0, 0, 0};
  cudaStreamSynchronize(run_stream(c));
  cudaMemcpy(body, c->d_body, sizeof(body), cudaMemcpyDeviceToHost);
  return c->launches + c->graph_replays * c->fixed_nodes_per_step + (int64_t)body[0] * c->body_nodes[0] +
         (int64_t)body[1] * c->body_nodes[1] + (int64_t)body[2] * c->body_nodes[2];
}

int nn_bind_state(nn_ctx* c, const nn_state* st) {
  if (!c || !st) return fail(c, NN_ERR_INVALID_ARG, "nn_bind_state: null argument");
  if (st->size != sizeof(nn_state)) return fail(c, NN_ERR_INVALID_ARG, "nn_state size %u != %zu", st->size, sizeof(nn_state));
  if (st->n < 0 || st->n > c->cap) return fail(c, NN_ERR_CAPACITY, "state has %d particles, capacity %d", st->n, c->cap);
  if (st->n > 0 && (!st->x || !st->x_0 || !st->v || !st->acceleration || !st->volume || !st->m || !st->density ||
                    !st->dfsph_factor || !st->density_adv || !st->material || !st->is_dynamic || !st->phase_id))
    return fail(c, NN_ERR_INVALID_ARG, "nn_bind_state: required field is NULL");
  nn_state prev = c->state;
  prev.n = st->n;
  if (std::memcmp(&prev, st, sizeof(nn_state)) != 0) drop_graphs(c);
  c->state = *st;
  c->bound = true;
  c->searched = false;
  c->resident_ok = false;
  return NN_OK;
}

int nn_set_scenes(nn_ctx* c, int32_t nscenes, const nn_scene_desc* scenes) {
  if (!c || (nscenes > 0 && !scenes) || nscenes < 0) return fail(c, NN_ERR_INVALID_ARG, "nn_set_scenes: bad arguments");
  if (!c->bound) return fail(c, NN_ERR_STATE, "nn_set_scenes: bind the state first");
  if (nscenes > c->max_scenes) return fail(c, NN_ERR_CAPACITY, "%d scenes > capacity %d", nscenes, c->max_scenes);
  const int n = c->state.n;
  std::vector<std::pair<int, int>> ranges;  // (start, scene): the scenes must tile [0, n)
  for (int k = 0; k < nscenes; ++k) {
    const nn_scene_desc& sd = scenes[k];
    if (sd.size != sizeof(nn_scene_desc) || sd.params.size != sizeof(nn_scene_params))
      return fail(c, NN_ERR_INVALID_ARG, "scene %d: struct size mismatch", k);
    if (sd.start < 0 || sd.n < 0 || sd.start + sd.n > n || sd.n_fluid < 0 || sd.n_fluid > sd.n)
      return fail(c, NN_ERR_INVALID_ARG, "scene %d: range [%d, %d) outside the state", k, sd.start, sd.start + sd.n);
    if (!(sd.params.support_radius > 0) || !(sd.params.dt > 0) || !(sd.params.density0 > 0))
      return fail(c, NN_ERR_INVALID_ARG, "scene %d: support_radius, dt and density0 must be positive", k);
    if (sd.n > 0) ranges.push_back({sd.start, k});
  }
  std::sort(ranges.begin(), ranges.end());
  int covered = 0;
  for (auto& r : ranges) {
    if (r.first < covered) return fail(c, NN_ERR_INVALID_ARG, "scene %d overlaps another scene", r.second);
    if (r.first > covered) return fail(c, NN_ERR_INVALID_ARG, "particle %d belongs to no scene", covered);
    covered = r.first + scenes[r.second].n;
  }
  if (covered != n) return fail(c, NN_ERR_INVALID_ARG, "particle %d belongs to no scene", covered);
  // host copies of the class fields lay out the elastic particles; scenes without the
  // elasticity flag need none (no transfer for pure-fluid batches)
  bool want_el = false;
  for (int k = 0; k < nscenes; ++k) want_el |= (scenes[k].params.flags & (NN_F_ELASTICITY | NN_F_RIGID)) != 0;
  std::vector<int32_t> mat, ph;
  if (n > 0 && want_el) {
    mat.resize(n);
    ph.resize(n);
    CK(cudaMemcpy(mat.data(), c->state.material, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ph.data(), c->state.phase_id, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
  }
  std::vector<SceneDev> sdev;
  std::vector<SceneDyn> sdyn(nscenes);
  std::vector<int32_t> el_id;
  struct RB { int scene, phase, round; };
  std::vector<RB> rb_list;
  int64_t cells = 0;
  c->any_fluid = c->any_div = c->any_nonnewton = c->any_implicit = c->any_cfl = false;
  c->forces_feat = 0;
  c->el_mult_max = 0;
  bool all_div = true;                 // every scene with fluid runs the divergence solve
  for (int k = 0; k < nscenes; ++k) {
    const nn_scene_desc& sd = scenes[k];
    const bool q = (sd.params.flags & NN_F_QUIRKS) != 0;
    std::vector<int> phases;
    if (sd.params.flags & NN_F_ELASTICITY)
      for (int i = sd.start; i < sd.start + sd.n; ++i)
        if (mat[i] == NN_SOLID && ph[i] >= NN_PHASE_ELASTIC_BASE) phases.push_back(ph[i]);
    std::sort(phases.begin(), phases.end());
    phases.erase(std::unique(phases.begin(), phases.end()), phases.end());
    int el_mult = 0;
    if ((sd.params.flags & NN_F_ELASTICITY) && !phases.empty()) el_mult = q ? (int)phases.size() : 1;
    if (el_mult > 0)
      for (int i = sd.start; i < sd.start + sd.n; ++i)
        if (q || (mat[i] == NN_SOLID && ph[i] >= NN_PHASE_ELASTIC_BASE)) el_id.push_back(i);
    SceneDev s = make_scene(sd, cells, el_mult, c->cell_factor, c->x_split);
    // rigid bodies of the scene (RIGID phases: dynamic solids with phase ids 2000..2999)
    if (sd.params.flags & NN_F_RIGID) {
      std::vector<int> rp;
      for (int i = sd.start; i < sd.start + sd.n; ++i)
        if (mat[i] == NN_SOLID && ph[i] >= NN_PHASE_RIGID_BASE && ph[i] < NN_PHASE_ELASTIC_BASE) rp.push_back(ph[i]);
      std::sort(rp.begin(), rp.end());
      rp.erase(std::unique(rp.begin(), rp.end()), rp.end());
      s.n_rigid = (int)rp.size();
      for (int r = 0; r < (int)rp.size(); ++r) rb_list.push_back({k, rp[r], r});
    }
    cells += (int64_t)s.gx * ((int64_t)1 << (2 * s.mbits));
    sdev.push_back(s);
    SceneDyn y{};
    y.dt = (real)sd.params.dt;
    y.inv_dt = (real)(1.0 / (double)y.dt);
    y.inv_dt2 = (real)(1.0 / ((double)y.dt * (double)y.dt));
    sdyn[k] = y;
    c->any_fluid |= sd.n_fluid > 0;
    c->any_div |= sd.n_fluid > 0 && (sd.params.flags & NN_F_DIVERGENCE);
    if (sd.n_fluid > 0 && !(sd.params.flags & NN_F_DIVERGENCE)) all_div = false;
    c->any_nonnewton |= (sd.params.flags & NN_F_NONNEWTON) != 0;
    c->any_implicit |= sd.n_fluid > 0 && (sd.params.flags & NN_F_IMPLICIT_VISCOSITY) && !q;
    c->any_cfl |= (sd.params.flags & NN_F_CFL) != 0;
    c->el_mult_max = std::max(c->el_mult_max, el_mult);
    if (sd.n_fluid > 0) {  // terms the force pass must compile in (the union over scenes)
      const bool implicit = (sd.params.flags & NN_F_IMPLICIT_VISCOSITY) && !q;
      if (sd.params.flags & NN_F_SURFACE_TENSION) c->forces_feat |= FF_ST;
      if ((sd.params.flags & NN_F_VISCOSITY) && !implicit) c->forces_feat |= FF_VI;
      if (sd.params.flags & NN_F_NONNEWTON) c->forces_feat |= FF_SR;
      if (q) c->forces_feat |= FF_Q;
    }
  }
  // the force pass's terms ride on the divergence loop's last density change unless a
  // scene skips the divergence solve or needs the explicit viscosity or quirk mode
  c->fold_np = c->any_fluid && all_div && (c->forces_feat & (FF_VI | FF_Q)) == 0;
  c->body_nodes[0] = c->fold_np ? 4 : 3;  // the folded density change is a second launch per body
  if (cells >= (int64_t)0x7fffffff) return fail(c, NN_ERR_CAPACITY, "%lld grid cells exceed the 32-bit key space", (long long)cells);
  if (cells > c->max_cells) drop_graphs(c);  // the scan grids were sized for the old table
  RC(ensure_cells(c, cells));
  c->ne = (int)el_id.size();
  // elastic buffers are reallocated below (their pointers and stride are graph arguments)
  if (feature_sig(c) != c->graph_sig || c->ne > 0) drop_graphs(c);
  c->scenes.assign(scenes, scenes + nscenes);
  c->sdev = sdev;
  c->n = n;
  c->ncells = (int)cells;
  c->ne = (int)el_id.size();
  free_elastic(c);
  c->el_stale = false;

  if (c->ne > 0) {
    c->el_stride = c->ne;
    const size_t E = (size_t)c->ne;
    if (dalloc(&c->el_id, E) != cudaSuccess || dalloc(&c->el_slot, E) != cudaSuccess ||
        dalloc(&c->el_nb, E * c->el_cap) != cudaSuccess || dalloc(&c->el_cnt, E) != cudaSuccess ||
        dalloc(&c->el_x0, E) != cudaSuccess || dalloc(&c->el_R, 9 * E) != cudaSuccess ||
        dalloc(&c->el_S, 6 * E) != cudaSuccess)
      return fail(c, NN_ERR_OOM, "elastic buffers");
    CK(cudaMemcpy(c->el_id, el_id.data(), E * sizeof(int32_t), cudaMemcpyHostToDevice));
    CK(cudaMemset(c->el_cnt, 0, E * sizeof(int32_t)));
  }
  if (c->ne > 0) {
    std::vector<int32_t> e_of_id(n, -1);
    for (size_t e = 0; e < el_id.size(); ++e) e_of_id[el_id[e]] = (int32_t)e;
    CK(cudaMemcpy(c->e_of_id, e_of_id.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
  } else if (n > 0) {
    CK(cudaMemset(c->e_of_id, 0xff, n * sizeof(int32_t)));  // all -1
  }
  if (nscenes > 0) {
    CK(cudaMemcpy(c->d_sc, sdev.data(), nscenes * sizeof(SceneDev), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_dyn, sdyn.data(), nscenes * sizeof(SceneDyn), cudaMemcpyHostToDevice));
  }
  int32_t hn[4] = {n, nscenes, (int)cells, c->ne};
  CK(cudaMemcpy(c->d_n, hn, sizeof(hn), cudaMemcpyHostToDevice));
  CK(cudaMemset(c->d_acc, 0, (size_t)c->max_scenes * ACC_COUNT * NN_STRIPES * sizeof(double)));
  // rigid bodies ("r-space")
  cudaFree(c->rb_of_id); cudaFree(c->rb_round); cudaFree(c->rb_acc); cudaFree(c->rb_rest); cudaFree(c->rb_cm);
  cudaFree(c->rb_R);
  c->rb_of_id = c->rb_round = nullptr;
  c->rb_acc = c->rb_rest = c->rb_cm = c->rb_R = nullptr;
  c->n_rb = (int)rb_list.size();
  c->rb_rounds = 0;
  c->coupling_max = 1;
  if (c->n_rb > 0) {
    std::vector<int32_t> rb_of(n, -1), rounds(c->n_rb);
    for (int b = 0; b < c->n_rb; ++b) {
      const nn_scene_desc& sd = scenes[rb_list[b].scene];
      for (int i = sd.start; i < sd.start + sd.n; ++i)
        if (mat[i] == NN_SOLID && ph[i] == rb_list[b].phase) rb_of[i] = b;
      rounds[b] = rb_list[b].round;
      c->rb_rounds = std::max(c->rb_rounds, rb_list[b].round + 1);
      c->coupling_max = std::max(c->coupling_max, std::max(sd.params.coupling_interval, 1));
    }
    const size_t B = (size_t)c->n_rb;
    if (dalloc(&c->rb_of_id, (size_t)n) != cudaSuccess || dalloc(&c->rb_round, B) != cudaSuccess ||
        dalloc(&c->rb_acc, B * 13) != cudaSuccess || dalloc(&c->rb_rest, B * 3) != cudaSuccess ||
        dalloc(&c->rb_cm, B * 3) != cudaSuccess || dalloc(&c->rb_R, B * 9) != cudaSuccess)
      return fail(c, NN_ERR_OOM, "rigid-body buffers");
    CK(cudaMemcpy(c->rb_of_id, rb_of.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->rb_round, rounds.data(), B * sizeof(int32_t), cudaMemcpyHostToDevice));
    CK(cudaMemset(c->rb_acc, 0, B * 13 * sizeof(double)));
    drop_graphs(c);  // body buffers and counts are graph arguments
  }
  if (nscenes > 0 && n > 0) {  // scene of every particle id, filled from the scene table on the device
    k_scene_of_id<<<std::min(nscenes, 65535), 256>>>(make_dev(c, c->cur));
    CK(cudaGetLastError());
  }
  c->searched = false;
  c->resident_ok = false;
  return NN_OK;
}

static int check_ready(nn_ctx* c) {
  if (!c) return fail(nullptr, NN_ERR_INVALID_ARG, "null context");
  if (!c->bound || c->scenes.empty()) return fail(c, NN_ERR_STATE, "bind a state and set scenes first");
  return NN_OK;
}
static int check_elastic(nn_ctx* c) {
  if (c->el_stale) return fail(c, NN_ERR_STATE, "elastic rest lists were re-sized: call nn_initialize first");
  return NN_OK;
}

int nn_initialize(nn_ctx* c) {
  RC(check_ready(c));
  c->resident_ok = false;
  cudaStream_t s = run_stream(c);
  // Elasticity constructors run before solver.initialize() (SPH/main.py:1889-1895, 1915).
  // Their rest neighbourhoods come from a search over the rest positions x_0 (equal to
  // x at t = 0, as in the reference; after a checkpoint restore they differ).
  if (c->ne > 0) {
    CK(cudaMemsetAsync(c->d_src_flag, 0, sizeof(int32_t), s));
    RC(launch1(c, s, k_set_int, c->d_src_flag, 2));
    RC(enq_search(c, s));
    Dev dr = make_dev(c, c->cur);
    RC(launch1(c, s, k_step_dt, dr, 0));
    RC(launch(c, s, k_el_init, 256, c->n, dr));
  }
  CK(cudaMemsetAsync(c->d_src_flag, 1, sizeof(int32_t), s));
  RC(enq_search(c, s));
  Dev d = make_dev(c, c->cur);
  RC(launch1(c, s, k_step_dt, d, 0));
  // RigidBodySolver.__init__: rest centre of mass of every body (SPH/main.py:1101-1106)
  for (int r = 0; r < c->rb_rounds; ++r) {
    RC(launch(c, s, k_rigid_com, 256, c->n, d, r, 1));
    RC(launch1(c, s, k_rigid_cm, d, r, 1));
  }
  RC(launch(c, s, KU(k_boundary_volume, U_BOUNDARY_VOLUME), c->block, c->n, d, 0));
  RC(launch(c, s, KU(k_boundary_volume, U_BOUNDARY_VOLUME), c->block, c->n, d, 1));
  RC(enq_sync_out(c, s, SM_VOL));
  CK(cudaStreamSynchronize(s));
  c->el_stale = false;
  return NN_OK;
}

int nn_step(nn_ctx* c, int32_t nsteps, uint32_t flags) {
  RC(check_ready(c));
  RC(check_elastic(c));
  if (nsteps < 0) return fail(c, NN_ERR_INVALID_ARG, "nsteps < 0");
  cudaStream_t s = run_stream(c);
  if (!s) return fail(c, NN_ERR_STATE, "no stream");
  const bool host = (flags & NN_STEP_HOST_LOOP) != 0;
  const bool resume = (flags & NN_STEP_RESUME) != 0;
  if (resume && !c->resident_ok)
    return fail(c, NN_ERR_STATE, "NN_STEP_RESUME: no state left resident by a previous nn_step");
  for (int k = 0; k < nsteps; ++k) {
    // the first step reads the caller's state, unless it resumes from the resident slots
    CK(cudaMemsetAsync(c->d_src_flag, (k == 0 && !resume) ? 1 : 0, sizeof(int32_t), s));
    if (host) {
      RC(enq_step(c, s));
    } else {
      const int parity = c->cur;
      if (!c->exec[parity]) RC(capture_step(c, s, parity));
      CK(cudaGraphLaunch(c->exec[parity], s));
      c->cur = 1 - parity;
      c->graph_replays++;
      c->searched = true;
    }
  }
  if (flags & NN_STEP_SYNC_STATE) RC(enq_sync_out(c, s, SM_ALL));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(c, NN_ERR_CUDA, "nn_step: %s", cudaGetErrorString(e));
  if (nsteps > 0) c->resident_ok = true;
  return NN_OK;
}

int nn_run_pass(nn_ctx* c, int32_t pass) {
  RC(check_ready(c));
  if (pass < 0 || pass >= NN_PASS_COUNT) return fail(c, NN_ERR_INVALID_ARG, "unknown pass %d", pass);
  c->resident_ok = false;
  cudaStream_t s = run_stream(c);
  if (pass == NN_PASS_SEARCH) {
    CK(cudaMemsetAsync(c->d_src_flag, 1, sizeof(int32_t), s));
    RC(launch1(c, s, k_step_reset, make_dev(c, c->cur)));
    RC(enq_search(c, s));
    CK(cudaStreamSynchronize(s));
    return NN_OK;
  }
  if (!c->searched) return fail(c, NN_ERR_STATE, "run the neighbour search first");
  RC(check_elastic(c));
  Dev d = make_dev(c, c->cur);
  RC(launch(c, s, k_sync_in, 256, c->n, d, (uint32_t)SM_ALL));
  RC(launch1(c, s, k_step_dt, d, 0));
  switch (pass) {
    case NN_PASS_STATIC_BOUNDARY_VOLUME: RC(launch(c, s, KU(k_boundary_volume, U_BOUNDARY_VOLUME), c->block, c->n, d, 0)); break;
    case NN_PASS_MOVING_BOUNDARY_VOLUME: RC(launch(c, s, KU(k_boundary_volume, U_BOUNDARY_VOLUME), c->block, c->n, d, 1)); break;
    case NN_PASS_CLEAR_ACCELERATIONS: RC(launch(c, s, k_clear_acc, 256, c->n, d, 0, 0)); break;
    case NN_PASS_DENSITIES: RC(launch(c, s, KU2(k_density_factor, false, U_DENSITY_FACTOR), c->block, c->n, d, 1, 0)); break;
    case NN_PASS_DFSPH_FACTOR: RC(launch(c, s, KU2(k_density_factor, false, U_DENSITY_FACTOR), c->block, c->n, d, 0, 1)); break;
    case NN_PASS_DIVERGENCE_SOLVE: if (c->any_div) RC(enq_divergence(c, s, false)); break;
    case NN_PASS_NON_PRESSURE_FORCES: if (c->any_fluid) RC(enq_nonpressure(c, s, 0, 0)); break;
    case NN_PASS_NON_PRESSURE_ADVECT: RC(launch(c, s, k_np_advect, 256, c->n, d)); break;
    case NN_PASS_PRESSURE_SOLVE: if (c->any_fluid) RC(enq_pressure(c, s, 0)); break;
    case NN_PASS_ELASTICITY: RC(enq_elastic(c, s)); break;
    case NN_PASS_ADVECT: RC(launch(c, s, k_advect_boundary, 256, c->n, d, 1, 0, 0)); break;
    case NN_PASS_ENFORCE_BOUNDARY: RC(launch(c, s, k_advect_boundary, 256, c->n, d, 0, 1, 0)); break;
    case NN_PASS_SUBSTEP: RC(enq_substep(c, s)); break;
    case NN_PASS_RIGID: RC(enq_rigid(c, s)); break;
    default: break;
  }
  RC(enq_sync_out(c, s, SM_ALL));
  CK(cudaStreamSynchronize(s));
  return NN_OK;
}

int nn_set_animation(nn_ctx* c, int32_t scene, const float* displacement) {
  RC(check_ready(c));
  if (!displacement || scene < 0 || scene >= (int32_t)c->scenes.size())
    return fail(c, NN_ERR_INVALID_ARG, "nn_set_animation: scene %d of %d", scene, (int)c->scenes.size());
  // pageable source: staged before the call returns, applied in stream order
  CK(cudaMemcpyAsync(&c->d_dyn[scene].anim[0], displacement, 3 * sizeof(float), cudaMemcpyHostToDevice,
                     run_stream(c)));
  return NN_OK;
}

int nn_time_kernel(nn_ctx* c, int32_t kernel, int32_t reps, float* ms_out) {
  RC(check_ready(c));
  if (!ms_out || reps <= 0 || kernel < 0 || kernel >= NN_K_COUNT) return fail(c, NN_ERR_INVALID_ARG, "nn_time_kernel: bad arguments");
  if (!c->searched) return fail(c, NN_ERR_STATE, "run a step first");
  c->resident_ok = false;  // the timed update kernels change the slots' velocities
  cudaStream_t s = run_stream(c);
  if (kernel == NN_K_BUILD_LISTS) {
    // the slots of the last search are sorted by the positions before its step's
    // advection: sort the current ones again (from the slots), so the timed builds see
    // the cell ranges a step's build sees
    CK(cudaMemsetAsync(c->d_src_flag, 0, sizeof(int32_t), s));
    RC(launch1(c, s, k_step_reset, make_dev(c, c->cur)));
    RC(enq_search(c, s));
  }
  Dev d = make_dev(c, c->cur);
  RC(launch1(c, s, k_force_active, d));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  auto one = [&]() -> int {
    const int B = c->block;
    switch (kernel) {
      case NN_K_PRESSURE_UPDATE: return launch(c, s, KU(k_pressure_update, U_PRESSURE_UPDATE), B, c->n, d);
      case NN_K_DENSITY_ADV: return launch(c, s, KU(k_density_adv, U_DENSITY_ADV), B, c->n, d, 1);
      case NN_K_DIVERGENCE_UPDATE: return launch(c, s, KU(k_divergence_update, U_DIVERGENCE_UPDATE), B, c->n, d);
      case NN_K_DENSITY_CHANGE: return launch(c, s, KU(k_density_change, U_DENSITY_CHANGE), B, c->n, d, 1, 0);
      case NN_K_DENSITY_CHANGE_NP: return launch(c, s, KU(k_density_change_np, U_DENSITY_CHANGE_NP), B, c->n, d, 1, 0);
      case NN_K_DENSITY_FACTOR:  // the instance the step runs (with the first density change)
        return c->any_div ? launch(c, s, KU2(k_density_factor, true, U_DENSITY_FACTOR), B, c->n, d, 1, 1)
                          : launch(c, s, KU2(k_density_factor, false, U_DENSITY_FACTOR), B, c->n, d, 1, 1);
      case NN_K_BUILD_LISTS: return launch(c, s, k_build_lists, NS_WARPS * 32, c->n, d);
      case NN_K_CG_MATVEC: return launch(c, s, KU(k_cg_matvec, U_CG_MATVEC), B, c->n, d);
      case NN_K_CG_SETUP: return launch(c, s, KU(k_cg_setup, U_CG_SETUP), B, c->n, d);
      default: return launch(c, s, forces_kernel(c), B, c->n, d, 0);
    }
  };
  RC(one());  // warm-up
  CK(cudaEventRecord(e0, s));
  for (int r = 0; r < reps; ++r) RC(one());
  CK(cudaEventRecord(e1, s));
  CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // leave the accumulators clean for the next step
  CK(cudaMemsetAsync(c->d_acc, 0, (size_t)c->max_scenes * ACC_COUNT * NN_STRIPES * sizeof(double), s));
  CK(cudaStreamSynchronize(s));
  *ms_out = ms / reps;
  return NN_OK;
}

int nn_get_neighbors(nn_ctx* c, int32_t* num, int32_t* lists, int32_t width) {
  RC(check_ready(c));
  if (!num || !lists || width <= 0) return fail(c, NN_ERR_INVALID_ARG, "nn_get_neighbors: bad arguments");
  if (!c->searched) return fail(c, NN_ERR_STATE, "run the neighbour search first");
  cudaStream_t s = run_stream(c);
  RC(launch(c, s, k_export_neighbors, 256, c->n, make_dev(c, c->cur), num, lists, width));
  CK(cudaStreamSynchronize(s));
  return NN_OK;
}

__global__ void k_clear_overflow(Dev d) {
  const int ns = d.d_n[1];
  for (int sc = threadIdx.x; sc < ns; sc += blockDim.x)
    if (d.dyn[sc].status == NN_ERR_NEIGHBOR_OVERFLOW) d.dyn[sc].status = NN_OK;
}

int nn_set_neighbor_cap(nn_ctx* c, int32_t max_neighbors) {
  if (!c) return fail(nullptr, NN_ERR_INVALID_ARG, "null context");
  if (max_neighbors <= 0 || max_neighbors > 1024)
    return fail(c, NN_ERR_INVALID_ARG, "nn_set_neighbor_cap: %d entries (1..1024)", max_neighbors);
  cudaStream_t s = run_stream(c);
  CK(cudaStreamSynchronize(s));
  if (max_neighbors != c->max_nb) {
    drop_graphs(c);  // the list pointer and its capacity are graph arguments
    cudaFree(c->nbr);
    c->nbr = nullptr;
    cudaError_t e = dalloc(&c->nbr, (size_t)c->cap * (size_t)max_neighbors);
    if (e != cudaSuccess) {
      c->max_nb = 0;
      return fail(c, NN_ERR_OOM, "nn_set_neighbor_cap: cudaMalloc of %d x %d entries: %s", c->cap, max_neighbors,
                  cudaGetErrorString(e));
    }
    c->max_nb = max_neighbors;
  }
  if (c->ne > 0 && max_neighbors != c->el_cap) {  // rest lists: rebuilt from x_0 by the next nn_initialize
    cudaFree(c->el_nb);
    c->el_nb = nullptr;
    if (dalloc(&c->el_nb, (size_t)c->el_stride * (size_t)max_neighbors) != cudaSuccess)
      return fail(c, NN_ERR_OOM, "nn_set_neighbor_cap: elastic rest lists");
    CK(cudaMemset(c->el_cnt, 0, (size_t)c->el_stride * sizeof(int32_t)));
    c->el_stale = true;
  }
  if (c->ne == 0 || c->el_stale) c->el_cap = max_neighbors;
  if (!c->scenes.empty()) RC(launch1(c, s, k_clear_overflow, make_dev(c, c->cur)));
  c->searched = false;
  c->resident_ok = false;
  CK(cudaStreamSynchronize(s));
  return NN_OK;
}

int nn_status_async(nn_ctx* c, int32_t scene, int32_t* host_out) {
  RC(check_ready(c));
  if (!host_out || scene < 0 || scene >= (int)c->scenes.size())
    return fail(c, NN_ERR_INVALID_ARG, "nn_status_async: bad arguments");
  static_assert(offsetof(SceneDyn, max_nb) == offsetof(SceneDyn, status) + sizeof(int32_t), "status, max_nb adjacent");
  cudaStream_t s = run_stream(c);
  CK(cudaMemcpyAsync(host_out, &c->d_dyn[scene].status, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaEventRecord(c->status_ev, s));
  return NN_OK;
}

int nn_status_wait(nn_ctx* c) {
  if (!c) return fail(nullptr, NN_ERR_INVALID_ARG, "null context");
  CK(cudaEventSynchronize(c->status_ev));
  return NN_OK;
}

static void fill_stats(const SceneDyn& y, nn_stats* out) {
  std::memset(out, 0, sizeof(*out));
  out->size = sizeof(*out);
  out->status = y.status;
  out->iterations_v = y.it_v;
  out->iterations = y.it_p;
  out->cg_iterations = y.it_cg;
  out->max_neighbors_seen = y.max_nb;
  out->avg_density_err_v = y.avg_v;
  out->avg_density_err = y.avg_p;
  out->cg_residual = y.cg_rel;
  out->dt = y.dt;
  unsigned bits = y.max_density_bits;
  float md;
  std::memcpy(&md, &bits, sizeof(md));
  out->max_density = md;
  out->steps = y.steps;
  out->max_avg_density_err = y.max_avg_p;
  out->nonpressure_folded = y.np_fresh;
}

int nn_get_stats_range(nn_ctx* c, int32_t first, int32_t count, nn_stats* out) {
  RC(check_ready(c));
  if (!out || first < 0 || count < 0 || first + count > (int)c->scenes.size())
    return fail(c, NN_ERR_INVALID_ARG, "bad scene range");
  if (count == 0) return NN_OK;
  cudaStream_t s = run_stream(c);
  std::vector<SceneDyn> y(count);
  CK(cudaMemcpyAsync(y.data(), c->d_dyn + first, count * sizeof(SceneDyn), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (int k = 0; k < count; ++k) fill_stats(y[k], out + k);
  return NN_OK;
}

int nn_get_stats(nn_ctx* c, int32_t scene, nn_stats* out) {
  RC(check_ready(c));
  if (!out || scene < 0 || scene >= (int)c->scenes.size()) return fail(c, NN_ERR_INVALID_ARG, "bad scene index");
  return nn_get_stats_range(c, scene, 1, out);
}

}  // extern "C"

// ---- neighbour search without device allocation ------------------------------------
// For callers that cannot call cudaMalloc (for example code running inside a host
// callback or a framework that owns every device allocation): the scratch of the
// search lives in one file-scope device array that the library carries. Every GPU
// that loads libnnsph.so holds NN_NOALLOC_SCRATCH_BYTES of device memory until the
// process exits. All calls share the array, so calls that overlap on the GPU (on
// different streams, or from several host threads) race; calls on one stream are
// ordered. The first call in each CUDA context looks up the array's device address
// in that context; make that first call before any stream capture.
namespace {
constexpr size_t kNaAlign = 256;
constexpr size_t na_round(size_t b) { return (b + kNaAlign - 1) / kNaAlign * kNaAlign; }
constexpr size_t kNaN = NN_NOALLOC_MAX_PARTICLES;
constexpr size_t kNaC = NN_NOALLOC_MAX_CELLS;
constexpr size_t kNaNb = NN_NOALLOC_MAX_NEIGHBORS;
// layout of the scratch array (byte offsets)
constexpr size_t kOffN = 0;
constexpr size_t kOffSc = kOffN + na_round(4 * sizeof(int32_t));
constexpr size_t kOffDyn = kOffSc + na_round(sizeof(SceneDev));
constexpr size_t kOffFlag = kOffDyn + na_round(sizeof(SceneDyn));
constexpr size_t kOffSceneOf = kOffFlag + na_round(sizeof(int32_t));
constexpr size_t kOffKey = kOffSceneOf + na_round(kNaN * 4);
constexpr size_t kOffRank = kOffKey + na_round(kNaN * 4);
constexpr size_t kOffSrc = kOffRank + na_round(kNaN * 4);
constexpr size_t kOffCells = kOffSrc + na_round(kNaN * 4);
constexpr size_t kOffTiles = kOffCells + na_round((kNaC + 1) * 4);
constexpr size_t kOffPos = kOffTiles + na_round(((kNaC + 1) / SCAN_TILE + 2) * 4);
constexpr size_t kOffFlags = kOffPos + na_round(kNaN * sizeof(real4));
constexpr size_t kOffId = kOffFlags + na_round(kNaN * 4);
constexpr size_t kOffNbr = kOffId + na_round(kNaN * 4);
constexpr size_t kOffCnt = kOffNbr + na_round(kNaN * kNaNb * 4);
constexpr size_t kOffRaw = kOffCnt + na_round(kNaN * 4);
constexpr size_t kNaEnd = kOffRaw + na_round(kNaN * 4);
static_assert(kNaEnd <= NN_NOALLOC_SCRATCH_BYTES, "no-alloc scratch layout exceeds the array");
}  // namespace

static __device__ __align__(256) unsigned char g_nn_noalloc_scratch[NN_NOALLOC_SCRATCH_BYTES];

// Sizes, scene constants and cleared per-call state, written by a kernel so the call
// needs no host-to-device copy.
__global__ void k_na_setup(Dev d, SceneDev s, int32_t n, int32_t cells) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int32_t* dn = const_cast<int32_t*>(d.d_n);
    dn[0] = n; dn[1] = 1; dn[2] = cells; dn[3] = 0;
    *const_cast<SceneDev*>(d.sc) = s;
    SceneDyn y{};
    *d.dyn = y;
    *const_cast<int32_t*>(d.src_from_truth) = 1;
  }
  int32_t* so = const_cast<int32_t*>(d.scene_of_id);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) so[i] = 0;
}

// Positions only: the slot set of the search (no velocities or masses involved).
__global__ void k_na_gather(Dev d) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const int s = d.src[i];
    d.w.pos[i] = make_real4(d.t.x[3 * s], d.t.x[3 * s + 1], d.t.x[3 * s + 2], 0.f);
    d.w.flags[i] = NN_CLS_VALID;
    d.w.id[i] = s;
  }
}

// Device address of the scratch array per CUDA context: a symbol's address belongs to
// the module loaded in one context, so a caller on another context of the same device
// (or after cudaDeviceReset) looks it up again. The current context comes from the
// driver's cuCtxGetCurrent, reached through the runtime (no link against libcuda).
static std::mutex g_na_mutex;
struct NaAddr { int dev; void* ctx; void* ptr; };
static std::vector<NaAddr> g_na_addr;
typedef int (*NaCtxGetCurrent)(void**);

static int na_current_context(void** ctx) {
  static NaCtxGetCurrent fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !f)
      return -1;
    fn = reinterpret_cast<NaCtxGetCurrent>(f);
  }
  *ctx = nullptr;
  return fn(ctx) == 0 && *ctx ? 0 : -1;
}

extern "C" int nn_neighbors_noalloc(const float* x, int32_t n, const double* domain_start,
                                    const double* domain_end, double support_radius, int32_t width,
                                    int32_t* num_neighbors, int32_t* neighbors, void* cuda_stream) {
  nn_ctx* c = nullptr;  // error messages go to nn_last_error(NULL)
  if (!x || !domain_start || !domain_end || !num_neighbors || !neighbors || n < 0 || width <= 0 || width > 1024 ||
      !(support_radius > 0))
    return fail(c, NN_ERR_INVALID_ARG, "nn_neighbors_noalloc: invalid argument");
  if (n > NN_NOALLOC_MAX_PARTICLES)
    return fail(c, NN_ERR_CAPACITY, "nn_neighbors_noalloc: %d particles exceed the maximum of %d", n,
                NN_NOALLOC_MAX_PARTICLES);
  nn_scene_desc sd{};
  sd.size = sizeof(sd);
  sd.n = n;
  sd.params.size = sizeof(nn_scene_params);
  for (int k = 0; k < 3; ++k) {
    if (!(domain_end[k] > domain_start[k])) return fail(c, NN_ERR_INVALID_ARG, "nn_neighbors_noalloc: empty domain");
    sd.params.domain_start[k] = domain_start[k];
    sd.params.domain_end[k] = domain_end[k];
  }
  sd.params.support_radius = support_radius;
  sd.params.density0 = 1000.0;
  sd.params.dt = 1e-3;
  const SceneDev s = make_scene(sd, 0, 0);
  const int64_t cells = (int64_t)s.gx * ((int64_t)1 << (2 * s.mbits));
  if (cells > NN_NOALLOC_MAX_CELLS)
    return fail(c, NN_ERR_CAPACITY, "nn_neighbors_noalloc: the domain needs %lld cells of edge h, maximum %d",
                (long long)cells, NN_NOALLOC_MAX_CELLS);
  // an error left by earlier, unrelated work is reported as such, before any launch
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(c, NN_ERR_CUDA, "nn_neighbors_noalloc: a CUDA error was pending from earlier work: %s",
                cudaGetErrorString(e));
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(c, NN_ERR_CUDA, "nn_neighbors_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_na_mutex);
    void* ctx = nullptr;
    if (na_current_context(&ctx) != 0) {
      // no context current yet: the runtime makes the device's primary context current
      // on its first use, here the address lookup
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_nn_noalloc_scratch);
      if (e != cudaSuccess)
        return fail(c, NN_ERR_CUDA, "nn_neighbors_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      if (na_current_context(&ctx) != 0) return fail(c, NN_ERR_CUDA, "nn_neighbors_noalloc: no current CUDA context");
    }
    for (const NaAddr& a : g_na_addr)
      if (a.dev == dev && a.ctx == ctx) base = static_cast<unsigned char*>(a.ptr);
    if (!base) {  // once per device and context, with that device current
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_nn_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return fail(c, NN_ERR_CUDA, "nn_neighbors_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      g_na_addr.push_back({dev, ctx, p});
      base = static_cast<unsigned char*>(p);
    }
  }
  if (n == 0) return NN_OK;
  Dev d{};
  d.d_n = reinterpret_cast<int32_t*>(base + kOffN);
  d.sc = reinterpret_cast<SceneDev*>(base + kOffSc);
  d.dyn = reinterpret_cast<SceneDyn*>(base + kOffDyn);
  d.src_from_truth = reinterpret_cast<int32_t*>(base + kOffFlag);
  d.scene_of_id = reinterpret_cast<int32_t*>(base + kOffSceneOf);
  d.key = reinterpret_cast<uint32_t*>(base + kOffKey);
  d.rank = reinterpret_cast<uint32_t*>(base + kOffRank);
  d.src = reinterpret_cast<int32_t*>(base + kOffSrc);
  d.cell_count = reinterpret_cast<uint32_t*>(base + kOffCells);
  d.tile_sums = reinterpret_cast<uint32_t*>(base + kOffTiles);
  d.w.pos = reinterpret_cast<real4*>(base + kOffPos);
  d.w.flags = reinterpret_cast<uint32_t*>(base + kOffFlags);
  d.w.id = reinterpret_cast<int32_t*>(base + kOffId);
  d.nbr = reinterpret_cast<int32_t*>(base + kOffNbr);
  d.nbr_cnt = reinterpret_cast<int32_t*>(base + kOffCnt);
  d.nbr_raw = reinterpret_cast<int32_t*>(base + kOffRaw);
  d.cap = NN_NOALLOC_MAX_PARTICLES;
  d.max_nb = NN_NOALLOC_MAX_NEIGHBORS;
  d.t.x = const_cast<float*>(x);
  cudaStream_t st = (cudaStream_t)cuda_stream;
  const int B = 256;
  const int gN = std::max(1, std::min((n + B - 1) / B, 1024));
  const int gC = std::max(1, std::min((int)((cells + 1 + B - 1) / B), 1024));
  const int tiles = (int)((cells + 1 + SCAN_TILE - 1) / SCAN_TILE);
  k_na_setup<<<gN, B, 0, st>>>(d, s, n, (int32_t)cells);
  k_zero_cells<<<gC, B, 0, st>>>(d, 0);
  k_keys<<<gN, B, 0, st>>>(d);
  k_scan_tiles<<<std::min(tiles, 256), SCAN_THREADS, 0, st>>>(d);
  k_scan_apply<<<std::min(tiles, 256), SCAN_THREADS, 0, st>>>(d);
  k_scatter<<<gN, B, 0, st>>>(d);
  k_cell_sort<<<gC, B, 0, st>>>(d);
  k_na_gather<<<gN, B, 0, st>>>(d);
  k_build_lists<<<gN, NS_WARPS * 32, 0, st>>>(d);
  k_export_neighbors<<<gN, B, 0, st>>>(d, num_neighbors, neighbors, width);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(c, NN_ERR_CUDA, "nn_neighbors_noalloc: %s", cudaGetErrorString(e));
  return NN_OK;
}

#ifndef NN_FP64
// Surface reconstruction (SRTool): kernels and its C ABI (FP32 build only).
#include "surf.cuh"
#endif
