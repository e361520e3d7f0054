// common.cuh — device data layout, SPH kernel functions and reductions shared by
// every pass of the B200 SPH step.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/nnsph.h"

#define NN_STRIPES 32          // striped FP64 accumulators per scene and quantity
#define NN_SCENE_SHIFT 8       // slot flags: bits 0..7 particle class, 8.. scene index
#define NN_CLS_SOLID 1u        // material == SOLID
#define NN_CLS_DYNAMIC 2u      // is_dynamic
#define NN_CLS_ELASTIC 4u      // member of the elastic model
#define NN_CLS_VALID 8u        // slot holds a particle

// Arithmetic type of the step. libnnsph.so is built with real = float, the
// reference's precision (Taichi's default f32). libnnsph64.so is the same source built
// with NN_FP64 (real = double): the FP64 run of the same kernels that the FP32 path's
// per-field error is stated against. The caller's state (meta.pd) is float32 in both.
#ifdef NN_FP64
typedef double real;
typedef double2 real2;
typedef double3 real3;
typedef double4 real4;
__host__ __device__ __forceinline__ real2 make_real2(real a, real b) { return make_double2(a, b); }
__host__ __device__ __forceinline__ real3 make_real3(real a, real b, real c) { return make_double3(a, b, c); }
__host__ __device__ __forceinline__ real4 make_real4(real a, real b, real c, real e) { return make_double4(a, b, c, e); }
__device__ __forceinline__ real mul_rn(real a, real b) { return __dmul_rn(a, b); }
__device__ __forceinline__ real add_rn(real a, real b) { return __dadd_rn(a, b); }
__device__ __forceinline__ real sqrt_rn(real a) { return __dsqrt_rn(a); }
__device__ __forceinline__ real fast_div(real a, real b) { return a / b; }
#define NN_REGS64                         // no register caps: double registers come in pairs
#else
typedef float real;
typedef float2 real2;
typedef float3 real3;
typedef float4 real4;
__host__ __device__ __forceinline__ real2 make_real2(real a, real b) { return make_float2(a, b); }
__host__ __device__ __forceinline__ real3 make_real3(real a, real b, real c) { return make_float3(a, b, c); }
__host__ __device__ __forceinline__ real4 make_real4(real a, real b, real c, real e) { return make_float4(a, b, c, e); }
__device__ __forceinline__ real mul_rn(real a, real b) { return __fmul_rn(a, b); }
__device__ __forceinline__ real add_rn(real a, real b) { return __fadd_rn(a, b); }
__device__ __forceinline__ real sqrt_rn(real a) { return __fsqrt_rn(a); }
__device__ __forceinline__ real fast_div(real a, real b) { return __fdividef(a, b); }
#define NN_REGS64 __maxnreg__(64)
#endif

// Read-only loads through the texture path (__ldg), double4 as two double2 loads.
template <typename T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }
#ifdef NN_FP64
template <>
__device__ __forceinline__ double4 ldg<double4>(const double4* p) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}
#endif

// Constants of one scene, derived once on the host (mirrors how Taichi folds the
// reference's Python floats into f32 literals: SPH/main.py:859-905, 1044-1051).
struct SceneDev {
  uint32_t flags;
  int32_t start, n, n_fluid;      // id range
  int64_t cell_base;              // first cell key of the scene
  int32_t gx, gy, gz, mbits;      // grid size; rows (y,z) are Morton-ordered with mbits per axis
  real origin[3];
  real cell;                     // cell edge in y and z (h / nf)
  int32_t nf;                     // stencil half-width in y and z cells (cell factor)
  real cellx;                    // cell edge in x (cell / x split)
  int32_t nfx;                    // stencil half-width in x cells (nf * x split)
  real h, k_w, k2_w, k_grad, W0; // cubic spline constants
  real inv_h;
  real h2_thr;                   // smallest value whose rounded sqrt is >= h (h^2 in the FP64 build)
  real rho0, inv_rho0;
  real g[3];
  real eps;
  real sigma, dia2, w_dia;       // surface tension
  real visc, visc_b, c01h2;      // explicit viscosity
  real xmin[3], xmax[3], cf, sticky;
  double eta_v_fac;               // maxErrorV * 0.01 * rho0 (multiplied by 1/dt)
  double eta_p;                   // maxError * 0.01 * rho0
  int32_t max_iter_v, max_iter, visco_max_iter, nn_method;
  double visco_tol;
  real nn_n, nn_K, nn_mu0, nn_muinf, nn_gc, nn_muc, nn_tauy;
  real mu_newton;                // viscosity * rho0 (implicit solver without a law)
  real mu_b;                     // visco_boundary * rho0
  real el_cd, el_co, el_cs;      // isotropic C of Becker 2009 (SPH/main.py:1276-1283)
  int32_t el_mult;                // elastic substeps per step (quirk: one per elastic phase)
  real cfl_factor, cfl_min_dt, cfl_max_dt, diameter;
  real V0, padding;              // volume0 and padding (rigid-body mass, ground clamp)
  int32_t n_rigid, coupling;      // rigid bodies of the scene, substeps per step
};

// Mutable per-scene state on the device.
struct SceneDyn {
  real dt, inv_dt;               // time step and f32(1/dt)
  real inv_dt2;                  // f32(1/(dt*dt))
  int32_t it_v, it_p, it_cg;      // loop counters (reference semantics)
  int32_t act_v, act_p, act_cg;   // 1 while the scene still iterates
  int32_t status;                 // first NN_ERR_* seen
  int32_t max_nb;                 // max neighbour count of the last search
  uint32_t max_density_bits;      // float bits (densities are positive)
  uint32_t vmax_bits;             // float bits of max |v| (CFL)
  double avg_v, avg_p;            // last average density errors
  double cg_rz, cg_bnorm2, cg_rel;
  int32_t div_ran;                // divergence solve ran this step (alpha bookkeeping)
  int32_t np_body;                // divergence loop body (0-based) whose density change also computes
                                  // the non-pressure terms: the last body of the previous step
  double cg_alpha, cg_beta;       // PCG scalars of the current iteration
  int64_t steps;
  float anim[3];                 // animate_particles displacement of the next step (set by the host)
  int32_t np_last;                // index of the last divergence loop body of the last step
  double max_avg_p;               // largest avg_p at the end of a step since the scene was set
  int32_t np_fresh;               // this step's non-pressure terms came from body np_body, the last
  int32_t pad;
};

// Accumulator slots per scene (each NN_STRIPES doubles).
enum { ACC_ERR = 0, ACC_RZ, ACC_PAP, ACC_RR, ACC_BB, ACC_COUNT };

struct Vec3 { real x, y, z; };
__device__ __forceinline__ real3 f3(real4 a) { return make_real3(a.x, a.y, a.z); }
__device__ __forceinline__ real3 operator-(real3 a, real3 b) { return make_real3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ real3 operator+(real3 a, real3 b) { return make_real3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ real3 operator*(real3 a, real s) { return make_real3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ real3 operator-(real3 a) { return make_real3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ void operator+=(real3& a, real3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
__device__ __forceinline__ void operator-=(real3& a, real3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
__device__ __forceinline__ real dot3(real3 a, real3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Exact f32 distance as the reference computes it for the in-range test:
// (x_i - x_j).norm() < support_radius (SPH/main.py:845), no FMA contraction.
__device__ __forceinline__ real exact_norm(real3 r) {
  real s = add_rn(add_rn(mul_rn(r.x, r.x), mul_rn(r.y, r.y)), mul_rn(r.z, r.z));
  return sqrt_rn(s);
}

// cubic_kernel, SPH/main.py:859-880
__device__ __forceinline__ real kernel_w(real rn, const SceneDev& s) {
  real q = rn / s.h;
  real res = 0.f;
  if (q <= 1.f) {
    if (q <= 0.5f) {
      real q2 = q * q;
      real q3 = q2 * q;
      res = s.k_w * (6.f * q3 - 6.f * q2 + 1.f);
    } else {
      real t = 1.f - q;
      res = s.k2_w * (t * t * t);
    }
  }
  return res;
}

// cubic_kernel_derivative, SPH/main.py:883-905 (rn = |r| passed in)
__device__ __forceinline__ real3 kernel_grad(real3 r, real rn, const SceneDev& s) {
  real q = rn / s.h;
  real3 res = make_real3(0.f, 0.f, 0.f);
  if (rn > 1e-5f && q <= 1.f) {
    real den = rn * s.h;
    real3 gq = make_real3(r.x / den, r.y / den, r.z / den);
    real f;
    if (q <= 0.5f) {
      f = s.k_grad * q * (3.f * q - 2.f);
    } else {
      real t = 1.f - q;
      f = s.k_grad * (-t * t);
    }
    res = gq * f;
  }
  return res;
}

// The same cubic spline and gradient as kernel_w / kernel_grad, from r^2 and without
// divisions (1/h precomputed, 1/|r| from rsqrt): used inside the neighbour loops,
// where it agrees with the reference expressions to a few ulp.
__device__ __forceinline__ void kwg_r2(real3 r, real r2, const SceneDev& s, real& w, real3& g) {
  const real inv_rn = r2 > 0.f ? rsqrt(r2) : 0.f;
  const real rn = r2 * inv_rn;
  const real q = rn * s.inv_h;
  const real t = 1.f - q;
  const bool in = q <= 1.f;
  const bool inner = q <= 0.5f;
  w = in ? (inner ? s.k_w * (6.f * q * q * (q - 1.f) + 1.f) : s.k2_w * (t * t * t)) : 0.f;
  const real f = inner ? s.k_grad * q * (3.f * q - 2.f) : -s.k_grad * t * t;
  const real c = (rn > 1e-5f && in) ? f * inv_rn * s.inv_h : 0.f;
  g = make_real3(r.x * c, r.y * c, r.z * c);
}
__device__ __forceinline__ real kw_r2(real r2, const SceneDev& s) {
  const real rn = r2 > 0.f ? r2 * rsqrt(r2) : 0.f;
  const real q = rn * s.inv_h;
  const real t = 1.f - q;
  const real w = q <= 0.5f ? s.k_w * (6.f * q * q * (q - 1.f) + 1.f) : s.k2_w * (t * t * t);
  return q <= 1.f ? w : 0.f;
}
__device__ __forceinline__ real3 kgrad_r2(real3 r, real r2, const SceneDev& s) {
  real w;
  real3 g;
  kwg_r2(r, r2, s, w, g);
  return g;
}

// Neighbour loop in batches of NB_U list entries: the NB_U list loads, then the NB_U
// gathers of `load`, are issued before any `use`, so several dependent load chains
// are in flight per thread (the passes are latency-bound on list -> gather).
// STREAM loads the list entries evict-first (__ldcs), leaving L2 to the gathered
// particle data; the passes of the pressure loop gain from it (see their call sites).
template <bool STREAM>
__device__ __forceinline__ int nb_list_load(const int32_t* p) {
  if constexpr (STREAM) return __ldcs(p);
  else return ldg(p);
}

template <int NB_U, bool STREAM = false, typename Load, typename Use>
__device__ __forceinline__ void nb_batches(const int32_t* __restrict__ list, int stride, int c, int self, Load load,
                                           Use use) {
  // software pipeline: list entries are loaded PD batches (8 entries) ahead of the
  // gathers, so the DRAM latency of the list stream overlaps several batches
  constexpr int PD = NB_U >= 8 ? 1 : 8 / NB_U;
  int q[PD][NB_U];
#pragma unroll
  for (int p = 0; p < PD; ++p)
#pragma unroll
    for (int u = 0; u < NB_U; ++u) q[p][u] = (p * NB_U + u < c) ? nb_list_load<STREAM>(list + (size_t)(p * NB_U + u) * stride) : self;
  for (int k = 0; k < c; k += NB_U) {
    int j[NB_U];
#pragma unroll
    for (int u = 0; u < NB_U; ++u) j[u] = q[0][u];
#pragma unroll
    for (int p = 0; p + 1 < PD; ++p)
#pragma unroll
      for (int u = 0; u < NB_U; ++u) q[p][u] = q[p + 1][u];
#pragma unroll
    for (int u = 0; u < NB_U; ++u) {
      const int kk = k + PD * NB_U + u;
      q[PD - 1][u] = (kk < c) ? nb_list_load<STREAM>(list + (size_t)kk * stride) : self;
    }
    decltype(load(0)) g[NB_U];
#pragma unroll
    for (int u = 0; u < NB_U; ++u) g[u] = load(j[u]);
#pragma unroll
    for (int u = 0; u < NB_U; ++u)
      if (k + u < c) use(j[u], g[u]);
  }
}

// Material of a slot is also kept in the sign of pos.w: the volume is stored
// positive for fluid and negative for solid particles, so neighbour loops need no
// separate class gather.
__device__ __forceinline__ bool w_fluid(real w) { return w > 0.f; }

__device__ __forceinline__ int slot_scene(uint32_t fl) { return (int)(fl >> NN_SCENE_SHIFT); }
__device__ __forceinline__ bool cls_fluid(uint32_t fl) { return (fl & (NN_CLS_VALID | NN_CLS_SOLID)) == NN_CLS_VALID; }
__device__ __forceinline__ bool cls_solid(uint32_t fl) { return (fl & NN_CLS_SOLID) != 0; }
__device__ __forceinline__ bool cls_dyn_solid(uint32_t fl) { return (fl & (NN_CLS_SOLID | NN_CLS_DYNAMIC)) == (NN_CLS_SOLID | NN_CLS_DYNAMIC); }
__device__ __forceinline__ bool cls_static_solid(uint32_t fl) { return (fl & (NN_CLS_SOLID | NN_CLS_DYNAMIC)) == NN_CLS_SOLID; }

__device__ __forceinline__ void set_status(SceneDyn* dyn, int code) { atomicCAS(&dyn->status, 0, code); }

// Per-scene FP64 sum of `val` over a warp: scene-uniform warps reduce with shuffles
// and issue one atomic on a striped accumulator; mixed warps fall back to per-lane
// atomics. Must be called by all 32 lanes (invalid lanes pass valid=false).
__device__ __forceinline__ void scene_add(double* acc, int quantity, int nscenes_stride, int scene, bool valid,
                                          double val) {
  const unsigned full = 0xffffffffu;
  int key = valid ? scene : -1;
  int k0 = __shfl_sync(full, key, 0);
  // find any valid scene in the warp to compare against
  unsigned vb = __ballot_sync(full, valid);
  if (vb == 0) return;
  int leader = __ffs(vb) - 1;
  int sl = __shfl_sync(full, key, leader);
  bool uniform = __all_sync(full, !valid || key == sl);
  (void)k0;
  int lane = threadIdx.x & 31;
  int stripe = ((blockIdx.x * (blockDim.x >> 5)) + (threadIdx.x >> 5)) & (NN_STRIPES - 1);
  if (uniform) {
    double v = valid ? val : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(full, v, o);
    if (lane == leader) atomicAdd(&acc[((size_t)sl * ACC_COUNT + quantity) * NN_STRIPES + stripe], v);
  } else if (valid) {
    atomicAdd(&acc[((size_t)scene * ACC_COUNT + quantity) * NN_STRIPES + stripe], val);
  }
  (void)nscenes_stride;
}

// FP64 partial sums of NQ quantities that a lane keeps for the scene it last worked
// on, across the iterations of a grid-stride loop: they go to the scene's striped
// accumulators (scene_add) when any lane of the warp moves on to another scene, and
// at the end of the kernel, instead of once per iteration. add() and flush() must be
// called by all 32 lanes.
template <int NQ>
struct LaneSums {
  double v[NQ];
  int scn = -1;
  __device__ __forceinline__ LaneSums() {
#pragma unroll
    for (int k = 0; k < NQ; ++k) v[k] = 0.0;
  }
  __device__ __forceinline__ void flush(double* acc, const int (&q)[NQ]) {
#pragma unroll
    for (int k = 0; k < NQ; ++k) scene_add(acc, q[k], 0, scn >= 0 ? scn : 0, scn >= 0, v[k]);
#pragma unroll
    for (int k = 0; k < NQ; ++k) v[k] = 0.0;
    scn = -1;
  }
  __device__ __forceinline__ void add(double* acc, const int (&q)[NQ], bool work, int scene, const double (&x)[NQ]) {
    if (__any_sync(0xffffffffu, work && scn >= 0 && scene != scn)) flush(acc, q);
    if (work) {
#pragma unroll
      for (int k = 0; k < NQ; ++k) v[k] += x[k];
      scn = scene;
    }
  }
};

// Warp-aggregated atomicMax: lanes that target the same address combine first.
// Must be called by all 32 lanes.
__device__ __forceinline__ void warp_max_to(unsigned* addr, unsigned val, bool valid) {
  const unsigned full = 0xffffffffu;
  unsigned long long key = valid ? (unsigned long long)addr : 0ull;
  unsigned peers = __match_any_sync(full, key);
  unsigned r = __reduce_max_sync(peers, valid ? val : 0u);
  if (valid && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicMax(addr, r);
}
__device__ __forceinline__ void warp_max_to(int* addr, int val, bool valid) {
  warp_max_to(reinterpret_cast<unsigned*>(addr), (unsigned)max(val, 0), valid);
}

__device__ __forceinline__ bool scene_implicit(const SceneDev& s) {
  return (s.flags & NN_F_IMPLICIT_VISCOSITY) && !(s.flags & NN_F_QUIRKS);
}

__device__ __forceinline__ double acc_sum(const double* acc, int scene, int quantity) {
  const double* a = &acc[((size_t)scene * ACC_COUNT + quantity) * NN_STRIPES];
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < NN_STRIPES; ++k) s += a[k];
  return s;
}
__device__ __forceinline__ void acc_zero(double* acc, int scene, int quantity) {
  double* a = &acc[((size_t)scene * ACC_COUNT + quantity) * NN_STRIPES];
#pragma unroll
  for (int k = 0; k < NN_STRIPES; ++k) a[k] = 0.0;
}

// Rotation of the polar decomposition (semantics of ti.polar_decompose used at
// SPH/main.py:1273): SVD with U, V in SO(3), R = U V^T, computed in double with a
// cyclic Jacobi eigen-decomposition of A^T A (same algorithm as the CPU oracle).
__device__ inline void closest_rotation(const double A[3][3], double R[3][3]) {
  double S[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) S[i][j] = A[0][i] * A[0][j] + A[1][i] * A[1][j] + A[2][i] * A[2][j];
  double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 12; ++sweep) {
    double off = S[0][1] * S[0][1] + S[0][2] * S[0][2] + S[1][2] * S[1][2];
    double diag = S[0][0] * S[0][0] + S[1][1] * S[1][1] + S[2][2] * S[2][2];
    if (off <= 1e-30 * diag || off == 0.0) break;
#pragma unroll
    for (int pq = 0; pq < 3; ++pq) {
      const int p = pq == 2 ? 1 : 0;
      const int q = pq == 0 ? 1 : 2;
      double apq = S[p][q];
      if (apq == 0.0) continue;
      double theta = (S[q][q] - S[p][p]) / (2.0 * apq);
      double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        double skp = S[k][p], skq = S[k][q];
        S[k][p] = c * skp - sn * skq;
        S[k][q] = sn * skp + c * skq;
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        double spk = S[p][k], sqk = S[q][k];
        S[p][k] = c * spk - sn * sqk;
        S[q][k] = sn * spk + c * sqk;
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        double vkp = V[k][p], vkq = V[k][q];
        V[k][p] = c * vkp - sn * vkq;
        V[k][q] = sn * vkp + c * vkq;
      }
    }
  }
  double lam[3] = {S[0][0], S[1][1], S[2][2]};
  int idx[3] = {0, 1, 2};
  // order by descending eigenvalue (same comparisons as the CPU oracle)
  for (int i = 0; i < 2; ++i)
    for (int j = i + 1; j < 3; ++j)
      if (lam[idx[j]] > lam[idx[i]]) { int t = idx[i]; idx[i] = idx[j]; idx[j] = t; }
  double Vs[3][3], sig[3];
  for (int c = 0; c < 3; ++c) {
    sig[c] = sqrt(fmax(lam[idx[c]], 0.0));
    for (int r = 0; r < 3; ++r) Vs[r][c] = V[r][idx[c]];
  }
  double detV = Vs[0][0] * (Vs[1][1] * Vs[2][2] - Vs[1][2] * Vs[2][1]) -
                Vs[0][1] * (Vs[1][0] * Vs[2][2] - Vs[1][2] * Vs[2][0]) +
                Vs[0][2] * (Vs[1][0] * Vs[2][1] - Vs[1][1] * Vs[2][0]);
  if (detV < 0)
    for (int r = 0; r < 3; ++r) Vs[r][2] = -Vs[r][2];
  if (!(sig[0] > 1e-30)) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) R[i][j] = (i == j) ? 1.0 : 0.0;
    return;
  }
  const double tiny = 1e-12 * sig[0];
  double u0[3], u1[3], u2[3];
  for (int r = 0; r < 3; ++r) u0[r] = (A[r][0] * Vs[0][0] + A[r][1] * Vs[1][0] + A[r][2] * Vs[2][0]) / sig[0];
  double n0 = sqrt(u0[0] * u0[0] + u0[1] * u0[1] + u0[2] * u0[2]);
  for (int r = 0; r < 3; ++r) u0[r] /= n0;
  if (sig[1] > tiny) {
    for (int r = 0; r < 3; ++r) u1[r] = A[r][0] * Vs[0][1] + A[r][1] * Vs[1][1] + A[r][2] * Vs[2][1];
  } else {
    int m = (fabs(u0[0]) < fabs(u0[1])) ? (fabs(u0[0]) < fabs(u0[2]) ? 0 : 2) : (fabs(u0[1]) < fabs(u0[2]) ? 1 : 2);
    u1[0] = u1[1] = u1[2] = 0;
    u1[m] = 1;
  }
  double d = u1[0] * u0[0] + u1[1] * u0[1] + u1[2] * u0[2];
  for (int r = 0; r < 3; ++r) u1[r] -= d * u0[r];
  double n1 = sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
  for (int r = 0; r < 3; ++r) u1[r] /= n1;
  u2[0] = u0[1] * u1[2] - u0[2] * u1[1];
  u2[1] = u0[2] * u1[0] - u0[0] * u1[2];
  u2[2] = u0[0] * u1[1] - u0[1] * u1[0];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R[i][j] = u0[i] * Vs[j][0] + u1[i] * Vs[j][1] + u2[i] * Vs[j][2];
}

// Morton interleave of two 16-bit row coordinates (y, z)
__device__ __host__ __forceinline__ uint32_t morton2(uint32_t a, uint32_t b) {
  auto spread = [](uint32_t v) {
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
  };
  return spread(a) | (spread(b) << 1);
}
