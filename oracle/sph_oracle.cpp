// sph_oracle.cpp — CPU restatement of the reference SPH step. TEST INFRASTRUCTURE.
//
// This file is the parity oracle and the timed CPU baseline of the B200 SPH step.
// It restates, function by function, the Taichi kernels of SPH/main.py in
// chunleili/nonNewton (cited per function below). It is NOT part of the product:
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
//
// Parity status: pinned against the reference's own step. Taichi is not installed
// here, so tests/golden/make_reference_run.py runs SPH/main.py itself in plain Python
// against a Taichi stand-in on seven small scenes (fluid in a boundary box; with the
// non-Newtonian model; with an elastic cube; with a rigid cube; the reference's own
// test_deformable.json, test_neighbor.json and test_anime.json) and stores the state
// after each step (tests/golden/ref_*.npz). In the reference-quirks mode this oracle
// reproduces every recorded field of those runs within 2e-5 of its scale
// (tests/test_reference_pin.py). The neighbour search and the density /
// boundary-volume / DFSPH-factor passes are also pinned by known answers derived from
// the reference's fixtures (tests/golden/make_golden.py) and by an independent numpy
// restatement.
//
// Templated on Real (float = the reference's ti.f32 default, double = the FP64
// comparison run). Every neighbour loop walks neighbours in ascending particle id.
// Reductions that decide convergence accumulate in double.
//
// Build: oracle/Makefile (g++ -O2 -fopenmp -ffp-contract=off).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/nnsph.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

template <typename R>
struct V3 {
  R x, y, z;
  V3() : x(0), y(0), z(0) {}
  V3(R a, R b, R c) : x(a), y(b), z(c) {}
  V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
  V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
  V3 operator-() const { return V3(-x, -y, -z); }
  V3 operator*(R s) const { return V3(x * s, y * s, z * s); }
  V3 operator/(R s) const { return V3(x / s, y / s, z / s); }
  V3& operator+=(const V3& o) { x += o.x; y += o.y; z += o.z; return *this; }
  V3& operator-=(const V3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  R dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
  R norm_sqr() const { return x * x + y * y + z * z; }
  R norm() const { return std::sqrt(x * x + y * y + z * z); }
  R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  R& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};
template <typename R>
V3<R> operator*(R s, const V3<R>& v) { return V3<R>(s * v.x, s * v.y, s * v.z); }

template <typename R>
struct M3 {
  R a[3][3];
  M3() { std::memset(a, 0, sizeof(a)); }
  static M3 eye() { M3 m; m.a[0][0] = m.a[1][1] = m.a[2][2] = R(1); return m; }
  static M3 outer(const V3<R>& u, const V3<R>& v) {
    M3 m;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) m.a[i][j] = u[i] * v[j];
    return m;
  }
  M3 operator+(const M3& o) const { M3 m; for (int i = 0; i < 9; ++i) (&m.a[0][0])[i] = (&a[0][0])[i] + (&o.a[0][0])[i]; return m; }
  M3 operator*(R s) const { M3 m; for (int i = 0; i < 9; ++i) (&m.a[0][0])[i] = (&a[0][0])[i] * s; return m; }
  M3& operator+=(const M3& o) { for (int i = 0; i < 9; ++i) (&a[0][0])[i] += (&o.a[0][0])[i]; return *this; }
  M3& operator-=(const M3& o) { for (int i = 0; i < 9; ++i) (&a[0][0])[i] -= (&o.a[0][0])[i]; return *this; }
  V3<R> mul(const V3<R>& v) const {
    return V3<R>(a[0][0] * v.x + a[0][1] * v.y + a[0][2] * v.z,
                 a[1][0] * v.x + a[1][1] * v.y + a[1][2] * v.z,
                 a[2][0] * v.x + a[2][1] * v.y + a[2][2] * v.z);
  }
  V3<R> mul_t(const V3<R>& v) const {  // transpose() @ v
    return V3<R>(a[0][0] * v.x + a[1][0] * v.y + a[2][0] * v.z,
                 a[0][1] * v.x + a[1][1] * v.y + a[2][1] * v.z,
                 a[0][2] * v.x + a[1][2] * v.y + a[2][2] * v.z);
  }
  R frob() const { double s = 0; for (int i = 0; i < 9; ++i) s += double((&a[0][0])[i]) * double((&a[0][0])[i]); return R(std::sqrt(s)); }
};

// Rotation part of the polar decomposition, the semantics of ti.polar_decompose
// used at SPH/main.py:1273: an SVD A = U S V^T with U, V proper rotations (the
// smallest singular value carries the sign of det A) and R = U V^T. Computed in
// double by a cyclic Jacobi eigen-decomposition of A^T A. The CUDA path runs the
// same algorithm.
inline void closest_rotation(const double A[3][3], double R[3][3]) {
  double S[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += A[k][i] * A[k][j];
      S[i][j] = s;
    }
  double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 12; ++sweep) {
    double off = S[0][1] * S[0][1] + S[0][2] * S[0][2] + S[1][2] * S[1][2];
    double diag = S[0][0] * S[0][0] + S[1][1] * S[1][1] + S[2][2] * S[2][2];
    if (off <= 1e-30 * diag || off == 0.0) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        double apq = S[p][q];
        if (apq == 0.0) continue;
        double theta = (S[q][q] - S[p][p]) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {  // S <- J^T S J
          double skp = S[k][p], skq = S[k][q];
          S[k][p] = c * skp - s * skq;
          S[k][q] = s * skp + c * skq;
        }
        for (int k = 0; k < 3; ++k) {
          double spk = S[p][k], sqk = S[q][k];
          S[p][k] = c * spk - s * sqk;
          S[q][k] = s * spk + c * sqk;
        }
        for (int k = 0; k < 3; ++k) {
          double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
  }
  // order eigenpairs by descending eigenvalue
  double lam[3] = {S[0][0], S[1][1], S[2][2]};
  int idx[3] = {0, 1, 2};
  for (int i = 0; i < 2; ++i)
    for (int j = i + 1; j < 3; ++j)
      if (lam[idx[j]] > lam[idx[i]]) std::swap(idx[i], idx[j]);
  double Vs[3][3], sig[3];
  for (int c = 0; c < 3; ++c) {
    sig[c] = std::sqrt(std::max(lam[idx[c]], 0.0));
    for (int r = 0; r < 3; ++r) Vs[r][c] = V[r][idx[c]];
  }
  double detV = Vs[0][0] * (Vs[1][1] * Vs[2][2] - Vs[1][2] * Vs[2][1]) -
                Vs[0][1] * (Vs[1][0] * Vs[2][2] - Vs[1][2] * Vs[2][0]) +
                Vs[0][2] * (Vs[1][0] * Vs[2][1] - Vs[1][1] * Vs[2][0]);
  if (detV < 0)
    for (int r = 0; r < 3; ++r) Vs[r][2] = -Vs[r][2];
  const double tiny = 1e-12 * std::max(sig[0], 1e-300);
  if (!(sig[0] > 1e-30)) {  // A == 0: identity (SVD of zero gives U = V = I)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) R[i][j] = (i == j) ? 1.0 : 0.0;
    return;
  }
  double U[3][3];
  double u0[3], u1[3], u2[3];
  for (int r = 0; r < 3; ++r) u0[r] = (A[r][0] * Vs[0][0] + A[r][1] * Vs[1][0] + A[r][2] * Vs[2][0]) / sig[0];
  double n0 = std::sqrt(u0[0] * u0[0] + u0[1] * u0[1] + u0[2] * u0[2]);
  for (int r = 0; r < 3; ++r) u0[r] /= n0;
  if (sig[1] > tiny) {
    for (int r = 0; r < 3; ++r) u1[r] = (A[r][0] * Vs[0][1] + A[r][1] * Vs[1][1] + A[r][2] * Vs[2][1]);
  } else {  // rank 1: any unit vector orthogonal to u0
    int m = (std::fabs(u0[0]) < std::fabs(u0[1])) ? (std::fabs(u0[0]) < std::fabs(u0[2]) ? 0 : 2)
                                                   : (std::fabs(u0[1]) < std::fabs(u0[2]) ? 1 : 2);
    u1[0] = u1[1] = u1[2] = 0;
    u1[m] = 1;
  }
  double d = u1[0] * u0[0] + u1[1] * u0[1] + u1[2] * u0[2];
  for (int r = 0; r < 3; ++r) u1[r] -= d * u0[r];
  double n1 = std::sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
  for (int r = 0; r < 3; ++r) u1[r] /= n1;
  u2[0] = u0[1] * u1[2] - u0[2] * u1[1];
  u2[1] = u0[2] * u1[0] - u0[0] * u1[2];
  u2[2] = u0[0] * u1[1] - u0[1] * u1[0];
  for (int r = 0; r < 3; ++r) { U[r][0] = u0[r]; U[r][1] = u1[r]; U[r][2] = u2[r]; }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R[i][j] = U[i][0] * Vs[j][0] + U[i][1] * Vs[j][1] + U[i][2] * Vs[j][2];
}

struct OrStats {
  int iterations_v = 0, iterations = 0, cg_iterations = 0, max_neighbors_seen = 0;
  double avg_density_err_v = 0, avg_density_err = 0, cg_residual = 0, dt = 0, max_density = 0;
  int64_t steps = 0;
  int status = 0;
};

class SimBase {
 public:
  virtual ~SimBase() {}
  virtual int run_pass(int pass) = 0;
  virtual int initialize() = 0;
  virtual int step(int nsteps) = 0;
  virtual int get_field(int field, double* out) = 0;
  virtual int set_field(int field, const double* in) = 0;
  virtual int get_neighbors(int32_t* counts, int32_t* lists, int32_t width) = 0;
  virtual int64_t neighbor_total() = 0;
  // displacement added to every particle by the next step (animate_particles)
  virtual void set_animation(const double* d) = 0;
  OrStats stats;
  std::string err;
};

enum Field {
  F_X = 0, F_X0, F_V, F_A, F_VOLUME, F_M, F_DENSITY, F_PRESSURE, F_DFSPH_FACTOR, F_DENSITY_ADV,
  F_MATERIAL, F_IS_DYNAMIC, F_PHASE_ID, F_STRAIN_RATE_NORM, F_NN_VISCOSITY, F_STRESS, F_ROTATIONS,
  F_REST_VOLUME, F_COUNT
};

template <typename R>
class Sim : public SimBase {
 public:
  nn_scene_params p;
  int n, n_fluid;
  std::vector<V3<R>> x, x0, v, a;
  std::vector<R> volume, m, density, pressure, alpha, rho_adv;
  std::vector<int> material, is_dynamic, phase_id;
  std::vector<int> nb_start, nb;           // CSR, each row ascending by id
  std::vector<R> srn, mu;                  // NonNewton
  std::vector<M3<R>> strain_rate;
  // elasticity (indices are particle ids)
  std::vector<int> el_active;              // particles the elastic model runs on
  std::vector<int> rest_start, rest_nb;    // rest neighbourhoods (CSR)
  std::vector<R> rest_volume;
  std::vector<M3<R>> rot, Fdef;
  std::vector<R> stress;                   // [n][6]
  int elastic_multiplicity = 0;
  bool elastic_ready = false;
  // constants (Taichi folds Python floats into f32 literals)
  R h, k_w, k2_w, k_grad, W0;

  bool quirks() const { return (p.flags & NN_F_QUIRKS) != 0; }
  bool has(uint32_t f) const { return (p.flags & f) != 0; }

  Sim(const nn_scene_params& prm, int n_, int nf, const double* x_in, const double* v_in, const int* mat,
      const int* dyn, const int* ph, const double* mass)
      : p(prm), n(n_), n_fluid(nf) {
    x.resize(n); x0.resize(n); v.resize(n); a.resize(n);
    volume.assign(n, R(p.volume0)); m.resize(n); density.assign(n, R(p.density0)); pressure.assign(n, 0);
    alpha.assign(n, 0); rho_adv.assign(n, 0);
    material.assign(mat, mat + n); is_dynamic.assign(dyn, dyn + n); phase_id.assign(ph, ph + n);
    for (int i = 0; i < n; ++i) {
      x[i] = V3<R>(R(x_in[3 * i]), R(x_in[3 * i + 1]), R(x_in[3 * i + 2]));
      x0[i] = x[i];
      v[i] = v_in ? V3<R>(R(v_in[3 * i]), R(v_in[3 * i + 1]), R(v_in[3 * i + 2])) : V3<R>();
      // m = volume0 * 1000 (SPH/main.py:743); a caller may pass per-particle masses
      m[i] = mass ? R(mass[i]) : R(p.volume0 * 1000.0);
    }
    srn.assign(n, 0); mu.assign(n, 0); strain_rate.assign(n, M3<R>());
    rot.assign(n, M3<R>::eye()); Fdef.assign(n, M3<R>::eye()); stress.assign(6 * (size_t)n, 0);
    rest_volume.assign(n, 0);
    h = R(p.support_radius);
    double k = 8.0 / kPi / (p.support_radius * p.support_radius * p.support_radius);
    k_w = R(k);
    k2_w = R(k * 2.0);
    k_grad = R(6.0 * (8.0 / kPi) / (p.support_radius * p.support_radius * p.support_radius));
    W0 = kernel_w(R(0));
    stats.dt = p.dt;
  }

  // cubic_kernel, SPH/main.py:859-880
  R kernel_w(R r_norm) const {
    R res = R(0);
    R q = r_norm / h;
    if (q <= R(1)) {
      if (q <= R(0.5)) {
        R q2 = q * q;
        R q3 = q2 * q;
        res = k_w * (R(6) * q3 - R(6) * q2 + R(1));
      } else {
        R t = R(1) - q;
        res = k2_w * (t * t * t);
      }
    }
    return res;
  }
  // cubic_kernel_derivative, SPH/main.py:883-905
  V3<R> kernel_grad(const V3<R>& r) const {
    R r_norm = r.norm();
    R q = r_norm / h;
    V3<R> res;
    if (r_norm > R(1e-5) && q <= R(1)) {
      V3<R> grad_q = r / (r_norm * h);
      if (q <= R(0.5)) {
        res = grad_q * (k_grad * q * (R(3) * q - R(2)));
      } else {
        R f = R(1) - q;
        res = grad_q * (k_grad * (-f * f));
      }
    }
    return res;
  }

  bool is_fluid(int i) const { return material[i] == NN_FLUID; }
  bool is_static_solid(int i) const { return material[i] == NN_SOLID && !is_dynamic[i]; }
  bool is_dynamic_solid(int i) const { return material[i] == NN_SOLID && is_dynamic[i]; }
  R dt() const { return R(stats.dt); }

  // ---- neighbour search: NeighborhoodSearchSparse.run_search, SPH/main.py:822-847.
  // Same pair set as the reference (p_i != p_j and |x_i - x_j| < h on absolute
  // positions, SPH/main.py:845); cells of size h; each list sorted by id.
  int run_search() {
    double hs = p.support_radius;
    double lo[3] = {1e300, 1e300, 1e300};
    for (int i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) lo[d] = std::min(lo[d], double(x[i][d]));
    std::vector<int64_t> key(n);
    int64_t gmax[3] = {0, 0, 0};
    std::vector<int> cx(3 * (size_t)n);
    for (int i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) {
        int c = (int)std::floor((double(x[i][d]) - lo[d]) / hs);
        cx[3 * i + d] = c;
        gmax[d] = std::max<int64_t>(gmax[d], c + 1);
      }
    for (int i = 0; i < n; ++i) key[i] = ((int64_t)cx[3 * i + 2] * gmax[1] + cx[3 * i + 1]) * gmax[0] + cx[3 * i];
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a_, int b_) { return key[a_] < key[b_]; });
    std::vector<int64_t> skey(n);
    for (int i = 0; i < n; ++i) skey[i] = key[order[i]];
    std::vector<std::vector<int>> lists(n);
    const R hr = h;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
      std::vector<int>& L = lists[i];
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int c0 = cx[3 * i] + dx, c1 = cx[3 * i + 1] + dy, c2 = cx[3 * i + 2] + dz;
            if (c0 < 0 || c1 < 0 || c2 < 0 || c0 >= gmax[0] || c1 >= gmax[1] || c2 >= gmax[2]) continue;
            int64_t kk = ((int64_t)c2 * gmax[1] + c1) * gmax[0] + c0;
            auto it = std::lower_bound(skey.begin(), skey.end(), kk);
            for (size_t s = it - skey.begin(); s < (size_t)n && skey[s] == kk; ++s) {
              int j = order[s];
              if (j != i && (x[i] - x[j]).norm() < hr) L.push_back(j);
            }
          }
      std::sort(L.begin(), L.end());
    }
    nb_start.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) nb_start[i + 1] = nb_start[i] + (int)lists[i].size();
    nb.resize(nb_start[n]);
    int mx = 0;
    for (int i = 0; i < n; ++i) {
      std::copy(lists[i].begin(), lists[i].end(), nb.begin() + nb_start[i]);
      mx = std::max(mx, (int)lists[i].size());
    }
    stats.max_neighbors_seen = mx;
    return 0;
  }
  int64_t neighbor_total() override { return nb_start.empty() ? 0 : nb_start[n]; }

  int get_neighbors(int32_t* counts, int32_t* lists, int32_t width) override {
    if (nb_start.empty()) return NN_ERR_STATE;
    int rc = 0;
    for (int i = 0; i < n; ++i) {
      int c = nb_start[i + 1] - nb_start[i];
      counts[i] = c;
      for (int k = 0; k < width; ++k) lists[(size_t)i * width + k] = k < c ? nb[nb_start[i] + k] : -1;
      if (c > width) rc = NN_ERR_NEIGHBOR_OVERFLOW;
    }
    return rc;
  }

  // ---- SPHBase ------------------------------------------------------------
  // compute_static_boundary_volume / compute_moving_boundary_volume, SPH/main.py:1010-1035
  void boundary_volume(bool moving) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      if (moving ? !is_dynamic_solid(i) : !is_static_solid(i)) continue;
      R delta = W0;
      for (int k = nb_start[i]; k < nb_start[i + 1]; ++k) {
        int j = nb[k];
        if (material[j] == NN_SOLID) delta += kernel_w((x[i] - x[j]).norm());
      }
      volume[i] = R(1) / delta * R(3);
    }
  }
  // clear_accelerations_kernel, SPH/main.py:945-951
  void clear_accelerations() {
    V3<R> g(R(p.gravity[0]), R(p.gravity[1]), R(p.gravity[2]));
    for (int i = 0; i < n; ++i) a[i] = is_static_solid(i) ? V3<R>() : g;
  }
  // compute_densities, SPH/main.py:962-984
  void compute_densities() {
    const R rho0 = R(p.density0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      R d = volume[i] * W0;
      R den = 0;
      for (int k = nb_start[i]; k < nb_start[i + 1]; ++k) {
        int j = nb[k];
        den += volume[j] * kernel_w((x[i] - x[j]).norm());
      }
      d += den;
      density[i] = d * rho0;
    }
  }
  // compute_DFSPH_factor, SPH/main.py:1569-1608
  void compute_factor() {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      V3<R> grad_p_i;
      R sum_grad = 0;
      for (int k = nb_start[i]; k < nb_start[i + 1]; ++k) {
        int j = nb[k];
        V3<R> gpj = kernel_grad(x[i] - x[j]) * (-volume[j]);
        if (is_fluid(j)) sum_grad += gpj.norm_sqr();
        grad_p_i -= gpj;
      }
      sum_grad += grad_p_i.norm_sqr();
      alpha[i] = sum_grad > R(1e-6) ? R(-1) / sum_grad : R(0);
    }
  }
  // compute_density_change, SPH/main.py:1610-1645
  void compute_density_change() {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      R d = 0;
      int cnt = 0;
      for (int k = nb_start[i]; k < nb_start[i + 1]; ++k) {
        int j = nb[k];
        d += volume[j] * (v[i] - v[j]).dot(kernel_grad(x[i] - x[j]));
        ++cnt;
      }
      d = std::max(d, R(0));
      if (cnt < 20) d = R(0);
      rho_adv[i] = d;
    }
  }
  // compute_density_adv, SPH/main.py:1647-1667
  void compute_density_adv() {
    const R rho0 = R(p.density0);
    const R dt_ = dt();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      R delta = 0;
      for (int k = nb_start[i]; k < nb_start[i + 1]; ++k) {
        int j = nb[k];
        delta += volume[j] * (v[i] - v[j]).dot(kernel_grad(x[i] - x[j]));
      }
      R da = density[i] / rho0 + dt_ * delta;
      rho_adv[i] = std::max(da, R(1));
    }
  }
  // compute_density_error, SPH/main.py:1669-1675 (FP64 accumulation)
  double density_error(double offset) const {
    double s = 0;
    const R rho0 = R(p.density0), off = R(offset);
    for (int i = 0; i < n; ++i)
      if (is_fluid(i)) s += double(rho0 * rho_adv[i] - off);
    return s;
  }
  // multiply_time_step, SPH/main.py:1677-1681
  void multiply_alpha(R s) {
    for (int i = 0; i < n; ++i)
      if (is_fluid(i)) alpha[i] *= s;
  }
  // divergence_solver_iteration_kernel, SPH/main.py:1721-1760. Pushes onto dynamic
  // solids (1755-1760) are discarded by the clear_accelerations at 1552, so they are
  // applied to `a` here only for fidelity of the intermediate state.
  void divergence_iteration() {
    const R dt_ = dt(), eps = R(p.eps);
    std::vector<V3<R>> dvs(n);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      R k_i = rho_adv[i] * alpha[i];
      V3<R> dv;
      for (int kk = nb_start[i]; kk < nb_start[i + 1]; ++kk) {
        int j = nb[kk];
        if (is_fluid(j)) {
          R k_j = rho_adv[j] * alpha[j];
          R k_sum = k_i + k_j;
          if (std::fabs(k_sum) > eps) {
            V3<R> gpj = kernel_grad(x[i] - x[j]) * (-volume[j]);
            dv -= gpj * (dt_ * k_sum);
          }
        } else {
          if (std::fabs(k_i) > eps) {
            V3<R> gpj = kernel_grad(x[i] - x[j]) * (-volume[j]);
            dv += gpj * ((-dt_ * R(1)) * k_i);
          }
        }
      }
      dvs[i] = dv;
    }
    // serial pushes onto dynamic solids, in id order (the reference uses atomics)
    const R inv_dt = R(1) / dt_;
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      R k_i = rho_adv[i] * alpha[i];
      if (!(std::fabs(k_i) > eps)) continue;
      for (int kk = nb_start[i]; kk < nb_start[i + 1]; ++kk) {
        int j = nb[kk];
        if (!is_dynamic_solid(j)) continue;
        V3<R> gpj = kernel_grad(x[i] - x[j]) * (-volume[j]);
        V3<R> vc = gpj * ((-dt_ * R(1)) * k_i);
        a[j] += (-vc) * inv_dt;
      }
    }
    for (int i = 0; i < n; ++i)
      if (is_fluid(i)) v[i] += dvs[i];
  }
  // divergence_solve, SPH/main.py:1683-1719
  void divergence_solve() {
    compute_density_change();
    const R dt_ = dt();
    multiply_alpha(R(1.0 / double(dt_)));
    int it = 0;
    double avg = 0;
    const double eta = 1.0 / double(dt_) * p.max_error_v * 0.01 * p.density0;
    while (it < 1 || it < p.max_iterations_v) {
      divergence_iteration();
      compute_density_change();
      avg = density_error(0.0) / double(n_fluid);
      if (avg <= eta) break;
      ++it;
    }
    stats.iterations_v = it;
    stats.avg_density_err_v = avg;
    multiply_alpha(dt_);
  }
  // pressure_solve_iteration_kernel, SPH/main.py:1799-1841
  void pressure_iteration() {
    const R dt_ = dt(), eps = R(p.eps);
    std::vector<R> kap(n, 0);
    for (int i = 0; i < n; ++i)
      if (is_fluid(i)) kap[i] = (rho_adv[i] - R(1)) * alpha[i];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      R k_i = kap[i];
      V3<R> vi = v[i];
      for (int kk = nb_start[i]; kk < nb_start[i + 1]; ++kk) {
        int j = nb[kk];
        if (is_fluid(j)) {
          R k_sum = k_i + kap[j];
          if (std::fabs(k_sum) > eps) {
            V3<R> gpj = kernel_grad(x[i] - x[j]) * (-volume[j]);
            vi -= gpj * (dt_ * k_sum);
          }
        } else if (std::fabs(k_i) > eps) {
          V3<R> gpj = kernel_grad(x[i] - x[j]) * (-volume[j]);
          vi += gpj * ((-dt_ * R(1)) * k_i);
        }
      }
      v[i] = vi;
    }
    // two-way coupling pushes (SPH/main.py:1835-1841), serial in id order
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      R k_i = kap[i];
      if (!(std::fabs(k_i) > eps)) continue;
      for (int kk = nb_start[i]; kk < nb_start[i + 1]; ++kk) {
        int j = nb[kk];
        if (!is_dynamic_solid(j)) continue;
        V3<R> gpj = kernel_grad(x[i] - x[j]) * (-volume[j]);
        V3<R> vc = gpj * ((-dt_ * R(1)) * k_i);
        a[j] += (-vc) * R(1) / dt_;
      }
    }
  }
  // pressure_solve, SPH/main.py:1762-1797
  void pressure_solve() {
    const R dt_ = dt();
    compute_density_adv();
    multiply_alpha(R(1.0 / (double(dt_) * double(dt_))));
    int it = 0;
    double avg = 0;
    const double eta = p.max_error * 0.01 * p.density0;
    while (it < 1 || it < p.max_iterations) {
      pressure_iteration();
      compute_density_adv();
      avg = density_error(p.density0) / double(n_fluid);
      if (avg <= eta) break;
      ++it;
    }
    stats.iterations = it;
    stats.avg_density_err = avg;
  }
  // SurfaceTension.compute_surface_tension_kernel, SPH/main.py:1387-1414
  void surface_tension() {
    const R sigma = R(p.surface_tension);
    const double dia = 2.0 * p.particle_radius;
    const R dia2 = R(dia * dia);
    const R w_dia = kernel_w(V3<R>(R(dia), 0, 0).norm());
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      V3<R> dv;
      for (int k = nb_start[i]; k < nb_start[i + 1]; ++k) {
        int j = nb[k];
        if (!is_fluid(j)) continue;
        V3<R> r = x[i] - x[j];
        R r2 = r.dot(r);
        R c = sigma / m[i] * m[j];
        if (r2 > dia2)
          dv -= (r * c) * kernel_w(r.norm());
        else
          dv -= (r * c) * w_dia;
      }
      a[i] += dv;
    }
  }
  // ViscosityModel.compute_viscosity_force_kernel, SPH/main.py:1426-1468
  void viscosity_explicit() {
    const R d = R(10);
    const R nu = R(p.viscosity), nub = R(p.boundary_viscosity), rho0 = R(p.density0);
    const R c01h2 = R(0.01 * p.support_radius * p.support_radius);
    std::vector<V3<R>> dvs(n);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      V3<R> dv;
      for (int k = nb_start[i]; k < nb_start[i + 1]; ++k) {
        int j = nb[k];
        V3<R> r = x[i] - x[j];
        R v_xy = (v[i] - v[j]).dot(r);
        R rn = r.norm();
        if (is_fluid(j)) {
          R s = d * nu * (m[j] / density[j]) * v_xy / (rn * rn + c01h2);
          dv += kernel_grad(r) * s;
        } else if (p.boundary_viscosity != 0.0) {
          R s = d * nub * (rho0 * volume[j] / density[i]) * v_xy / (rn * rn + c01h2);
          dv += kernel_grad(r) * s;
        }
      }
      dvs[i] = dv;
    }
    if (p.boundary_viscosity != 0.0) {  // push -f_v onto dynamic solids (1459-1460)
      for (int i = 0; i < n; ++i) {
        if (!is_fluid(i)) continue;
        for (int k = nb_start[i]; k < nb_start[i + 1]; ++k) {
          int j = nb[k];
          if (!is_dynamic_solid(j)) continue;
          V3<R> r = x[i] - x[j];
          R v_xy = (v[i] - v[j]).dot(r);
          R rn = r.norm();
          R s = d * nub * (rho0 * volume[j] / density[i]) * v_xy / (rn * rn + c01h2);
          a[j] -= kernel_grad(r) * s;
        }
      }
    }
    for (int i = 0; i < n; ++i)
      if (is_fluid(i)) a[i] += dvs[i];
  }

  // NonNewton.calcStrainRate, SPH/main.py:461-492. Quirk mode keeps the reference's
  // bugs: the accumulator is overwritten by each neighbour and the norm is taken
  // before the 0.5/rho scaling. Otherwise the sum is accumulated and the norm is
  // taken of the scaled tensor D = (0.5/rho_i) sum_j m_j (v_ji (x) gW + gW (x) v_ji).
  void strain_rate_pass() {
    const bool q = quirks();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!q && !is_fluid(i)) { srn[i] = 0; strain_rate[i] = M3<R>(); continue; }
      M3<R> sr;
      for (int k = nb_start[i]; k < nb_start[i + 1]; ++k) {
        int j = nb[k];
        V3<R> gw = kernel_grad(x[i] - x[j]);
        V3<R> vji = v[j] - v[i];
        M3<R> vg = M3<R>::outer(vji, gw);
        M3<R> term;
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) term.a[r][c] = (vg.a[r][c] + vg.a[c][r]) * m[j];
        if (q) sr = term; else sr += term;
      }
      M3<R> D = sr * (R(0.5) / density[i]);
      strain_rate[i] = D;
      srn[i] = q ? sr.frob() : D.frob();
    }
  }
  // NonNewton viscosity laws, SPH/main.py:404-459. Quirk mode: the JSON int never
  // equals the Enum members (387-402), so the Newtonian branch always runs.
  R law(R g) const {
    int method = quirks() ? NN_NEWTONIAN : p.nonnewton_method;
    const R n_ = R(p.power_index), K = R(p.consistency_index), mu0 = R(p.viscosity0), muinf = R(p.viscosity_inf);
    const R gc = R(p.critical_strain_rate);
    switch (method) {
      case NN_POWER_LAW: return K * std::pow(g, n_ - R(1));
      case NN_CROSS: return muinf + (mu0 - muinf) / (R(1) + std::pow(K * g, n_));
      case NN_CASSON: { R s = std::sqrt(R(p.mu_c)) + std::sqrt(R(p.yield_stress) / g); return s * s; }
      case NN_CARREAU:
        if (has(NN_F_CARREAU_TEXTBOOK)) return muinf + (mu0 - muinf) * std::pow(R(1) + (K * g) * (K * g), (n_ - R(1)) / R(2));
        return muinf + (mu0 - muinf) / (R(1) + std::pow(K * g * g, (R(1) - n_) / R(2)));
      case NN_BINGHAM:
        if (g < gc) return mu0;
        return gc * (mu0 - muinf) / g + muinf;
      case NN_HERSCHEL_BULKLEY:
        if (g < gc) return mu0;
        return (mu0 * gc - K * std::pow(gc, n_)) / g + K * std::pow(g, n_ - R(1));
      default: return mu0;
    }
  }
  void nonnewton_pass() {
    strain_rate_pass();
    for (int i = 0; i < n; ++i) mu[i] = (quirks() || is_fluid(i)) ? law(srn[i]) : R(0);
  }

  // Implicit viscosity after Weiler, Koschier, Brand, Bender 2018 ("A Physically
  // Consistent Implicit Viscosity Solver for SPH Fluids"); the reference only stubs
  // it (SPH/main.py:1471-1513). Unknowns: new velocities of fluid particles. Row i
  // multiplied by m_i gives the symmetric positive definite system
  //   m_i x_i - dt d sum_fluid mu_ij (m_i m_j)/(rho_i rho_j) K_ij (x_i - x_j)
  //           - dt d sum_solid mu_b (m_i rho0 V_j)/(rho_i rho_i) K_ij (x_i - v_j) = m_i v_i
  // with d = 10, K_ij = gradW_ij x_ij^T / (|x_ij|^2 + 0.01 h^2), mu_ij = (mu_i+mu_j)/2
  // (dynamic viscosities from the non-Newtonian law, or viscosity*rho0), and
  // mu_b = visco_boundary * rho0. Solved by CG with a 3x3 block-Jacobi
  // preconditioner, FP64 dot products; the result adds (x_i - v_i)/dt to a_i.
  void implicit_viscosity() {
    const double dt_ = double(dt());
    const double d = 10.0, h2 = p.support_radius * p.support_radius;
    const double rho0 = p.density0, mub = p.visco_boundary * rho0;
    const bool use_law = has(NN_F_NONNEWTON);
    auto mu_of = [&](int i) -> double { return use_law ? double(mu[i]) : p.viscosity * rho0; };
    std::vector<int> idx;  // fluid particles
    for (int i = 0; i < n; ++i) if (is_fluid(i)) idx.push_back(i);
    const int nf = (int)idx.size();
    if (nf == 0) return;
    // matrix-free operator on R-precision vectors (like the GPU: FP32 vectors, FP64 dots)
    auto pair_coef = [&](int i, int j, const V3<R>& r, V3<R>& gw, R& w) {
      gw = kernel_grad(r);
      R rn = r.norm();
      w = R(1) / (rn * rn + R(0.01 * h2));
    };
    std::vector<V3<R>> xs(n), rr(n), zz(n), pp(n), Ap(n), bb(n);
    std::vector<double> pinv(9 * (size_t)n, 0.0);
    // rhs and preconditioner
#pragma omp parallel for schedule(static)
    for (int t = 0; t < nf; ++t) {
      int i = idx[t];
      double D[3][3] = {{double(m[i]), 0, 0}, {0, double(m[i]), 0}, {0, 0, double(m[i])}};
      V3<R> b = v[i] * m[i];
      for (int k = nb_start[i]; k < nb_start[i + 1]; ++k) {
        int j = nb[k];
        V3<R> r = x[i] - x[j];
        V3<R> gw; R w;
        pair_coef(i, j, r, gw, w);
        double c;
        if (is_fluid(j))
          c = dt_ * d * 0.5 * (mu_of(i) + mu_of(j)) * double(m[i]) * double(m[j]) / (double(density[i]) * double(density[j]));
        else
          c = dt_ * d * mub * double(m[i]) * rho0 * double(volume[j]) / (double(density[i]) * double(density[i]));
        // -c K_ij: K = gw r^T w (symmetric since gw is parallel to r)
        for (int a_ = 0; a_ < 3; ++a_)
          for (int b_ = 0; b_ < 3; ++b_) D[a_][b_] -= c * double(gw[a_]) * double(r[b_]) * double(w);
        if (!is_fluid(j) && is_dynamic_solid(j)) {  // moving boundary velocity on the rhs
          R kv = r.dot(v[j]) * w;
          b -= gw * R(c * double(kv));  // known boundary velocity: rhs -= c K v_j
        }
      }
      bb[i] = b;
      // invert D (symmetric 3x3)
      double det = D[0][0] * (D[1][1] * D[2][2] - D[1][2] * D[2][1]) - D[0][1] * (D[1][0] * D[2][2] - D[1][2] * D[2][0]) +
                   D[0][2] * (D[1][0] * D[2][1] - D[1][1] * D[2][0]);
      double inv[9];
      inv[0] = (D[1][1] * D[2][2] - D[1][2] * D[2][1]) / det;
      inv[1] = (D[0][2] * D[2][1] - D[0][1] * D[2][2]) / det;
      inv[2] = (D[0][1] * D[1][2] - D[0][2] * D[1][1]) / det;
      inv[3] = (D[1][2] * D[2][0] - D[1][0] * D[2][2]) / det;
      inv[4] = (D[0][0] * D[2][2] - D[0][2] * D[2][0]) / det;
      inv[5] = (D[0][2] * D[1][0] - D[0][0] * D[1][2]) / det;
      inv[6] = (D[1][0] * D[2][1] - D[1][1] * D[2][0]) / det;
      inv[7] = (D[0][1] * D[2][0] - D[0][0] * D[2][1]) / det;
      inv[8] = (D[0][0] * D[1][1] - D[0][1] * D[1][0]) / det;
      std::memcpy(&pinv[9 * (size_t)i], inv, sizeof(inv));
    }
    auto matvec = [&](const std::vector<V3<R>>& in, std::vector<V3<R>>& out) {
#pragma omp parallel for schedule(static)
      for (int t = 0; t < nf; ++t) {
        int i = idx[t];
        V3<R> acc = in[i] * m[i];
        for (int k = nb_start[i]; k < nb_start[i + 1]; ++k) {
          int j = nb[k];
          V3<R> r = x[i] - x[j];
          V3<R> gw; R w;
          pair_coef(i, j, r, gw, w);
          R c;
          V3<R> diff;
          if (is_fluid(j)) {
            c = R(dt_ * d * 0.5 * (mu_of(i) + mu_of(j)) * double(m[i]) * double(m[j]) / (double(density[i]) * double(density[j])));
            diff = in[i] - in[j];
          } else {
            c = R(dt_ * d * mub * double(m[i]) * rho0 * double(volume[j]) / (double(density[i]) * double(density[i])));
            diff = in[i];
          }
          acc -= gw * (c * r.dot(diff) * w);
        }
        out[i] = acc;
      }
    };
    auto apply_prec = [&](const std::vector<V3<R>>& in, std::vector<V3<R>>& out) {
      for (int t = 0; t < nf; ++t) {
        int i = idx[t];
        const double* P = &pinv[9 * (size_t)i];
        for (int r = 0; r < 3; ++r)
          out[i][r] = R(P[3 * r] * double(in[i].x) + P[3 * r + 1] * double(in[i].y) + P[3 * r + 2] * double(in[i].z));
      }
    };
    auto dot = [&](const std::vector<V3<R>>& u, const std::vector<V3<R>>& w) {
      double s = 0;
      for (int t = 0; t < nf; ++t) { int i = idx[t]; s += double(u[i].x) * double(w[i].x) + double(u[i].y) * double(w[i].y) + double(u[i].z) * double(w[i].z); }
      return s;
    };
    for (int t = 0; t < nf; ++t) xs[idx[t]] = v[idx[t]];  // initial guess: current velocity
    matvec(xs, Ap);
    for (int t = 0; t < nf; ++t) { int i = idx[t]; rr[i] = bb[i] - Ap[i]; }
    double bnorm = std::sqrt(dot(bb, bb));
    double rnorm = std::sqrt(dot(rr, rr));
    int it = 0;
    const double tol = p.visco_max_error;
    double rel = bnorm > 0 ? rnorm / bnorm : 0.0;
    if (rel > tol) {
      apply_prec(rr, zz);
      for (int t = 0; t < nf; ++t) pp[idx[t]] = zz[idx[t]];
      double rz = dot(rr, zz);
      while (it < p.visco_max_iter) {
        matvec(pp, Ap);
        double pAp = dot(pp, Ap);
        double al = pAp != 0 ? rz / pAp : 0.0;
        for (int t = 0; t < nf; ++t) {
          int i = idx[t];
          xs[i] += pp[i] * R(al);
          rr[i] -= Ap[i] * R(al);
        }
        ++it;
        rnorm = std::sqrt(dot(rr, rr));
        rel = bnorm > 0 ? rnorm / bnorm : 0.0;
        if (rel <= tol) break;
        apply_prec(rr, zz);
        double rz_new = dot(rr, zz);
        double be = rz != 0 ? rz_new / rz : 0.0;
        rz = rz_new;
        for (int t = 0; t < nf; ++t) { int i = idx[t]; pp[i] = zz[i] + pp[i] * R(be); }
      }
    }
    stats.cg_iterations = it;
    stats.cg_residual = rel;
    const R inv_dt = R(1.0 / dt_);
    for (int t = 0; t < nf; ++t) { int i = idx[t]; a[i] += (xs[i] - v[i]) * inv_dt; }
  }

  // compute_non_pressure_forces, SPH/main.py:1557-1567
  void non_pressure_forces() {
    if (has(NN_F_SURFACE_TENSION)) surface_tension();
    if (has(NN_F_NONNEWTON)) nonnewton_pass();
    if (has(NN_F_IMPLICIT_VISCOSITY) && !quirks())
      implicit_viscosity();
    else if (has(NN_F_VISCOSITY))
      viscosity_explicit();
  }
  // non_pressure_advect, SPH/main.py:1843-1848
  void non_pressure_advect() {
    const R dt_ = dt();
    for (int i = 0; i < n; ++i)
      if (is_dynamic[i] && is_fluid(i)) v[i] += a[i] * dt_;
  }
  // advect, SPH/main.py:1086-1093
  void advect() {
    const R dt_ = dt();
    for (int i = 0; i < n; ++i) {
      if (!is_dynamic[i]) continue;
      if (is_dynamic_solid(i)) v[i] += a[i] * dt_;
      x[i] += v[i] * dt_;
    }
  }
  // enforce_boundary_3D + simulate_collisions, SPH/main.py:1037-1080
  void enforce_boundary(int type) {
    R mx[3], mn[3];
    for (int d = 0; d < 3; ++d) { mx[d] = R(p.domain_end[d] - p.padding); mn[d] = R(p.domain_start[d] + p.padding); }
    const R cf = R(p.collision_coeff), st = R(p.sticky_coeff);
    for (int i = 0; i < n; ++i) {
      if (!(is_dynamic[i] && material[i] == type)) continue;
      V3<R> pos = x[i];
      V3<R> nrm;
      for (int d = 0; d < 3; ++d) {
        if (pos[d] > mx[d]) { nrm[d] += R(1); x[i][d] = mx[d]; }
        if (pos[d] <= mn[d]) { nrm[d] += R(-1); x[i][d] = mn[d]; }
      }
      R len = nrm.norm();
      if (len > R(1e-6)) {
        V3<R> nn = nrm / len;
        v[i] -= nn * ((R(1) + cf) * v[i].dot(nn));
        v[i] = v[i] * st;
      }
    }
  }
  // CFL time step (extension; the reference keeps dt fixed)
  void cfl_update() {
    if (!has(NN_F_CFL)) return;
    double vmax = 0;
    for (int i = 0; i < n; ++i)
      if (is_dynamic[i]) vmax = std::max(vmax, double(v[i].norm()));
    double dt_new = p.cfl_max_dt;
    if (vmax > 1e-9) dt_new = p.cfl_factor * 0.4 * (2.0 * p.particle_radius) / vmax;
    dt_new = std::min(std::max(dt_new, p.cfl_min_dt), p.cfl_max_dt);
    stats.dt = double(R(dt_new));
  }

  // ---- Elasticity (Becker 2009), SPH/main.py:1182-1375 -----------------------
  bool elastic_member(int i) const {
    if (quirks()) return true;  // Elasticity(meta.particle_max_num) loops over all (1893)
    return material[i] == NN_SOLID && phase_id[i] >= NN_PHASE_ELASTIC_BASE;
  }
  // Elasticity.initValues_kernel, SPH/main.py:1220-1239 (+ compute_density_func 1170-1179)
  void elastic_init() {
    std::vector<int> phases;
    for (int i = 0; i < n; ++i)
      if (material[i] == NN_SOLID && phase_id[i] >= NN_PHASE_ELASTIC_BASE) phases.push_back(phase_id[i]);
    std::sort(phases.begin(), phases.end());
    phases.erase(std::unique(phases.begin(), phases.end()), phases.end());
    elastic_multiplicity = quirks() ? (int)phases.size() : (phases.empty() ? 0 : 1);
    if (elastic_multiplicity == 0) { elastic_ready = false; return; }
    run_search();
    const int cap = quirks() ? 50 : (1 << 30);  // m_initialNeighbors is [N, 50] (1192, 1197)
    rest_start.assign(n + 1, 0);
    std::vector<std::vector<int>> L(n);
    for (int i = 0; i < n; ++i) {
      if (!elastic_member(i)) continue;
      for (int k = nb_start[i]; k < nb_start[i + 1]; ++k) {
        int j = nb[k];
        if (!quirks() && !(elastic_member(j) && phase_id[j] == phase_id[i])) continue;
        if ((int)L[i].size() < cap) L[i].push_back(j);
      }
    }
    for (int i = 0; i < n; ++i) rest_start[i + 1] = rest_start[i] + (int)L[i].size();
    rest_nb.resize(rest_start[n]);
    for (int i = 0; i < n; ++i) std::copy(L[i].begin(), L[i].end(), rest_nb.begin() + rest_start[i]);
    for (int i = 0; i < n; ++i) {
      if (!elastic_member(i)) continue;
      // rest density from the rest neighbourhood, mass based
      R den = m[i] * W0;
      if (quirks()) {
        for (int k = nb_start[i]; k < nb_start[i + 1]; ++k) { int j = nb[k]; den += m[j] * kernel_w((x[i] - x[j]).norm()); }
      } else {
        for (int k = rest_start[i]; k < rest_start[i + 1]; ++k) { int j = rest_nb[k]; den += m[j] * kernel_w((x[i] - x[j]).norm()); }
      }
      rest_volume[i] = m[i] / den;
      rot[i] = M3<R>::eye();
    }
    elastic_ready = true;
  }
  void elastic_constants(double& E, double& nu) const {
    if (quirks()) { E = 25e4; nu = 0.33; }  // hard-coded at SPH/main.py:1188-1189
    else { E = p.youngs_modulus; nu = p.poisson_ratio; }
  }
  // computeRotations_kernel, SPH/main.py:1249-1274
  void compute_rotations() {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!elastic_member(i)) continue;
      M3<R> A;
      for (int k = rest_start[i]; k < rest_start[i + 1]; ++k) {
        int j = rest_nb[k];
        V3<R> xji = x[j] - x[i], xji0 = x0[j] - x0[i];
        A += M3<R>::outer(xji, xji0) * (m[i] * kernel_w(xji0.norm()));
      }
      double Ad[3][3], Rd[3][3];
      for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) Ad[r][c] = double(A.a[r][c]);
      closest_rotation(Ad, Rd);
      for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) rot[i].a[r][c] = R(Rd[r][c]);
    }
  }
  // computeStress / computeStress_kernel, SPH/main.py:1276-1323
  void compute_stress() {
    double E, nu;
    elastic_constants(E, nu);
    double f = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    R c_d = R(f * (1.0 - nu)), c_o = R(f * nu), c_s = R(f * 0.5 * (1.0 - 2.0 * nu));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!elastic_member(i)) continue;
      M3<R> gu;
      for (int k = rest_start[i]; k < rest_start[i + 1]; ++k) {
        int j = rest_nb[k];
        V3<R> xji = x[j] - x[i], xji0 = x0[j] - x0[i];
        V3<R> uji = rot[i].mul_t(xji) - xji0;
        gu -= M3<R>::outer(uji * rest_volume[j], kernel_grad(xji0));
      }
      Fdef[i] = gu + M3<R>::eye();
      R e[6] = {gu.a[0][0], gu.a[1][1], gu.a[2][2], R(0.5) * (gu.a[0][1] + gu.a[1][0]),
                R(0.5) * (gu.a[0][2] + gu.a[2][0]), R(0.5) * (gu.a[1][2] + gu.a[2][1])};
      R* s = &stress[6 * (size_t)i];
      s[0] = c_d * e[0] + c_o * e[1] + c_o * e[2];
      s[1] = c_o * e[0] + c_d * e[1] + c_o * e[2];
      s[2] = c_o * e[0] + c_o * e[1] + c_d * e[2];
      s[3] = c_s * e[3];
      s[4] = c_s * e[4];
      s[5] = c_s * e[5];
    }
  }
  static V3<R> sym_mul(const R* M, const V3<R>& v) {  // symMatTimesVec, SPH/main.py:1328-1332
    return V3<R>(M[0] * v.x + M[3] * v.y + M[4] * v.z, M[3] * v.x + M[1] * v.y + M[5] * v.z,
                 M[4] * v.x + M[5] * v.y + M[2] * v.z);
  }
  // computeForces_kernel, SPH/main.py:1334-1375
  void compute_elastic_forces() {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!elastic_member(i)) continue;
      V3<R> fi;
      for (int k = rest_start[i]; k < rest_start[i + 1]; ++k) {
        int j = rest_nb[k];
        V3<R> xji0 = x0[j] - x0[i];
        V3<R> gw0 = kernel_grad(xji0);
        V3<R> dji = gw0 * rest_volume[i];
        V3<R> dij = gw0 * (-rest_volume[j]);
        V3<R> fij = sym_mul(&stress[6 * (size_t)j], dji) * (-rest_volume[j]);
        V3<R> fji = sym_mul(&stress[6 * (size_t)i], dij) * (-rest_volume[i]);
        fi += rot[j].mul(fij) - rot[i].mul(fji);
      }
      fi = fi * R(0.5);
      a[i] += fi / m[i];
    }
  }
  void elasticity_substep() {
    if (!elastic_ready) return;
    for (int rep = 0; rep < elastic_multiplicity; ++rep) {
      compute_rotations();
      compute_stress();
      compute_elastic_forces();
    }
  }

  // ---- Rigid bodies: RigidBodySolver, SPH/main.py:1099-1158 ---------------------
  std::vector<int> rigid_phases;
  std::vector<V3<double>> rigid_rest_cm;
  bool is_rigid(int i) const {
    return material[i] == NN_SOLID && is_dynamic[i] && phase_id[i] >= NN_PHASE_RIGID_BASE &&
           phase_id[i] < NN_PHASE_ELASTIC_BASE;
  }
  // compute_com, SPH/main.py:1120-1130 (mass = volume0 * density; FP64 accumulation)
  V3<double> rigid_com(int ph, bool rest) const {
    double sm = 0, c[3] = {0, 0, 0};
    const double V0 = double(R(p.volume0));
    for (int i = 0; i < n; ++i) {
      if (!(material[i] == NN_SOLID && is_dynamic[i] && phase_id[i] == ph)) continue;
      const double mass = double(R(V0) * density[i]);
      const V3<R>& xi = rest ? x0[i] : x[i];
      for (int d = 0; d < 3; ++d) c[d] += mass * double(xi[d]);
      sm += mass;
    }
    return V3<double>(c[0] / sm, c[1] / sm, c[2] / sm);
  }
  // RigidBodySolver.__init__ / compute_rigid_rest_cm, SPH/main.py:1101-1106, 1132-1134
  void rigid_init() {
    rigid_phases.clear();
    rigid_rest_cm.clear();
    if (!has(NN_F_RIGID)) return;
    for (int i = 0; i < n; ++i)
      if (is_rigid(i)) rigid_phases.push_back(phase_id[i]);
    std::sort(rigid_phases.begin(), rigid_phases.end());
    rigid_phases.erase(std::unique(rigid_phases.begin(), rigid_phases.end()), rigid_phases.end());
    for (int ph : rigid_phases) rigid_rest_cm.push_back(rigid_com(ph, true));
  }
  // RigidBodySolver.substep: ground_collision + solve_constraints, SPH/main.py:1108-1158
  void rigid_substep() {
    const R pad = R(p.padding);
    const double V0 = double(R(p.volume0));
    for (size_t b = 0; b < rigid_phases.size(); ++b) {
      const int ph = rigid_phases[b];
      for (int i = 0; i < n; ++i)  // ground_collision, 1113-1118: every solid particle
        if (material[i] == NN_SOLID && x[i][1] < pad) x[i][1] = pad;
      const V3<double> cm = rigid_com(ph, false);
      const V3<double>& rc = rigid_rest_cm[b];
      double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int i = 0; i < n; ++i) {
        if (!(material[i] == NN_SOLID && is_dynamic[i] && phase_id[i] == ph)) continue;
        const double mass = double(R(V0) * density[i]);
        double q[3], pp[3];
        for (int d = 0; d < 3; ++d) { q[d] = double(x0[i][d]) - rc[d]; pp[d] = double(x[i][d]) - cm[d]; }
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) A[r][c] += mass * pp[r] * q[c];
      }
      double Rm[3][3];
      closest_rotation(A, Rm);
      bool small = true;
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) small = small && std::fabs(Rm[r][c]) < 1e-6;
      if (small)
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) Rm[r][c] = r == c ? 1.0 : 0.0;
      for (int i = 0; i < n; ++i) {
        if (!(material[i] == NN_SOLID && is_dynamic[i] && phase_id[i] == ph)) continue;
        double q[3];
        for (int d = 0; d < 3; ++d) q[d] = double(x0[i][d]) - rc[d];
        for (int d = 0; d < 3; ++d) {
          const double goal = cm[d] + Rm[d][0] * q[0] + Rm[d][1] * q[1] + Rm[d][2] * q[2];
          x[i][d] = R(goal);
        }
      }
    }
  }
  void rigid_step() {
    const int reps = std::max(p.coupling_interval, 1);
    for (int k = 0; k < reps; ++k) rigid_substep();
  }

  // DFSPHSolver.substep, SPH/main.py:1546-1555
  void substep() {
    compute_densities();
    double mx = 0;
    for (int i = 0; i < n; ++i) if (is_fluid(i)) mx = std::max(mx, double(density[i]));
    stats.max_density = mx;
    compute_factor();
    if (has(NN_F_DIVERGENCE)) divergence_solve();
    clear_accelerations();
    non_pressure_forces();
    non_pressure_advect();
    pressure_solve();
  }
  // SPHBase.step, SPH/main.py:915-937
  int one_step() {
    cfl_update();
    run_search();
    boundary_volume(true);
    clear_accelerations();
    if (n_fluid > 0) substep();
    elasticity_substep();
    rigid_step();  // for rb in meta.rbs: coupling_interval x rb.substep() (SPH/main.py:929-931)
    advect();
    // animate_particles (SPH/main.py:283-309): every particle, static ones too, moves by
    // the frame's displacement after advection and before the boundary clamp
    if (anim[0] != R(0) || anim[1] != R(0) || anim[2] != R(0))
      for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) x[i][d] += anim[d];
    anim[0] = anim[1] = anim[2] = R(0);  // one step only
    enforce_boundary(NN_FLUID);
    enforce_boundary(NN_SOLID);
    stats.steps += 1;
    return 0;
  }
  R anim[3] = {R(0), R(0), R(0)};
  void set_animation(const double* d) override {
    for (int k = 0; k < 3; ++k) anim[k] = R(float(d[k]));
  }

  // ---- API -------------------------------------------------------------------
  int initialize() override {
    // initialize() builds Elasticity objects before solver.initialize() (1889-1895, 1915)
    elastic_init();
    rigid_init();
    run_search();
    boundary_volume(false);
    boundary_volume(true);
    return 0;
  }
  int step(int nsteps) override {
    for (int s = 0; s < nsteps; ++s) one_step();
    return 0;
  }
  int run_pass(int pass) override {
    if (pass != NN_PASS_SEARCH && pass != NN_PASS_CLEAR_ACCELERATIONS && pass != NN_PASS_ADVECT &&
        pass != NN_PASS_ENFORCE_BOUNDARY && pass != NN_PASS_NON_PRESSURE_ADVECT && nb_start.empty())
      return NN_ERR_STATE;
    switch (pass) {
      case NN_PASS_SEARCH: return run_search();
      case NN_PASS_STATIC_BOUNDARY_VOLUME: boundary_volume(false); return 0;
      case NN_PASS_MOVING_BOUNDARY_VOLUME: boundary_volume(true); return 0;
      case NN_PASS_CLEAR_ACCELERATIONS: clear_accelerations(); return 0;
      case NN_PASS_DENSITIES: compute_densities(); return 0;
      case NN_PASS_DFSPH_FACTOR: compute_factor(); return 0;
      case NN_PASS_DIVERGENCE_SOLVE: divergence_solve(); return 0;
      case NN_PASS_NON_PRESSURE_FORCES: non_pressure_forces(); return 0;
      case NN_PASS_NON_PRESSURE_ADVECT: non_pressure_advect(); return 0;
      case NN_PASS_PRESSURE_SOLVE: pressure_solve(); return 0;
      case NN_PASS_ELASTICITY: elasticity_substep(); return 0;
      case NN_PASS_ADVECT: advect(); return 0;
      case NN_PASS_ENFORCE_BOUNDARY: enforce_boundary(NN_FLUID); enforce_boundary(NN_SOLID); return 0;
      case NN_PASS_SUBSTEP: if (n_fluid > 0) substep(); return 0;
      case NN_PASS_RIGID: rigid_step(); return 0;
      default: return NN_ERR_INVALID_ARG;
    }
  }
  template <typename T>
  static void put3(const std::vector<V3<R>>& f, T* out, int n) {
    for (int i = 0; i < n; ++i) for (int d = 0; d < 3; ++d) out[3 * i + d] = T(f[i][d]);
  }
  int get_field(int field, double* out) override {
    switch (field) {
      case F_X: put3(x, out, n); return 0;
      case F_X0: put3(x0, out, n); return 0;
      case F_V: put3(v, out, n); return 0;
      case F_A: put3(a, out, n); return 0;
      case F_VOLUME: for (int i = 0; i < n; ++i) out[i] = volume[i]; return 0;
      case F_M: for (int i = 0; i < n; ++i) out[i] = m[i]; return 0;
      case F_DENSITY: for (int i = 0; i < n; ++i) out[i] = density[i]; return 0;
      case F_PRESSURE: for (int i = 0; i < n; ++i) out[i] = pressure[i]; return 0;
      case F_DFSPH_FACTOR: for (int i = 0; i < n; ++i) out[i] = alpha[i]; return 0;
      case F_DENSITY_ADV: for (int i = 0; i < n; ++i) out[i] = rho_adv[i]; return 0;
      case F_MATERIAL: for (int i = 0; i < n; ++i) out[i] = material[i]; return 0;
      case F_IS_DYNAMIC: for (int i = 0; i < n; ++i) out[i] = is_dynamic[i]; return 0;
      case F_PHASE_ID: for (int i = 0; i < n; ++i) out[i] = phase_id[i]; return 0;
      case F_STRAIN_RATE_NORM: for (int i = 0; i < n; ++i) out[i] = srn[i]; return 0;
      case F_NN_VISCOSITY: for (int i = 0; i < n; ++i) out[i] = mu[i]; return 0;
      case F_STRESS: for (size_t i = 0; i < 6 * (size_t)n; ++i) out[i] = stress[i]; return 0;
      case F_ROTATIONS:
        for (int i = 0; i < n; ++i) for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) out[9 * i + 3 * r + c] = rot[i].a[r][c];
        return 0;
      case F_REST_VOLUME: for (int i = 0; i < n; ++i) out[i] = rest_volume[i]; return 0;
      default: return NN_ERR_INVALID_ARG;
    }
  }
  int set_field(int field, const double* in) override {
    auto get3 = [&](std::vector<V3<R>>& f) { for (int i = 0; i < n; ++i) f[i] = V3<R>(R(in[3 * i]), R(in[3 * i + 1]), R(in[3 * i + 2])); };
    switch (field) {
      case F_X: get3(x); return 0;
      case F_X0: get3(x0); return 0;
      case F_V: get3(v); return 0;
      case F_A: get3(a); return 0;
      case F_VOLUME: for (int i = 0; i < n; ++i) volume[i] = R(in[i]); return 0;
      case F_M: for (int i = 0; i < n; ++i) m[i] = R(in[i]); return 0;
      case F_DENSITY: for (int i = 0; i < n; ++i) density[i] = R(in[i]); return 0;
      case F_DFSPH_FACTOR: for (int i = 0; i < n; ++i) alpha[i] = R(in[i]); return 0;
      case F_DENSITY_ADV: for (int i = 0; i < n; ++i) rho_adv[i] = R(in[i]); return 0;
      default: return NN_ERR_INVALID_ARG;
    }
  }
};

}  // namespace

extern "C" {

// Create an oracle simulation of one scene. use_double selects the FP64 build.
void* or_create(int use_double, const nn_scene_params* p, int n, int n_fluid, const double* x, const double* v,
                const int* material, const int* is_dynamic, const int* phase_id, const double* mass) {
  if (!p || n < 0 || !x || !material || !is_dynamic || !phase_id) return nullptr;
  if (use_double) return new Sim<double>(*p, n, n_fluid, x, v, material, is_dynamic, phase_id, mass);
  return new Sim<float>(*p, n, n_fluid, x, v, material, is_dynamic, phase_id, mass);
}
void or_destroy(void* s) { delete static_cast<SimBase*>(s); }
int or_initialize(void* s) { return static_cast<SimBase*>(s)->initialize(); }
int or_step(void* s, int nsteps) { return static_cast<SimBase*>(s)->step(nsteps); }
int or_run_pass(void* s, int pass) { return static_cast<SimBase*>(s)->run_pass(pass); }
int or_set_animation(void* s, const double* d) {
  static_cast<SimBase*>(s)->set_animation(d);
  return 0;
}
int or_get_field(void* s, int field, double* out) { return static_cast<SimBase*>(s)->get_field(field, out); }
int or_set_field(void* s, int field, const double* in) { return static_cast<SimBase*>(s)->set_field(field, in); }
int or_get_neighbors(void* s, int32_t* counts, int32_t* lists, int32_t width) {
  return static_cast<SimBase*>(s)->get_neighbors(counts, lists, width);
}
int64_t or_neighbor_total(void* s) { return static_cast<SimBase*>(s)->neighbor_total(); }
int or_get_stats(void* s, nn_stats* out) {
  SimBase* b = static_cast<SimBase*>(s);
  if (!out) return NN_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof(*out));
  out->size = sizeof(*out);
  out->status = b->stats.status;
  out->iterations_v = b->stats.iterations_v;
  out->iterations = b->stats.iterations;
  out->cg_iterations = b->stats.cg_iterations;
  out->max_neighbors_seen = b->stats.max_neighbors_seen;
  out->avg_density_err_v = b->stats.avg_density_err_v;
  out->avg_density_err = b->stats.avg_density_err;
  out->cg_residual = b->stats.cg_residual;
  out->dt = b->stats.dt;
  out->max_density = b->stats.max_density;
  out->steps = b->stats.steps;
  return 0;
}
void or_set_threads(int t) {
#ifdef _OPENMP
  if (t > 0) omp_set_num_threads(t);
#else
  (void)t;
#endif
}
int or_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void or_polar_rotation(const double* A, double* R) {
  double a[3][3], r[3][3];
  for (int i = 0; i < 9; ++i) a[i / 3][i % 3] = A[i];
  closest_rotation(a, r);
  for (int i = 0; i < 9; ++i) R[i] = r[i / 3][i % 3];
}

}  // extern "C"
