// surf.cuh — surface reconstruction of a particle set on the GPU: the reference's
// SRTool.dual_contouring (SPH/surf_recon/srtool.py:1264-1304).
//
// Pipeline (one launch sequence per call, all on the caller's stream):
//   1. particles binned by voxel (counting sort, id order inside a voxel)
//      — update_particles, srtool.py:1192-1195
//   2. isotropic poly6 splat onto the 27 vertices around each particle's voxel
//      — generate_fluid_field, srtool.py:1238-1251
//   3. anisotropic kernel per particle: weighted mean x_bar and covariance C over the
//      particles within 2 * smooth_radius, eigen-decomposition, G = (1/r_s) U S^-1 U^T
//      — pre_process_data, srtool.py:1006-1095 (particle 0 is skipped, as there)
//   4. anisotropic splat of the reference's kernel onto every vertex of every voxel in
//      the smoothing range, once per adjacent voxel (the multiplicity is computed, not
//      looped) — generate_smooth_fluid_field_impl, srtool.py:1135-1157
//   5. one value-weighted Gaussian smoothing pass with the standard deviation of the
//      negative vertex values — smooth_sdf, srtool.py:1425-1484
//   6. dual contouring: a QEF point per crossing cube (vertex ids by a scan in cube
//      order), then two triangles per crossing x/y/z edge of each cube's first corner
//      — dual_contouring_impl / dual_contouring_polygen, srtool.py:1531-1763
//   7. optional vertex normals — process_normal, srtool.py:1383-1410
//
// Layout: the vertex grid is dense, x fastest; blocks of NN_SR_BLOCK^3 vertices carry
// an "active" flag that emulates the reference's sparse fields (a block becomes active
// when any of its vertices is written; the smoothing and contouring visit every vertex
// of the active blocks and read 0 elsewhere). Splats accumulate in 64-bit fixed point
// (2^-32 units) with integer atomics, so the field is the same bits on every run
// whatever the order of the atomics.
//
// Restatement choices where the reference is undefined or nondeterministic: the QEF
// uses every crossing edge (the reference's 4x4 matrix overflows past 4 edges) through
// the normal equations with the reference's 0.1 clamp on the singular values;
// vertices and triangles are numbered in cube order.
#pragma once
#include "ns.cuh"

#define SR_FIX 4294967296.0  // fixed-point units per field unit
#define SR_PI 3.14159265358979323846

struct SrGrid {
  int nx, ny, nz, bx, by, bz;
  float ox, oy, oz, vs;        // f32, as the reference's get_voxel_index computes
  double dox, doy, doz, dvs;   // the same values in double
  __device__ __forceinline__ int64_t idx(int x, int y, int z) const {
    return x + (int64_t)nx * (y + (int64_t)ny * z);
  }
  __device__ __forceinline__ bool in(int x, int y, int z) const {
    return x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz;
  }
  __device__ __forceinline__ int64_t bidx(int x, int y, int z) const {
    return x / NN_SR_BLOCK + (int64_t)bx * (y / NN_SR_BLOCK + (int64_t)by * (z / NN_SR_BLOCK));
  }
  // get_voxel_index (srtool.py:799-803): f32, int() truncates toward zero
  __device__ __forceinline__ void voxel_of(float px, float py, float pz, int& x, int& y, int& z) const {
    x = (int)((px - ox) / vs);
    y = (int)((py - oy) / vs);
    z = (int)((pz - oz) / vs);
  }
};

struct SrDev {
  SrGrid g;
  int n;
  const float* pos;         // [n,3]
  int32_t* status;
  uint32_t* vcount;         // [cells+1] voxel counts, then starts
  uint32_t* vkey;           // [n]
  uint32_t* vrank;          // [n]
  int32_t* vsrc;            // [n] particles in voxel order
  float4* spos;             // [n] their positions, in the same order
  unsigned long long* fix;  // [cells] fixed-point field
  float* splat;             // [cells] field after the splats
  float* field;             // [cells] field after smoothing
  float* tmp;               // [cells]
  uint8_t* active;          // [blocks]
  float* G;                 // [n,9]
  float* xbar;              // [n,3]
  double* stats;            // sum, count, var, sd
  uint32_t* vflag;          // [cells+1] crossing-cube flags, then vertex ids
  uint32_t* tcount;         // [cells+1] index counts, then offsets
  uint32_t* cube_of;        // [max_v] cube (linear index) of each vertex id
  float* vert;              // [max_v,3]
  int32_t* tri;             // [max_i]
  float* nrm;               // [max_v,3]
  const float* vel;         // [n,3] particle velocities, or null (no velocity recording)
  unsigned long long* vfix; // [3][cells] fixed-point vertex velocities
  float* mvel;              // [max_v,3] mesh-vertex velocities
  int32_t max_v, max_i;
  float iso, sr, volume, acoeff;
  float q1_thr, q05_thr;     // largest f32 whose rounded square root is <= 1, <= 0.5
  float rr_thr;              // smallest f32 whose rounded square root is >= 2 smooth_radius
  int range, off, smooth_cells, record_normals;
};

// corner w of cube (x, y, z) is vertex (x, y, z) + off (srtool.py:775-783)
__constant__ int8_t c_sr_off[8][3] = {{0, 1, 0}, {1, 1, 0}, {1, 0, 0}, {0, 0, 0},
                                      {0, 1, 1}, {1, 1, 1}, {1, 0, 1}, {0, 0, 1}};
// corners of edge w (srtool.py:931-942)
__constant__ int8_t c_sr_edge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                        {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

__device__ __forceinline__ void sr_fail(const SrDev& s, int code) { atomicCAS(s.status, 0, code); }

__device__ __forceinline__ void sr_add(const SrDev& s, int64_t c, double val) {
  if (!isfinite(val)) { sr_fail(s, NN_ERR_NAN); return; }
  val = fmin(fmax(val, -1e8), 1e8);
  atomicAdd(&s.fix[c], (unsigned long long)(long long)llrint(val * SR_FIX));
}

// ---- 1. voxel binning --------------------------------------------------------------
__global__ void k_sr_keys(SrDev s) {
  GRID_STRIDE(i, s.n) {
    int x, y, z;
    s.g.voxel_of(s.pos[3 * i], s.pos[3 * i + 1], s.pos[3 * i + 2], x, y, z);
    if (!s.g.in(x, y, z)) { sr_fail(s, NN_ERR_INVALID_ARG); s.vkey[i] = 0xffffffffu; continue; }
    const uint32_t k = (uint32_t)s.g.idx(x, y, z);
    s.vkey[i] = k;
    s.vrank[i] = atomicAdd(&s.vcount[k], 1u);
    if (s.vrank[i] >= NN_SR_MAX_PER_VOXEL) sr_fail(s, NN_ERR_CAPACITY);
  }
}
__global__ void k_sr_scatter(SrDev s) {
  GRID_STRIDE(i, s.n) {
    const uint32_t k = s.vkey[i];
    if (k != 0xffffffffu) s.vsrc[s.vcount[k] + s.vrank[i]] = i;
  }
}
// id order inside a voxel (at most a few particles)
__global__ void k_sr_voxel_sort(SrDev s, int64_t cells) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells; c += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t b = s.vcount[c], e = s.vcount[c + 1];
    for (uint32_t i = b + 1; i < e; ++i) {
      const int v = s.vsrc[i];
      uint32_t j = i;
      while (j > b && s.vsrc[j - 1] > v) { s.vsrc[j] = s.vsrc[j - 1]; --j; }
      s.vsrc[j] = v;
    }
  }
}

// Positions in voxel order; only the first vcount[cells] entries of vsrc are filled
// (particles outside the grid are not binned, and the call then fails).
__global__ void k_sr_sorted_pos(SrDev s, int64_t cells) {
  const int nb = (int)min((int64_t)s.vcount[cells], (int64_t)s.n);
  GRID_STRIDE(k, nb) {
    const int i = s.vsrc[k];
    if (i < 0 || i >= s.n) continue;
    s.spos[k] = make_float4(s.pos[3 * i], s.pos[3 * i + 1], s.pos[3 * i + 2], 0.f);
  }
}

// ---- 2. isotropic splat (generate_fluid_field) --------------------------------------
__global__ void k_sr_iso(SrDev s) {
  GRID_STRIDE(i, s.n) {
    const float px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
    int cx, cy, cz;
    s.g.voxel_of(px, py, pz, cx, cy, cz);
    if (!s.g.in(cx, cy, cz)) continue;
    const float h = s.sr, h2 = h * h;
    const float h9 = h2 * h2 * h2 * h2 * h;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int x = cx + dx, y = cy + dy, z = cz + dz;
          if (x < 0 || y < 0 || z < 0) continue;
          if (!s.g.in(x, y, z)) { sr_fail(s, NN_ERR_CAPACITY); continue; }
          const float rx = px - (x * s.g.vs + s.g.ox), ry = py - (y * s.g.vs + s.g.oy), rz = pz - (z * s.g.vs + s.g.oz);
          const float r2 = rx * rx + ry * ry + rz * rz;
          float w = 0.f;  // poly6_weight, srtool.py:1212-1227
          if (sqrtf(r2) <= h) {
            const float t = h2 - r2;
            w = s.acoeff * (t * t * t) / h9;
          }
          s.active[s.g.bidx(x, y, z)] = 1;
          sr_add(s, s.g.idx(x, y, z), (double)(s.volume * w));
        }
  }
}

// ---- 3. anisotropic kernels (pre_process_data) ---------------------------------------
// symmetric 3x3 eigen-decomposition (cyclic Jacobi, double), descending eigenvalues,
// eigenvectors as the columns of V
__device__ void sr_sym_eig(const double S0[3][3], double lam[3], double V[3][3]) {
  double S[3][3], W[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) S[i][j] = S0[i][j];
  for (int sweep = 0; sweep < 16; ++sweep) {
    const double off = S[0][1] * S[0][1] + S[0][2] * S[0][2] + S[1][2] * S[1][2];
    const double dg = S[0][0] * S[0][0] + S[1][1] * S[1][1] + S[2][2] * S[2][2];
    if (off == 0.0 || off <= 1e-30 * dg) break;
#pragma unroll
    for (int pq = 0; pq < 3; ++pq) {
      const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
      if (S[p][q] == 0.0) continue;
      const double th = (S[q][q] - S[p][p]) / (2.0 * S[p][q]);
      const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
      const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
#pragma unroll
      for (int k = 0; k < 3; ++k) { const double a = S[k][p], b = S[k][q]; S[k][p] = c * a - sn * b; S[k][q] = sn * a + c * b; }
#pragma unroll
      for (int k = 0; k < 3; ++k) { const double a = S[p][k], b = S[q][k]; S[p][k] = c * a - sn * b; S[q][k] = sn * a + c * b; }
#pragma unroll
      for (int k = 0; k < 3; ++k) { const double a = W[k][p], b = W[k][q]; W[k][p] = c * a - sn * b; W[k][q] = sn * a + c * b; }
    }
  }
  const double d[3] = {S[0][0], S[1][1], S[2][2]};
  int o0 = 0, o1 = 1, o2 = 2;  // sort descending
  if (d[o1] > d[o0]) { int t = o0; o0 = o1; o1 = t; }
  if (d[o2] > d[o1]) { int t = o1; o1 = o2; o2 = t; }
  if (d[o1] > d[o0]) { int t = o0; o0 = o1; o1 = t; }
  const int o[3] = {o0, o1, o2};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    lam[c] = d[o[c]];
#pragma unroll
    for (int r = 0; r < 3; ++r) V[r][c] = W[r][o[c]];
  }
}

// Visits the particles within the smoothing range of voxel (cx, cy, cz) whose voxel
// can hold a point closer than `reach`, row by row (the voxels of one (y, z) row are
// one contiguous stretch of the voxel-sorted arrays, whose index k is passed to f);
// lane `lane` of `lanes` takes every lanes-th row.
// The particles of the voxel rows (x-runs) of the range around voxel (cx, cy, cz)
// whose y-z slab comes within `reach` of p, visited by a whole warp. Only about one
// row in four of the range crosses a particle lattice at half the voxel density, so
// lanes owning rows would mostly idle: each lane takes one row of a group of 32, a
// warp scan of the row counts lays their particles end to end, and lane l handles
// particles l, l + 32, ... of the group, finding its row by a search over the scan.
// f(k) gets the voxel-sorted index of each particle; `valid` lanes only.
template <typename F>
__device__ __forceinline__ void sr_range_particles(const SrDev& s, int cx, int cy, int cz, float px, float py,
                                                   float pz, float reach, int lane, F f) {
  const SrGrid& g = s.g;
  const unsigned full = 0xffffffffu;
  const int lo = -s.off, hi = s.range - 1 - s.off;
  const float r2 = reach * reach;
  const int x0 = max(cx + lo, 0), x1 = min(cx + hi, g.nx - 1);
  if (x0 > x1) return;  // warp-uniform
  const int nrows = s.range * s.range;
  for (int r0 = 0; r0 < nrows; r0 += 32) {
    const int r = r0 + lane;
    uint32_t b = 0, cnt = 0;
    if (r < nrows) {
      const int z = cz + lo + r / s.range, y = cy + lo + r % s.range;
      if (z >= 0 && z < g.nz && y >= 0 && y < g.ny) {
        const float zc = fmaxf(fmaxf(g.oz + z * g.vs - pz, pz - (g.oz + (z + 1) * g.vs)), 0.f);
        const float yc = fmaxf(fmaxf(g.oy + y * g.vs - py, py - (g.oy + (y + 1) * g.vs)), 0.f);
        if (yc * yc + zc * zc <= r2) {
          b = s.vcount[g.idx(x0, y, z)];
          cnt = s.vcount[g.idx(x1, y, z) + 1] - b;
        }
      }
    }
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(full, incl, o);
      if (lane >= o) incl += v;
    }
    const uint32_t total = __shfl_sync(full, incl, 31);
    for (uint32_t base = 0; base < total; base += 32) {
      const uint32_t t = base + lane;
      int l = 0;  // the first row lane whose inclusive count exceeds t
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1)
        if (__shfl_sync(full, incl, l + step - 1) <= t) l += step;
      const uint32_t bl = __shfl_sync(full, b, l), il = __shfl_sync(full, incl, l), cl = __shfl_sync(full, cnt, l);
      if (t < total) f(bl + (t - (il - cl)));
    }
  }
}

// One warp per particle: lanes split the particles of the range and the moments are
// reduced across the warp with shuffles.
__global__ void k_sr_aniso_pre(SrDev s) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < s.n; i += warps) {
    if (i == 0) continue;  // the reference's loop starts at 1 (srtool.py:1013)
    const float px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
    int cx, cy, cz;
    s.g.voxel_of(px, py, pz, cx, cy, cz);
    const float rr = 2.f * s.sr;  // isoweight radius
    // one pass over the neighbourhood: weights, and the first and second moments of
    // the offsets d_j = x_j - x_i, from which x_w = x_i + <d> and
    // C = sum w (x_j - x_w)(x_j - x_w)^T / sum w = <d d^T> - <d><d>^T (srtool.py:1021-1061)
    double tw = 0.0, m1[3] = {0.0, 0.0, 0.0}, m2[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    int nnb = 0;
    // a margin of one voxel on the pruning distance keeps every pair with w > 0
    sr_range_particles(s, cx, cy, cz, px, py, pz, rr + s.g.vs, lane, [&](uint32_t k) {
      const float4 pj = s.spos[k];
      const float dx = __fsub_rn(px, pj.x), dy = __fsub_rn(py, pj.y), dz = __fsub_rn(pz, pj.z);
      const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
      // |x_i - x_j| in f32 (unfused, as any f32 evaluation of it) < 2 r_s, decided on
      // the square: rn(sqrt(d2)) < rr exactly when d2 < rr_thr
      if (d2 < s.rr_thr) {
        const float dn = __fsqrt_rn(d2);
        const float q = dn / rr;
        const double w = 1.0 - (double)(q * q * q);  // isoweight, srtool.py:993-999
        const double d[3] = {(double)pj.x - px, (double)pj.y - py, (double)pj.z - pz};
        tw += w;
        m1[0] += w * d[0]; m1[1] += w * d[1]; m1[2] += w * d[2];
        if (w > 0) {
          ++nnb;
          m2[0] += w * d[0] * d[0]; m2[1] += w * d[1] * d[1]; m2[2] += w * d[2] * d[2];
          m2[3] += w * d[0] * d[1]; m2[4] += w * d[0] * d[2]; m2[5] += w * d[1] * d[2];
        }
      }
    });
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      tw += __shfl_xor_sync(0xffffffffu, tw, o);
#pragma unroll
      for (int k = 0; k < 3; ++k) m1[k] += __shfl_xor_sync(0xffffffffu, m1[k], o);
#pragma unroll
      for (int k = 0; k < 6; ++k) m2[k] += __shfl_xor_sync(0xffffffffu, m2[k], o);
      nnb += __shfl_xor_sync(0xffffffffu, nnb, o);
    }
    if (lane != 0) continue;
    double db[3] = {0.0, 0.0, 0.0}, C[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (tw != 0.0) {
      db[0] = m1[0] / tw; db[1] = m1[1] / tw; db[2] = m1[2] / tw;
      C[0][0] = m2[0] / tw - db[0] * db[0]; C[1][1] = m2[1] / tw - db[1] * db[1]; C[2][2] = m2[2] / tw - db[2] * db[2];
      C[0][1] = C[1][0] = m2[3] / tw - db[0] * db[1];
      C[0][2] = C[2][0] = m2[4] / tw - db[0] * db[2];
      C[1][2] = C[2][1] = m2[5] / tw - db[1] * db[2];
    }
    const double xw[3] = {tw != 0.0 ? px + db[0] : 0.0, tw != 0.0 ? py + db[1] : 0.0, tw != 0.0 ? pz + db[2] : 0.0};
    const double lam_ = 0.9;  // akLambda
    s.xbar[3 * i] = (float)((1 - lam_) * px + lam_ * xw[0]);
    s.xbar[3 * i + 1] = (float)((1 - lam_) * py + lam_ * xw[1]);
    s.xbar[3 * i + 2] = (float)((1 - lam_) * pz + lam_ * xw[2]);
    double lam[3], V[3][3];
    sr_sym_eig(C, lam, V);
    double sg[3] = {lam[0], lam[1], lam[2]};
    if (nnb > 25) {  // Nvep, kr = 4, ks = 1400 (srtool.py:910-914, 1072-1079)
      sg[1] = fmax(sg[1], sg[0] / 4.0);
      sg[2] = fmax(sg[2], sg[0] / 4.0);
      sg[0] *= 1400.0; sg[1] *= 1400.0; sg[2] *= 1400.0;
    } else {
      sg[0] = sg[1] = sg[2] = 0.5;  // kn
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const double m = V[a][0] * V[b][0] / sg[0] + V[a][1] * V[b][1] / sg[1] + V[a][2] * V[b][2] / sg[2];
        s.G[9 * i + 3 * a + b] = (float)(tw != 0.0 ? m / (double)s.sr : (a == b ? 1.0 : 0.0));
      }
  }
}

// ---- 4. anisotropic splat (generate_smooth_fluid_field_impl) -------------------------
// One warp per particle; lanes stride over the vertices of the kernel's support box.
__global__ void k_sr_aniso_splat(SrDev s) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < s.n; i += warps) {
    const SrGrid& g = s.g;
    int cx, cy, cz;
    g.voxel_of(s.pos[3 * i], s.pos[3 * i + 1], s.pos[3 * i + 2], cx, cy, cz);
    // voxels [c - off, c - off + range - 1]; their vertices one further
    const int lo[3] = {cx - s.off, cy - s.off, cz - s.off};
    const int hi[3] = {lo[0] + s.range - 1, lo[1] + s.range - 1, lo[2] + s.range - 1};
    if (hi[0] + 1 >= g.nx || hi[1] + 1 >= g.ny || hi[2] + 1 >= g.nz) {
      if (lane == 0) sr_fail(s, NN_ERR_CAPACITY);
      continue;
    }
    const int v0[3] = {max(lo[0], 0), max(lo[1], 0), max(lo[2], 0)};
    const int v1[3] = {hi[0] + 1, hi[1] + 1, hi[2] + 1};
    if (v1[0] < 0 || v1[1] < 0 || v1[2] < 0) continue;
    {  // every vertex of the box is written (+= 0 included): activate its blocks
      const int b0 = v0[0] / NN_SR_BLOCK, b1 = v1[0] / NN_SR_BLOCK, c0 = v0[1] / NN_SR_BLOCK,
                c1 = v1[1] / NN_SR_BLOCK, e0 = v0[2] / NN_SR_BLOCK, e1 = v1[2] / NN_SR_BLOCK;
      const int nbx = b1 - b0 + 1, nby = c1 - c0 + 1, nb = nbx * nby * (e1 - e0 + 1);
      for (int t = lane; t < nb; t += 32) {
        const int bx = b0 + t % nbx, by = c0 + (t / nbx) % nby, bz = e0 + t / (nbx * nby);
        s.active[bx + (int64_t)g.bx * (by + (int64_t)g.by * bz)] = 1;
      }
    }
    float Gm[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) Gm[k] = s.G[9 * i + k];
    const double det = (double)Gm[0] * ((double)Gm[4] * Gm[8] - (double)Gm[5] * Gm[7]) -
                       (double)Gm[1] * ((double)Gm[3] * Gm[8] - (double)Gm[5] * Gm[6]) +
                       (double)Gm[2] * ((double)Gm[3] * Gm[7] - (double)Gm[4] * Gm[6]);
    if (det == 0.0) continue;  // G = 0 (particle 0): the kernel is 0 everywhere
    // support |G d| <= 1 is an ellipsoid; its bounding half-widths are the row norms of G^-1
    double Gi[3][3];
    Gi[0][0] = ((double)Gm[4] * Gm[8] - (double)Gm[5] * Gm[7]) / det;
    Gi[0][1] = ((double)Gm[2] * Gm[7] - (double)Gm[1] * Gm[8]) / det;
    Gi[0][2] = ((double)Gm[1] * Gm[5] - (double)Gm[2] * Gm[4]) / det;
    Gi[1][0] = ((double)Gm[5] * Gm[6] - (double)Gm[3] * Gm[8]) / det;
    Gi[1][1] = ((double)Gm[0] * Gm[8] - (double)Gm[2] * Gm[6]) / det;
    Gi[1][2] = ((double)Gm[2] * Gm[3] - (double)Gm[0] * Gm[5]) / det;
    Gi[2][0] = ((double)Gm[3] * Gm[7] - (double)Gm[4] * Gm[6]) / det;
    Gi[2][1] = ((double)Gm[1] * Gm[6] - (double)Gm[0] * Gm[7]) / det;
    Gi[2][2] = ((double)Gm[0] * Gm[4] - (double)Gm[1] * Gm[3]) / det;
    const float xb[3] = {s.xbar[3 * i], s.xbar[3 * i + 1], s.xbar[3 * i + 2]};
    const double org[3] = {g.dox, g.doy, g.doz};
    int w0[3], w1[3];
    bool empty = false;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double hw = sqrt(Gi[a][0] * Gi[a][0] + Gi[a][1] * Gi[a][1] + Gi[a][2] * Gi[a][2]);
      const double lo_v = (xb[a] - hw - org[a]) / g.dvs, hi_v = (xb[a] + hw - org[a]) / g.dvs;
      w0[a] = max(v0[a], (int)fmax(floor(lo_v) - 1.0, -1e9));
      w1[a] = min(v1[a], (int)fmin(ceil(hi_v) + 1.0, 1e9));
      empty |= w0[a] > w1[a];
    }
    if (empty) continue;
    const float k1 = (float)(48.0 / SR_PI * det), k2 = (float)(16.0 / SR_PI * det);
    // each lane owns (x, y) columns of the box and walks z; the x and y terms of
    // G d are per column and the sums keep the order ((G0 d0 + G1 d1) + G2 d2)
    const int nxw = w1[0] - w0[0] + 1, ncol = nxw * (w1[1] - w0[1] + 1);
    const int64_t plane = (int64_t)g.nx * g.ny;
    for (int col = lane; col < ncol; col += 32) {
      const int x = w0[0] + col % nxw, y = w0[1] + col / nxw;
      const int mxy = ((x - 1 >= lo[0] && x - 1 <= hi[0]) + (x >= lo[0] && x <= hi[0])) *
                      ((y - 1 >= lo[1] && y - 1 <= hi[1]) + (y >= lo[1] && y <= hi[1]));
      if (mxy == 0) continue;
      const float d0 = __fsub_rn(xb[0], __fadd_rn(__fmul_rn((float)x, g.vs), g.ox));
      const float d1 = __fsub_rn(xb[1], __fadd_rn(__fmul_rn((float)y, g.vs), g.oy));
      const float a0 = __fadd_rn(__fmul_rn(Gm[0], d0), __fmul_rn(Gm[1], d1));
      const float a1 = __fadd_rn(__fmul_rn(Gm[3], d0), __fmul_rn(Gm[4], d1));
      const float a2 = __fadd_rn(__fmul_rn(Gm[6], d0), __fmul_rn(Gm[7], d1));
      const int64_t base = g.idx(x, y, 0);
      for (int z = w0[2]; z <= w1[2]; ++z) {
        // q = |G (x_bar - vertex)| in f32 with unfused operations: the kernel as written
        // jumps at q = 0.5, so q must round the same way in every f32 evaluation
        const float d2 = __fsub_rn(xb[2], __fadd_rn(__fmul_rn((float)z, g.vs), g.oz));
        const float q0 = __fadd_rn(a0, __fmul_rn(Gm[2], d2));
        const float q1 = __fadd_rn(a1, __fmul_rn(Gm[5], d2));
        const float q2 = __fadd_rn(a2, __fmul_rn(Gm[8], d2));
        const float q2s = __fadd_rn(__fadd_rn(__fmul_rn(q0, q0), __fmul_rn(q1, q1)), __fmul_rn(q2, q2));
        // outside the support: rn(sqrt(q2s)) > 1 exactly when q2s > q1_thr
        if (!(q2s <= s.q1_thr) || !(q2s > 0.f)) continue;
        // the branch of cubic_spline_kernel (srtool.py:1114-1124) is decided exactly
        // (rn(sqrt(q2s)) <= 0.5 exactly when q2s <= q05_thr); its value, continuous
        // within a branch, takes q from the hardware reciprocal square root
        const float q = q2s * rsqrtf(q2s);
        const float res = q2s <= s.q05_thr ? k1 * (q * q * q - q * q) + 1.f : k2 * (1.f - q) * (1.f - q) * (1.f - q);
        // vertex (x, y, z) belongs to the voxels x - 1 and x of the box, per axis; the
        // multiplicity is 1, 2, 4 or 8, a power of two, so scaling by it is exact
        const int m = mxy * ((z - 1 >= lo[2] && z - 1 <= hi[2]) + (z >= lo[2] && z <= hi[2]));
        if (m == 0) continue;
        const float c = s.volume * res;
        if (!isfinite(c)) { sr_fail(s, NN_ERR_NAN); continue; }
        const long long u = __float2ll_rn(fminf(fmaxf(c, -1e8f), 1e8f) * (4294967296.f * (float)m));
        atomicAdd(&s.fix[base + z * plane], (unsigned long long)u);
      }
    }
  }
}

// Velocity splat (generate_smooth_fluid_field_with_velocity_impl, srtool.py:1159-1190):
// every vertex of every voxel in the smoothing range, once per adjacent voxel, gets
// v_i * poly6(x_i - vertex, r_s) * voxel_size^3. One warp per particle; lanes own
// (x, y) columns of the poly6 support's box and walk z.
__global__ void k_sr_vel_splat(SrDev s) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const float h = s.sr, h2 = h * h, h9 = h2 * h2 * h2 * h2 * h;
  const float coeff = s.g.vs * s.g.vs * s.g.vs;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < s.n; i += warps) {
    const SrGrid& g = s.g;
    const float px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
    int cx, cy, cz;
    g.voxel_of(px, py, pz, cx, cy, cz);
    const int lo[3] = {cx - s.off, cy - s.off, cz - s.off};
    const int hi[3] = {lo[0] + s.range - 1, lo[1] + s.range - 1, lo[2] + s.range - 1};
    if (hi[0] + 1 >= g.nx || hi[1] + 1 >= g.ny || hi[2] + 1 >= g.nz) continue;  // flagged by the field splat
    const float p[3] = {px, py, pz};
    const float org[3] = {g.ox, g.oy, g.oz};
    int w0[3], w1[3];
    bool empty = false;
#pragma unroll
    for (int a = 0; a < 3; ++a) {  // the poly6 support |x_i - vertex| <= r_s, one vertex of margin
      w0[a] = max(max(lo[a], 0), (int)floorf((p[a] - h - org[a]) / g.vs) - 1);
      w1[a] = min(hi[a] + 1, (int)ceilf((p[a] + h - org[a]) / g.vs) + 1);
      empty |= w0[a] > w1[a];
    }
    if (empty) continue;
    const float v[3] = {s.vel[3 * i], s.vel[3 * i + 1], s.vel[3 * i + 2]};
    const int nxw = w1[0] - w0[0] + 1, ncol = nxw * (w1[1] - w0[1] + 1);
    const int64_t plane = (int64_t)g.nx * g.ny, cells = plane * g.nz;
    for (int col = lane; col < ncol; col += 32) {
      const int x = w0[0] + col % nxw, y = w0[1] + col / nxw;
      const int mxy = ((x - 1 >= lo[0] && x - 1 <= hi[0]) + (x >= lo[0] && x <= hi[0])) *
                      ((y - 1 >= lo[1] && y - 1 <= hi[1]) + (y >= lo[1] && y <= hi[1]));
      if (mxy == 0) continue;
      const float rx = px - (x * g.vs + g.ox), ry = py - (y * g.vs + g.oy);
      const int64_t base = g.idx(x, y, 0);
      for (int z = w0[2]; z <= w1[2]; ++z) {
        const float rz = pz - (z * g.vs + g.oz);
        const float r2 = rx * rx + ry * ry + rz * rz;
        if (!(sqrtf(r2) <= h)) continue;  // poly6_weight, srtool.py:1212-1227
        const float t = h2 - r2;
        const float w = s.acoeff * (t * t * t) / h9 * coeff;
        const int m = mxy * ((z - 1 >= lo[2] && z - 1 <= hi[2]) + (z >= lo[2] && z <= hi[2]));
        if (m == 0) continue;
        const int64_t c = base + z * plane;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float cv = v[k] * w;
          if (!isfinite(cv)) { sr_fail(s, NN_ERR_NAN); continue; }
          const long long u = __float2ll_rn(fminf(fmaxf(cv, -1e8f), 1e8f) * (4294967296.f * (float)m));
          atomicAdd(&s.vfix[k * cells + c], (unsigned long long)u);
        }
      }
    }
  }
}

// process_velocity (srtool.py:1351-1381): trilinear blend of the 8 vertex velocities
// around each mesh vertex
__global__ void k_sr_mesh_velocity(SrDev s, int nv) {
  const int64_t plane = (int64_t)s.g.nx * s.g.ny, cells = plane * s.g.nz;
  GRID_STRIDE(i, min(nv, s.max_v)) {
    const double p[3] = {s.vert[3 * i], s.vert[3 * i + 1], s.vert[3 * i + 2]};
    int x0, y0, z0;
    s.g.voxel_of((float)p[0], (float)p[1], (float)p[2], x0, y0, z0);
    const double xd = (p[0] - (x0 * s.g.dvs + s.g.dox)) / s.g.dvs, yd = (p[1] - (y0 * s.g.dvs + s.g.doy)) / s.g.dvs,
                 zd = (p[2] - (z0 * s.g.dvs + s.g.doz)) / s.g.dvs;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int e = 0; e < 2; ++e) {
          const int x = x0 + a, y = y0 + b, z = z0 + e;
          if (!s.g.in(x, y, z)) continue;
          const double wgt = (a ? xd : 1 - xd) * (b ? yd : 1 - yd) * (e ? zd : 1 - zd);
          const int64_t c = s.g.idx(x, y, z);
          for (int k = 0; k < 3; ++k) acc[k] += wgt * ((double)(long long)s.vfix[k * cells + c] / SR_FIX);
        }
    for (int k = 0; k < 3; ++k) s.mvel[3 * i + k] = (float)acc[k];
  }
}

__global__ void k_sr_fix_to_field(SrDev s, int64_t cells) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells; c += (int64_t)gridDim.x * blockDim.x) {
    const float v = (float)((double)(long long)s.fix[c] / SR_FIX);
    s.splat[c] = v;
    s.field[c] = v;
  }
}

// ---- 5. smoothing (smooth_sdf) --------------------------------------------------------
__device__ __forceinline__ bool sr_act(const SrDev& s, int x, int y, int z) {
  return s.g.in(x, y, z) && s.active[s.g.bidx(x, y, z)];
}
__device__ __forceinline__ float sr_get(const SrDev& s, const float* f, int x, int y, int z) {
  return sr_act(s, x, y, z) ? f[s.g.idx(x, y, z)] : 0.f;
}

// density_field_stats (srtool.py:1436-1456): pass 0 sums the negative values of the
// active vertices and counts them, pass 1 their squared deviations from the mean
__global__ void k_sr_stats(SrDev s, int64_t cells, int pass) {
  double a = 0.0, b = 0.0;
  const double mean = pass ? s.stats[0] / s.stats[1] : 0.0;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells; c += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(c % s.g.nx), y = (int)((c / s.g.nx) % s.g.ny), z = (int)(c / ((int64_t)s.g.nx * s.g.ny));
    if (!s.active[s.g.bidx(x, y, z)]) continue;
    const float v = s.field[c];
    if (v < 0.f) {
      if (pass == 0) { a += v; b += 1.0; }
      else { const double d = v - mean; a += d * d; }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (pass == 0) { atomicAdd(&s.stats[0], a); atomicAdd(&s.stats[1], b); }
    else atomicAdd(&s.stats[2], a);
  }
}
__global__ void k_sr_sd(SrDev s) {
  // 0/0 = NaN without negative values, as in the reference (the smoothing then
  // produces NaN and the contouring finds no crossing)
  if (threadIdx.x == 0) s.stats[3] = sqrt(s.stats[2] / s.stats[1]);
}

__global__ void k_sr_smooth(SrDev s, int64_t cells) {
  const float sd = (float)s.stats[3];
  const float inv2s2 = 1.f / (2.f * sd * sd);
  const float norm = powf(2.f * (float)SR_PI * sd * sd, 1.5f);
  const int R = s.smooth_cells;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells; c += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(c % s.g.nx), y = (int)((c / s.g.nx) % s.g.ny), z = (int)(c / ((int64_t)s.g.nx * s.g.ny));
    if (!s.active[s.g.bidx(x, y, z)]) { s.tmp[c] = 0.f; continue; }
    const float v0 = s.field[c];
    float avg = 0.f, wsum = 0.f;
    for (int dz = -R; dz <= R; ++dz)
      for (int dy = -R; dy <= R; ++dy)
        for (int dx = -R; dx <= R; ++dx) {
          const int a = x + dx, b = y + dy, e = z + dz;
          if (a < 0 || b < 0 || e < 0) continue;
          const float vv = sr_get(s, s.field, a, b, e);
          const float diff = fabsf(v0 - vv);
          const float gw = expf(-diff * diff * inv2s2) / norm;  // gaussian_blur, srtool.py:1432-1434
          avg += gw * vv;
          wsum += gw;
        }
    if (wsum != 0.f) avg /= wsum;
    s.tmp[c] = avg;
  }
}

// ---- 6. dual contouring ---------------------------------------------------------------
__device__ __forceinline__ int sr_cube_mask(const SrDev& s, int x, int y, int z) {
  int ci = 0;
#pragma unroll
  for (int w = 0; w < 8; ++w)
    if (sr_get(s, s.field, x + c_sr_off[w][0], y + c_sr_off[w][1], z + c_sr_off[w][2]) < s.iso) ci |= 1 << w;
  return ci;
}
__device__ __forceinline__ bool sr_edge_cross(int ci, int w) {
  return ((ci >> c_sr_edge[w][0]) ^ (ci >> c_sr_edge[w][1])) & 1;
}

__global__ void k_sr_dc_flag(SrDev s, int64_t cells) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells; c += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(c % s.g.nx), y = (int)((c / s.g.nx) % s.g.ny), z = (int)(c / ((int64_t)s.g.nx * s.g.ny));
    uint32_t f = 0u;
    if (s.active[s.g.bidx(x, y, z)]) {
      const int ci = sr_cube_mask(s, x, y, z);
      f = (ci != 0 && ci != 255) ? 1u : 0u;
    }
    s.vflag[c] = f;
  }
}

// calc_vertex_normal (srtool.py:1306-1321), normalised
__device__ void sr_vertex_normal(const SrDev& s, int x, int y, int z, double n[3]) {
  const float* f = s.field;
  n[0] = (x == 0) ? -(double)sr_get(s, f, x + 1, y, z) : (double)sr_get(s, f, x - 1, y, z) - sr_get(s, f, x + 1, y, z);
  n[1] = (y == 0) ? -(double)sr_get(s, f, x, y + 1, z) : (double)sr_get(s, f, x, y - 1, z) - sr_get(s, f, x, y + 1, z);
  n[2] = (z == 0) ? -(double)sr_get(s, f, x, y, z + 1) : (double)sr_get(s, f, x, y, z - 1) - sr_get(s, f, x, y, z + 1);
  const double l = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  if (l != 0.0) { n[0] /= l; n[1] /= l; n[2] /= l; }
}
// process_normal_at (srtool.py:1335-1349)
__device__ void sr_normal_at(const SrDev& s, const double p[3], double n[3]) {
  int x0, y0, z0;
  s.g.voxel_of((float)p[0], (float)p[1], (float)p[2], x0, y0, z0);
  const double xd = (p[0] - (x0 * s.g.dvs + s.g.dox)) / s.g.dvs, yd = (p[1] - (y0 * s.g.dvs + s.g.doy)) / s.g.dvs,
               zd = (p[2] - (z0 * s.g.dvs + s.g.doz)) / s.g.dvs;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int e = 0; e < 2; ++e) {
        double c[3];
        sr_vertex_normal(s, x0 + a, y0 + b, z0 + e, c);
        const double wgt = (a ? xd : 1 - xd) * (b ? yd : 1 - yd) * (e ? zd : 1 - zd);
        acc[0] += wgt * c[0]; acc[1] += wgt * c[1]; acc[2] += wgt * c[2];
      }
  const double l = sqrt(acc[0] * acc[0] + acc[1] * acc[1] + acc[2] * acc[2]);
  if (l != 0.0) { n[0] = acc[0] / l; n[1] = acc[1] / l; n[2] = acc[2] / l; }
  else n[0] = n[1] = n[2] = 0.0;
}

// The crossing cubes in vertex-id order, so that the QEF kernel runs on dense work.
__global__ void k_sr_dc_list(SrDev s, int64_t cells) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells; c += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t id = s.vflag[c];
    if (s.vflag[c + 1] != id && (int64_t)id < s.max_v) s.cube_of[id] = (uint32_t)c;
  }
}

// One point per crossing cube: the mass point of the edge crossings plus the clamped
// QEF solution, kept only if it stays in its cube (srtool.py:1536-1596)
__global__ void k_sr_dc_point(SrDev s, int64_t cells) {
  const int64_t nv = min((int64_t)s.vflag[cells], (int64_t)s.max_v);
  for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < nv; id += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = s.cube_of[id];
    const int x = (int)(c % s.g.nx), y = (int)((c / s.g.nx) % s.g.ny), z = (int)(c / ((int64_t)s.g.nx * s.g.ny));
    const int ci = sr_cube_mask(s, x, y, z);
    double P[12][3];
    int cnt = 0;
    double mean[3] = {0.0, 0.0, 0.0};
    for (int w = 0; w < 12; ++w) {
      if (!sr_edge_cross(ci, w)) continue;
      const int a = c_sr_edge[w][0], b = c_sr_edge[w][1];
      const int ax = x + c_sr_off[a][0], ay = y + c_sr_off[a][1], az = z + c_sr_off[a][2];
      const int bx = x + c_sr_off[b][0], by = y + c_sr_off[b][1], bz = z + c_sr_off[b][2];
      const double v1 = sr_get(s, s.field, ax, ay, az), v2 = sr_get(s, s.field, bx, by, bz);
      const double delta = v2 - v1;
      const double t = fabs(delta) < 1e-5 ? 0.5 : ((double)s.iso - v1) / delta;  // vertex_interpolate
      const double p1[3] = {ax * s.g.dvs + s.g.dox, ay * s.g.dvs + s.g.doy, az * s.g.dvs + s.g.doz};
      const double p2[3] = {bx * s.g.dvs + s.g.dox, by * s.g.dvs + s.g.doy, bz * s.g.dvs + s.g.doz};
      for (int k = 0; k < 3; ++k) { P[cnt][k] = p1[k] + t * (p2[k] - p1[k]); mean[k] += P[cnt][k]; }
      ++cnt;
    }
    for (int k = 0; k < 3; ++k) mean[k] /= cnt;
    double NtN[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Ntb[3] = {0, 0, 0};
    for (int r = 0; r < cnt; ++r) {
      double n[3];
      sr_normal_at(s, P[r], n);
      const double bb = n[0] * (P[r][0] - mean[0]) + n[1] * (P[r][1] - mean[1]) + n[2] * (P[r][2] - mean[2]);
      for (int i = 0; i < 3; ++i) {
        Ntb[i] += n[i] * bb;
        for (int j = 0; j < 3; ++j) NtN[i][j] += n[i] * n[j];
      }
    }
    double lam[3], V[3][3], res[3] = {0.0, 0.0, 0.0};
    sr_sym_eig(NtN, lam, V);
    for (int i = 0; i < 3; ++i) {
      const double sv = sqrt(fmax(lam[i], 0.0));
      if (!(sv > 0.0)) continue;
      const double f = (V[0][i] * Ntb[0] + V[1][i] * Ntb[1] + V[2][i] * Ntb[2]) / (sv * fmax(sv, 0.1));
      for (int k = 0; k < 3; ++k) res[k] += f * V[k][i];
    }
    int qx, qy, qz;
    s.g.voxel_of((float)(res[0] + mean[0]), (float)(res[1] + mean[1]), (float)(res[2] + mean[2]), qx, qy, qz);
    const bool keep = qx == x && qy == y && qz == z;
    for (int k = 0; k < 3; ++k) s.vert[3 * id + k] = (float)(keep ? res[k] + mean[k] : mean[k]);
  }
}

// get_edge_adjacent_cubes (srtool.py:1612-1705) for edges 2 (x), 3 (y), 11 (z) of corner 3
__device__ __forceinline__ void sr_edge_cubes(int w, int d[4][3]) {
  const int t2[4][3] = {{0, 0, 0}, {0, 0, -1}, {0, -1, -1}, {0, -1, 0}};
  const int t3[4][3] = {{0, 0, 0}, {0, 0, -1}, {-1, 0, -1}, {-1, 0, 0}};
  const int t11[4][3] = {{0, 0, 0}, {0, -1, 0}, {-1, -1, 0}, {-1, 0, 0}};
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) d[i][k] = w == 2 ? t2[i][k] : w == 3 ? t3[i][k] : t11[i][k];
}
// the vertex id of cube (x, y, z), or -1
__device__ __forceinline__ int64_t sr_vid(const SrDev& s, int x, int y, int z) {
  if (!s.g.in(x, y, z)) return -1;
  const int64_t c = s.g.idx(x, y, z);
  return s.vflag[c + 1] != s.vflag[c] ? (int64_t)s.vflag[c] : -1;
}

// pass 0 counts the indices each cube emits, pass 1 writes them at the scanned offsets
__global__ void k_sr_tris(SrDev s, int64_t cells, int pass) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells; c += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(c % s.g.nx), y = (int)((c / s.g.nx) % s.g.ny), z = (int)(c / ((int64_t)s.g.nx * s.g.ny));
    uint32_t cnt = 0;
    if (s.vflag[c + 1] != s.vflag[c]) {
      const int ci = sr_cube_mask(s, x, y, z);
      int64_t o = pass ? (int64_t)s.tcount[c] : 0;
      for (int k = 0; k < 3; ++k) {
        const int w = k == 0 ? 2 : k == 1 ? 3 : 11;
        if (!sr_edge_cross(ci, w)) continue;
        int d[4][3];
        sr_edge_cubes(w, d);
        int64_t id[4];
        bool ok = true;
        for (int q = 0; q < 4; ++q) {
          id[q] = sr_vid(s, x + d[q][0], y + d[q][1], z + d[q][2]);
          ok = ok && id[q] >= 0;
        }
        if (!ok) continue;
        cnt += 6;
        if (pass) {
          if (o + 6 > s.max_i) { sr_fail(s, NN_ERR_CAPACITY); continue; }
          const bool cond0 = (ci >> c_sr_edge[w][0]) & 1;
          const bool flip = cond0 != (w == 11);
          const int64_t t[6] = {id[2], id[1], id[0], id[3], id[2], id[0]};
          const int64_t tf[6] = {id[0], id[1], id[2], id[0], id[2], id[3]};
          for (int q = 0; q < 6; ++q) s.tri[o + q] = (int32_t)(flip ? tf[q] : t[q]);
          o += 6;
        }
      }
    }
    if (!pass) s.tcount[c] = cnt;
  }
}

// ---- 6b. marching cubes (marching_cube_impl, srtool.py:1765-1800) ----------------------
// The reference's 256-case triangle table is not reproduced. This build's table is
// computed at compile time from the corner states of each case ("in": value <
// isolevel): faces list their corners counter-clockwise seen from outside; on a face,
// every run of in-corners gets one segment from the edge where the walk leaves the run
// to the edge where it entered it (in-corners stay separate on ambiguous faces, which
// depends on the face alone, so neighbouring cubes agree and the surface is closed);
// the segments chain into loops over the crossing edges; loops are taken in order of
// their smallest edge id, start there, and are fanned as (l0, l[k+1], l[k]).
#define SR_MC_MAXT 5
struct SrMcTable {
  uint16_t edges[256];               // crossing edges of each case
  uint8_t ntri[256];
  int8_t tri[256][SR_MC_MAXT][3];    // edge ids
  bool overflow;                     // a case needs more than SR_MC_MAXT triangles
};

constexpr int sr_mc_edge_of(const int8_t (&e)[12][2], int c0, int c1) {
  for (int w = 0; w < 12; ++w)
    if ((e[w][0] == c0 && e[w][1] == c1) || (e[w][0] == c1 && e[w][1] == c0)) return w;
  return -1;
}

constexpr SrMcTable sr_make_mc_table() {
  // the same corner offsets and edges as c_sr_off and c_sr_edge (srtool.py:775-783, 931-942)
  const int8_t off[8][3] = {{0, 1, 0}, {1, 1, 0}, {1, 0, 0}, {0, 0, 0}, {0, 1, 1}, {1, 1, 1}, {1, 0, 1}, {0, 0, 1}};
  const int8_t edge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  SrMcTable t{};
  for (int ci = 0; ci < 256; ++ci) {
    int next[12] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
    for (int a = 0; a < 3; ++a)
      for (int side = 0; side < 2; ++side) {
        const int u = (a + 1) % 3, v = (a + 2) % 3;
        int uv[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};  // counter-clockwise around +e_a
        if (side == 0) { uv[1][0] = 0; uv[1][1] = 1; uv[3][0] = 1; uv[3][1] = 0; }
        int q[4] = {0, 0, 0, 0};
        for (int k = 0; k < 4; ++k)
          for (int c = 0; c < 8; ++c)
            if (off[c][a] == side && off[c][u] == uv[k][0] && off[c][v] == uv[k][1]) q[k] = c;
        bool in[4] = {false, false, false, false};
        for (int k = 0; k < 4; ++k) in[k] = (ci >> q[k]) & 1;
        for (int k = 0; k < 4; ++k) {
          if (!in[k] || in[(k + 1) % 4]) continue;  // the walk leaves a run of in-corners at q[k]
          int j = k;
          while (in[(j + 3) % 4]) j = (j + 3) % 4;  // the run starts at q[j]
          next[sr_mc_edge_of(edge, q[k], q[(k + 1) % 4])] = sr_mc_edge_of(edge, q[(j + 3) % 4], q[j]);
        }
      }
    bool seen[12] = {false, false, false, false, false, false, false, false, false, false, false, false};
    int nt = 0;
    for (int e = 0; e < 12; ++e) {
      if (next[e] < 0) continue;
      t.edges[ci] = (uint16_t)(t.edges[ci] | (1u << e));
      if (seen[e]) continue;
      int loop[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
      int m = 0;
      for (int f = e; !seen[f]; f = next[f]) {
        seen[f] = true;
        loop[m++] = f;
      }
      for (int k = 1; k + 1 < m; ++k) {
        if (nt == SR_MC_MAXT) { t.overflow = true; break; }
        t.tri[ci][nt][0] = (int8_t)loop[0];
        t.tri[ci][nt][1] = (int8_t)loop[k + 1];
        t.tri[ci][nt][2] = (int8_t)loop[k];
        ++nt;
      }
    }
    t.ntri[ci] = (uint8_t)nt;
  }
  return t;
}
static_assert(!sr_make_mc_table().overflow, "a marching-cubes case needs more than SR_MC_MAXT triangles");
__constant__ SrMcTable c_sr_mc = sr_make_mc_table();

// pass 0: vertices (crossing edges) and indices per cube into vflag / tcount;
// pass 1: both written at the scanned offsets, in edge order within a cube
__global__ void k_sr_mc(SrDev s, int64_t cells, int pass) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells; c += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(c % s.g.nx), y = (int)((c / s.g.nx) % s.g.ny), z = (int)(c / ((int64_t)s.g.nx * s.g.ny));
    if (pass == 1 && s.vflag[c + 1] == s.vflag[c]) continue;
    // a cube with a crossing has a nonzero corner, which lies in an active block: the
    // reference's visit of the cubes around the active vertices reaches every such cube
    const int ci = sr_cube_mask(s, x, y, z);
    const uint32_t em = c_sr_mc.edges[ci];
    if (pass == 0) {
      s.vflag[c] = __popc(em);
      s.tcount[c] = 3u * c_sr_mc.ntri[ci];
      continue;
    }
    const int64_t vb = s.vflag[c], tb = s.tcount[c];
    const int nt = c_sr_mc.ntri[ci];
    if (vb + __popc(em) > s.max_v || tb + 3 * nt > s.max_i) { sr_fail(s, NN_ERR_CAPACITY); continue; }
    for (int w = 0; w < 12; ++w) {
      if (!((em >> w) & 1u)) continue;
      const int a = c_sr_edge[w][0], b = c_sr_edge[w][1];
      const int ax = x + c_sr_off[a][0], ay = y + c_sr_off[a][1], az = z + c_sr_off[a][2];
      const int bx = x + c_sr_off[b][0], by = y + c_sr_off[b][1], bz = z + c_sr_off[b][2];
      const double v1 = sr_get(s, s.field, ax, ay, az), v2 = sr_get(s, s.field, bx, by, bz);
      const double delta = v2 - v1;
      const double t = fabs(delta) < 1e-5 ? 0.5 : ((double)s.iso - v1) / delta;  // vertex_interpolate
      const double p1[3] = {ax * s.g.dvs + s.g.dox, ay * s.g.dvs + s.g.doy, az * s.g.dvs + s.g.doz};
      const double p2[3] = {bx * s.g.dvs + s.g.dox, by * s.g.dvs + s.g.doy, bz * s.g.dvs + s.g.doz};
      const int64_t v = vb + __popc(em & ((1u << w) - 1u));
      for (int k = 0; k < 3; ++k) s.vert[3 * v + k] = (float)(p1[k] + t * (p2[k] - p1[k]));
    }
    for (int q = 0; q < nt; ++q)
      for (int k = 0; k < 3; ++k) {
        const int w = c_sr_mc.tri[ci][q][k];
        s.tri[tb + 3 * q + k] = (int32_t)(vb + __popc(em & ((1u << w) - 1u)));
      }
  }
}

// ---- 7. vertex normals (process_normal) ----------------------------------------------
__global__ void k_sr_normals(SrDev s, int nv) {
  GRID_STRIDE(i, min(nv, s.max_v)) {
    const double p[3] = {s.vert[3 * i], s.vert[3 * i + 1], s.vert[3 * i + 2]};
    double n[3];
    sr_normal_at(s, p, n);
    s.nrm[3 * i] = (float)n[0]; s.nrm[3 * i + 1] = (float)n[1]; s.nrm[3 * i + 2] = (float)n[2];
  }
}

// ---- host side: context and C ABI -------------------------------------------------------
struct nn_sr_ctx {
  int dev_id = 0;
  int sms = 148;
  int32_t max_particles = 0, max_v = 0, max_i = 0;
  int64_t max_cells = 0, blocks = 0;
  int32_t* d_n = nullptr;  // scan sizes ([2] = last index of the current scan)
  int32_t* status = nullptr;
  uint32_t *vcount = nullptr, *vkey = nullptr, *vrank = nullptr, *vflag = nullptr, *tcount = nullptr,
           *tile_sums = nullptr, *cube_of = nullptr;
  int32_t *vsrc = nullptr, *tri = nullptr;
  float4* spos = nullptr;
  unsigned long long* vfix = nullptr;  // [3][cells], with NN_SR_VELOCITY only
  float* mvel = nullptr;
  unsigned long long* fix = nullptr;
  float *splat = nullptr, *fa = nullptr, *fb = nullptr, *G = nullptr, *xbar = nullptr, *vert = nullptr, *nrm = nullptr;
  uint8_t* active = nullptr;
  double* stats = nullptr;
  // last call
  SrDev last{};
  int64_t cells = 0;
  int32_t nv = 0, ni = 0, n = 0;
  double sd = 0.0;
  bool have = false;
  std::string err;
};

static int sr_fail_host(nn_sr_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}
#define SRCK(call)                                                                                         \
  do {                                                                                                     \
    cudaError_t _e = (call);                                                                               \
    if (_e != cudaSuccess) return sr_fail_host(c, NN_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e));   \
  } while (0)

static void sr_free(nn_sr_ctx* c) {
  void* bufs[] = {c->d_n, c->status, c->vcount, c->vkey, c->vrank, c->vflag, c->tcount, c->tile_sums, c->vsrc,
                  c->tri, c->fix, c->splat, c->fa, c->fb, c->G, c->xbar, c->vert, c->nrm, c->active, c->stats,
                  c->cube_of, c->spos, c->vfix, c->mvel};
  for (void* b : bufs) cudaFree(b);
}

// An exclusive scan of a[0 .. len) in place with the neighbour search's scan kernels.
static int sr_scan(nn_sr_ctx* c, uint32_t* a, int64_t len, cudaStream_t st) {
  Dev d{};
  d.d_n = c->d_n;
  d.cell_count = a;
  d.tile_sums = c->tile_sums;
  const int32_t hn[3] = {0, 0, (int32_t)(len - 1)};
  SRCK(cudaMemcpyAsync(c->d_n, hn, sizeof(hn), cudaMemcpyHostToDevice, st));
  const int tiles = (int)((len + SCAN_TILE - 1) / SCAN_TILE);
  k_scan_tiles<<<std::max(1, std::min(tiles, c->sms * 2)), SCAN_THREADS, 0, st>>>(d);
  k_scan_apply<<<std::max(1, std::min(tiles, c->sms * 2)), SCAN_THREADS, 0, st>>>(d);
  SRCK(cudaGetLastError());
  return NN_OK;
}

extern "C" {

int nn_sr_create(int32_t max_particles, int64_t max_cells, int32_t max_vertices, int32_t max_indices,
                 int32_t options, nn_sr_ctx** out) {
  if (!out) return NN_ERR_INVALID_ARG;
  *out = nullptr;
  if (max_particles <= 0 || max_cells <= 0 || max_cells >= (int64_t)INT32_MAX - SCAN_TILE || max_vertices <= 0 ||
      max_indices <= 0 || (options & ~NN_SR_VELOCITY))
    return NN_ERR_INVALID_ARG;
  nn_sr_ctx* c = new nn_sr_ctx();
  cudaGetDevice(&c->dev_id);
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->dev_id);
  c->max_particles = max_particles;
  c->max_cells = max_cells;
  c->max_v = max_vertices;
  c->max_i = max_indices;
  const size_t N = (size_t)max_particles, CL = (size_t)max_cells + 1;
  const size_t blocks = (size_t)max_cells / 512 + 4096;  // block flags: checked against each grid's shape
  const size_t tiles = CL / SCAN_TILE + 2;
  cudaError_t e = cudaSuccess;
  auto al = [&](auto** p, size_t cnt) {
    if (e == cudaSuccess) e = cudaMalloc((void**)p, cnt * sizeof(**p));
  };
  al(&c->d_n, 4); al(&c->status, 1); al(&c->stats, 4);
  al(&c->vcount, CL); al(&c->vflag, CL); al(&c->tcount, CL); al(&c->tile_sums, tiles);
  al(&c->vkey, N); al(&c->vrank, N); al(&c->vsrc, N); al(&c->spos, N); al(&c->G, 9 * N); al(&c->xbar, 3 * N);
  al(&c->fix, CL); al(&c->splat, CL); al(&c->fa, CL); al(&c->fb, CL); al(&c->active, blocks);
  al(&c->vert, 3 * (size_t)max_vertices); al(&c->nrm, 3 * (size_t)max_vertices); al(&c->tri, (size_t)max_indices);
  al(&c->cube_of, (size_t)max_vertices); al(&c->mvel, 3 * (size_t)max_vertices);
  if (options & NN_SR_VELOCITY) al(&c->vfix, 3 * CL);
  if (e != cudaSuccess) {
    sr_free(c);
    delete c;
    return NN_ERR_OOM;
  }
  c->blocks = (int64_t)blocks;
  *out = c;
  return NN_OK;
}

int nn_sr_destroy(nn_sr_ctx* c) {
  if (!c) return NN_ERR_INVALID_ARG;
  sr_free(c);
  delete c;
  return NN_OK;
}

const char* nn_sr_last_error(const nn_sr_ctx* c) { return c ? c->err.c_str() : "null context"; }

// The shared pipeline of SRTool.dual_contouring (srtool.py:1264-1304): binning, splats,
// smoothing, then dual contouring or marching cubes, normals and velocities.
static int sr_run(nn_sr_ctx* c, const nn_sr_params* p, const float* pos, const float* vel, int32_t n, void* stream,
                  bool marching_cubes) {
  if (!c) return NN_ERR_INVALID_ARG;
  const char* fn = marching_cubes ? "nn_sr_marching_cubes" : "nn_sr_dual_contouring";
  c->have = false;
  if (!p || p->size != (int32_t)sizeof(nn_sr_params) || (!pos && n > 0) || n < 0)
    return sr_fail_host(c, NN_ERR_INVALID_ARG, "%s: invalid argument", fn);
  if (n > c->max_particles)
    return sr_fail_host(c, NN_ERR_CAPACITY, "%d particles exceed the context's %d", n, c->max_particles);
  if (vel && !c->vfix)
    return sr_fail_host(c, NN_ERR_STATE, "velocities given to a context created without NN_SR_VELOCITY");
  if (!(p->voxel_size > 0) || !(p->smooth_radius > 0) || !(p->particle_radius > 0) || p->dims[0] <= 0 ||
      p->dims[1] <= 0 || p->dims[2] <= 0 || p->smooth_iterations < 0 || p->smooth_cells < 0)
    return sr_fail_host(c, NN_ERR_INVALID_ARG, "%s: bad parameters", fn);
  const int64_t cells = (int64_t)p->dims[0] * p->dims[1] * p->dims[2];
  const int bx = (p->dims[0] + NN_SR_BLOCK - 1) / NN_SR_BLOCK, by = (p->dims[1] + NN_SR_BLOCK - 1) / NN_SR_BLOCK,
            bz = (p->dims[2] + NN_SR_BLOCK - 1) / NN_SR_BLOCK;
  const int64_t blocks = (int64_t)bx * by * bz;
  if (cells > c->max_cells || blocks > c->blocks)
    return sr_fail_host(c, NN_ERR_CAPACITY, "grid of %lld vertices exceeds the context's %lld", (long long)cells,
                        (long long)c->max_cells);
  cudaStream_t st = (cudaStream_t)stream;
  SrDev s{};
  s.g.nx = p->dims[0]; s.g.ny = p->dims[1]; s.g.nz = p->dims[2];
  s.g.bx = bx; s.g.by = by; s.g.bz = bz;
  s.g.ox = (float)p->origin[0]; s.g.oy = (float)p->origin[1]; s.g.oz = (float)p->origin[2];
  s.g.vs = (float)p->voxel_size;
  s.g.dox = s.g.ox; s.g.doy = s.g.oy; s.g.doz = s.g.oz; s.g.dvs = s.g.vs;
  s.n = n; s.pos = pos; s.status = c->status;
  s.vcount = c->vcount; s.vkey = c->vkey; s.vrank = c->vrank; s.vsrc = c->vsrc; s.spos = c->spos;
  s.fix = c->fix; s.splat = c->splat; s.field = c->fa; s.tmp = c->fb; s.active = c->active;
  s.G = c->G; s.xbar = c->xbar; s.stats = c->stats; s.vflag = c->vflag; s.tcount = c->tcount;
  s.vert = c->vert; s.tri = c->tri; s.nrm = c->nrm; s.max_v = c->max_v; s.max_i = c->max_i;
  s.cube_of = c->cube_of;
  s.vel = vel; s.vfix = c->vfix; s.mvel = c->mvel;
  s.iso = (float)p->isolevel;
  s.sr = (float)p->smooth_radius;
  const double r = p->particle_radius;
  s.volume = (float)(r * r * r * SR_PI * 4.0 / 3.0);  // srtool.py:920
  s.acoeff = (float)(315.0 / (64.0 * SR_PI));        // srtool.py:921
  s.range = (int)std::ceil(4.0 * (double)s.sr / (double)s.g.vs) + 1;  // srtool.py:1137
  s.off = s.range / 2;
  s.smooth_cells = p->smooth_cells;
  {  // the pre-pass's in-range test rn(sqrt(r2)) < 2 r_s  <=>  r2 < rr_thr
    const float rr = 2.f * s.sr;
    float t = rr * rr;
    while (std::sqrt(t) >= rr) t = std::nextafter(t, 0.f);
    while (std::sqrt(t) < rr) t = std::nextafter(t, INFINITY);
    s.rr_thr = t;
  }
  {  // exact branch tests without the square root: rn(sqrt(t)) <= 1 (0.5)  <=>  t <= q1_thr (q05_thr)
    float t = 1.f;
    while (std::sqrt(std::nextafter(t, INFINITY)) <= 1.f) t = std::nextafter(t, INFINITY);
    while (std::sqrt(t) > 1.f) t = std::nextafter(t, 0.f);
    s.q1_thr = t;
    t = 0.25f;
    while (std::sqrt(std::nextafter(t, INFINITY)) <= 0.5f) t = std::nextafter(t, INFINITY);
    while (std::sqrt(t) > 0.5f) t = std::nextafter(t, 0.f);
    s.q05_thr = t;
  }
  s.record_normals = p->record_normals;
  const int B = 256;
  const int grid_n = std::max(1, std::min((n + B - 1) / B, c->sms * 8));
  const int grid_c = (int)std::max<int64_t>(1, std::min<int64_t>((cells + B - 1) / B, (int64_t)c->sms * 16));
  SRCK(cudaMemsetAsync(c->status, 0, sizeof(int32_t), st));
  SRCK(cudaMemsetAsync(c->stats, 0, 4 * sizeof(double), st));
  SRCK(cudaMemsetAsync(c->vcount, 0, (cells + 1) * sizeof(uint32_t), st));
  SRCK(cudaMemsetAsync(c->fix, 0, cells * sizeof(unsigned long long), st));
  if (vel) SRCK(cudaMemsetAsync(c->vfix, 0, 3 * cells * sizeof(unsigned long long), st));
  SRCK(cudaMemsetAsync(c->active, 0, blocks, st));
  SRCK(cudaMemsetAsync(c->G, 0, 9 * (size_t)std::max(n, 1) * sizeof(float), st));
  SRCK(cudaMemsetAsync(c->xbar, 0, 3 * (size_t)std::max(n, 1) * sizeof(float), st));
  if (n > 0) {
    // 1. binning
    k_sr_keys<<<grid_n, B, 0, st>>>(s);
    RC(sr_scan(c, c->vcount, cells + 1, st));
    k_sr_scatter<<<grid_n, B, 0, st>>>(s);
    k_sr_voxel_sort<<<grid_c, B, 0, st>>>(s, cells);
    k_sr_sorted_pos<<<grid_n, B, 0, st>>>(s, cells);
    // 2. isotropic splat
    k_sr_iso<<<grid_n, B, 0, st>>>(s);
    if (p->use_smooth_field) {
      // 3-4. anisotropic kernels and splat (one warp per particle each)
      const int grid_w = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)n * 32 + B - 1) / B, c->sms * 16));
      k_sr_aniso_pre<<<grid_w, B, 0, st>>>(s);
      k_sr_aniso_splat<<<grid_w, B, 0, st>>>(s);
      if (vel) k_sr_vel_splat<<<grid_w, B, 0, st>>>(s);
    }
  }
  k_sr_fix_to_field<<<grid_c, B, 0, st>>>(s, cells);
  // 5. smoothing
  for (int it = 0; it < p->smooth_iterations; ++it) {
    SRCK(cudaMemsetAsync(c->stats, 0, 4 * sizeof(double), st));
    k_sr_stats<<<grid_c, B, 0, st>>>(s, cells, 0);
    k_sr_stats<<<grid_c, B, 0, st>>>(s, cells, 1);
    k_sr_sd<<<1, 32, 0, st>>>(s);
    k_sr_smooth<<<grid_c, B, 0, st>>>(s, cells);
    std::swap(s.field, s.tmp);
  }
  SRCK(cudaMemsetAsync(c->vflag, 0, (cells + 1) * sizeof(uint32_t), st));
  SRCK(cudaMemsetAsync(c->tcount, 0, (cells + 1) * sizeof(uint32_t), st));
  if (marching_cubes) {
    // 6b. marching cubes: count, scan, write
    k_sr_mc<<<grid_c, B, 0, st>>>(s, cells, 0);
    RC(sr_scan(c, c->vflag, cells + 1, st));
    RC(sr_scan(c, c->tcount, cells + 1, st));
    k_sr_mc<<<grid_c, B, 0, st>>>(s, cells, 1);
  } else {
    // 6. dual contouring
    k_sr_dc_flag<<<grid_c, B, 0, st>>>(s, cells);
    RC(sr_scan(c, c->vflag, cells + 1, st));
    k_sr_dc_list<<<grid_c, B, 0, st>>>(s, cells);
    k_sr_dc_point<<<c->sms * 4, 128, 0, st>>>(s, cells);
    k_sr_tris<<<grid_c, B, 0, st>>>(s, cells, 0);
    RC(sr_scan(c, c->tcount, cells + 1, st));
    k_sr_tris<<<grid_c, B, 0, st>>>(s, cells, 1);
  }
  SRCK(cudaGetLastError());
  uint32_t counts[2];
  int32_t status = 0;
  double sd = 0.0;
  SRCK(cudaMemcpyAsync(&counts[0], c->vflag + cells, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  SRCK(cudaMemcpyAsync(&counts[1], c->tcount + cells, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  SRCK(cudaMemcpyAsync(&status, c->status, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SRCK(cudaMemcpyAsync(&sd, c->stats + 3, sizeof(double), cudaMemcpyDeviceToHost, st));
  SRCK(cudaStreamSynchronize(st));
  c->nv = (int32_t)counts[0];
  c->ni = (int32_t)counts[1];
  c->sd = sd;
  if (status == 0 && (c->nv > c->max_v || c->ni > c->max_i)) status = NN_ERR_CAPACITY;
  if (status != 0) {
    if (status == NN_ERR_INVALID_ARG) return sr_fail_host(c, status, "a particle lies outside the grid");
    if (status == NN_ERR_NAN) return sr_fail_host(c, status, "non-finite splat contribution");
    return sr_fail_host(c, status, "grid, voxel list or mesh capacity exceeded (%d vertices, %d indices)", c->nv,
                        c->ni);
  }
  if (p->record_normals && c->nv > 0) {
    k_sr_normals<<<std::max(1, std::min((c->nv + B - 1) / B, c->sms * 8)), B, 0, st>>>(s, c->nv);
    SRCK(cudaGetLastError());
  }
  if (vel && c->nv > 0) {  // process_velocity (srtool.py:1298-1300); a zero field without the smooth splat
    k_sr_mesh_velocity<<<std::max(1, std::min((c->nv + B - 1) / B, c->sms * 8)), B, 0, st>>>(s, c->nv);
    SRCK(cudaGetLastError());
  }
  c->last = s;
  c->cells = cells;
  c->n = n;
  c->have = true;
  return NN_OK;
}

int nn_sr_dual_contouring(nn_sr_ctx* c, const nn_sr_params* p, const float* pos, const float* vel, int32_t n,
                          void* stream) {
  return sr_run(c, p, pos, vel, n, stream, false);
}

int nn_sr_marching_cubes(nn_sr_ctx* c, const nn_sr_params* p, const float* pos, const float* vel, int32_t n,
                         void* stream) {
  return sr_run(c, p, pos, vel, n, stream, true);
}

int nn_sr_get_mesh(nn_sr_ctx* c, int32_t* num_vertices, int32_t* num_indices, float* vertices, int32_t* indices,
                   float* normals, float* velocities, void* stream) {
  if (!c) return NN_ERR_INVALID_ARG;
  if (!c->have) return sr_fail_host(c, NN_ERR_STATE, "no mesh: run nn_sr_dual_contouring or nn_sr_marching_cubes first");
  cudaStream_t st = (cudaStream_t)stream;
  if (num_vertices) *num_vertices = c->nv;
  if (num_indices) *num_indices = c->ni;
  if (vertices && c->nv)
    SRCK(cudaMemcpyAsync(vertices, c->vert, 3 * (size_t)c->nv * sizeof(float), cudaMemcpyDeviceToDevice, st));
  if (indices && c->ni)
    SRCK(cudaMemcpyAsync(indices, c->tri, (size_t)c->ni * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
  if (normals && c->nv) {
    if (!c->last.record_normals) return sr_fail_host(c, NN_ERR_STATE, "normals were not recorded");
    SRCK(cudaMemcpyAsync(normals, c->nrm, 3 * (size_t)c->nv * sizeof(float), cudaMemcpyDeviceToDevice, st));
  }
  if (velocities && c->nv) {
    if (!c->last.vel) return sr_fail_host(c, NN_ERR_STATE, "velocities were not recorded");
    SRCK(cudaMemcpyAsync(velocities, c->mvel, 3 * (size_t)c->nv * sizeof(float), cudaMemcpyDeviceToDevice, st));
  }
  return NN_OK;
}

int nn_sr_get_stage(nn_sr_ctx* c, int32_t stage, float* field, uint8_t* active_blocks, float* G, float* xbar,
                    double* sd, void* stream) {
  if (!c) return NN_ERR_INVALID_ARG;
  if (!c->have) return sr_fail_host(c, NN_ERR_STATE, "no result: run nn_sr_dual_contouring first");
  if (stage != 0 && stage != 1) return sr_fail_host(c, NN_ERR_INVALID_ARG, "stage must be 0 or 1");
  cudaStream_t st = (cudaStream_t)stream;
  const SrDev& s = c->last;
  const int64_t blocks = (int64_t)s.g.bx * s.g.by * s.g.bz;
  if (field)
    SRCK(cudaMemcpyAsync(field, stage == 0 ? c->splat : s.field, c->cells * sizeof(float), cudaMemcpyDeviceToDevice, st));
  if (active_blocks) SRCK(cudaMemcpyAsync(active_blocks, c->active, blocks, cudaMemcpyDeviceToDevice, st));
  if (G && c->n) SRCK(cudaMemcpyAsync(G, c->G, 9 * (size_t)c->n * sizeof(float), cudaMemcpyDeviceToDevice, st));
  if (xbar && c->n)
    SRCK(cudaMemcpyAsync(xbar, c->xbar, 3 * (size_t)c->n * sizeof(float), cudaMemcpyDeviceToDevice, st));
  if (sd) *sd = c->sd;
  return NN_OK;
}

}  // extern "C"
