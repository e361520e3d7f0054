// surf_oracle.cpp — CPU restatement of the reference's particle surface reconstruction
// (SPH/surf_recon/srtool.py, SRTool.dual_contouring, srtool.py:1264-1304).
//
// TEST INFRASTRUCTURE: only tests/ and bench.py's CPU-baseline leg load this library,
// as the checker or the CPU baseline. Nothing in the product links or calls it.
//
// Sums are accumulated in double, in particle-id order (the reference accumulates in
// f32 with atomics, in no fixed order). Pinned against the reference's own SRTool
// stages, run in plain Python through a Taichi stand-in on a 154-particle ball
// (tests/golden/make_reference_surface.py, tests/golden/ref_surface.npz): G and x_bar
// within 1e-6 of scale, the same active blocks, the splat field within 3e-4 (the
// reference's f32 sums; 3.2e-5 against the same run in f64), sd within 1e-4 and the
// smoothed field within 2e-4 (tests/test_reference_pin.py). The contouring is pinned
// by closed-mesh properties only: the reference's QEF indexes past its 4x4 matrix for
// cubes with more than four crossing edges, which plain Python cannot execute.
//
// Follows, step by step:
//   update_particles      srtool.py:1192-1195, _SRVoxel.add_particle 819-823
//   generate_fluid_field  srtool.py:1238-1251 (poly6 1212-1227)
//   pre_process_data      srtool.py:1006-1095 (isoweight 993-999)
//   generate_smooth_fluid_field_impl 1135-1157 (cubic_spline_kernel 1114-1124)
//   smooth_sdf            srtool.py:1425-1484, density_field_stats 1436-1456
//   dual_contouring_impl  srtool.py:1531-1596 (vertex_interpolate 1253-1262,
//                         process_normal_at 1335-1349, calc_vertex_normal 1306-1321)
//   dual_contouring_polygen 1707-1763 (get_edge_adjacent_cubes 1612-1705)
//   process_normal        srtool.py:1383-1410
//   generate_smooth_fluid_field_with_velocity_impl (velocity part) 1159-1190,
//   process_velocity      srtool.py:1351-1381
//
// Taichi's sparse fields are emulated with one "active" flag per 32^3 block of
// vertices (the reference's leaf blocks are dense 32^3 under pointer levels): a
// write, `+= 0` included, activates the block; struct-for loops visit every vertex
// of the active blocks; reads elsewhere give 0.
//
// Restatement choices where the reference's own behaviour is undefined or
// nondeterministic:
//   - the QEF (srtool.py:1549-1581) writes one row per crossing edge into a 4x4
//     matrix, so cubes with more than 4 crossing edges index past it. Here every
//     crossing edge is a row. The least-squares solution comes from the normal
//     equations: eigen-decomposition N^T N = V diag(s^2) V^T, x = sum_i v_i
//     (v_i . N^T b) / (s_i * max(s_i, 0.1)). This keeps the reference's clamp of the
//     singular values at 0.1 (solve_qef 70-81); a zero singular value adds nothing.
//   - vertices and triangles are numbered in cube order (linear index of the cube;
//     edges 2, 3, 11 within a cube), not in atomic-counter order.
//   - every DC point is written to the vertex array (the reference writes only the
//     points a triangle uses and leaves stale data in the other slots).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/nnsph.h"

namespace {

constexpr double kPi = 3.14159265358979323846;
// SRTool.__init__ constants (srtool.py:902-918)
constexpr double kKr = 4.0, kKs = 1400.0, kKn = 0.5, kLambda = 0.9;
constexpr int kNvep = 25;

// _SRVoxel.voxel_vertex_offset_map (srtool.py:775-783): corner w of cube (x, y, z)
// is vertex (x, y, z) + kOff[w].
constexpr int kOff[8][3] = {{0, 1, 0}, {1, 1, 0}, {1, 0, 0}, {0, 0, 0}, {0, 1, 1}, {1, 1, 1}, {1, 0, 1}, {0, 0, 1}};
// SRTool.interpolation_table (srtool.py:931-942): the corners of edge w
constexpr int kEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                              {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

struct Grid {
  int nx, ny, nz, bx, by, bz;
  double ox, oy, oz, vs;
  std::vector<double> v;         // vertex values
  std::vector<uint8_t> active;   // per NN_SR_BLOCK^3 block
  int64_t idx(int x, int y, int z) const { return x + (int64_t)nx * (y + (int64_t)ny * z); }
  bool in(int x, int y, int z) const { return x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz; }
  int64_t bidx(int x, int y, int z) const {
    return x / NN_SR_BLOCK + (int64_t)bx * (y / NN_SR_BLOCK + (int64_t)by * (z / NN_SR_BLOCK));
  }
  bool act(int x, int y, int z) const { return in(x, y, z) && active[bidx(x, y, z)]; }
  double get(int x, int y, int z) const { return act(x, y, z) ? v[idx(x, y, z)] : 0.0; }
  // a write (`+=` included) activates the vertex's block
  void add(int x, int y, int z, double a) {
    active[bidx(x, y, z)] = 1;
    v[idx(x, y, z)] += a;
  }
};

// get_voxel_index (srtool.py:799-803): f32, int() truncates toward zero
inline void voxel_of(const Grid& g, const float* p, int& x, int& y, int& z) {
  x = (int)((p[0] - (float)g.ox) / (float)g.vs);
  y = (int)((p[1] - (float)g.oy) / (float)g.vs);
  z = (int)((p[2] - (float)g.oz) / (float)g.vs);
}

double poly6(double r2, double h, double acoeff) {  // srtool.py:1212-1227
  double rn = std::sqrt(r2);
  if (rn > h) return 0.0;
  double t = h * h - r2;
  return acoeff * t * t * t / (h * h * h * h * h * h * h * h * h);
}

// cyclic Jacobi eigen-decomposition of a symmetric 3x3 matrix; eigenvalues in
// descending order, eigenvectors as the columns of V
void sym_eig(const double S0[3][3], double lam[3], double V[3][3]) {
  double S[3][3];
  std::memcpy(S, S0, sizeof(S));
  double W[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 16; ++sweep) {
    double off = S[0][1] * S[0][1] + S[0][2] * S[0][2] + S[1][2] * S[1][2];
    double dg = S[0][0] * S[0][0] + S[1][1] * S[1][1] + S[2][2] * S[2][2];
    if (off == 0.0 || off <= 1e-30 * dg) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (S[p][q] == 0.0) continue;
        double th = (S[q][q] - S[p][p]) / (2.0 * S[p][q]);
        double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {
          double a = S[k][p], b = S[k][q];
          S[k][p] = c * a - s * b;
          S[k][q] = s * a + c * b;
        }
        for (int k = 0; k < 3; ++k) {
          double a = S[p][k], b = S[q][k];
          S[p][k] = c * a - s * b;
          S[q][k] = s * a + c * b;
        }
        for (int k = 0; k < 3; ++k) {
          double a = W[k][p], b = W[k][q];
          W[k][p] = c * a - s * b;
          W[k][q] = s * a + c * b;
        }
      }
  }
  int o[3] = {0, 1, 2};
  double d[3] = {S[0][0], S[1][1], S[2][2]};
  std::sort(o, o + 3, [&](int a, int b) { return d[a] > d[b]; });
  for (int c = 0; c < 3; ++c) {
    lam[c] = d[o[c]];
    for (int r = 0; r < 3; ++r) V[r][c] = W[r][o[c]];
  }
}

// calc_vertex_normal (srtool.py:1306-1321) and normalize (1412-1417)
void vertex_normal(const Grid& g, int x, int y, int z, double n[3]) {
  n[0] = (x == 0) ? -g.get(x + 1, y, z) : g.get(x - 1, y, z) - g.get(x + 1, y, z);
  n[1] = (y == 0) ? -g.get(x, y + 1, z) : g.get(x, y - 1, z) - g.get(x, y + 1, z);
  n[2] = (z == 0) ? -g.get(x, y, z + 1) : g.get(x, y, z - 1) - g.get(x, y, z + 1);
  double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  if (l != 0.0)
    for (int k = 0; k < 3; ++k) n[k] /= l;
  else
    n[0] = n[1] = n[2] = 0.0;
}

// process_normal_at (srtool.py:1335-1349): trilinear blend of the 8 corner normals
void normal_at(const Grid& g, const double p[3], double n[3]) {
  float pf[3] = {(float)p[0], (float)p[1], (float)p[2]};
  int x0, y0, z0;
  voxel_of(g, pf, x0, y0, z0);
  const double vs = (double)(float)g.vs, ox = (double)(float)g.ox, oy = (double)(float)g.oy,
               oz = (double)(float)g.oz;
  double xd = (p[0] - (x0 * vs + ox)) / vs, yd = (p[1] - (y0 * vs + oy)) / vs, zd = (p[2] - (z0 * vs + oz)) / vs;
  double acc[3] = {0, 0, 0};
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int e = 0; e < 2; ++e) {
        double c[3];
        vertex_normal(g, x0 + a, y0 + b, z0 + e, c);
        const double w = (a ? xd : 1 - xd) * (b ? yd : 1 - yd) * (e ? zd : 1 - zd);
        for (int k = 0; k < 3; ++k) acc[k] += w * c[k];
      }
  double l = std::sqrt(acc[0] * acc[0] + acc[1] * acc[1] + acc[2] * acc[2]);
  if (l != 0.0)
    for (int k = 0; k < 3; ++k) n[k] = acc[k] / l;
  else
    n[0] = n[1] = n[2] = 0.0;
}

int cube_mask(const Grid& g, int x, int y, int z, double iso) {
  int ci = 0;
  for (int w = 0; w < 8; ++w)
    if (g.get(x + kOff[w][0], y + kOff[w][1], z + kOff[w][2]) < iso) ci |= 1 << w;
  return ci;
}

inline bool edge_cross(int ci, int w) { return ((ci >> kEdge[w][0]) ^ (ci >> kEdge[w][1])) & 1; }

// The dual-contouring point of a crossing cube (dual_contouring_impl, 1536-1596)
void dc_point(const Grid& g, int x, int y, int z, int ci, double iso, double out[3]) {
  const double vs = (double)(float)g.vs, ox = (double)(float)g.ox, oy = (double)(float)g.oy,
               oz = (double)(float)g.oz;
  double P[12][3];
  int cnt = 0;
  double mean[3] = {0, 0, 0};
  for (int w = 0; w < 12; ++w) {
    if (!edge_cross(ci, w)) continue;
    const int a = kEdge[w][0], b = kEdge[w][1];
    double p1[3] = {(x + kOff[a][0]) * vs + ox, (y + kOff[a][1]) * vs + oy, (z + kOff[a][2]) * vs + oz};
    double p2[3] = {(x + kOff[b][0]) * vs + ox, (y + kOff[b][1]) * vs + oy, (z + kOff[b][2]) * vs + oz};
    double v1 = g.get(x + kOff[a][0], y + kOff[a][1], z + kOff[a][2]);
    double v2 = g.get(x + kOff[b][0], y + kOff[b][1], z + kOff[b][2]);
    double delta = v2 - v1;
    double t = std::fabs(delta) < 1e-5 ? 0.5 : (iso - v1) / delta;  // vertex_interpolate
    for (int k = 0; k < 3; ++k) {
      P[cnt][k] = p1[k] + t * (p2[k] - p1[k]);
      mean[k] += P[cnt][k];
    }
    ++cnt;
  }
  for (int k = 0; k < 3; ++k) mean[k] /= cnt;
  double NtN[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Ntb[3] = {0, 0, 0};
  for (int r = 0; r < cnt; ++r) {
    double n[3];
    normal_at(g, P[r], n);
    double b = n[0] * (P[r][0] - mean[0]) + n[1] * (P[r][1] - mean[1]) + n[2] * (P[r][2] - mean[2]);
    for (int i = 0; i < 3; ++i) {
      Ntb[i] += n[i] * b;
      for (int j = 0; j < 3; ++j) NtN[i][j] += n[i] * n[j];
    }
  }
  double lam[3], V[3][3];
  sym_eig(NtN, lam, V);
  double res[3] = {0, 0, 0};
  for (int i = 0; i < 3; ++i) {
    double s = std::sqrt(std::max(lam[i], 0.0));
    if (!(s > 0.0)) continue;
    double proj = V[0][i] * Ntb[0] + V[1][i] * Ntb[1] + V[2][i] * Ntb[2];
    double f = proj / (s * std::max(s, 0.1));
    for (int k = 0; k < 3; ++k) res[k] += f * V[k][i];
  }
  // keep the QEF point only inside its own cube (1586-1590)
  float q[3] = {(float)(res[0] + mean[0]), (float)(res[1] + mean[1]), (float)(res[2] + mean[2])};
  int qx, qy, qz;
  voxel_of(g, q, qx, qy, qz);
  for (int k = 0; k < 3; ++k) out[k] = (qx != x || qy != y || qz != z) ? mean[k] : res[k] + mean[k];
}

// get_edge_adjacent_cubes (srtool.py:1612-1705) for the three edges used by polygen:
// edge 2 (corners 2-3, along x), edge 3 (0-3, along y), edge 11 (3-7, along z)
void edge_cubes(int w, int c[4][3]) {
  static const int d2[4][3] = {{0, 0, 0}, {0, 0, -1}, {0, -1, -1}, {0, -1, 0}};
  static const int d3[4][3] = {{0, 0, 0}, {0, 0, -1}, {-1, 0, -1}, {-1, 0, 0}};
  static const int d11[4][3] = {{0, 0, 0}, {0, -1, 0}, {-1, -1, 0}, {-1, 0, 0}};
  const int(*d)[3] = w == 2 ? d2 : w == 3 ? d3 : d11;
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 3; ++k) c[i][k] = d[i][k];
}

// dual_contouring_impl + dual_contouring_polygen + process_normal on a finished field
int contour(const Grid& g, double iso, int record_normals, double* vertices, int32_t max_v, int32_t* indices,
            int32_t max_i, double* normals, int32_t* nv, int32_t* ni) {
  const int64_t cells = (int64_t)g.nx * g.ny * g.nz;
  std::vector<int32_t> vid(cells, -1);
  std::vector<double> pts;
  int32_t nvert = 0;
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x) {
        if (!g.act(x, y, z)) continue;
        const int ci = cube_mask(g, x, y, z, iso);
        if (ci == 0 || ci == 255) continue;
        double p[3];
        dc_point(g, x, y, z, ci, iso, p);
        vid[g.idx(x, y, z)] = nvert++;
        pts.insert(pts.end(), p, p + 3);
      }
  if (nvert > max_v) return -8;
  // two triangles per crossing x/y/z edge of a cube's corner 3 (dual_contouring_polygen)
  int32_t nidx = 0;
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x) {
        if (!g.act(x, y, z)) continue;
        const int ci = cube_mask(g, x, y, z, iso);
        if (ci == 0 || ci == 255) continue;
        for (int w : {2, 3, 11}) {
          if (!edge_cross(ci, w)) continue;
          int dc[4][3];
          edge_cubes(w, dc);
          int32_t id[4];
          bool ok = true;
          for (int k = 0; k < 4; ++k) {
            int a = x + dc[k][0], b = y + dc[k][1], e = z + dc[k][2];
            id[k] = g.in(a, b, e) ? vid[g.idx(a, b, e)] : -1;
            ok = ok && id[k] >= 0;
          }
          if (!ok) continue;
          const bool cond0 = (ci >> kEdge[w][0]) & 1;
          const bool flip = cond0 != (w == 11);
          const int32_t t[6] = {id[2], id[1], id[0], id[3], id[2], id[0]};
          const int32_t tf[6] = {id[0], id[1], id[2], id[0], id[2], id[3]};
          if (nidx + 6 > max_i) return -8;
          for (int k = 0; k < 6; ++k) indices[nidx + k] = flip ? tf[k] : t[k];
          nidx += 6;
        }
      }
  if (vertices) std::memcpy(vertices, pts.data(), sizeof(double) * pts.size());
  if (normals && record_normals)
    for (int i = 0; i < nvert; ++i) normal_at(g, &pts[3 * i], &normals[3 * i]);
  *nv = nvert;
  *ni = nidx;
  return 0;
}

// Marching cubes (marching_cube_impl, srtool.py:1765-1800) with this build's own
// triangulation in place of the reference's 256-case table, which is not reproduced.
// The triangles of a cube come from its corner states ("in": value < isolevel):
//   - faces (axis a, side s) list their corners counter-clockwise seen from outside;
//   - on a face, every run of in-corners gets one segment, from the edge where the
//     walk leaves the run to the edge where it entered it (in-corners stay separate on
//     ambiguous faces, a rule that depends on the face alone, so neighbours agree);
//   - the segments chain into closed loops over the crossing edges; loops are taken
//     in order of their smallest edge id, each starting there, and fanned from that
//     edge: (l0, l[k+1], l[k]).
// Vertices are the crossing edges of each cube in edge order (the reference's atomic
// counter order is replaced by cube order, as for dual contouring).
int mc_cube(int ci, int tri[][3]) {
  int next[12];
  for (int& e : next) e = -1;
  for (int a = 0; a < 3; ++a)
    for (int side = 0; side < 2; ++side) {
      const int u = (a + 1) % 3, v = (a + 2) % 3;
      // (u, v) corners of the face in counter-clockwise order around +e_a
      int uv[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
      if (side == 0) std::swap(uv[1], uv[3]);
      int q[4];
      for (int k = 0; k < 4; ++k)
        for (int c = 0; c < 8; ++c)
          if (kOff[c][a] == side && kOff[c][u] == uv[k][0] && kOff[c][v] == uv[k][1]) q[k] = c;
      auto edge_of = [](int c0, int c1) {
        for (int w = 0; w < 12; ++w)
          if ((kEdge[w][0] == c0 && kEdge[w][1] == c1) || (kEdge[w][0] == c1 && kEdge[w][1] == c0)) return w;
        return -1;
      };
      auto in = [&](int k) { return (ci >> q[((k % 4) + 4) % 4]) & 1; };
      for (int k = 0; k < 4; ++k) {
        if (!(in(k) && !in(k + 1))) continue;  // leaves a run of in-corners at q[k]
        int j = k;
        while (in(j - 1)) --j;  // the run starts at q[j]
        next[edge_of(q[k], q[(k + 1) % 4])] = edge_of(q[((j - 1) % 4 + 4) % 4], q[((j % 4) + 4) % 4]);
      }
    }
  int nt = 0;
  bool seen[12] = {false};
  for (int e = 0; e < 12; ++e) {
    if (next[e] < 0 || seen[e]) continue;
    int loop[12], m = 0;
    for (int f = e; !seen[f]; f = next[f]) {
      seen[f] = true;
      loop[m++] = f;
    }
    for (int k = 1; k + 1 < m; ++k) {
      tri[nt][0] = loop[0];
      tri[nt][1] = loop[k + 1];
      tri[nt][2] = loop[k];
      ++nt;
    }
  }
  return nt;
}

int marching_cubes(const Grid& g, double iso, int record_normals, double* vertices, int32_t max_v, int32_t* indices,
                   int32_t max_i, double* normals, int32_t* nv, int32_t* ni) {
  const double vs = (double)(float)g.vs, ox = (double)(float)g.ox, oy = (double)(float)g.oy,
               oz = (double)(float)g.oz;
  std::vector<double> pts;
  std::vector<int32_t> idx;
  // every cube with a crossing has a corner of nonzero value, so a corner in an active
  // block: the reference's visit of the cubes around active vertices finds it
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x) {
        const int ci = cube_mask(g, x, y, z, iso);
        if (ci == 0 || ci == 255) continue;
        int local[12];
        const int32_t base = (int32_t)(pts.size() / 3);
        int cnt = 0;
        for (int w = 0; w < 12; ++w) {
          local[w] = -1;
          if (!edge_cross(ci, w)) continue;
          const int a = kEdge[w][0], b = kEdge[w][1];
          const double p1[3] = {(x + kOff[a][0]) * vs + ox, (y + kOff[a][1]) * vs + oy, (z + kOff[a][2]) * vs + oz};
          const double p2[3] = {(x + kOff[b][0]) * vs + ox, (y + kOff[b][1]) * vs + oy, (z + kOff[b][2]) * vs + oz};
          const double v1 = g.get(x + kOff[a][0], y + kOff[a][1], z + kOff[a][2]);
          const double v2 = g.get(x + kOff[b][0], y + kOff[b][1], z + kOff[b][2]);
          const double delta = v2 - v1;
          const double t = std::fabs(delta) < 1e-5 ? 0.5 : (iso - v1) / delta;  // vertex_interpolate
          for (int k = 0; k < 3; ++k) pts.push_back(p1[k] + t * (p2[k] - p1[k]));
          local[w] = cnt++;
        }
        int tri[12][3];
        const int nt = mc_cube(ci, tri);
        for (int t = 0; t < nt; ++t)
          for (int k = 0; k < 3; ++k) idx.push_back(base + local[tri[t][k]]);
      }
  const int32_t nvert = (int32_t)(pts.size() / 3);
  if (nvert > max_v || (int64_t)idx.size() > max_i) return -8;
  if (vertices) std::memcpy(vertices, pts.data(), sizeof(double) * pts.size());
  if (indices) std::memcpy(indices, idx.data(), sizeof(int32_t) * idx.size());
  if (normals && record_normals)
    for (int i = 0; i < nvert; ++i) normal_at(g, &pts[3 * i], &normals[3 * i]);
  *nv = nvert;
  *ni = (int32_t)idx.size();
  return 0;
}

// Grid of the parameters, all blocks inactive and every value 0.
Grid make_grid(const nn_sr_params* prm) {
  Grid g;
  g.nx = prm->dims[0]; g.ny = prm->dims[1]; g.nz = prm->dims[2];
  g.bx = (g.nx + NN_SR_BLOCK - 1) / NN_SR_BLOCK;
  g.by = (g.ny + NN_SR_BLOCK - 1) / NN_SR_BLOCK;
  g.bz = (g.nz + NN_SR_BLOCK - 1) / NN_SR_BLOCK;
  g.ox = prm->origin[0]; g.oy = prm->origin[1]; g.oz = prm->origin[2];
  g.vs = prm->voxel_size;
  g.v.assign((size_t)g.nx * g.ny * g.nz, 0.0);
  g.active.assign((size_t)g.bx * g.by * g.bz, 0);
  return g;
}

// update_particles: per-voxel particle lists in id order (at most 64 each)
int bin_particles(const Grid& g, const float* pos, int n, std::vector<int>& vox, std::vector<std::vector<int>>& hash) {
  vox.assign(3 * (size_t)n, 0);
  hash.assign((size_t)g.nx * g.ny * g.nz, {});
  for (int i = 0; i < n; ++i) {
    int x, y, z;
    voxel_of(g, pos + 3 * i, x, y, z);
    if (!g.in(x, y, z)) return -1;
    vox[3 * i] = x; vox[3 * i + 1] = y; vox[3 * i + 2] = z;
    auto& l = hash[g.idx(x, y, z)];
    if ((int)l.size() >= NN_SR_MAX_PER_VOXEL) return -8;
    l.push_back(i);
  }
  return 0;
}

int smoothing_range(const nn_sr_params* prm) {  // srtool.py:1137
  return (int)std::ceil(4.0 * (double)(float)prm->smooth_radius / (double)(float)prm->voxel_size) + 1;
}

// pre_process_data (srtool.py:1006-1095). Distances and the in-range test are f32
// with unfused operations (as the reference's f32 arithmetic); sums are double.
// Particle 0 is skipped (the loop starts at 1): its G and x_bar stay 0.
int prepass(const nn_sr_params* prm, const float* pos, int n, float* G, float* xbar) {
  Grid g = make_grid(prm);
  std::vector<int> vox;
  std::vector<std::vector<int>> hash;
  int rc = bin_particles(g, pos, n, vox, hash);
  if (rc) return rc;
  const float sr = (float)prm->smooth_radius, rr = 2.f * sr;
  const int range = smoothing_range(prm), off = range / 2;
  std::fill(G, G + 9 * (size_t)n, 0.f);
  std::fill(xbar, xbar + 3 * (size_t)n, 0.f);
  for (int i = 1; i < n; ++i) {
    const float* pi = pos + 3 * i;
    double tw = 0.0, xw[3] = {0, 0, 0};
    std::vector<int> nb;
    std::vector<double> wt;
    for (int dz = -off; dz < range - off; ++dz)
      for (int dy = -off; dy < range - off; ++dy)
        for (int dx = -off; dx < range - off; ++dx) {
          int x = vox[3 * i] + dx, y = vox[3 * i + 1] + dy, z = vox[3 * i + 2] + dz;
          if (x < 0 || y < 0 || z < 0 || !g.in(x, y, z)) continue;
          for (int j : hash[g.idx(x, y, z)]) {
            const float d0 = pi[0] - pos[3 * j], d1 = pi[1] - pos[3 * j + 1], d2 = pi[2] - pos[3 * j + 2];
            const float dn = std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
            if (!(dn < rr)) continue;  // isoweight is 0 outside 2 * smooth_radius
            const float q = dn / rr;
            const double w = 1.0 - (double)(q * q * q);
            tw += w;
            for (int k = 0; k < 3; ++k) xw[k] += w * pos[3 * j + k];
            if (w > 0) { nb.push_back(j); wt.push_back(w); }
          }
        }
    if (tw != 0)
      for (int k = 0; k < 3; ++k) xw[k] /= tw;
    for (int k = 0; k < 3; ++k) xbar[3 * i + k] = (float)((1 - kLambda) * pi[k] + kLambda * xw[k]);
    double C[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (size_t q = 0; q < nb.size(); ++q) {
      double dp[3] = {pos[3 * nb[q]] - xw[0], pos[3 * nb[q] + 1] - xw[1], pos[3 * nb[q] + 2] - xw[2]};
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) C[a][b] += wt[q] * dp[a] * dp[b];
    }
    if (tw != 0)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) C[a][b] /= tw;
    double lam[3], V[3][3];
    sym_eig(C, lam, V);
    double sg[3] = {lam[0], lam[1], lam[2]};
    if ((int)nb.size() > kNvep) {
      sg[1] = std::max(sg[1], sg[0] / kKr);
      sg[2] = std::max(sg[2], sg[0] / kKr);
      for (int k = 0; k < 3; ++k) sg[k] *= kKs;
    } else {
      sg[0] = sg[1] = sg[2] = kKn;
    }
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double m = 0;
        for (int k = 0; k < 3; ++k) m += V[a][k] * V[b][k] / sg[k];
        G[9 * i + 3 * a + b] = (float)((tw != 0) ? m / (double)sr : (a == b ? 1.0 : 0.0));
      }
  }
  return 0;
}

// generate_fluid_field (srtool.py:1238-1251) and, with G / x_bar given,
// generate_smooth_fluid_field_impl (1135-1157). The kernel argument q = |G d| is
// evaluated in f32 with unfused operations, so its branch (the kernel as written
// jumps at q = 0.5) is decided the same way wherever the same f32 inputs are used.
int splat(const nn_sr_params* prm, const float* pos, int n, const float* G, const float* xbar, Grid& g) {
  std::vector<int> vox;
  std::vector<std::vector<int>> hash;
  int rc = bin_particles(g, pos, n, vox, hash);
  if (rc) return rc;
  const double r = prm->particle_radius, sr = prm->smooth_radius;
  const double volume = r * r * r * kPi * 4.0 / 3.0;  // srtool.py:920
  const double acoeff = 315.0 / (64.0 * kPi);         // srtool.py:921
  for (int i = 0; i < n; ++i) {
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int x = vox[3 * i] + dx, y = vox[3 * i + 1] + dy, z = vox[3 * i + 2] + dz;
          if (x < 0 || y < 0 || z < 0) continue;
          if (!g.in(x, y, z)) return -8;
          const double q[3] = {x * g.vs + g.ox, y * g.vs + g.oy, z * g.vs + g.oz};
          double d0 = pos[3 * i] - q[0], d1 = pos[3 * i + 1] - q[1], d2 = pos[3 * i + 2] - q[2];
          g.add(x, y, z, volume * poly6(d0 * d0 + d1 * d1 + d2 * d2, sr, acoeff));
        }
  }
  if (!G) return 0;
  const int range = smoothing_range(prm), off = range / 2;
  const float vs = (float)g.vs, ox = (float)g.ox, oy = (float)g.oy, oz = (float)g.oz;
  for (int i = 0; i < n; ++i) {
    const float* Gi = &G[9 * i];
    const double det = (double)Gi[0] * ((double)Gi[4] * Gi[8] - (double)Gi[5] * Gi[7]) -
                       (double)Gi[1] * ((double)Gi[3] * Gi[8] - (double)Gi[5] * Gi[6]) +
                       (double)Gi[2] * ((double)Gi[3] * Gi[7] - (double)Gi[4] * Gi[6]);
    for (int dz = 0; dz < range; ++dz)
      for (int dy = 0; dy < range; ++dy)
        for (int dx = 0; dx < range; ++dx) {
          int nx = vox[3 * i] + dx - off, ny = vox[3 * i + 1] + dy - off, nz = vox[3 * i + 2] + dz - off;
          for (int w = 0; w < 8; ++w) {
            int x = nx + kOff[w][0], y = ny + kOff[w][1], z = nz + kOff[w][2];
            if (x < 0 || y < 0 || z < 0) continue;
            if (!g.in(x, y, z)) return -8;
            const float d[3] = {xbar[3 * i] - ((float)x * vs + ox), xbar[3 * i + 1] - ((float)y * vs + oy),
                                xbar[3 * i + 2] - ((float)z * vs + oz)};
            float gd[3];
            for (int a = 0; a < 3; ++a) gd[a] = Gi[3 * a] * d[0] + Gi[3 * a + 1] * d[1] + Gi[3 * a + 2] * d[2];
            const float qn = std::sqrt(gd[0] * gd[0] + gd[1] * gd[1] + gd[2] * gd[2]);
            double res = 0.0;  // cubic_spline_kernel, srtool.py:1114-1124, as written
            if (0 < qn && qn <= 0.5f)
              res = 48.0 / kPi * det * ((double)qn * qn * qn - (double)qn * qn) + 1.0;
            else if (0.5f < qn && qn <= 1.f)
              res = 16.0 / kPi * det * (1 - (double)qn) * (1 - (double)qn) * (1 - (double)qn);
            g.add(x, y, z, volume * res);
          }
        }
  }
  return 0;
}

// smooth_sdf (srtool.py:1425-1484): statistics of the negative values of the active
// vertices, then the value-weighted Gaussian average over the (2 R + 1)^3 vertices
double smooth(Grid& g, int R) {
  const int64_t cells = (int64_t)g.nx * g.ny * g.nz;
  double mean = 0.0, var = 0.0;
  int64_t cnt = 0;
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x)
        if (g.act(x, y, z) && g.v[g.idx(x, y, z)] < 0) { mean += g.v[g.idx(x, y, z)]; ++cnt; }
  mean /= (double)cnt;  // 0/0 = NaN without negative values, as in the reference
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x)
        if (g.act(x, y, z) && g.v[g.idx(x, y, z)] < 0) {
          double dd = g.v[g.idx(x, y, z)] - mean;
          var += dd * dd;
        }
  const double sd = std::sqrt(var / (double)cnt);
  std::vector<double> out(cells, 0.0);
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x) {
        if (!g.act(x, y, z)) continue;
        const double c = g.v[g.idx(x, y, z)];
        double avg = 0.0, wsum = 0.0;
        for (int dz = -R; dz <= R; ++dz)
          for (int dy = -R; dy <= R; ++dy)
            for (int dx = -R; dx <= R; ++dx) {
              int a = x + dx, b = y + dy, e = z + dz;
              if (a < 0 || b < 0 || e < 0) continue;
              double vv = g.get(a, b, e);
              double diff = std::fabs(c - vv);
              double gw = std::exp(-diff * diff / (2 * sd * sd)) / std::pow(2 * kPi * sd * sd, 1.5);
              avg += gw * vv;
              wsum += gw;
            }
        if (wsum != 0.0) avg /= wsum;
        out[g.idx(x, y, z)] = avg;
      }
  g.v.swap(out);  // copy_and_clear: the same blocks stay active
  return sd;
}

}  // namespace

extern "C" {

// pre_process_data alone: G [n,9] and x_bar [n,3] (f32, as the CUDA path stores them).
int sro_prepass(const nn_sr_params* prm, const float* pos, int32_t n, float* G, float* xbar) {
  return prepass(prm, pos, n, G, xbar);
}

// The splats alone, with the anisotropic kernels given (G, xbar NULL: isotropic
// only): field [cells] and the active-block flags.
int sro_splat(const nn_sr_params* prm, const float* pos, int32_t n, const float* G, const float* xbar, double* field,
              uint8_t* active) {
  Grid g = make_grid(prm);
  int rc = splat(prm, pos, n, G, xbar, g);
  if (rc) return rc;
  std::memcpy(field, g.v.data(), sizeof(double) * g.v.size());
  std::memcpy(active, g.active.data(), g.active.size());
  return 0;
}

// The smoothing alone on a given field and active flags; returns the field in place.
int sro_smooth(const nn_sr_params* prm, double* field, const uint8_t* active, double* sd_out) {
  Grid g = make_grid(prm);
  g.v.assign(field, field + g.v.size());
  g.active.assign(active, active + g.active.size());
  double sd = 0.0;
  for (int it = 0; it < prm->smooth_iterations; ++it) sd = smooth(g, prm->smooth_cells);
  if (sd_out) *sd_out = sd;
  std::memcpy(field, g.v.data(), sizeof(double) * g.v.size());
  return 0;
}

// The contouring stages alone, on a given field (x-fastest [cells]) and active-block
// flags: checks the CUDA contouring on exactly the field the CUDA path produced.
int sro_contour(const nn_sr_params* prm, const double* field, const uint8_t* active, double* vertices,
                int32_t max_v, int32_t* indices, int32_t max_i, double* normals, int32_t* nv, int32_t* ni) {
  Grid g = make_grid(prm);
  g.v.assign(field, field + g.v.size());
  g.active.assign(active, active + g.active.size());
  return contour(g, prm->isolevel, prm->record_normals, vertices, max_v, indices, max_i, normals, nv, ni);
}

// Marching cubes on a given field (values [cells], active flags [blocks]).
int sro_marching_cubes(const nn_sr_params* prm, const double* field, const uint8_t* active, double* vertices,
                       int32_t max_v, int32_t* indices, int32_t max_i, double* normals, int32_t* nv, int32_t* ni) {
  Grid g = make_grid(prm);
  g.v.assign(field, field + g.v.size());
  g.active.assign(active, active + g.active.size());
  return marching_cubes(g, prm->isolevel, prm->record_normals, vertices, max_v, indices, max_i, normals, nv, ni);
}

// The triangle table that mc_cube gives: per cube index, the triangle count and the
// edge ids (12 triangles at most; unused entries -1).
int sro_mc_table(int32_t* ntri, int32_t* tris) {
  for (int ci = 0; ci < 256; ++ci) {
    int tri[12][3];
    ntri[ci] = mc_cube(ci, tri);
    for (int t = 0; t < 12; ++t)
      for (int k = 0; k < 3; ++k) tris[(ci * 12 + t) * 3 + k] = t < ntri[ci] ? tri[t][k] : -1;
  }
  return 0;
}

// The whole of SRTool.dual_contouring for n particles. Outputs (each optional):
// field_splat / field [cells] (after the splats / after smoothing), active [blocks],
// G [n,9], xbar [n,3], sd (smoothing standard deviation), vertices [max_v,3],
// indices [max_i], normals [max_v,3]; counts in *nv, *ni. Returns 0, or -8 when a
// capacity is exceeded, -1 for particles outside the grid.
int sro_dual_contouring(const nn_sr_params* prm, const float* pos, int32_t n, double* field_splat, double* field,
                        uint8_t* active, float* G_out, float* xbar_out, double* sd_out, double* vertices,
                        int32_t max_v, int32_t* indices, int32_t max_i, double* normals, int32_t* nv,
                        int32_t* ni) {
  std::vector<float> G(9 * (size_t)std::max(n, 1), 0.f), xbar(3 * (size_t)std::max(n, 1), 0.f);
  int rc = 0;
  if (prm->use_smooth_field) {
    rc = prepass(prm, pos, n, G.data(), xbar.data());
    if (rc) return rc;
  }
  Grid g = make_grid(prm);
  rc = splat(prm, pos, n, prm->use_smooth_field ? G.data() : nullptr, xbar.data(), g);
  if (rc) return rc;
  if (field_splat) std::memcpy(field_splat, g.v.data(), sizeof(double) * g.v.size());
  double sd = 0.0;
  for (int it = 0; it < prm->smooth_iterations; ++it) sd = smooth(g, prm->smooth_cells);
  if (sd_out) *sd_out = sd;
  if (field) std::memcpy(field, g.v.data(), sizeof(double) * g.v.size());
  if (active) std::memcpy(active, g.active.data(), g.active.size());
  if (G_out) std::memcpy(G_out, G.data(), sizeof(float) * 9 * n);
  if (xbar_out) std::memcpy(xbar_out, xbar.data(), sizeof(float) * 3 * n);
  return contour(g, prm->isolevel, prm->record_normals, vertices, max_v, indices, max_i, normals, nv, ni);
}

// generate_smooth_fluid_field_with_velocity_impl's velocity part (srtool.py:1159-1190):
// vfield [3][cells] (x-fastest per component) gets, for every vertex of every voxel in
// the smoothing range (once per adjacent voxel), v_i * poly6(x_i - vertex) * vs^3.
int sro_vel_field(const nn_sr_params* prm, const float* pos, const float* vel, int32_t n, double* vfield) {
  Grid g = make_grid(prm);
  std::vector<int> vox;
  std::vector<std::vector<int>> hash;
  int rc = bin_particles(g, pos, n, vox, hash);
  if (rc) return rc;
  const int64_t cells = (int64_t)g.nx * g.ny * g.nz;
  std::fill(vfield, vfield + 3 * cells, 0.0);
  const double sr = prm->smooth_radius, acoeff = 315.0 / (64.0 * kPi), coeff = g.vs * g.vs * g.vs;
  const int range = smoothing_range(prm), off = range / 2;
  for (int i = 0; i < n; ++i)
    for (int dz = 0; dz < range; ++dz)
      for (int dy = 0; dy < range; ++dy)
        for (int dx = 0; dx < range; ++dx) {
          int nx = vox[3 * i] + dx - off, ny = vox[3 * i + 1] + dy - off, nz = vox[3 * i + 2] + dz - off;
          for (int w = 0; w < 8; ++w) {
            int x = nx + kOff[w][0], y = ny + kOff[w][1], z = nz + kOff[w][2];
            if (x < 0 || y < 0 || z < 0) continue;
            if (!g.in(x, y, z)) return -8;
            double d0 = pos[3 * i] - (x * g.vs + g.ox), d1 = pos[3 * i + 1] - (y * g.vs + g.oy),
                   d2 = pos[3 * i + 2] - (z * g.vs + g.oz);
            const double f = poly6(d0 * d0 + d1 * d1 + d2 * d2, sr, acoeff) * coeff;
            if (f == 0.0) continue;
            for (int k = 0; k < 3; ++k) vfield[k * cells + g.idx(x, y, z)] += vel[3 * i + k] * f;
          }
        }
  return 0;
}

// process_velocity (srtool.py:1351-1381) at the given mesh vertices [nv,3].
int sro_mesh_velocity(const nn_sr_params* prm, const double* vfield, const double* vertices, int32_t nv,
                      double* out) {
  Grid g = make_grid(prm);
  const int64_t cells = (int64_t)g.nx * g.ny * g.nz;
  const double vs = (double)(float)g.vs, ox = (double)(float)g.ox, oy = (double)(float)g.oy,
               oz = (double)(float)g.oz;
  for (int i = 0; i < nv; ++i) {
    const double* p = vertices + 3 * i;
    float pf[3] = {(float)p[0], (float)p[1], (float)p[2]};
    int x0, y0, z0;
    voxel_of(g, pf, x0, y0, z0);
    const double xd = (p[0] - (x0 * vs + ox)) / vs, yd = (p[1] - (y0 * vs + oy)) / vs, zd = (p[2] - (z0 * vs + oz)) / vs;
    double acc[3] = {0, 0, 0};
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int e = 0; e < 2; ++e) {
          const int x = x0 + a, y = y0 + b, z = z0 + e;
          if (!g.in(x, y, z)) continue;
          const double w = (a ? xd : 1 - xd) * (b ? yd : 1 - yd) * (e ? zd : 1 - zd);
          for (int k = 0; k < 3; ++k) acc[k] += w * vfield[k * cells + g.idx(x, y, z)];
        }
    for (int k = 0; k < 3; ++k) out[3 * i + k] = acc[k];
  }
  return 0;
}

}  // extern "C"
