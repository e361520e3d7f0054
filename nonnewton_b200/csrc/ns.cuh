// ns.cuh — cell-linked neighbour search: Z-order counting sort of particles into
// cells of edge h, deterministic in-cell order (by particle id), gather of the state
// into the new slot order, and per-slot neighbour lists from the 9 contiguous
// cell rows of the 27-cell stencil.
//
// Replaces NeighborhoodSearchSparse.update_grid / store_neighbors
// (SPH/main.py:815-847): same pair set (p_i != p_j and |x_i - x_j| < h on absolute
// f32 positions, SPH/main.py:845), no per-cell cap (the reference stores at most 50
// particles per cell, SPH/main.py:778) and a checked neighbour cap.
#pragma once
#include "dev.cuh"

#define GRID_STRIDE(i, n) for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

// Grid-stride loop whose trip count is uniform across a warp (for warp collectives):
// `valid` is false on the lanes past the end.
#define FOR_SLOTS_WARP(i, valid, n)                                                        \
  for (int _base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; _base < (n);             \
       _base += gridDim.x * blockDim.x)                                                     \
    for (int i = _base + (threadIdx.x & 31), _once = 1; _once; _once = 0)                   \
      for (bool valid = i < (n); _once; _once = 0)

// Cell key of a position in scene s: Morton(cy, cz) * gx + cx + cell_base.
__device__ __forceinline__ uint32_t cell_key(const SceneDev& s, real x, real y, real z, int* cx_out, int* cy_out,
                                             int* cz_out) {
  int cx = (int)floor((x - s.origin[0]) / s.cellx);
  int cy = (int)floor((y - s.origin[1]) / s.cell);
  int cz = (int)floor((z - s.origin[2]) / s.cell);
  cx = min(max(cx, 0), s.gx - 1);
  cy = min(max(cy, 0), s.gy - 1);
  cz = min(max(cz, 0), s.gz - 1);
  if (cx_out) { *cx_out = cx; *cy_out = cy; *cz_out = cz; }
  return (uint32_t)(s.cell_base + (int64_t)morton2((uint32_t)cy, (uint32_t)cz) * s.gx + cx);
}

// Per-step counters reset (before the neighbour search).
__device__ __forceinline__ void step_reset_scenes(const Dev& d) {
  const int ns = d.d_n[1];
  for (int sc = threadIdx.x; sc < ns; sc += blockDim.x) {
    SceneDyn& y = d.dyn[sc];
    y.max_density_bits = 0u;
    y.max_nb = 0;
    y.it_v = y.it_p = y.it_cg = 0;
    y.div_ran = 0;
    y.np_fresh = 0;
  }
}

// `reset_step`: block 0 also resets the step's per-scene counters (the step's first
// launch; nothing before the list build reads them).
__global__ void k_zero_cells(Dev d, int reset_step) {
  if (reset_step && blockIdx.x == 0) step_reset_scenes(d);
  const int nc = d.d_n[2];
  GRID_STRIDE(i, nc + 1) d.cell_count[i] = 0u;
}

// Keys and in-cell ranks of every source particle (truth id order or previous slots).
__global__ void k_keys(Dev d) {
  const int n = d.d_n[0];
  const int mode = *d.src_from_truth;  // 0 previous slots, 1 caller state, 2 caller rest positions
  const bool truth = mode != 0;
  const float* __restrict__ X = mode == 2 ? d.t.x_0 : d.t.x;
  GRID_STRIDE(s, n) {
    real x, y, z;
    int sc;
    if (truth) {
      x = X[3 * s]; y = X[3 * s + 1]; z = X[3 * s + 2];
      sc = d.scene_of_id[s];
    } else {
      real4 p = d.wo.pos[s];
      x = p.x; y = p.y; z = p.z;
      sc = slot_scene(d.wo.flags[s]);
    }
    uint32_t k = cell_key(d.sc[sc], x, y, z, nullptr, nullptr, nullptr);
    d.key[s] = k;
    d.rank[s] = atomicAdd(&d.cell_count[k], 1u);
  }
}

// Exclusive scan of cell_count[0 .. cells] in place (two phases over tiles).
#define SCAN_TILE 4096
#define SCAN_THREADS 1024
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t w = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    sh[lane] = w;
  }
  __syncthreads();
  uint32_t base = wid > 0 ? sh[wid - 1] : 0u;
  uint32_t incl = base + x;
  if (total) *total = sh[(blockDim.x >> 5) - 1];
  __syncthreads();
  return incl - v;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(Dev d) {
  __shared__ uint32_t sh[32];
  const int len = d.d_n[2] + 1;
  const int ntiles = (len + SCAN_TILE - 1) / SCAN_TILE;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    uint32_t s = 0;
    for (int k = threadIdx.x; k < SCAN_TILE; k += blockDim.x) {
      int i = t * SCAN_TILE + k;
      if (i < len) s += d.cell_count[i];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t tot = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += sh[w];
      d.tile_sums[t] = tot;
    }
    __syncthreads();
  }
}

// Second phase: each block adds up the tile sums before its tile itself (the blocks
// walk the tiles in order, so each reads about as many tile sums as there are tiles),
// then scans its tile. A separate one-block scan of the tile sums would cost a launch.
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply(Dev d) {
  __shared__ uint32_t sh[32];
  const int len = d.d_n[2] + 1;
  const int ntiles = (len + SCAN_TILE - 1) / SCAN_TILE;
  constexpr int PER = SCAN_TILE / SCAN_THREADS;
  uint32_t before = 0;  // sum of tile_sums[0 .. done)
  int done = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    uint32_t part = 0, tot = 0;
    for (int k = done + (int)threadIdx.x; k < t; k += blockDim.x) part += d.tile_sums[k];
    block_excl_scan(part, sh, &tot);
    before += tot;
    done = t;
    uint32_t v[PER];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      int i = t * SCAN_TILE + threadIdx.x * PER + k;
      v[k] = i < len ? d.cell_count[i] : 0u;
      s += v[k];
    }
    uint32_t ex = block_excl_scan(s, sh, nullptr) + before;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      int i = t * SCAN_TILE + threadIdx.x * PER + k;
      if (i < len) d.cell_count[i] = ex;
      ex += v[k];
    }
    __syncthreads();
  }
}

__global__ void k_scatter(Dev d) {
  const int n = d.d_n[0];
  GRID_STRIDE(s, n) d.src[d.cell_count[d.key[s]] + d.rank[s]] = s;
}

// In-cell order by particle id, so that the slot order (and every neighbour sum)
// does not depend on the atomics of k_keys. A cell of up to NS_SORT_REG particles is
// sorted by its own thread in registers, one of up to NS_SORT_SMALL by its own thread
// in place (insertion sort); a crowded cell (a cluster) by the
// whole warp: each lane ranks some of its particles by counting the smaller ids, so
// a cell of n particles takes n^2 / 32 steps per lane instead of about n^2 / 4 on one
// thread. Particle ids are distinct, so the ranks are a permutation. The scratch of
// the warp path is the key array, which nothing reads after k_scatter.
#define NS_SORT_SMALL 24
#define NS_SORT_REG 8
__global__ void k_cell_sort(Dev d) {
  const int nc = d.d_n[2];
  const bool truth = *d.src_from_truth != 0;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  FOR_SLOTS_WARP(c, valid, nc) {
    uint32_t b = 0, e = 0;
    if (valid) { b = d.cell_count[c]; e = d.cell_count[c + 1]; }
    const uint32_t n = e - b;
    if (n >= 2 && n <= NS_SORT_REG) {
      // in registers: the sources and their ids load together (no chain of dependent
      // loads per comparison), an odd-even transposition network sorts NS_SORT_REG slots
      // whose unused tail holds the largest key, and the sources go back in id order
      int sv[NS_SORT_REG], kv[NS_SORT_REG];
#pragma unroll
      for (int q = 0; q < NS_SORT_REG; ++q) sv[q] = (uint32_t)q < n ? d.src[b + q] : 0;
#pragma unroll
      for (int q = 0; q < NS_SORT_REG; ++q) kv[q] = (uint32_t)q < n ? (truth ? sv[q] : d.wo.id[sv[q]]) : INT_MAX;
#pragma unroll
      for (int r = 0; r < NS_SORT_REG; ++r)
#pragma unroll
        for (int q = r & 1; q + 1 < NS_SORT_REG; q += 2)
          if (kv[q] > kv[q + 1]) {
            const int tk = kv[q]; kv[q] = kv[q + 1]; kv[q + 1] = tk;
            const int ts = sv[q]; sv[q] = sv[q + 1]; sv[q + 1] = ts;
          }
#pragma unroll
      for (int q = 0; q < NS_SORT_REG; ++q)
        if ((uint32_t)q < n) d.src[b + q] = sv[q];
    } else if (n > NS_SORT_REG && n <= NS_SORT_SMALL) {
      for (uint32_t i = b + 1; i < e; ++i) {
        int s = d.src[i];
        int ids = truth ? s : d.wo.id[s];
        uint32_t j = i;
        while (j > b) {
          int sp = d.src[j - 1];
          int idp = truth ? sp : d.wo.id[sp];
          if (idp <= ids) break;
          d.src[j] = sp;
          --j;
        }
        d.src[j] = s;
      }
    }
    unsigned big = __ballot_sync(full, n > NS_SORT_SMALL);
    while (big) {
      const int l = __ffs(big) - 1;
      big &= big - 1;
      const uint32_t bb = __shfl_sync(full, b, l), ee = __shfl_sync(full, e, l);
      for (uint32_t k = bb + lane; k < ee; k += 32) d.key[k] = (uint32_t)d.src[k];
      __syncwarp();
      for (uint32_t k = bb + lane; k < ee; k += 32) {
        const int s = (int)d.key[k];
        const int ids = truth ? s : d.wo.id[s];
        uint32_t rank = 0;
        for (uint32_t j = bb; j < ee; ++j) {
          const int sj = (int)d.key[j];
          rank += (uint32_t)((truth ? sj : d.wo.id[sj]) < ids);
        }
        d.src[bb + rank] = s;
      }
      __syncwarp();
    }
  }
}

__device__ __forceinline__ uint32_t class_bits(int material, int dynamic, int phase, const SceneDev& s) {
  uint32_t c = NN_CLS_VALID;
  if (material == NN_SOLID) c |= NN_CLS_SOLID;
  if (dynamic) c |= NN_CLS_DYNAMIC;
  if (s.el_mult > 0) {
    if ((s.flags & NN_F_QUIRKS) || (material == NN_SOLID && phase >= NN_PHASE_ELASTIC_BASE)) c |= NN_CLS_ELASTIC;
  }
  return c;
}

// Gather the state into the new slot order (from Truth by id, or from the previous
// slots), and record max |v| per scene for the CFL step.
__global__ void k_gather(Dev d) {
  const int n = d.d_n[0];
  const int mode = *d.src_from_truth;
  const bool truth = mode != 0;
  const float* __restrict__ X = mode == 2 ? d.t.x_0 : d.t.x;
  FOR_SLOTS_WARP(i, valid, n) {
    uint32_t fl = 0u;
    real vm = 0.f;
    if (valid) {
      int s = d.src[i];
      int id;
      real4 p, v;
      real m, rho;
      if (truth) {
        id = s;
        int sc = d.scene_of_id[id];
        const real vol = d.t.volume[id];
        p = make_real4(X[3 * id], X[3 * id + 1], X[3 * id + 2],
                        d.t.material[id] == NN_SOLID ? -vol : vol);  // signed volume: solid < 0
        m = d.t.m[id];
        v = make_real4(d.t.v[3 * id], d.t.v[3 * id + 1], d.t.v[3 * id + 2], m);  // vel.w carries the mass
        rho = d.t.density[id];
        fl = class_bits(d.t.material[id], d.t.is_dynamic[id], d.t.phase_id[id], d.sc[sc]) |
             ((uint32_t)sc << NN_SCENE_SHIFT);
      } else {
        id = d.wo.id[s];
        p = d.wo.pos[s];
        v = d.wo.vel[s];
        m = d.wo.mass[s];
        rho = d.wo.dens[s];
        fl = d.wo.flags[s];
      }
      d.w.pos[i] = p;
      d.w.vel[i] = v;
      d.w.mass[i] = m;
      d.w.dens[i] = rho;
      d.w.flags[i] = fl;
      d.w.id[i] = id;
      d.slot_of_id[id] = i;
      vm = sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    }
    const bool cfl = valid && (fl & NN_CLS_DYNAMIC) && (d.sc[slot_scene(fl)].flags & NN_F_CFL);
    warp_max_to(&d.dyn[slot_scene(fl)].vmax_bits, __float_as_uint((float)vm), cfl);
  }
}

// Neighbour lists: for every slot, the 9 (dy, dz) rows of three x-adjacent cells are
// contiguous slot ranges; candidates are tested with the reference's exact f32
// expression. Lists hold slot indices, transposed [k][cap] for coalesced reads.
//
// A warp whose 32 slots lie in one (y, z) row of one scene (the common case, since
// slots are cell-sorted) stages each candidate row, covering all its lanes' windows,
// into shared memory with coalesced loads, in chunks of NS_CHUNK; each lane then tests
// its own 3-cell window from shared memory. Other warps read candidates directly.
// The in-range test sqrt_rn(r2) < h is evaluated as r2 < h2_thr, where h2_thr is the
// smallest float whose correctly rounded square root is >= h (exactly equivalent; the
// FP64 build tests r2 < h^2 in double).
#define NS_WARPS 8
#define NS_CHUNK 128
__device__ __forceinline__ real exact_r2(real3 r) {
  return add_rn(add_rn(mul_rn(r.x, r.x), mul_rn(r.y, r.y)), mul_rn(r.z, r.z));
}

#ifndef NN_FP64
// Staged candidates of the FP32 build are tested two at a time with sm_100's packed
// f32x2 arithmetic, half the arithmetic instructions of the issue-bound test loop, and
// with results bit-identical to exact_r2 (so the lists are unchanged):
//  - x_j + (-x_i) is the exact negation of x_i - x_j (one add.rn.f32x2);
//  - each square is fma.rn.f32x2(d, d, +0), which rounds d*d once, as mul.rn does.
//    A packed mul.rn.f32x2 feeding the packed add was measured to be contracted into a
//    fused multiply-add by ptxas, which moves r2 by a rounding step in about a quarter
//    of the pairs; an fma with a +0 addend cannot be folded into the add that follows,
//    since that would change its result;
//  - the two sums are add.rn.f32x2, in the reference's order.
// The stage holds x, y and z planes, so one 8-byte shared load yields a pair (t even);
// the lower 32 bits hold candidate t.
#define NS_PACKED 1
__device__ __forceinline__ uint64_t add_rn_x2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t sq_rn_x2(uint64_t a) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %1, %2;" : "=l"(d) : "l"(a), "l"(0ull));
  return d;
}
__device__ __forceinline__ uint64_t splat_x2(float v) {
  const uint64_t u = __float_as_uint(v);
  return u | (u << 32);
}
__device__ __forceinline__ uint32_t pair_hits(const float* sx, const float* sy, const float* sz, uint32_t t,
                                              uint64_t nx, uint64_t ny, uint64_t nz, float thr) {
  const uint64_t dx = add_rn_x2(*reinterpret_cast<const uint64_t*>(sx + t), nx);
  const uint64_t dy = add_rn_x2(*reinterpret_cast<const uint64_t*>(sy + t), ny);
  const uint64_t dz = add_rn_x2(*reinterpret_cast<const uint64_t*>(sz + t), nz);
  const uint64_t r2 = add_rn_x2(add_rn_x2(sq_rn_x2(dx), sq_rn_x2(dy)), sq_rn_x2(dz));
  return (uint32_t)(__uint_as_float((uint32_t)r2) < thr) |
         ((uint32_t)(__uint_as_float((uint32_t)(r2 >> 32)) < thr) << 1);
}
#endif

__global__ void __launch_bounds__(NS_WARPS * 32) k_build_lists(Dev d) {
#ifdef NS_PACKED
  __shared__ __align__(16) float stage_xyz[3][NS_WARPS][NS_CHUNK];
  float* sx = stage_xyz[0][threadIdx.x >> 5];
  float* sy = stage_xyz[1][threadIdx.x >> 5];
  float* sz = stage_xyz[2][threadIdx.x >> 5];
#else
  __shared__ real4 stage_all[NS_WARPS][NS_CHUNK];
  real4* stage = stage_all[threadIdx.x >> 5];
#endif
  const int lane = threadIdx.x & 31;
  const unsigned full = 0xffffffffu;
  const int n = d.d_n[0];
  FOR_SLOTS_WARP(i, valid, n) {
    int cnt = 0, scn = 0, cx = 0, cy = 0, cz = 0;
    real4 pi = make_real4(0.f, 0.f, 0.f, 0.f);
    if (valid) {
      scn = slot_scene(d.w.flags[i]);
      pi = d.w.pos[i];
      cell_key(d.sc[scn], pi.x, pi.y, pi.z, &cx, &cy, &cz);
    }
    const SceneDev& s = d.sc[scn];
    const real3 xi = f3(pi);
    const real thr = s.h2_thr;
#ifdef NS_PACKED
    const uint64_t nx = splat_x2(-xi.x), ny = splat_x2(-xi.y), nz = splat_x2(-xi.z);
#endif
    const int x0 = max(cx - s.nfx, 0), x1 = min(cx + s.nfx, s.gx - 1);
    // lane 0 is always valid (the warp's first slot is below n)
    const int ly = __shfl_sync(full, cy, 0), lz = __shfl_sync(full, cz, 0), ls = __shfl_sync(full, scn, 0);
    const bool uniform = __all_sync(full, !valid || (cy == ly && cz == lz && scn == ls));
    auto append = [&](int j) {
      if (cnt < d.max_nb) __stcs(&d.nbr[(size_t)cnt * d.cap + i], j);  // streaming store (see k_density_adv)
      ++cnt;
    };
    if (uniform) {
      // every bound below is warp-uniform: the lanes past the end of the array carry
      // scene 0, so the scene of lane 0 is used (all valid lanes share it)
      const SceneDev& su = d.sc[ls];
      const int wx0 = max(__reduce_min_sync(full, valid ? cx : 0x7fffffff) - su.nfx, 0);
      const int wx1 = min(__reduce_max_sync(full, valid ? cx : -1) + su.nfx, su.gx - 1);
      for (int dz = -su.nf; dz <= su.nf; ++dz) {
        const int zz = lz + dz;
        if (zz < 0 || zz >= su.gz) continue;
        for (int dy = -su.nf; dy <= su.nf; ++dy) {
          const int yy = ly + dy;
          if (yy < 0 || yy >= su.gy) continue;
          const int64_t row = su.cell_base + (int64_t)morton2((uint32_t)yy, (uint32_t)zz) * su.gx;
          const uint32_t rb = d.cell_count[row + wx0], re = d.cell_count[row + wx1 + 1];
          uint32_t b = 0, e = 0;
          if (valid) { b = d.cell_count[row + x0]; e = d.cell_count[row + x1 + 1]; }
          for (uint32_t c0 = rb; c0 < re; c0 += NS_CHUNK) {
            const uint32_t c1 = min(c0 + NS_CHUNK, re);
#ifdef NS_PACKED
            for (uint32_t t = lane; t < c1 - c0; t += 32) {
              const real4 p = ldg(&d.w.pos[c0 + t]);
              sx[t] = p.x; sy[t] = p.y; sz[t] = p.z;
            }
            // a pair that ends past an odd chunk end reads one more entry (< NS_CHUNK,
            // which is even): give it a defined value; its bit is masked below
            if (lane == 0 && ((c1 - c0) & 1u)) { sx[c1 - c0] = 0.f; sy[c1 - c0] = 0.f; sz[c1 - c0] = 0.f; }
            __syncwarp();
            const uint32_t lo = max(b, c0), hi = min(e, c1);
            // groups of up to 32 candidates from an even stage index (one below lo when
            // lo - c0 is odd; that bit is cleared), tested in pairs
            for (uint32_t g = (lo - c0) & ~1u; lo < hi && g < hi - c0; g += 32) {
              const uint32_t len = min(32u, hi - c0 - g);
              uint32_t m = 0u, k = 0u;
              for (; k + 4 <= len; k += 4) {  // two independent pairs
                const uint32_t p0 = pair_hits(sx, sy, sz, g + k, nx, ny, nz, thr);
                const uint32_t p1 = pair_hits(sx, sy, sz, g + k + 2, nx, ny, nz, thr);
                m |= (p0 | (p1 << 2)) << k;
              }
              for (; k < len; k += 2) m |= pair_hits(sx, sy, sz, g + k, nx, ny, nz, thr) << k;
              if (len < 32u) m &= (1u << len) - 1u;
              if (c0 + g < lo) m &= ~1u;
              const uint32_t self = (uint32_t)i - (c0 + g);
              if (self < 32u) m &= ~(1u << self);
              while (m) {
                append((int)(c0 + g + __ffs(m) - 1));
                m &= m - 1u;
              }
            }
#else
            for (uint32_t t = lane; t < c1 - c0; t += 32) stage[t] = ldg(&d.w.pos[c0 + t]);
            __syncwarp();
            const uint32_t lo = max(b, c0), hi = min(e, c1);
            // tests first, into a hit mask per group of 32 candidates (no stores in the
            // test loop, where every store site would run whenever any lane hits), then
            // the hits appended in ascending slot order
            for (uint32_t g0 = lo; g0 < hi; g0 += 32) {
              const uint32_t len = min(32u, hi - g0);
              const real4* st = stage + (g0 - c0);
              uint32_t m = 0u, k = 0u;
              for (; k + 4 <= len; k += 4) {  // four independent tests
                const uint32_t h0 = exact_r2(xi - f3(st[k])) < thr;
                const uint32_t h1 = exact_r2(xi - f3(st[k + 1])) < thr;
                const uint32_t h2 = exact_r2(xi - f3(st[k + 2])) < thr;
                const uint32_t h3 = exact_r2(xi - f3(st[k + 3])) < thr;
                m |= (h0 | (h1 << 1) | (h2 << 2) | (h3 << 3)) << k;
              }
              for (; k < len; ++k) m |= (uint32_t)(exact_r2(xi - f3(st[k])) < thr) << k;
              const uint32_t self = (uint32_t)i - g0;
              if (self < len) m &= ~(1u << self);
              while (m) {
                append((int)(g0 + __ffs(m) - 1));
                m &= m - 1u;
              }
            }
#endif
            __syncwarp();
          }
        }
      }
    } else if (valid) {
      for (int dz = -s.nf; dz <= s.nf; ++dz) {
        const int zz = cz + dz;
        if (zz < 0 || zz >= s.gz) continue;
        for (int dy = -s.nf; dy <= s.nf; ++dy) {
          const int yy = cy + dy;
          if (yy < 0 || yy >= s.gy) continue;
          const int64_t row = s.cell_base + (int64_t)morton2((uint32_t)yy, (uint32_t)zz) * s.gx;
          const uint32_t b = d.cell_count[row + x0], e = d.cell_count[row + x1 + 1];
          for (uint32_t j = b; j < e; ++j) {
            if ((int)j == i) continue;
            if (exact_r2(xi - f3(ldg(&d.w.pos[j]))) < thr) append((int)j);
          }
        }
      }
    }
    if (valid) {
      d.nbr_cnt[i] = min(cnt, d.max_nb);
      if (d.nbr_raw) d.nbr_raw[i] = cnt;
      if (cnt > d.max_nb) set_status(&d.dyn[scn], NN_ERR_NEIGHBOR_OVERFLOW);
    }
    warp_max_to(&d.dyn[scn].max_nb, cnt, valid);
  }
}

// meta.ns.num_neighbors / neighbors in particle-id space, rows sorted by id
// (materialised on demand for parity checks and the elastic rest state). `num` gets
// the stored count, or the full count where the search kept it (nbr_raw).
__global__ void k_export_neighbors(Dev d, int32_t* num, int32_t* lists, int width) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const int id = d.w.id[i];
    const int c = d.nbr_cnt[i];
    int32_t* row = lists + (size_t)id * width;
    int w = min(c, width);
    // insertion sort of the neighbour ids into the output row
    for (int k = 0; k < w; ++k) {
      int v = d.w.id[d.nbr[(size_t)k * d.cap + i]];
      int p = k;
      while (p > 0 && row[p - 1] > v) { row[p] = row[p - 1]; --p; }
      row[p] = v;
    }
    if (c > width) {  // keep the `width` smallest ids
      for (int k = width; k < c; ++k) {
        int v = d.w.id[d.nbr[(size_t)k * d.cap + i]];
        if (v >= row[width - 1]) continue;
        int p = width - 1;
        while (p > 0 && row[p - 1] > v) { row[p] = row[p - 1]; --p; }
        row[p] = v;
      }
    }
    for (int k = w; k < width; ++k) row[k] = -1;
    num[id] = d.nbr_raw ? d.nbr_raw[i] : c;
  }
}
