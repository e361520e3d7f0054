// sph.cuh — the SPH passes of one step on the sorted working set. Each kernel is a
// grid-stride loop over slots (sizes read from the device, so one captured graph
// serves any batch composition), walks the slot's neighbour list, and reads per-scene
// constants from SceneDev. Reductions that decide convergence are FP64.
#pragma once
#include "dev.cuh"

// Register cap of the solver-loop passes (occupancy vs. spills; set at build time).
#ifdef NN_PASS_MAXREG
#define NN_PASS_REGS __maxnreg__(NN_PASS_MAXREG)
#else
#define NN_PASS_REGS
#endif

#define NB_LOOP(d, i, j)                                   \
  for (int _k = 0, _c = (d).nbr_cnt[i]; _k < _c; ++_k)     \
    for (int j = (d).nbr[(size_t)_k * (d).cap + (i)], _o = 1; _o; _o = 0)

struct GPV { real4 p, v; };

// ---------------------------------------------------------------------------
// compute_static_boundary_volume / compute_moving_boundary_volume (SPH/main.py:1010-1035)
template <int U>
__global__ void k_boundary_volume(Dev d, int moving) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const uint32_t fl = d.w.flags[i];
    if (moving ? !cls_dyn_solid(fl) : !cls_static_solid(fl)) continue;
    const SceneDev& s = d.sc[slot_scene(fl)];
    const real3 xi = f3(d.w.pos[i]);
    real delta = s.W0;
    // plain loads: this pass writes pos.w of solid slots (the sign never changes)
    nb_batches<U>(d.nbr + i, d.cap, d.nbr_cnt[i], i, [&](int j) { return d.w.pos[j]; },
               [&](int, real4 pj) {
                 if (!w_fluid(pj.w)) {
                   const real3 r = xi - f3(pj);
                   delta += kw_r2(dot3(r, r), s);
                 }
               });
    d.w.pos[i].w = -(1.f / delta * 3.f);
  }
}

// clear_accelerations_kernel (SPH/main.py:945-951). With `solid_terms` also what the
// force pass would write for the solid slots of scenes with fluid (strain rate and
// viscosity 0, CG coefficients (0, 1 if dynamic)): the step sets it when the fluid's
// non-pressure terms come from the divergence loop's last density change instead.
// `step_start`: block 0 also takes the step's time step (k_step_dt with the CFL rule)
// and the divergence and pressure solves' loop start, which nothing reads before them.
__device__ __forceinline__ void step_dt_scenes(const Dev& d, int do_cfl);
__device__ __forceinline__ void solver_begin_scene(SceneDyn& y, const SceneDev& s, int which);
__global__ void k_clear_acc(Dev d, int solid_terms, int step_start) {
  if (step_start && blockIdx.x == 0) {
    step_dt_scenes(d, 1);
    for (int sc = threadIdx.x; sc < d.d_n[1]; sc += blockDim.x) {
      solver_begin_scene(d.dyn[sc], d.sc[sc], 0);
      solver_begin_scene(d.dyn[sc], d.sc[sc], 1);
    }
  }
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const uint32_t fl = d.w.flags[i];
    const SceneDev& s = d.sc[slot_scene(fl)];
    d.acc4[i] = cls_static_solid(fl) ? make_real4(0.f, 0.f, 0.f, 0.f) : make_real4(s.g[0], s.g[1], s.g[2], 0.f);
    if (solid_terms && !cls_fluid(fl) && s.n_fluid > 0) {
      if (s.flags & NN_F_NONNEWTON) { d.srn[i] = 0.f; d.mu[i] = 0.f; }
      if (scene_implicit(s)) d.cg_aux[i] = make_real2(0.f, cls_dyn_solid(fl) ? 1.f : 0.f);
    }
  }
}

// compute_densities (SPH/main.py:975-984) fused with compute_DFSPH_factor
// (SPH/main.py:1569-1608): both walk the same neighbours with fixed positions.
// compute_densities (SPH/main.py:975-984), compute_DFSPH_factor (SPH/main.py:1569-1608)
// and, with CHANGE, the divergence solve's first compute_density_change and
// alpha *= 1/dt (SPH/main.py:1686-1688): all read the same neighbours at the same
// positions and velocities, and each only needs the particle's own factor.
template <int U, bool CHANGE>
__global__ void k_density_factor(Dev d, int do_density, int do_factor) {
  const int n = d.d_n[0];
  FOR_SLOTS_WARP(i, valid, n) {
    const uint32_t fl = valid ? d.w.flags[i] : 0u;
    const bool work = valid && cls_fluid(fl);
    const int scn = slot_scene(fl);
    real rho = 0.f;
    if (work) {
      const SceneDev& s = d.sc[scn];
      const real4 pi = d.w.pos[i];
      const real3 xi = f3(pi);
      const real3 vi = f3(d.w.vel[i]);
      const int c = d.nbr_cnt[i];
      real den = 0.f, sum_grad = 0.f, dd = 0.f;
      real3 gpi = make_real3(0.f, 0.f, 0.f);
      auto body = [&](real4 pj, real4 vj) {
        const real3 r = xi - f3(pj);
        real w;
        real3 g;
        kwg_r2(r, dot3(r, r), s, w, g);
        const real V = fabs(pj.w);
        den += V * w;
        const real3 gpj = g * (-V);
        if (w_fluid(pj.w)) sum_grad += dot3(gpj, gpj);
        gpi -= gpj;
        if (CHANGE) dd += V * dot3(vi - f3(vj), g);
      };
      if constexpr (CHANGE) {
        nb_batches<U>(d.nbr + i, d.cap, c, i, [&](int j) { return GPV{pos_of(d, j), ldg(&d.w.vel[j])}; },
                      [&](int, const GPV& g) { body(g.p, g.v); });
      } else {
        nb_batches<U>(d.nbr + i, d.cap, c, i, [&](int j) { return pos_of(d, j); },
                      [&](int, real4 pj) { body(pj, pj); });
      }
      if (do_density) {
        rho = pi.w * s.W0;
        rho += den;
        rho = rho * s.rho0;
        d.w.dens[i] = rho;
      }
      if (do_factor) {
        sum_grad += dot3(gpi, gpi);
        real alpha = sum_grad > 1e-6f ? -1.f / sum_grad : 0.f;
        if (CHANGE && d.dyn[scn].act_v) {
          dd = fmax(dd, real(0));
          if (c < 20) dd = 0.f;
          d.rho_adv[i] = dd;
          alpha = alpha * d.dyn[scn].inv_dt;
          d.kappa[i] = dd * alpha;
        }
        d.alpha[i] = alpha;
      }
    }
    if (do_density) warp_max_to(&d.dyn[scn].max_density_bits, __float_as_uint((float)rho), work);
  }
}

__device__ __forceinline__ real nn_law(real g, const SceneDev& s);
__device__ __forceinline__ real strain_rate_norm(const real (&S)[6], real rho_i, bool quirks);

// compute_density_change (SPH/main.py:1610-1645). mode 0: first call of
// divergence_solve, also applies alpha *= 1/dt (1688); mode 1: solver iteration,
// accumulates the FP64 density error (1669-1675, 1717-1719).
//
// NP: the fluid's non-pressure terms of compute_non_pressure_forces (SPH/main.py:
// 1557-1567) in the same pass: surface tension (1387-1414), the strain rate and the
// viscosity law (461-492, 404-459) and the implicit viscosity's coefficients. They read
// the positions and the velocities that the force pass would read: the velocities left
// by the divergence solve, whose loop always ends with this pass after its last update
// (it runs at least once, SPH/main.py:1695). Results are the force pass's, term for term
// and in neighbour order. Only the body predicted to be the scene's last (np_body: the
// last body of its previous step) runs this instance; when the prediction holds,
// k_solver_check marks the terms fresh and the force pass skips the scene. The step
// uses it when no scene needs the force pass's other terms (explicit viscosity, quirk
// mode); the solids' outputs come from k_clear_acc.
// `sel` = 1 in such a loop: the plain instance skips, and the NP instance takes, the
// scenes whose np_body this body is; 0: every scene.
template <int U, bool NP>
__device__ __forceinline__ void density_change_body(Dev d, int mode, int sel) {
  const int n = d.d_n[0];
  FOR_SLOTS_WARP(i, valid, n) {
    uint32_t fl = valid ? d.w.flags[i] : 0u;
    const int scn = slot_scene(fl);
    const SceneDyn& y = d.dyn[scn];
    const bool np_here = sel && y.it_v == y.np_body;
    bool work = valid && cls_fluid(fl) && y.act_v && (NP ? (np_here || !sel) : !np_here);
    double err = 0.0;
    if (work) {
      const SceneDev& s = d.sc[scn];
      const real3 xi = f3(d.w.pos[i]);
      const real3 vi = f3(d.w.vel[i]);
      const int c = d.nbr_cnt[i];
      real dd = 0.f;
      if constexpr (!NP) {
        nb_batches<U>(d.nbr + i, d.cap, c, i, [&](int j) { return GPV{pos_of(d, j), ldg(&d.w.vel[j])}; },
                   [&](int, const GPV& g) {
                     const real3 r = xi - f3(g.p);
                     dd += fabs(g.p.w) * dot3(vi - f3(g.v), kgrad_r2(r, dot3(r, r), s));
                   });
      } else {
        const bool st_on = (s.flags & NN_F_SURFACE_TENSION) != 0;
        const bool sr_on = (s.flags & NN_F_NONNEWTON) != 0;
        const real mi = d.w.mass[i];
        real3 st = make_real3(0.f, 0.f, 0.f);
        real S[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // strain-rate sum: 00 11 22 01 02 12
        nb_batches<U>(d.nbr + i, d.cap, c, i, [&](int j) { return GPV{pos_of(d, j), ldg(&d.w.vel[j])}; },
                   [&](int, const GPV& g) {
                     const real3 r = xi - f3(g.p);
                     const real r2 = dot3(r, r);
                     real w;
                     real3 gw;
                     kwg_r2(r, r2, s, w, gw);
                     dd += fabs(g.p.w) * dot3(vi - f3(g.v), gw);
                     const real mj = g.v.w;
                     if (st_on && w_fluid(g.p.w)) st -= (r * (s.sigma / mi * mj)) * (r2 > s.dia2 ? w : s.w_dia);
                     if (sr_on) {
                       const real3 vji = f3(g.v) - vi;
                       const real t[6] = {(vji.x * gw.x + vji.x * gw.x) * mj, (vji.y * gw.y + vji.y * gw.y) * mj,
                                           (vji.z * gw.z + vji.z * gw.z) * mj, (vji.x * gw.y + vji.y * gw.x) * mj,
                                           (vji.x * gw.z + vji.z * gw.x) * mj, (vji.y * gw.z + vji.z * gw.y) * mj};
#pragma unroll
                       for (int k = 0; k < 6; ++k) S[k] += t[k];
                     }
                   });
        real4 a = make_real4(s.g[0], s.g[1], s.g[2], 0.f);
        if (st_on) { a.x += st.x; a.y += st.y; a.z += st.z; }
        d.acc4[i] = a;
        const real rho_i = d.w.dens[i];
        real mu = s.mu_newton;
        if (sr_on) {
          const real g = strain_rate_norm(S, rho_i, false);
          mu = nn_law(g, s);
          d.srn[i] = g;
          d.mu[i] = mu;
        }
        if (scene_implicit(s)) d.cg_aux[i] = make_real2(mu, mi / rho_i);
      }
      dd = fmax(dd, real(0));
      if (c < 20) dd = 0.f;
      d.rho_adv[i] = dd;
      real a = d.alpha[i];
      if (mode == 0) {
        a = a * d.dyn[scn].inv_dt;
        d.alpha[i] = a;
      }
      d.kappa[i] = dd * a;
      err = (double)(s.rho0 * dd - 0.f);
    }
    // one reduction per warp and slot group: per-lane partial sums kept across the
    // loop (as in k_density_adv) measured 18 % slower here
    if (mode == 1) scene_add(d.acc, ACC_ERR, 0, scn, work, err);
  }
}
template <int U>
__global__ void NN_PASS_REGS k_density_change(Dev d, int mode, int sel) { density_change_body<U, false>(d, mode, sel); }
// The NP instance is capped at 64 registers: uncapped it takes 79 (6 blocks of 128 per
// SM) and ran 0.455 ms on the 2.4M scene, capped 0.428 ms (44 bytes spilled).
template <int U>
__global__ void NN_REGS64 k_density_change_np(Dev d, int mode, int sel) { density_change_body<U, true>(d, mode, sel); }

// divergence_solver_iteration_kernel (SPH/main.py:1721-1760). The pushes onto
// dynamic solids (1755-1760) are omitted: clear_accelerations (1552) discards them.
struct GPK { real4 p; real k; };
template <int U>
__global__ void NN_PASS_REGS k_divergence_update(Dev d) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const uint32_t fl = d.w.flags[i];
    if (!cls_fluid(fl)) continue;
    const int scn = slot_scene(fl);
    if (!d.dyn[scn].act_v) continue;
    const SceneDev& s = d.sc[scn];
    const real dt = d.dyn[scn].dt;
    const real3 xi = f3(d.w.pos[i]);
    const real k_i = d.kappa[i];
    real3 dv = make_real3(0.f, 0.f, 0.f);
    nb_batches<U>(d.nbr + i, d.cap, d.nbr_cnt[i], i, [&](int j) { return GPK{pos_of(d, j), ldg(&d.kappa[j])}; },
               [&](int, const GPK& g) {
                 const real3 r = xi - f3(g.p);
                 if (w_fluid(g.p.w)) {
                   const real k_sum = k_i + g.k;
                   if (fabs(k_sum) > s.eps) dv -= kgrad_r2(r, dot3(r, r), s) * (-g.p.w) * (dt * k_sum);
                 } else if (fabs(k_i) > s.eps) {
                   dv += kgrad_r2(r, dot3(r, r), s) * g.p.w * ((-dt * 1.f) * k_i);
                 }
               });
    real4 v = d.w.vel[i];
    v.x += dv.x; v.y += dv.y; v.z += dv.z;
    d.w.vel[i] = v;
  }
}

// multiply_time_step (SPH/main.py:1677-1681): alpha *= dt after the divergence loop.
__global__ void k_alpha_times_dt(Dev d) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const uint32_t fl = d.w.flags[i];
    if (!cls_fluid(fl)) continue;
    const int scn = slot_scene(fl);
    if (!d.dyn[scn].div_ran) continue;
    d.alpha[i] = d.alpha[i] * d.dyn[scn].dt;
  }
}

// compute_density_adv (SPH/main.py:1647-1667). mode 0: first call of pressure_solve,
// also alpha *= 1/dt^2 (1771); mode 1: iteration, FP64 error (1793-1797).
// This pass and k_pressure_update, the pressure loop, read their lists evict-first
// (nb_batches<U, true>) and the list build writes them streaming: -2 % here and
// -10 % in k_pressure_update, the step 3.475 -> 3.435 ms on the 2.4M scene (the other
// passes measured flat or slower with it).
template <int U>
__global__ void NN_PASS_REGS k_density_adv(Dev d, int mode) {
  const int n = d.d_n[0];
  LaneSums<1> sums;
  const int q[1] = {ACC_ERR};
  FOR_SLOTS_WARP(i, valid, n) {
    uint32_t fl = valid ? d.w.flags[i] : 0u;
    const int scn = slot_scene(fl);
    bool work = valid && cls_fluid(fl) && d.dyn[scn].act_p;
    double err = 0.0;
    if (work) {
      const SceneDev& s = d.sc[scn];
      const real dt = d.dyn[scn].dt;
      const real3 xi = f3(d.w.pos[i]);
      const real3 vi = f3(d.w.vel[i]);
      real delta = 0.f;
      nb_batches<U, true>(d.nbr + i, d.cap, d.nbr_cnt[i], i,
                 [&](int j) { return GPV{pos_of(d, j), ldg(&d.w.vel[j])}; },
                 [&](int, const GPV& g) {
                   const real3 r = xi - f3(g.p);
                   delta += fabs(g.p.w) * dot3(vi - f3(g.v), kgrad_r2(r, dot3(r, r), s));
                 });
      real da = d.w.dens[i] * s.inv_rho0 + dt * delta;
      da = fmax(da, real(1));
      d.rho_adv[i] = da;
      real a = d.alpha[i];
      if (mode != 1) {
        // mode 2 also applies the divergence solve's closing alpha *= dt (1713)
        if (mode == 2 && d.dyn[scn].div_ran) a = a * d.dyn[scn].dt;
        a = a * d.dyn[scn].inv_dt2;
        d.alpha[i] = a;
      }
      d.kappa[i] = (da - 1.f) * a;
      err = (double)(s.rho0 * da - s.rho0);
    }
    if (mode == 1) sums.add(d.acc, q, work, scn, {err});
  }
  if (mode == 1) sums.flush(d.acc, q);
}

// pressure_solve_iteration_kernel (SPH/main.py:1799-1841). Fluid slots update v in
// place per neighbour; dynamic solid slots gather the two-way coupling acceleration
// from their fluid neighbours (the reference scatters it with atomics, 1835-1841).
template <int U>
__global__ void NN_PASS_REGS k_pressure_update(Dev d) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const uint32_t fl = d.w.flags[i];
    const bool fluid = cls_fluid(fl);
    if (!fluid && !cls_dyn_solid(fl)) continue;
    const int scn = slot_scene(fl);
    if (!d.dyn[scn].act_p) continue;
    const SceneDev& s = d.sc[scn];
    const real dt = d.dyn[scn].dt;
    const real4 pi = d.w.pos[i];
    const real3 xi = f3(pi);
    auto load = [&](int j) { return GPK{pos_of(d, j), ldg(&d.kappa[j])}; };
    if (fluid) {
      const real k_i = d.kappa[i];
      real4 v4 = d.w.vel[i];
      real3 vi = f3(v4);
      nb_batches<U, true>(d.nbr + i, d.cap, d.nbr_cnt[i], i, load, [&](int, const GPK& g) {
        const real3 r = xi - f3(g.p);
        if (w_fluid(g.p.w)) {
          const real k_sum = k_i + g.k;
          if (fabs(k_sum) > s.eps) vi -= kgrad_r2(r, dot3(r, r), s) * (-g.p.w) * (dt * k_sum);
        } else if (fabs(k_i) > s.eps) {
          vi += kgrad_r2(r, dot3(r, r), s) * g.p.w * ((-dt * 1.f) * k_i);
        }
      });
      d.w.vel[i] = make_real4(vi.x, vi.y, vi.z, v4.w);
    } else {
      const real Vi = fabs(pi.w);
      const real inv_dt = 1.f / dt;
      real3 ai = make_real3(0.f, 0.f, 0.f);
      nb_batches<U, true>(d.nbr + i, d.cap, d.nbr_cnt[i], i, load, [&](int, const GPK& g) {
        if (!w_fluid(g.p.w) || !(fabs(g.k) > s.eps)) return;
        const real3 r = f3(g.p) - xi;  // x_fluid - x_solid, as the fluid computes it
        const real3 vc = kgrad_r2(r, dot3(r, r), s) * (-Vi) * ((-dt * 1.f) * g.k);
        ai -= vc * inv_dt;
      });
      real4 a = d.acc4[i];
      a.x += ai.x; a.y += ai.y; a.z += ai.z;
      d.acc4[i] = a;
    }
  }
}

// Loop control after each solver iteration: per-scene average error against eta,
// the reference's iteration counting (SPH/main.py:1695-1703, 1778-1784), and the
// CUDA graph while-condition (any scene still iterating).
// `fold`: the divergence loop runs the non-pressure terms in body np_body (k_density_change
// NP); when a scene stops, its terms are fresh if that body was its last.
__global__ void k_solver_check(Dev d, int which /*0 div, 1 pressure*/, int fold) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  const int ns = d.d_n[1];
  for (int sc = threadIdx.x; sc < ns; sc += blockDim.x) {
    SceneDyn& y = d.dyn[sc];
    const SceneDev& s = d.sc[sc];
    int* act = which == 0 ? &y.act_v : &y.act_p;
    if (!*act) continue;
    double err = acc_sum(d.acc, sc, ACC_ERR);
    acc_zero(d.acc, sc, ACC_ERR);
    double avg = err / (double)s.n_fluid;
    double eta = which == 0 ? (1.0 / (double)y.dt) * s.eta_v_fac : s.eta_p;
    int* it = which == 0 ? &y.it_v : &y.it_p;
    const int body = *it;  // 0-based index of the body that just ran
    int mx = which == 0 ? s.max_iter_v : s.max_iter;
    if (which == 0) y.avg_v = avg; else y.avg_p = avg;
    if (avg <= eta) {
      *act = 0;
    } else {
      *it += 1;
      if (*it >= max(mx, 1)) *act = 0;
    }
    if (!(avg == avg)) { set_status(&y, NN_ERR_NAN); *act = 0; }
    if (which == 0 && !*act) {
      y.np_last = body;
      y.np_fresh = fold && body == y.np_body;
    }
    if (*act) any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *d.any_active = any;
    atomicAdd(&d.body_count[which], 1);
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 900)
    if (d.loop_handle) cudaGraphSetConditional((cudaGraphConditionalHandle)d.loop_handle, any ? 1u : 0u);
#endif
  }
}

// Per-scene loop start: which scenes iterate, counters reset.
__device__ __forceinline__ void solver_begin_scene(SceneDyn& y, const SceneDev& s, int which) {
  int on = s.n_fluid > 0;
  if (which == 0) {
    on = on && (s.flags & NN_F_DIVERGENCE);
    y.act_v = on; y.it_v = 0; y.div_ran = on;
    y.np_body = min(max(y.np_last, 0), max(s.max_iter_v, 1) - 1);  // as many bodies as last step
  }
  else if (which == 1) { y.act_p = on; y.it_p = 0; }
  else { y.it_cg = 0; }
}
__global__ void k_solver_begin(Dev d, int which /*0 div, 1 pressure, 2 cg*/) {
  const int ns = d.d_n[1];
  for (int sc = threadIdx.x; sc < ns; sc += blockDim.x) solver_begin_scene(d.dyn[sc], d.sc[sc], which);
}

__global__ void k_step_reset(Dev d) { step_reset_scenes(d); }

// Time step of the step: the CFL step from max |v| of the gather (extension; the
// reference keeps dt fixed), and the f32 constants the reference passes to its
// kernels (1/dt and 1/dt^2 computed in f64 from the f32 dt field, SPH/main.py:1687,1764).
__device__ __forceinline__ void step_dt_scenes(const Dev& d, int do_cfl) {
  const int ns = d.d_n[1];
  for (int sc = threadIdx.x; sc < ns; sc += blockDim.x) {
    SceneDyn& y = d.dyn[sc];
    const SceneDev& s = d.sc[sc];
    if (do_cfl && (s.flags & NN_F_CFL)) {
      const real vm = __uint_as_float(y.vmax_bits);
      double dtn = s.cfl_max_dt;
      if (vm > 1e-9f) dtn = (double)s.cfl_factor * 0.4 * (double)s.diameter / (double)vm;
      dtn = fmin(fmax(dtn, (double)s.cfl_min_dt), (double)s.cfl_max_dt);
      y.dt = (real)dtn;
    }
    y.inv_dt = (real)(1.0 / (double)y.dt);
    y.inv_dt2 = (real)(1.0 / ((double)y.dt * (double)y.dt));
    y.vmax_bits = 0u;
  }
}
__global__ void k_step_dt(Dev d, int do_cfl) { step_dt_scenes(d, do_cfl); }

// non_pressure_advect (SPH/main.py:1843-1848) as a pass of its own.
__global__ void k_np_advect(Dev d) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const uint32_t fl = d.w.flags[i];
    if (!cls_fluid(fl) || !(fl & NN_CLS_DYNAMIC)) continue;
    const real dt = d.dyn[slot_scene(fl)].dt;
    const real4 a = d.acc4[i];
    real4 v = d.w.vel[i];
    v.x += dt * a.x; v.y += dt * a.y; v.z += dt * a.z;
    d.w.vel[i] = v;
  }
}

__global__ void k_force_active(Dev d) {
  const int ns = d.d_n[1];
  for (int sc = threadIdx.x; sc < ns; sc += blockDim.x) {
    SceneDyn& y = d.dyn[sc];
    const bool on = d.sc[sc].n_fluid > 0;
    y.act_v = y.act_p = on;
    y.act_cg = on && scene_implicit(d.sc[sc]);
    y.np_fresh = 0;
  }
}

// Scene index of every particle id, from the scene table (block b walks scenes b, b+grid, ...).
__global__ void k_scene_of_id(Dev d) {
  const int ns = d.d_n[1];
  int32_t* so = const_cast<int32_t*>(d.scene_of_id);
  for (int sc = blockIdx.x; sc < ns; sc += gridDim.x) {
    const int b = d.sc[sc].start, n = d.sc[sc].n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) so[b + i] = sc;
  }
}

__global__ void k_set_int(int32_t* p, int32_t v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *const_cast<int32_t*>(p) = v;
}

__global__ void k_step_end(Dev d) {
  const int ns = d.d_n[1];
  for (int sc = threadIdx.x; sc < ns; sc += blockDim.x) {
    d.dyn[sc].steps += 1;
    if (d.sc[sc].n_fluid > 0) d.dyn[sc].max_avg_p = fmax(d.dyn[sc].max_avg_p, d.dyn[sc].avg_p);
    d.dyn[sc].anim[0] = d.dyn[sc].anim[1] = d.dyn[sc].anim[2] = 0.f;  // one step only
  }
}

// ---------------------------------------------------------------------------
// NonNewton viscosity laws (SPH/main.py:404-459); quirk mode keeps the Newtonian
// branch that the reference's int-vs-Enum dispatch always takes (387-402).
__device__ __forceinline__ real nn_law(real g, const SceneDev& s) {
  const int method = (s.flags & NN_F_QUIRKS) ? NN_NEWTONIAN : s.nn_method;
  switch (method) {
    case NN_POWER_LAW: return s.nn_K * pow(g, s.nn_n - 1.f);
    case NN_CROSS: return s.nn_muinf + (s.nn_mu0 - s.nn_muinf) / (1.f + pow(s.nn_K * g, s.nn_n));
    case NN_CASSON: { real q = sqrt(s.nn_muc) + sqrt(s.nn_tauy / g); return q * q; }
    case NN_CARREAU:
      if (s.flags & NN_F_CARREAU_TEXTBOOK)
        return s.nn_muinf + (s.nn_mu0 - s.nn_muinf) * pow(1.f + (s.nn_K * g) * (s.nn_K * g), (s.nn_n - 1.f) / 2.f);
      return s.nn_muinf + (s.nn_mu0 - s.nn_muinf) / (1.f + pow(s.nn_K * g * g, (1.f - s.nn_n) / 2.f));
    case NN_BINGHAM:
      if (g < s.nn_gc) return s.nn_mu0;
      return s.nn_gc * (s.nn_mu0 - s.nn_muinf) / g + s.nn_muinf;
    case NN_HERSCHEL_BULKLEY:
      if (g < s.nn_gc) return s.nn_mu0;
      return (s.nn_mu0 * s.nn_gc - s.nn_K * pow(s.nn_gc, s.nn_n)) / g + s.nn_K * pow(g, s.nn_n - 1.f);
    default: return s.nn_mu0;
  }
}



// calcStrainRate's norm (SPH/main.py:461-492) of the strain-rate sum S (00 11 22 01 02
// 12): sqrt(D:D) with D = S / (2 rho_i); in quirk mode the norm of S itself, since the
// reference takes the norm before the 0.5 / rho scaling (491-492).
__device__ __forceinline__ real strain_rate_norm(const real (&S)[6], real rho_i, bool quirks) {
  real nrm2;
  if (quirks) {
    nrm2 = S[0] * S[0] + S[1] * S[1] + S[2] * S[2] + 2.f * (S[3] * S[3] + S[4] * S[4] + S[5] * S[5]);
  } else {
    const real sc = 0.5f / rho_i;
    real D[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) D[k] = S[k] * sc;
    nrm2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2] + 2.f * (D[3] * D[3] + D[4] * D[4] + D[5] * D[5]);
  }
  return sqrt(nrm2);
}

// compute_non_pressure_forces (SPH/main.py:1557-1567) in one neighbour pass:
// [clear_accelerations (1552)] + SurfaceTension (1387-1414) + NonNewton strain rate
// and law (461-492, 404-459) + ViscosityModel (1426-1468), and the per-particle
// coefficients (mu_i, m_i / rho_i) of the implicit viscosity. Dynamic solids gather
// the boundary-viscosity reaction from their fluid neighbours (the reference scatters
// it, 1459-1460). The velocity update of non_pressure_advect cannot join this pass:
// the viscosity reads the neighbours' velocities.
struct GF { real4 p, v; real rho; int id; };  // v.w = mass
// Terms compiled into an instance of the force pass (the host picks the instance
// that covers every scene of the batch; the scene flags still gate each term).
#define FF_ST 1  // surface tension
#define FF_VI 2  // explicit viscosity (fluid and boundary) and its reaction on dynamic solids
#define FF_SR 4  // strain rate and viscosity law
#define FF_Q 8   // reference quirk mode
template <int U, int FF>
__device__ __forceinline__ void forces_body(Dev d, int clear) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const uint32_t fl = d.w.flags[i];
    const bool fluid = cls_fluid(fl);
    const int scn = slot_scene(fl);
    const SceneDev& s = d.sc[scn];
    if (s.n_fluid == 0) continue;  // the reference runs the substep only with fluid
    if (d.dyn[scn].np_fresh) continue;  // computed by the divergence loop's last density change
    const bool implicit = scene_implicit(s);
    const bool quirks = (FF & FF_Q) && (s.flags & NN_F_QUIRKS);
    const bool st_on = (FF & FF_ST) && fluid && (s.flags & NN_F_SURFACE_TENSION);
    const bool vi_on = (FF & FF_VI) && fluid && !implicit && (s.flags & NN_F_VISCOSITY);
    const bool vb_on =
        (FF & FF_VI) && cls_dyn_solid(fl) && !implicit && (s.flags & NN_F_VISCOSITY) && s.visc_b != 0.f;
    const bool nn_on = (FF & FF_SR) && (s.flags & NN_F_NONNEWTON);
    const bool sr_on = nn_on && (fluid || quirks);
    const real4 pi = d.w.pos[i];
    const real3 xi = f3(pi);
    const real3 vi = f3(d.w.vel[i]);
    real4 a;
    if (clear) a = cls_static_solid(fl) ? make_real4(0.f, 0.f, 0.f, 0.f) : make_real4(s.g[0], s.g[1], s.g[2], 0.f);
    else a = d.acc4[i];
    real3 st = make_real3(0.f, 0.f, 0.f), vs = make_real3(0.f, 0.f, 0.f), rf = make_real3(0.f, 0.f, 0.f);
    real S[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // strain-rate sum: 00 11 22 01 02 12
    int last_id = -1;                             // quirk: the last neighbour in id order survives
    if (st_on || vi_on || vb_on || sr_on) {
      const real mi = d.w.mass[i];
      const real rho_i = d.w.dens[i];
      const real Vi = fabs(pi.w);
      const bool need_rho = vi_on || vb_on;  // density and id only where a term reads them
      nb_batches<U>(d.nbr + i, d.cap, d.nbr_cnt[i], i,
                    [&](int j) {
                      return GF{pos_of(d, j), ldg(&d.w.vel[j]), need_rho ? ldg(&d.w.dens[j]) : 1.f,
                                quirks ? ldg(&d.w.id[j]) : 0};
                    },
                    [&](int, const GF& g) {
                      const real3 r = xi - f3(g.p);
                      const real r2 = dot3(r, r);
                      real w;
                      real3 gw;
                      kwg_r2(r, r2, s, w, gw);
                      const bool jf = w_fluid(g.p.w);
                      const real mj = g.v.w;
                      if (jf && st_on) st -= (r * (s.sigma / mi * mj)) * (r2 > s.dia2 ? w : s.w_dia);
                      if (vi_on) {
                        const real v_xy = dot3(vi - f3(g.v), r);
                        if (jf) vs += gw * (10.f * s.visc * (mj / g.rho) * v_xy / (r2 + s.c01h2));
                        else if (s.visc_b != 0.f)
                          vs += gw * (10.f * s.visc_b * (s.rho0 * fabs(g.p.w) / rho_i) * v_xy / (r2 + s.c01h2));
                      }
                      if (vb_on && jf) {  // reaction on a dynamic solid: the fluid's term with i <-> j
                        const real3 rr = -r;
                        const real v_xy = dot3(f3(g.v) - vi, rr);
                        rf += (-gw) * (10.f * s.visc_b * (s.rho0 * Vi / g.rho) * v_xy / (r2 + s.c01h2));
                      }
                      if (sr_on) {
                        const real3 vji = f3(g.v) - vi;
                        const real t[6] = {(vji.x * gw.x + vji.x * gw.x) * mj, (vji.y * gw.y + vji.y * gw.y) * mj,
                                            (vji.z * gw.z + vji.z * gw.z) * mj, (vji.x * gw.y + vji.y * gw.x) * mj,
                                            (vji.x * gw.z + vji.z * gw.x) * mj, (vji.y * gw.z + vji.z * gw.y) * mj};
                        const bool take = g.id > last_id;
                        if (quirks && take) last_id = g.id;
#pragma unroll
                        for (int k = 0; k < 6; ++k) S[k] = quirks ? (take ? t[k] : S[k]) : S[k] + t[k];
                      }
                    });
    }
    if (st_on) { a.x += st.x; a.y += st.y; a.z += st.z; }
    if (vi_on) { a.x += vs.x; a.y += vs.y; a.z += vs.z; }
    if (vb_on) { a.x -= rf.x; a.y -= rf.y; a.z -= rf.z; }
    d.acc4[i] = a;
    real mu = s.mu_newton;
    if (nn_on) {
      real g = 0.f;
      if (sr_on) {
        g = strain_rate_norm(S, d.w.dens[i], quirks);
        mu = nn_law(g, s);
      } else {
        mu = 0.f;
      }
      d.srn[i] = g;
      d.mu[i] = mu;
    }
    // CG coefficients: (mu, m / rho) of a fluid slot; (0, 1) marks a dynamic solid
    if (implicit)
      d.cg_aux[i] = fluid ? make_real2(mu, d.w.mass[i] / d.w.dens[i])
                          : make_real2(0.f, cls_dyn_solid(fl) ? 1.f : 0.f);
  }
}

// Register budget per instance: without the explicit viscosity, 64 registers (a few
// spilled bytes) give 8 blocks of 128 per SM instead of 6, and the gathers hide better:
// 0.457 -> 0.404 ms on the 2.4M scene, -21 % on the shear-thinning drop. With it, the
// spills cost more than the occupancy gains (+8 % on the dam break), so that instance
// keeps the compiler's own budget (forces_kernel_of picks the wrapper).
template <int U, int FF>
__global__ void k_forces(Dev d, int clear) { forces_body<U, FF>(d, clear); }
template <int U, int FF>
__global__ void NN_REGS64 k_forces_r64(Dev d, int clear) { forces_body<U, FF>(d, clear); }
template <int U, int FF>
constexpr void (*forces_kernel_of())(Dev, int) {
  if constexpr ((FF & FF_VI) != 0) return &k_forces<U, FF>;
  else return &k_forces_r64<U, FF>;
}

// ---------------------------------------------------------------------------
// Implicit viscosity (Weiler, Koschier, Brand, Bender 2018), matrix-free PCG on the
// mass-weighted SPD system (the reference stubs it, SPH/main.py:1471-1513):
//   m_i x_i - sum_fluid c_ij K_ij (x_i - x_j) - sum_solid c_ib K_ib (x_i - v_b) = m_i v_i
//   c_ij = dt * 10 * (mu_i + mu_j)/2 * (m_i/rho_i) (m_j/rho_j),  c_ib = dt*10*mu_b*m_i*rho0*V_b/rho_i^2
//   K_ij = gradW_ij x_ij^T / (|x_ij|^2 + 0.01 h^2)
// FP32 vectors, FP64 dot products, 3x3 block-Jacobi preconditioner.


__device__ __forceinline__ bool cg_row(const Dev& d, int i, uint32_t fl) {
  if (!cls_fluid(fl)) return false;
  return scene_implicit(d.sc[slot_scene(fl)]);
}

// A p for one row; in the setup also the diagonal block D and the right-hand-side
// correction of moving boundaries (SETUP: `vec` is the velocity field).
// The setup gathers a neighbour's pos, v and coefficients (mu_j, m_j / rho_j). It leaves
// mu_i in p.w and writes cg_pos = (x_i, m_i / rho_i) for fluid and pos = (x_i, -V_i) for
// solids, so the matvec reads the same operands in two float4 gathers (32 B per pair)
// instead of three loads (40 B): the matvec 0.302 -> 0.265 ms on the 2.4M scene.
struct GCG { real4 p, x; real2 a; };
template <int U, bool SETUP>
__device__ __forceinline__ real3 cg_apply(const Dev& d, int i, const real4* __restrict__ vec, real3 vi,
                                           const SceneDev& s, real dt, real* D, real3* bcorr) {
  const real3 xi = f3(d.w.pos[i]);
  const real2 ai = d.cg_aux[i];
  const real mi = d.w.mass[i];
  const real rho_i = d.w.dens[i];
  real3 acc = vi * mi;
  const real cdt = dt * 10.f;
  const real cb = cdt * s.mu_b * mi * s.rho0 / (rho_i * rho_i);
  nb_batches<U>(d.nbr + i, d.cap, d.nbr_cnt[i], i,
             [&](int j) {
               GCG g;
               if (SETUP) {
                 g.p = pos_of(d, j);
                 g.x = ldg(&vec[j]);
                 g.a = ldg(&d.cg_aux[j]);
               } else {
                 g.p = ldg(&d.cg_pos[j]);
                 g.x = ldg(&vec[j]);
                 g.a = make_real2(g.x.w, g.p.w);  // fluid j: (mu_j, m_j / rho_j)
               }
               return g;
             },
             [&](int, const GCG& g) {
               const real3 r = xi - f3(g.p);
               const real r2 = dot3(r, r);
               const real3 gw = kgrad_r2(r, r2, s);
               const real w = fast_div(1.f, r2 + s.c01h2);
               real c;
               real3 diff;
               if (w_fluid(g.p.w)) {
                 c = cdt * 0.5f * (ai.x + g.a.x) * ai.y * g.a.y;
                 diff = vi - f3(g.x);
               } else {
                 c = cb * fabs(g.p.w);
                 diff = vi;
                 if (SETUP && g.a.y > 0.f) *bcorr -= gw * (c * dot3(r, f3(g.x)) * w);  // dynamic solid
               }
               acc -= gw * (c * dot3(r, diff) * w);
               if (SETUP) {
                 const real cw = c * w;
                 D[0] -= cw * gw.x * r.x; D[1] -= cw * gw.y * r.y; D[2] -= cw * gw.z * r.z;
                 D[3] -= cw * gw.x * r.y; D[4] -= cw * gw.x * r.z; D[5] -= cw * gw.y * r.z;
               }
             });
  return acc;
}

__device__ __forceinline__ real3 sym_apply(const real* P, real3 v) {  // P: 00 11 22 01 02 12
  return make_real3(P[0] * v.x + P[3] * v.y + P[4] * v.z, P[3] * v.x + P[1] * v.y + P[5] * v.z,
                     P[4] * v.x + P[5] * v.y + P[2] * v.z);
}

// 64 registers (from 72): 8 blocks of 128 per SM instead of 7
template <int U>
__global__ void NN_REGS64 k_cg_setup(Dev d) {
  const int n = d.d_n[0];
  FOR_SLOTS_WARP(i, valid, n) {
    const uint32_t fl = valid ? d.w.flags[i] : 0u;
    const int scn = slot_scene(fl);
    const bool work = valid && cg_row(d, i, fl);
    double rr = 0, bb = 0, rz = 0;
    // a solid neighbour's matvec operands: its pos (x, -V); its p is not read
    if (valid && cls_solid(fl) && scene_implicit(d.sc[scn])) d.cg_pos[i] = d.w.pos[i];
    if (work) {
      const SceneDev& s = d.sc[scn];
      const real dt = d.dyn[scn].dt;
      const real mi = d.w.mass[i];
      const real3 vi = f3(d.w.vel[i]);
      real D[6] = {mi, mi, mi, 0.f, 0.f, 0.f};
      real3 bc = make_real3(0.f, 0.f, 0.f);
      const real3 Av = cg_apply<U, true>(d, i, d.w.vel, vi, s, dt, D, &bc);
      const real3 b = vi * mi + bc;
      // symmetric 3x3 inverse in double
      double a00 = D[0], a11 = D[1], a22 = D[2], a01 = D[3], a02 = D[4], a12 = D[5];
      double c00 = a11 * a22 - a12 * a12, c01 = a02 * a12 - a01 * a22, c02 = a01 * a12 - a02 * a11;
      double det = a00 * c00 + a01 * c01 + a02 * c02;
      double id = 1.0 / det;
      real P[6] = {(real)(c00 * id), (real)((a00 * a22 - a02 * a02) * id), (real)((a00 * a11 - a01 * a01) * id),
                    (real)(c01 * id), (real)(c02 * id), (real)((a01 * a02 - a00 * a12) * id)};
#pragma unroll
      for (int k = 0; k < 6; ++k) d.cg_pinv[(size_t)k * d.cap + i] = P[k];
      const real3 r = b - Av;
      const real3 z = sym_apply(P, r);
      d.cg_x[i] = make_real4(vi.x, vi.y, vi.z, 0.f);
      d.cg_r[i] = make_real4(r.x, r.y, r.z, 0.f);
      d.cg_z[i] = make_real4(z.x, z.y, z.z, 0.f);
      const real2 ai = d.cg_aux[i];
      const real3 xi = f3(d.w.pos[i]);
      d.cg_pos[i] = make_real4(xi.x, xi.y, xi.z, ai.y);
      d.cg_p[i] = make_real4(z.x, z.y, z.z, ai.x);
      rr = (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z;
      bb = (double)b.x * b.x + (double)b.y * b.y + (double)b.z * b.z;
      rz = (double)r.x * z.x + (double)r.y * z.y + (double)r.z * z.z;
    }
    // per iteration: partial sums kept across iterations spill under the 64-register cap
    scene_add(d.acc, ACC_RR, 0, scn, work, rr);
    scene_add(d.acc, ACC_BB, 0, scn, work, bb);
    scene_add(d.acc, ACC_RZ, 0, scn, work, rz);
  }
}

// After setup: relative residual of the initial guess decides whether to iterate.
__global__ void k_cg_check0(Dev d) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  const int ns = d.d_n[1];
  for (int sc = threadIdx.x; sc < ns; sc += blockDim.x) {
    SceneDyn& y = d.dyn[sc];
    const SceneDev& s = d.sc[sc];
    const bool on = s.n_fluid > 0 && scene_implicit(s);
    double rr = acc_sum(d.acc, sc, ACC_RR), bb = acc_sum(d.acc, sc, ACC_BB), rz = acc_sum(d.acc, sc, ACC_RZ);
    acc_zero(d.acc, sc, ACC_RR); acc_zero(d.acc, sc, ACC_BB); acc_zero(d.acc, sc, ACC_RZ);
    y.it_cg = 0;
    y.cg_bnorm2 = bb;
    y.cg_rz = rz;
    y.cg_rel = bb > 0 ? sqrt(rr / bb) : 0.0;
    y.act_cg = on && (y.cg_rel > s.visco_tol) && s.visco_max_iter > 0;
    if (y.act_cg) any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *d.any_active = any;
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 900)
    if (d.loop_handle) cudaGraphSetConditional((cudaGraphConditionalHandle)d.loop_handle, any ? 1u : 0u);
#endif
  }
}

template <int U>
__global__ void k_cg_matvec(Dev d) {
  const int n = d.d_n[0];
  LaneSums<1> sums;
  const int q[1] = {ACC_PAP};
  FOR_SLOTS_WARP(i, valid, n) {
    const uint32_t fl = valid ? d.w.flags[i] : 0u;
    const int scn = slot_scene(fl);
    const bool work = valid && cg_row(d, i, fl) && d.dyn[scn].act_cg;
    double pap = 0;
    if (work) {
      const SceneDev& s = d.sc[scn];
      const real3 p = f3(d.cg_p[i]);
      const real3 Ap = cg_apply<U, false>(d, i, d.cg_p, p, s, d.dyn[scn].dt, nullptr, nullptr);
      d.cg_Ap[i] = make_real4(Ap.x, Ap.y, Ap.z, 0.f);
      pap = (double)p.x * Ap.x + (double)p.y * Ap.y + (double)p.z * Ap.z;
    }
    sums.add(d.acc, q, work, scn, {pap});
  }
  sums.flush(d.acc, q);
}

__global__ void k_cg_update(Dev d) {
  const int n = d.d_n[0];
  LaneSums<2> sums;
  const int q[2] = {ACC_RR, ACC_RZ};
  FOR_SLOTS_WARP(i, valid, n) {
    const uint32_t fl = valid ? d.w.flags[i] : 0u;
    const int scn = slot_scene(fl);
    const bool work = valid && cg_row(d, i, fl) && d.dyn[scn].act_cg;
    double rr = 0, rz = 0;
    if (work) {
      const real al = (real)d.dyn[scn].cg_alpha;
      real3 x = f3(d.cg_x[i]), r = f3(d.cg_r[i]);
      const real3 p = f3(d.cg_p[i]), Ap = f3(d.cg_Ap[i]);
      x += p * al;
      r -= Ap * al;
      real P[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) P[k] = d.cg_pinv[(size_t)k * d.cap + i];
      const real3 z = sym_apply(P, r);
      d.cg_x[i] = make_real4(x.x, x.y, x.z, 0.f);
      d.cg_r[i] = make_real4(r.x, r.y, r.z, 0.f);
      d.cg_z[i] = make_real4(z.x, z.y, z.z, 0.f);
      rr = (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z;
      rz = (double)r.x * z.x + (double)r.y * z.y + (double)r.z * z.z;
    }
    sums.add(d.acc, q, work, scn, {rr, rz});
  }
  sums.flush(d.acc, q);
}

// PCG step length per scene: alpha = (r.z) / (p.Ap).
__global__ void k_cg_alpha(Dev d) {
  const int ns = d.d_n[1];
  for (int sc = threadIdx.x; sc < ns; sc += blockDim.x) {
    SceneDyn& y = d.dyn[sc];
    if (!y.act_cg) continue;
    const double pap = acc_sum(d.acc, sc, ACC_PAP);
    acc_zero(d.acc, sc, ACC_PAP);
    y.cg_alpha = pap != 0.0 ? y.cg_rz / pap : 0.0;
  }
}

// PCG convergence check per scene (relative residual, FP64) and beta.
__global__ void k_cg_check(Dev d) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  const int ns = d.d_n[1];
  for (int sc = threadIdx.x; sc < ns; sc += blockDim.x) {
    SceneDyn& y = d.dyn[sc];
    const SceneDev& s = d.sc[sc];
    if (!y.act_cg) continue;
    const double rr = acc_sum(d.acc, sc, ACC_RR), rz = acc_sum(d.acc, sc, ACC_RZ);
    acc_zero(d.acc, sc, ACC_RR);
    acc_zero(d.acc, sc, ACC_RZ);
    y.it_cg += 1;
    y.cg_rel = y.cg_bnorm2 > 0 ? sqrt(rr / y.cg_bnorm2) : 0.0;
    y.cg_beta = y.cg_rz != 0.0 ? rz / y.cg_rz : 0.0;
    y.cg_rz = rz;
    if (y.cg_rel <= s.visco_tol || y.it_cg >= s.visco_max_iter || !(y.cg_rel == y.cg_rel)) y.act_cg = 0;
    if (y.act_cg) any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *d.any_active = any;
    atomicAdd(&d.body_count[2], 1);
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 900)
    if (d.loop_handle) cudaGraphSetConditional((cudaGraphConditionalHandle)d.loop_handle, any ? 1u : 0u);
#endif
  }
}

__global__ void k_cg_pupdate(Dev d) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const uint32_t fl = d.w.flags[i];
    const int scn = slot_scene(fl);
    if (!cg_row(d, i, fl) || !d.dyn[scn].act_cg) continue;
    const real be = (real)d.dyn[scn].cg_beta;
    const real3 z = f3(d.cg_z[i]);
    const real4 p4 = d.cg_p[i];
    const real3 np = z + f3(p4) * be;
    d.cg_p[i] = make_real4(np.x, np.y, np.z, p4.w);  // w: mu_i
  }
}

// Implicit scenes: a_i += (x_i - v_i)/dt (the viscous acceleration of the CG
// solution); then, for every scene, non_pressure_advect (SPH/main.py:1843-1848).
// No neighbour reads, so the velocity update is safe here.
__global__ void k_cg_finish(Dev d, int advect) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const uint32_t fl = d.w.flags[i];
    if (!cls_fluid(fl)) continue;
    const int scn = slot_scene(fl);
    const SceneDev& s = d.sc[scn];
    if (s.n_fluid == 0) continue;
    const real dt = d.dyn[scn].dt;
    real4 a = d.acc4[i];
    const real4 v4 = d.w.vel[i];
    if (scene_implicit(s)) {
      const real inv_dt = d.dyn[scn].inv_dt;
      const real3 x = f3(d.cg_x[i]);
      a.x += (x.x - v4.x) * inv_dt;
      a.y += (x.y - v4.y) * inv_dt;
      a.z += (x.z - v4.z) * inv_dt;
      d.acc4[i] = a;
    }
    if (advect && (fl & NN_CLS_DYNAMIC)) d.w.vel[i] = make_real4(v4.x + dt * a.x, v4.y + dt * a.y, v4.z + dt * a.z, v4.w);
  }
}

// ---------------------------------------------------------------------------
// Elasticity (Becker et al. 2009), SPH/main.py:1182-1375, on elastic particles
// ("e-space", id order); current positions through the slot map of the last sort.
__global__ void k_el_slots(Dev d) {
  const int ne = d.d_n[3];
  GRID_STRIDE(e, ne) d.el_slot[e] = d.slot_of_id[d.el_id[e]];
}

// computeRotations_kernel, SPH/main.py:1249-1274
__global__ void k_el_rotations(Dev d, int rep) {
  const int ne = d.d_n[3];
  GRID_STRIDE(e, ne) {
    const int i = d.el_slot[e];
    const uint32_t fl = d.w.flags[i];
    const SceneDev& s = d.sc[slot_scene(fl)];
    if (rep >= s.el_mult) continue;
    const real3 xi = f3(d.w.pos[i]);
    const real3 x0i = f3(d.el_x0[e]);
    const real mi = d.w.mass[i];
    real A[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int c = d.el_cnt[e];
    for (int k = 0; k < c; ++k) {
      const int je = d.el_nb[(size_t)k * d.el_stride + e];
      const real3 xji = f3(d.w.pos[d.el_slot[je]]) - xi;
      const real3 xji0 = f3(d.el_x0[je]) - x0i;
      const real wgt = mi * kernel_w(sqrt(dot3(xji0, xji0)), s);
      A[0] += xji.x * xji0.x * wgt; A[1] += xji.x * xji0.y * wgt; A[2] += xji.x * xji0.z * wgt;
      A[3] += xji.y * xji0.x * wgt; A[4] += xji.y * xji0.y * wgt; A[5] += xji.y * xji0.z * wgt;
      A[6] += xji.z * xji0.x * wgt; A[7] += xji.z * xji0.y * wgt; A[8] += xji.z * xji0.z * wgt;
    }
    double Ad[3][3], Rd[3][3];
    for (int k = 0; k < 9; ++k) Ad[k / 3][k % 3] = (double)A[k];
    closest_rotation(Ad, Rd);
    for (int k = 0; k < 9; ++k) d.el_R[(size_t)k * d.el_stride + e] = (real)Rd[k / 3][k % 3];
  }
}

// computeStress_kernel, SPH/main.py:1285-1323
__global__ void k_el_stress(Dev d, int rep) {
  const int ne = d.d_n[3];
  GRID_STRIDE(e, ne) {
    const int i = d.el_slot[e];
    const uint32_t fl = d.w.flags[i];
    const SceneDev& s = d.sc[slot_scene(fl)];
    if (rep >= s.el_mult) continue;
    const real3 xi = f3(d.w.pos[i]);
    const real3 x0i = f3(d.el_x0[e]);
    real R[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) R[k] = d.el_R[(size_t)k * d.el_stride + e];
    real G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int c = d.el_cnt[e];
    for (int k = 0; k < c; ++k) {
      const int je = d.el_nb[(size_t)k * d.el_stride + e];
      const real4 x0j = d.el_x0[je];
      const real3 xji = f3(d.w.pos[d.el_slot[je]]) - xi;
      const real3 xji0 = f3(x0j) - x0i;
      // u_ji = R^T x_ji - x0_ji
      real3 u = make_real3(R[0] * xji.x + R[3] * xji.y + R[6] * xji.z - xji0.x,
                             R[1] * xji.x + R[4] * xji.y + R[7] * xji.z - xji0.y,
                             R[2] * xji.x + R[5] * xji.y + R[8] * xji.z - xji0.z);
      u = u * x0j.w;
      const real3 gw = kernel_grad(xji0, sqrt(dot3(xji0, xji0)), s);
      G[0] -= u.x * gw.x; G[1] -= u.x * gw.y; G[2] -= u.x * gw.z;
      G[3] -= u.y * gw.x; G[4] -= u.y * gw.y; G[5] -= u.y * gw.z;
      G[6] -= u.z * gw.x; G[7] -= u.z * gw.y; G[8] -= u.z * gw.z;
    }
    const real e0 = G[0], e1 = G[4], e2 = G[8];
    const real e3 = 0.5f * (G[1] + G[3]), e4 = 0.5f * (G[2] + G[6]), e5 = 0.5f * (G[5] + G[7]);
    real S[6];
    S[0] = s.el_cd * e0 + s.el_co * e1 + s.el_co * e2;
    S[1] = s.el_co * e0 + s.el_cd * e1 + s.el_co * e2;
    S[2] = s.el_co * e0 + s.el_co * e1 + s.el_cd * e2;
    S[3] = s.el_cs * e3;
    S[4] = s.el_cs * e4;
    S[5] = s.el_cs * e5;
#pragma unroll
    for (int k = 0; k < 6; ++k) d.el_S[(size_t)k * d.el_stride + e] = S[k];
  }
}

__device__ __forceinline__ real3 sym6_mul(const real* M, real3 v) {  // symMatTimesVec 1328-1332
  return make_real3(M[0] * v.x + M[3] * v.y + M[4] * v.z, M[3] * v.x + M[1] * v.y + M[5] * v.z,
                     M[4] * v.x + M[5] * v.y + M[2] * v.z);
}

// computeForces_kernel, SPH/main.py:1334-1375
__global__ void k_el_forces(Dev d, int rep) {
  const int ne = d.d_n[3];
  GRID_STRIDE(e, ne) {
    const int i = d.el_slot[e];
    const uint32_t fl = d.w.flags[i];
    const SceneDev& s = d.sc[slot_scene(fl)];
    if (rep >= s.el_mult) continue;
    const real4 x0i4 = d.el_x0[e];
    const real3 x0i = f3(x0i4);
    const real Vi = x0i4.w;
    real Ri[9], Si[6];
#pragma unroll
    for (int k = 0; k < 9; ++k) Ri[k] = d.el_R[(size_t)k * d.el_stride + e];
#pragma unroll
    for (int k = 0; k < 6; ++k) Si[k] = d.el_S[(size_t)k * d.el_stride + e];
    real3 f = make_real3(0.f, 0.f, 0.f);
    const int c = d.el_cnt[e];
    for (int k = 0; k < c; ++k) {
      const int je = d.el_nb[(size_t)k * d.el_stride + e];
      const real4 x0j = d.el_x0[je];
      const real3 xji0 = f3(x0j) - x0i;
      const real3 gw0 = kernel_grad(xji0, sqrt(dot3(xji0, xji0)), s);
      const real3 dji = gw0 * Vi;
      const real3 dij = gw0 * (-x0j.w);
      real Sj[6], Rj[9];
#pragma unroll
      for (int q = 0; q < 6; ++q) Sj[q] = d.el_S[(size_t)q * d.el_stride + je];
#pragma unroll
      for (int q = 0; q < 9; ++q) Rj[q] = d.el_R[(size_t)q * d.el_stride + je];
      const real3 fij = sym6_mul(Sj, dji) * (-x0j.w);
      const real3 fji = sym6_mul(Si, dij) * (-Vi);
      f.x += (Rj[0] * fij.x + Rj[1] * fij.y + Rj[2] * fij.z) - (Ri[0] * fji.x + Ri[1] * fji.y + Ri[2] * fji.z);
      f.y += (Rj[3] * fij.x + Rj[4] * fij.y + Rj[5] * fij.z) - (Ri[3] * fji.x + Ri[4] * fji.y + Ri[5] * fji.z);
      f.z += (Rj[6] * fij.x + Rj[7] * fij.y + Rj[8] * fij.z) - (Ri[6] * fji.x + Ri[7] * fji.y + Ri[8] * fji.z);
    }
    f = f * 0.5f;
    const real mi = d.w.mass[i];
    real4 a = d.acc4[i];
    a.x += f.x / mi; a.y += f.y / mi; a.z += f.z / mi;
    d.acc4[i] = a;
  }
}

// Elasticity.initValues_kernel (SPH/main.py:1220-1239): rest neighbourhood from the
// current lists (quirk: all neighbours, at most 50, SPH/main.py:1192; otherwise the
// elastic neighbours of the same phase) and rest volume m_i / rho_i (mass-based
// density, compute_density_func SPH/main.py:1170-1179).
__global__ void k_el_init(Dev d) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const uint32_t fl = d.w.flags[i];
    if (!(fl & NN_CLS_ELASTIC)) continue;
    const int id = d.w.id[i];
    const int e = d.e_of_id[id];
    if (e < 0) continue;
    const SceneDev& s = d.sc[slot_scene(fl)];
    const bool q = (s.flags & NN_F_QUIRKS) != 0;
    const int cap = q ? min(50, d.el_cap) : d.el_cap;
    const int ph = d.t.phase_id[id];
    const real3 xi = f3(d.w.pos[i]);
    const real mi = d.w.mass[i];
    real den = mi * s.W0;
    int c = 0;
    NB_LOOP(d, i, j) {
      const int jid = d.w.id[j];
      const int je = d.e_of_id[jid];
      const bool member = q ? (je >= 0) : (je >= 0 && d.t.phase_id[jid] == ph);
      const real3 r = xi - f3(d.w.pos[j]);
      const real wj = d.w.mass[j] * kernel_w(sqrt(dot3(r, r)), s);
      if (q || member) den += wj;
      if (member) {
        if (c < cap) d.el_nb[(size_t)c * d.el_stride + e] = je;
        ++c;
      }
    }
    d.el_cnt[e] = min(c, cap);
    const real3 x0 = make_real3(d.t.x_0[3 * id], d.t.x_0[3 * id + 1], d.t.x_0[3 * id + 2]);
    d.el_x0[e] = make_real4(x0.x, x0.y, x0.z, mi / den);
#pragma unroll
    for (int k = 0; k < 9; ++k) d.el_R[(size_t)k * d.el_stride + e] = (k % 4 == 0) ? 1.f : 0.f;
#pragma unroll
    for (int k = 0; k < 6; ++k) d.el_S[(size_t)k * d.el_stride + e] = 0.f;
  }
}

// ---------------------------------------------------------------------------
// advect (SPH/main.py:1086-1093) + enforce_boundary_3D for FLUID then SOLID
// (SPH/main.py:1044-1080; each particle is handled by the loop of its material).
// do_anim (the step's call only): animate_particles (SPH/main.py:283-309, called by
// SPHBase.step between advect and the boundary clamp) moves every particle of the
// scene, static ones too, by the displacement nn_set_animation stored for this step.
__global__ void k_advect_boundary(Dev d, int do_advect, int do_boundary, int do_anim) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const uint32_t fl = d.w.flags[i];
    const int scn = slot_scene(fl);
    const float* an = d.dyn[scn].anim;
    const bool move = do_anim && (an[0] != 0.f || an[1] != 0.f || an[2] != 0.f);
    if (!(fl & NN_CLS_DYNAMIC)) {
      if (move) {
        real4 p = d.w.pos[i];
        p.x += an[0]; p.y += an[1]; p.z += an[2];
        d.w.pos[i] = p;
      }
      continue;
    }
    const SceneDev& s = d.sc[scn];
    const real dt = d.dyn[scn].dt;
    real4 p = d.w.pos[i];
    real4 v = d.w.vel[i];
    if (do_advect) {
      if (cls_dyn_solid(fl)) {
        const real4 a = d.acc4[i];
        v.x += dt * a.x; v.y += dt * a.y; v.z += dt * a.z;
      }
      p.x += dt * v.x; p.y += dt * v.y; p.z += dt * v.z;
    }
    if (move) { p.x += an[0]; p.y += an[1]; p.z += an[2]; }
    if (do_boundary) {
      real pos[3] = {p.x, p.y, p.z};
      real nrm[3] = {0.f, 0.f, 0.f};
      real q[3] = {p.x, p.y, p.z};
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (pos[k] > s.xmax[k]) { nrm[k] += 1.f; q[k] = s.xmax[k]; }
        if (pos[k] <= s.xmin[k]) { nrm[k] += -1.f; q[k] = s.xmin[k]; }
      }
      p.x = q[0]; p.y = q[1]; p.z = q[2];
      const real len = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
      if (len > 1e-6f) {
        const real3 nn = make_real3(nrm[0] / len, nrm[1] / len, nrm[2] / len);
        const real vd = (1.f + s.cf) * (v.x * nn.x + v.y * nn.y + v.z * nn.z);
        v.x -= nn.x * vd; v.y -= nn.y * vd; v.z -= nn.z * vd;
        v.x *= s.sticky; v.y *= s.sticky; v.z *= s.sticky;
      }
    }
    if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(v.x) && isfinite(v.y) && isfinite(v.z)))
      set_status(&d.dyn[scn], NN_ERR_NAN);
    d.w.pos[i] = p;
    d.w.vel[i] = v;
  }
}

// ---------------------------------------------------------------------------
// Synchronisation with the caller's id-order state (meta.pd).
// Walks the caller's arrays in id order, so its stores are coalesced; the loads come
// from the slots through slot_of_id (a float4 load uses half of its sector, where a
// 4-byte store by slot would take a sector for itself).
__global__ void k_sync_out(Dev d, uint32_t mask) {
  const int n = d.d_n[0];
  GRID_STRIDE(id, n) {
    const int i = d.slot_of_id[id];
    const real4 p = d.w.pos[i];
    if (mask & 1u) { d.t.x[3 * id] = p.x; d.t.x[3 * id + 1] = p.y; d.t.x[3 * id + 2] = p.z; }
    if (mask & 2u) { const real4 v = d.w.vel[i]; d.t.v[3 * id] = v.x; d.t.v[3 * id + 1] = v.y; d.t.v[3 * id + 2] = v.z; }
    if (mask & 4u) { const real4 a = d.acc4[i]; d.t.a[3 * id] = a.x; d.t.a[3 * id + 1] = a.y; d.t.a[3 * id + 2] = a.z; }
    if (mask & 8u) d.t.volume[id] = fabs(p.w);
    if (mask & 16u) d.t.density[id] = d.w.dens[i];
    if (mask & 32u) d.t.dfsph_factor[id] = d.alpha[i];
    if (mask & 64u) d.t.density_adv[id] = d.rho_adv[i];
    if ((mask & 128u) && d.t.srn) d.t.srn[id] = d.srn[i];
    if ((mask & 128u) && d.t.mu) d.t.mu[id] = d.mu[i];
  }
}

__global__ void k_sync_out_elastic(Dev d) {
  const int ne = d.d_n[3];
  GRID_STRIDE(e, ne) {
    const int id = d.el_id[e];
    if (d.t.stress)
      for (int k = 0; k < 6; ++k) d.t.stress[6 * (size_t)id + k] = d.el_S[(size_t)k * d.el_stride + e];
    if (d.t.rot)
      for (int k = 0; k < 9; ++k) d.t.rot[9 * (size_t)id + k] = d.el_R[(size_t)k * d.el_stride + e];
  }
}

// Gather the per-pass fields from the caller's state into the current slots.
__global__ void k_sync_in(Dev d, uint32_t mask) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const int id = d.w.id[i];
    real4 p = d.w.pos[i];
    if (mask & 1u) { p.x = d.t.x[3 * id]; p.y = d.t.x[3 * id + 1]; p.z = d.t.x[3 * id + 2]; }
    if (mask & 8u) p.w = cls_solid(d.w.flags[i]) ? -d.t.volume[id] : d.t.volume[id];
    d.w.pos[i] = p;
    real m = d.w.mass[i];  // vel.w carries the mass
    if (mask & 256u) { m = d.t.m[id]; d.w.mass[i] = m; }
    if (mask & 2u) d.w.vel[i] = make_real4(d.t.v[3 * id], d.t.v[3 * id + 1], d.t.v[3 * id + 2], m);
    else if (mask & 256u) d.w.vel[i].w = m;
    if (mask & 4u) d.acc4[i] = make_real4(d.t.a[3 * id], d.t.a[3 * id + 1], d.t.a[3 * id + 2], 0.f);
    if (mask & 16u) d.w.dens[i] = d.t.density[id];
    if (mask & 32u) d.alpha[i] = d.t.dfsph_factor[id];
    if (mask & 64u) d.rho_adv[i] = d.t.density_adv[id];
  }
}

// ---------------------------------------------------------------------------
// Rigid bodies: RigidBodySolver.substep (SPH/main.py:1108-1158), shape matching per
// body. Bodies are numbered per context ("r-space"); round r processes the r-th body
// of every scene, so each scene's bodies run in the reference's order.
#define RB_ACC 13  // per body: sum m x (3), sum m (1), sum m p (x) q (9)

// FP64 sums of `nv` values per body over a warp: body-uniform warps reduce with
// shuffles and one lane issues the atomics; mixed warps use per-lane atomics.
template <int NV>
__device__ __forceinline__ void body_add(double* acc, int body, const double (&v)[NV]) {
  const unsigned full = 0xffffffffu;
  const unsigned vb = __ballot_sync(full, body >= 0);
  if (vb == 0) return;
  const int leader = __ffs(vb) - 1;
  const int b0 = __shfl_sync(full, body, leader);
  const bool uniform = __all_sync(full, body < 0 || body == b0);
  if (uniform) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double x = body >= 0 ? v[k] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(full, x, o);
      if ((int)(threadIdx.x & 31) == leader) atomicAdd(&acc[(size_t)b0 * RB_ACC + k], x);
    }
  } else if (body >= 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) atomicAdd(&acc[(size_t)body * RB_ACC + k], v[k]);
  }
}

__device__ __forceinline__ int rigid_body_of_slot(const Dev& d, int i, int round) {
  const int b = d.rb_of_id[d.w.id[i]];
  return (b >= 0 && d.rb_round[b] == round) ? b : -1;
}

// ground_collision (SPH/main.py:1113-1118): every solid particle of a scene with
// rigid bodies is lifted to y >= padding (once per body substep, like the reference).
__global__ void k_rigid_ground(Dev d, int round, int rep) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const uint32_t fl = d.w.flags[i];
    if (!cls_solid(fl)) continue;
    const SceneDev& s = d.sc[slot_scene(fl)];
    if (!(s.flags & NN_F_RIGID) || round >= s.n_rigid || rep >= s.coupling) continue;
    real4 p = d.w.pos[i];
    if (p.y < s.padding) { p.y = s.padding; d.w.pos[i] = p; }
  }
}

// compute_com (SPH/main.py:1120-1130) over the current (rest = 0) or rest positions.
__global__ void k_rigid_com(Dev d, int round, int rest) {
  const int n = d.d_n[0];
  FOR_SLOTS_WARP(i, valid, n) {
    int b = valid ? rigid_body_of_slot(d, i, round) : -1;
    double v[4] = {0, 0, 0, 0};
    if (b >= 0) {
      const SceneDev& s = d.sc[slot_scene(d.w.flags[i])];
      const double m = (double)(s.V0 * d.w.dens[i]);
      real3 x;
      if (rest) {
        const int id = d.w.id[i];
        x = make_real3(d.t.x_0[3 * id], d.t.x_0[3 * id + 1], d.t.x_0[3 * id + 2]);
      } else {
        x = f3(d.w.pos[i]);
      }
      v[0] = m * x.x; v[1] = m * x.y; v[2] = m * x.z; v[3] = m;
    }
    body_add<4>(d.rb_acc, b, v);
  }
}

// Per body: centre of mass (into rb_rest for the rest state, rb_cm otherwise).
__global__ void k_rigid_cm(Dev d, int round, int rest) {
  for (int b = threadIdx.x; b < d.n_rb; b += blockDim.x) {
    if (d.rb_round[b] != round) continue;
    double* a = &d.rb_acc[(size_t)b * RB_ACC];
    double* out = rest ? &d.rb_rest[3 * b] : &d.rb_cm[3 * b];
    for (int k = 0; k < 3; ++k) out[k] = a[3] > 0 ? a[k] / a[3] : 0.0;
    for (int k = 0; k < RB_ACC; ++k) a[k] = 0.0;
  }
}

// A = sum m (x - cm) (x) (x0 - rest_cm) (SPH/main.py:1141-1146).
__global__ void k_rigid_A(Dev d, int round) {
  const int n = d.d_n[0];
  FOR_SLOTS_WARP(i, valid, n) {
    int b = valid ? rigid_body_of_slot(d, i, round) : -1;
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (b >= 0) {
      const SceneDev& s = d.sc[slot_scene(d.w.flags[i])];
      const double m = (double)(s.V0 * d.w.dens[i]);
      const int id = d.w.id[i];
      const real4 x = d.w.pos[i];
      const double p[3] = {(double)x.x - d.rb_cm[3 * b], (double)x.y - d.rb_cm[3 * b + 1],
                           (double)x.z - d.rb_cm[3 * b + 2]};
      const double q[3] = {(double)d.t.x_0[3 * id] - d.rb_rest[3 * b], (double)d.t.x_0[3 * id + 1] - d.rb_rest[3 * b + 1],
                           (double)d.t.x_0[3 * id + 2] - d.rb_rest[3 * b + 2]};
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) v[3 * r + c] = m * p[r] * q[c];
    }
    double* acc = d.rb_acc + 4;  // the A block of each body's accumulator
    body_add<9>(acc, b, v);
  }
}

// R = polar(A) (SPH/main.py:1148-1151), identity if every entry is below 1e-6.
__global__ void k_rigid_R(Dev d, int round) {
  for (int b = threadIdx.x; b < d.n_rb; b += blockDim.x) {
    if (d.rb_round[b] != round) continue;
    double* a = &d.rb_acc[(size_t)b * RB_ACC + 4];
    double A[3][3], R[3][3];
    for (int k = 0; k < 9; ++k) A[k / 3][k % 3] = a[k];
    closest_rotation(A, R);
    bool small = true;
    for (int k = 0; k < 9; ++k) small = small && fabs(R[k / 3][k % 3]) < 1e-6;
    for (int k = 0; k < 9; ++k) d.rb_R[9 * b + k] = small ? ((k % 4 == 0) ? 1.0 : 0.0) : R[k / 3][k % 3];
    for (int k = 0; k < RB_ACC; ++k) d.rb_acc[(size_t)b * RB_ACC + k] = 0.0;
  }
}

// x = cm + R (x0 - rest_cm) (SPH/main.py:1153-1157).
__global__ void k_rigid_apply(Dev d, int round) {
  const int n = d.d_n[0];
  GRID_STRIDE(i, n) {
    const int b = rigid_body_of_slot(d, i, round);
    if (b < 0) continue;
    const int id = d.w.id[i];
    const double q[3] = {(double)d.t.x_0[3 * id] - d.rb_rest[3 * b], (double)d.t.x_0[3 * id + 1] - d.rb_rest[3 * b + 1],
                         (double)d.t.x_0[3 * id + 2] - d.rb_rest[3 * b + 2]};
    const double* R = &d.rb_R[9 * b];
    real4 p = d.w.pos[i];
    p.x = (real)(d.rb_cm[3 * b] + R[0] * q[0] + R[1] * q[1] + R[2] * q[2]);
    p.y = (real)(d.rb_cm[3 * b + 1] + R[3] * q[0] + R[4] * q[1] + R[5] * q[2]);
    p.z = (real)(d.rb_cm[3 * b + 2] + R[6] * q[0] + R[7] * q[1] + R[8] * q[2]);
    d.w.pos[i] = p;
  }
}
