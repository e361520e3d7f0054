// dev.cuh — device pointer bundle passed by value to every kernel.
#pragma once
#include "common.cuh"

// Sorted working set: particles in cell order ("slots").
struct WorkSet {
  real4* pos;       // x, y, z, volume (negative for solids)
  real4* vel;       // v, w = mass (a copy of `mass`, so neighbour loops get it with v)
  real* mass;
  real* dens;
  uint32_t* flags;   // class bits | scene << NN_SCENE_SHIFT
  int32_t* id;       // particle id of the slot
};

// Caller-owned state in particle-id order (meta.pd): float32 in both builds.
struct Truth {
  float* x; float* x_0; float* v; float* a;
  float* volume; float* m; float* density; float* dfsph_factor; float* density_adv;
  int32_t* material; int32_t* is_dynamic; int32_t* phase_id;
  float* srn; float* mu; float* stress; float* rot;
};

struct Dev {
  // sizes (device-resident so a captured graph serves any batch composition)
  const int32_t* d_n;          // [0] particles, [1] scenes, [2] total cells, [3] elastic particles
  const SceneDev* sc;
  SceneDyn* dyn;
  double* acc;                 // [scene][ACC_COUNT][NN_STRIPES]
  const int32_t* scene_of_id;  // scene of each particle id
  Truth t;
  WorkSet w;                   // current sorted set
  WorkSet wo;                  // previous sorted set (resident re-sort source)
  const int32_t* src_from_truth; // device flag: 1 = gather from Truth, 0 = from wo
  real4* acc4;                 // accelerations (slot order)
  real* alpha;
  real* rho_adv;
  real* kappa;
  int32_t* slot_of_id;
  // neighbour search
  uint32_t* key;               // per source index
  uint32_t* rank;              // per source index
  int32_t* src;                // source index of each new slot
  uint32_t* cell_count;        // [cells + 1] counts, then exclusive starts
  uint32_t* tile_sums;
  int32_t* nbr;                // [max_nb][cap]
  int32_t* nbr_cnt;            // [cap] stored entries, min(count, max_nb)
  int32_t* nbr_raw;            // [cap] full neighbour count, or null (only the allocation-free search keeps it)
  int32_t cap;                 // slot capacity (neighbour list stride)
  int32_t max_nb;
  // non-Newtonian
  real* srn;
  real* mu;
  // implicit viscosity CG (slot order)
  real4* cg_x; real4* cg_r; real4* cg_z; real4* cg_Ap;
  real4* cg_p;                 // search direction; w = mu_i (read by the matvec)
  real4* cg_pos;               // matvec positions: fluid (x_i, m_i / rho_i), solid (x_i, -V_i) as pos
  real2* cg_aux;               // fluid: mu_i, m_i / rho_i; solid: 0, 1 if dynamic
  real* cg_pinv;               // [6][cap] symmetric inverse of the diagonal block
  // elasticity (e-space: elastic particles in id order)
  int32_t* el_id;              // [Ne] particle id
  int32_t* el_slot;            // [Ne] current slot
  int32_t* e_of_id;            // [cap] elastic index or -1
  real4* el_x0;                // [Ne] rest position, rest volume
  int32_t* el_nb;              // [rest_cap][Ne] rest neighbours (elastic indices)
  int32_t* el_cnt;             // [Ne]
  int32_t el_cap;              // rest list capacity
  int32_t el_stride;           // Ne capacity
  real* el_R;                  // [9][Ne]
  real* el_S;                  // [6][Ne]
  // rigid bodies ("r-space")
  int32_t n_rb;
  const int32_t* rb_of_id;     // [cap] body index or -1
  const int32_t* rb_round;     // [n_rb] position of the body among its scene's bodies
  double* rb_acc;              // [n_rb][13] reductions
  double* rb_rest;             // [n_rb][3] rest centre of mass
  double* rb_cm;               // [n_rb][3] current centre of mass
  double* rb_R;                // [n_rb][9] rotation
  // loop control
  int32_t* any_active;         // host-visible flag of the last check
  unsigned long long loop_handle; // cudaGraphConditionalHandle (0 when not in a graph)
  int32_t* body_count;         // [4] executed loop bodies (div, pressure, cg, elastic)
};

// A neighbour's position + volume in the neighbour passes (read-only there).
__device__ __forceinline__ real4 pos_of(const Dev& d, int j) { return ldg(&d.w.pos[j]); }
