"""ctypes mirror of include/nnsph.h (the C ABI of libnnsph.so).

The field order and types follow the header exactly; `tests/test_abi.py` checks the
sizes against the compiled library.
"""
import ctypes as C

NN_OK = 0
NN_ERR_INVALID_ARG = -1
NN_ERR_CUDA = -2
NN_ERR_OOM = -3
NN_ERR_NEIGHBOR_OVERFLOW = -4
NN_ERR_NOT_CONVERGED = -5
NN_ERR_NAN = -6
NN_ERR_STATE = -7
NN_ERR_CAPACITY = -8

ERROR_NAMES = {
    NN_ERR_INVALID_ARG: "invalid argument",
    NN_ERR_CUDA: "CUDA error",
    NN_ERR_OOM: "out of device memory",
    NN_ERR_NEIGHBOR_OVERFLOW: "neighbour list overflow",
    NN_ERR_NOT_CONVERGED: "solver did not converge",
    NN_ERR_NAN: "non-finite value in the state",
    NN_ERR_STATE: "call out of order",
    NN_ERR_CAPACITY: "context capacity exceeded",
}

NN_FLUID = 0
NN_SOLID = 1
NN_PHASE_STATIC_BASE = 1000
NN_PHASE_RIGID_BASE = 2000
NN_PHASE_ELASTIC_BASE = 3000

NN_F_SURFACE_TENSION = 1 << 0
NN_F_VISCOSITY = 1 << 1
NN_F_NONNEWTON = 1 << 2
NN_F_IMPLICIT_VISCOSITY = 1 << 3
NN_F_ELASTICITY = 1 << 4
NN_F_DIVERGENCE = 1 << 5
NN_F_CFL = 1 << 6
NN_F_QUIRKS = 1 << 7
NN_F_CARREAU_TEXTBOOK = 1 << 8
NN_F_RIGID = 1 << 9

NN_NEWTONIAN = 0
NN_POWER_LAW = 1
NN_CROSS = 2
NN_CASSON = 3
NN_CARREAU = 4
NN_BINGHAM = 5
NN_HERSCHEL_BULKLEY = 6

(NN_PASS_SEARCH, NN_PASS_STATIC_BOUNDARY_VOLUME, NN_PASS_MOVING_BOUNDARY_VOLUME,
 NN_PASS_CLEAR_ACCELERATIONS, NN_PASS_DENSITIES, NN_PASS_DFSPH_FACTOR,
 NN_PASS_DIVERGENCE_SOLVE, NN_PASS_NON_PRESSURE_FORCES, NN_PASS_NON_PRESSURE_ADVECT,
 NN_PASS_PRESSURE_SOLVE, NN_PASS_ELASTICITY, NN_PASS_ADVECT, NN_PASS_ENFORCE_BOUNDARY,
 NN_PASS_SUBSTEP, NN_PASS_RIGID, NN_PASS_COUNT) = range(16)

(NN_K_PRESSURE_UPDATE, NN_K_DENSITY_ADV, NN_K_DIVERGENCE_UPDATE, NN_K_DENSITY_CHANGE, NN_K_DENSITY_FACTOR,
 NN_K_BUILD_LISTS, NN_K_CG_MATVEC, NN_K_NONPRESSURE, NN_K_DENSITY_CHANGE_NP, NN_K_CG_SETUP, NN_K_COUNT) = range(11)

NN_STEP_SYNC_STATE = 1 << 0
NN_STEP_HOST_LOOP = 1 << 1
NN_STEP_RESUME = 1 << 2


class nn_scene_params(C.Structure):
    _fields_ = [
        ("size", C.c_uint32),
        ("flags", C.c_uint32),
        ("domain_start", C.c_double * 3),
        ("domain_end", C.c_double * 3),
        ("particle_radius", C.c_double),
        ("support_radius", C.c_double),
        ("volume0", C.c_double),
        ("density0", C.c_double),
        ("gravity", C.c_double * 3),
        ("dt", C.c_double),
        ("sticky_coeff", C.c_double),
        ("collision_coeff", C.c_double),
        ("padding", C.c_double),
        ("viscosity", C.c_double),
        ("boundary_viscosity", C.c_double),
        ("surface_tension", C.c_double),
        ("eps", C.c_double),
        ("max_iterations_v", C.c_int32),
        ("max_iterations", C.c_int32),
        ("max_error_v", C.c_double),
        ("max_error", C.c_double),
        ("nonnewton_method", C.c_int32),
        ("pad0", C.c_int32),
        ("power_index", C.c_double),
        ("consistency_index", C.c_double),
        ("viscosity0", C.c_double),
        ("viscosity_inf", C.c_double),
        ("critical_strain_rate", C.c_double),
        ("mu_c", C.c_double),
        ("yield_stress", C.c_double),
        ("visco_max_iter", C.c_int32),
        ("pad1", C.c_int32),
        ("visco_max_error", C.c_double),
        ("visco_boundary", C.c_double),
        ("youngs_modulus", C.c_double),
        ("poisson_ratio", C.c_double),
        ("cfl_factor", C.c_double),
        ("cfl_min_dt", C.c_double),
        ("cfl_max_dt", C.c_double),
        ("coupling_interval", C.c_int32),
        ("pad2", C.c_int32),
    ]


class nn_scene_desc(C.Structure):
    _fields_ = [
        ("size", C.c_uint32),
        ("start", C.c_int32),
        ("n", C.c_int32),
        ("n_fluid", C.c_int32),
        ("params", nn_scene_params),
    ]


class nn_state(C.Structure):
    _fields_ = [
        ("size", C.c_uint32),
        ("n", C.c_int32),
        ("x", C.c_void_p),
        ("x_0", C.c_void_p),
        ("v", C.c_void_p),
        ("acceleration", C.c_void_p),
        ("volume", C.c_void_p),
        ("m", C.c_void_p),
        ("density", C.c_void_p),
        ("pressure", C.c_void_p),
        ("dfsph_factor", C.c_void_p),
        ("density_adv", C.c_void_p),
        ("material", C.c_void_p),
        ("is_dynamic", C.c_void_p),
        ("phase_id", C.c_void_p),
        ("strain_rate_norm", C.c_void_p),
        ("nonnewton_viscosity", C.c_void_p),
        ("stress", C.c_void_p),
        ("rotations", C.c_void_p),
    ]


class nn_stats(C.Structure):
    _fields_ = [
        ("size", C.c_uint32),
        ("status", C.c_int32),
        ("iterations_v", C.c_int32),
        ("iterations", C.c_int32),
        ("cg_iterations", C.c_int32),
        ("max_neighbors_seen", C.c_int32),
        ("avg_density_err_v", C.c_double),
        ("avg_density_err", C.c_double),
        ("cg_residual", C.c_double),
        ("dt", C.c_double),
        ("max_density", C.c_double),
        ("steps", C.c_int64),
        ("max_avg_density_err", C.c_double),
        ("nonpressure_folded", C.c_int32),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "size"}


def make_params(**kw) -> nn_scene_params:
    p = nn_scene_params()
    p.size = C.sizeof(nn_scene_params)
    for k, v in kw.items():
        if k in ("domain_start", "domain_end", "gravity"):
            getattr(p, k)[:] = [float(t) for t in v]
        else:
            setattr(p, k, v)
    return p


NN_SR_BLOCK = 32
NN_SR_VELOCITY = 1
NN_SR_MAX_PER_VOXEL = 64


class nn_sr_params(C.Structure):
    """Mirror of nn_sr_params (surface reconstruction)."""
    _fields_ = [
        ("size", C.c_int32),
        ("dims", C.c_int32 * 3),
        ("origin", C.c_double * 3),
        ("voxel_size", C.c_double),
        ("particle_radius", C.c_double),
        ("smooth_radius", C.c_double),
        ("isolevel", C.c_double),
        ("use_smooth_field", C.c_int32),
        ("smooth_iterations", C.c_int32),
        ("smooth_cells", C.c_int32),
        ("record_normals", C.c_int32),
    ]


def make_sr_params(dims, origin, voxel_size, particle_radius, smooth_radius, isolevel, use_smooth_field=True,
                   smooth_iterations=1, smooth_cells=1, record_normals=False) -> nn_sr_params:
    p = nn_sr_params()
    p.size = C.sizeof(nn_sr_params)
    p.dims[:] = [int(t) for t in dims]
    p.origin[:] = [float(t) for t in origin]
    p.voxel_size = float(voxel_size)
    p.particle_radius = float(particle_radius)
    p.smooth_radius = float(smooth_radius)
    p.isolevel = float(isolevel)
    p.use_smooth_field = int(bool(use_smooth_field))
    p.smooth_iterations = int(smooth_iterations)
    p.smooth_cells = int(smooth_cells)
    p.record_normals = int(bool(record_normals))
    return p
