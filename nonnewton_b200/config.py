"""Scene configuration: the reference's JSON schema and defaults.

Mirrors `SimConfig` / `get_cfg` (SPH/main.py:59-96) and `Parameter`
(SPH/main.py:594-621). Keys and defaults are the reference's; keys the reference
reads nowhere (viscosityMethod, viscoMaxError, youngsModulus, cfl*, ...) are
read here for the extensions (implicit viscosity, configurable elasticity, CFL),
using the SPlisHSPlasH-style names the reference's own scene files already carry.
Unlike the reference, a missing scene path is an error instead of a tkinter dialog
(SPH/main.py:47-56), and `noGUI` defaults to true (there is no GUI here).
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field

import numpy as np

from . import _abi

# NonNewton.NON_NEWTON_METHOD (SPH/main.py:347-355)
NON_NEWTON_METHODS = {
    "NEWTONIAN_": _abi.NN_NEWTONIAN, "POWER_LAW_": _abi.NN_POWER_LAW, "CROSS_": _abi.NN_CROSS,
    "CASSON_": _abi.NN_CASSON, "CARREAU_": _abi.NN_CARREAU, "BINGHAM_": _abi.NN_BINGHAM,
    "HERSCHEL_BULKLEY_": _abi.NN_HERSCHEL_BULKLEY,
}

# viscosityMethod values that select the implicit Weiler 2018 solver: SPlisHSPlasH's
# id 7 (Weiler et al. 2018) and 13, the id the reference's test_nonNewton.json uses.
IMPLICIT_VISCOSITY_METHODS = (7, 13, "Weiler2018", "weiler2018")


class SimConfig:
    """`SimConfig` (SPH/main.py:59-72): a JSON scene with a `Configuration` block."""

    def __init__(self, scene_path: str = "", config: dict | None = None) -> None:
        if config is not None:
            self.config = config
        else:
            if not scene_path:
                raise ValueError("a scene path is required (the reference opens a file dialog here)")
            with open(scene_path, "r") as f:
                self.config = json.load(f)
        self.scene_path = scene_path
        self.config.setdefault("Configuration", {})

    def get_cfg(self, name, default=None):
        c = self.config["Configuration"]
        return default if name not in c else c[name]

    def get_fluid_cfg(self):
        return self.config.get("FluidParticles", [])

    def get_solid_cfg(self):
        return self.config.get("SolidParticles", [])

    def get_cfg_list(self, name, default=None):
        return self.config.get(name, default)


@dataclass
class Parameter:
    """`Parameter` (SPH/main.py:594-621) plus the extension keys, as plain floats."""

    domain_start: np.ndarray
    domain_end: np.ndarray
    simulation_method: int
    particle_radius: float
    density0: float
    gravity: np.ndarray
    boundary_viscosity: float
    dt: float
    sticky_coeff: float
    collision_coeff: float
    coupling_interval: int
    solid_dt: float
    viscosity: float
    # DFSPH (SPH/main.py:1524-1535)
    max_iterations_v: int = 100
    max_iterations: int = 100
    max_error_v: float = 0.1
    max_error: float = 0.05
    m_eps: float = 1e-5
    use_surface_tension: bool = True
    use_nonnewtonian: bool = False
    use_viscosity: bool = True
    use_elasticity_model: bool = False
    enable_divergence_solver: bool = True
    # NonNewton (SPH/main.py:357-365), first fluid block
    nonnewton_method: int = _abi.NN_NEWTONIAN
    power_index: float = 0.667
    consistency_index: float = 100.0
    viscosity0: float = 2000.0
    viscosity_inf: float = 1.0
    critical_strain_rate: float = 20.0
    mu_c: float = 10.0
    yield_stress: float = 200.0
    carreau_textbook: bool = False
    # implicit viscosity (Weiler 2018; SPH/main.py:1481-1485 defaults)
    implicit_viscosity: bool = False
    visco_max_iter: int = 100
    visco_max_error: float = 0.01
    visco_boundary: float = 0.0
    # elasticity (SPH/main.py:1188-1189 defaults)
    youngs_modulus: float = 25e4
    poisson_ratio: float = 0.33
    # CFL (extension)
    cfl: bool = False
    cfl_factor: float = 1.0
    cfl_min_dt: float = 1e-4
    cfl_max_dt: float = 5e-3
    quirks: bool = False
    has_elastic: bool = False
    has_rigid: bool = False
    surface_tension: float = 0.01
    extra: dict = field(default_factory=dict)

    # derived, SPH/main.py:601-615
    @property
    def domain_size(self):
        return self.domain_end - self.domain_start

    @property
    def dim(self):
        return 3

    @property
    def particle_diameter(self):
        return 2.0 * self.particle_radius

    @property
    def support_radius(self):
        return self.particle_radius * 4.0

    @property
    def volume0(self):
        return 0.8 * self.particle_diameter ** 3

    @property
    def padding(self):
        return self.support_radius

    @classmethod
    def from_config(cls, cfg: SimConfig, quirks: bool = False) -> "Parameter":
        g = cfg.get_cfg
        dt = float(g("timeStepSize", 1e-4))
        fl = cfg.get_fluid_cfg()
        f0 = fl[0] if fl else {}
        method = f0.get("nonNewtonMethod", 0)
        if isinstance(method, str):
            method = NON_NEWTON_METHODS.get(method, _abi.NN_NEWTONIAN)
        visc_method = f0.get("viscosityMethod", g("viscosityMethod", None))
        solids = cfg.get_solid_cfg()
        el = [s for s in solids if s.get("solidType") == "ELASTIC"]
        e0 = el[0] if el else {}
        p = cls(
            domain_start=np.array(g("domainStart", [0.0, 0.0, 0.0]), dtype=np.float64),
            domain_end=np.array(g("domainEnd", [1.0, 1.0, 1.0]), dtype=np.float64),
            simulation_method=g("simulationMethod"),
            particle_radius=float(g("particleRadius", 0.01)),
            density0=float(g("density0", 1000.0)),
            gravity=np.array(g("gravitation", [0.0, -9.8, 0.0]), dtype=np.float64),
            boundary_viscosity=float(g("boundaryViscosity", 0.0)),
            dt=dt,
            sticky_coeff=float(g("stickyCoefficient", 0.999)),
            collision_coeff=float(g("collisionCoefficient", 0.5)),
            coupling_interval=int(g("couplingInterval", 1)),
            solid_dt=float(g("solidTimeStepSize", dt)),
            viscosity=float(g("viscosity", 0.01)),
            max_iterations_v=int(g("maxIterationsV", 100)),
            max_iterations=int(g("maxIterations", 100)),
            max_error_v=float(g("maxErrorV", 0.1)),
            max_error=float(g("maxError", 0.05)),
            use_surface_tension=bool(g("useSurfaceTensionModel", True)),
            use_nonnewtonian=bool(g("useNonNewtonianModel", False)),
            use_viscosity=bool(g("useViscosityModel", True)),
            use_elasticity_model=bool(g("useElasticityModel", False)),
            enable_divergence_solver=bool(g("enableDivergenceSolver", True)),
            nonnewton_method=int(method),
            power_index=float(f0.get("power_index", 0.667)),
            consistency_index=float(f0.get("consistency_index", 100.0)),
            viscosity0=float(f0.get("viscosity0", 2000.0)),
            viscosity_inf=float(f0.get("viscosity_inf", 1.0)),
            critical_strain_rate=float(f0.get("criticalStrainRate", 20.0)),
            mu_c=float(f0.get("muC", 10.0)),
            yield_stress=float(f0.get("yieldStress", 200.0)),
            carreau_textbook=bool(f0.get("carreauTextbook", False)),
            implicit_viscosity=visc_method in IMPLICIT_VISCOSITY_METHODS,
            visco_max_iter=int(f0.get("viscoMaxIter", g("viscoMaxIter", 100))),
            visco_max_error=float(f0.get("viscoMaxError", g("viscoMaxError", 0.01))),
            visco_boundary=float(f0.get("viscosityBoundary", g("viscosityBoundary", 0.0))),
            youngs_modulus=float(e0.get("youngsModulus", 25e4)),
            poisson_ratio=float(e0.get("poissonsRatio", 0.33)),
            cfl=int(g("cflMethod", 0)) != 0,
            cfl_factor=float(g("cflFactor", 1.0)),
            cfl_min_dt=float(g("cflMinTimeStepSize", 1e-4)),
            cfl_max_dt=float(g("cflMaxTimeStepSize", 5e-3)),
            quirks=bool(g("referenceQuirks", quirks)),
            has_elastic=bool(el),
            has_rigid=any(s_.get("solidType") == "RIGID" for s_ in solids),
        )
        if p.simulation_method not in (4, None):
            # build_solver (SPH/main.py:196-203)
            raise NotImplementedError(f"Solver type {p.simulation_method} has not been implemented.")
        if bool(g("useDragForceModel", False)):
            # the reference's DragForce model is commented out (SPH/main.py:1543-1544), so its
            # compute_non_pressure_forces (1564-1565) fails on the missing model
            raise NotImplementedError("useDragForceModel: the reference has no drag force model")
        return p

    def flags(self) -> int:
        f = 0
        if self.use_surface_tension:
            f |= _abi.NN_F_SURFACE_TENSION
        if self.use_viscosity:
            f |= _abi.NN_F_VISCOSITY
        if self.use_nonnewtonian:
            f |= _abi.NN_F_NONNEWTON
        if self.implicit_viscosity:
            f |= _abi.NN_F_IMPLICIT_VISCOSITY
        if self.enable_divergence_solver:
            f |= _abi.NN_F_DIVERGENCE
        if self.cfl:
            f |= _abi.NN_F_CFL
        if self.quirks:
            f |= _abi.NN_F_QUIRKS
        if self.carreau_textbook:
            f |= _abi.NN_F_CARREAU_TEXTBOOK
        if self.has_elastic:
            f |= _abi.NN_F_ELASTICITY
        if self.has_rigid:
            f |= _abi.NN_F_RIGID
        return f

    def to_c(self) -> _abi.nn_scene_params:
        return _abi.make_params(
            flags=self.flags(),
            domain_start=self.domain_start, domain_end=self.domain_end,
            particle_radius=self.particle_radius, support_radius=self.support_radius,
            volume0=self.volume0, density0=self.density0, gravity=self.gravity, dt=self.dt,
            sticky_coeff=self.sticky_coeff, collision_coeff=self.collision_coeff,
            padding=self.padding, viscosity=self.viscosity,
            boundary_viscosity=self.boundary_viscosity, surface_tension=self.surface_tension,
            eps=self.m_eps, max_iterations_v=self.max_iterations_v,
            max_iterations=self.max_iterations, max_error_v=self.max_error_v,
            max_error=self.max_error, nonnewton_method=self.nonnewton_method,
            power_index=self.power_index, consistency_index=self.consistency_index,
            viscosity0=self.viscosity0, viscosity_inf=self.viscosity_inf,
            critical_strain_rate=self.critical_strain_rate, mu_c=self.mu_c,
            yield_stress=self.yield_stress, visco_max_iter=self.visco_max_iter,
            visco_max_error=self.visco_max_error, visco_boundary=self.visco_boundary,
            youngs_modulus=self.youngs_modulus, poisson_ratio=self.poisson_ratio,
            cfl_factor=self.cfl_factor, cfl_min_dt=self.cfl_min_dt, cfl_max_dt=self.cfl_max_dt,
            coupling_interval=self.coupling_interval,
        )


def sph_root_path() -> str:
    return os.path.dirname(os.path.abspath(__file__))
