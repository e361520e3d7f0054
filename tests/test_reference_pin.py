"""The oracle against the reference's own step: tests/golden/ref_<scene>.npz hold the
particle state after each step of SPH/main.py itself, run through a plain-Python Taichi
stand-in (tests/golden/make_reference_run.py) on four small scenes of the reference's
kinds: a fluid block in a boundary box (surface tension and explicit viscosity on, as
the reference defaults them), the same with the non-Newtonian model on, with an elastic
cube, and with a rigid cube. The oracle runs in the reference-quirks mode from the same
initial state; every recorded field stays within 2e-5 of its scale (f32 rounding and
summation order; observed up to 2e-6). No GPU."""
import pytest

from .helpers import REF_SCENES, reference_errors, reference_run, reference_steps

TOL = 2e-5


@pytest.mark.parametrize("name", REF_SCENES)
def test_oracle_matches_the_reference_run(name):
    from oracle import oracle as O

    R, cfg, param, ps = reference_run(name)
    o = O.OracleSim(ps, param, "f32")
    o.initialize()
    assert abs(o.get("volume") - R["init_volume"]).max() <= TOL * abs(R["init_volume"]).max()
    # the reference's first search runs on the same positions: the same neighbour counts
    assert (o.neighbors(60)[0] == R["step0_num_neighbors"]).all()
    for s in range(reference_steps(R)):
        o.step(1)
        err = reference_errors(R, s, o.get, ps.n_fluid)
        assert err and max(err.values()) < TOL, (s, err)
