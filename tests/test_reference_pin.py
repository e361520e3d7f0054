"""The oracle against the reference's own step: tests/golden/ref_<scene>.npz hold the
particle state after each step of SPH/main.py itself, run through a plain-Python Taichi
stand-in (tests/golden/make_reference_run.py) on seven small scenes: a fluid block in a
boundary box (surface tension and explicit viscosity on, as the reference defaults
them), the same with the non-Newtonian model on, with an elastic cube, and with a rigid
cube, and the reference's own fixture scenes test_deformable.json (343 elastic
particles), test_neighbor.json (9 fluid particles) and test_anime.json (one particle
moved by an animeFile's per-frame displacements, the frame being the step index, as the
GUI loop counts it). The oracle runs in the reference-quirks mode from the same
initial state; every recorded field stays within 2e-5 of its scale (f32 rounding and
summation order; observed up to 2e-6). No GPU."""
import pytest

from .helpers import REF_SCENES, frame_displacement, reference_animation, reference_errors, reference_run, reference_steps

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
    anime = reference_animation(R)
    for s in range(reference_steps(R)):
        d = frame_displacement(anime, s)
        if d is not None:
            o.set_animation(d)
        o.step(1)
        err = reference_errors(R, s, o.get, ps.n_fluid)
        assert err and max(err.values()) < TOL, (s, err)


def test_surface_oracle_matches_the_reference_run():
    """The surface oracle against the reference's own SRTool stages
    (tests/golden/ref_surface.npz, srtool.py run through the Taichi stand-in on a
    154-particle ball): anisotropic kernels G and x_bar within 1e-6 of scale, the same
    active blocks, the field after the splats within 3e-4 of its scale, the smoothing's
    sd within 1e-4 and the smoothed field within 2e-4. The reference sums the splats in
    f32 and the oracle in double; run in f64, the reference comes within 3.2e-5 of the
    oracle's splat field, so most of the difference is the reference's own rounding."""
    import os

    import numpy as np

    from nonnewton_b200 import _abi
    from oracle import surf as S

    R = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_surface.npz"))
    vs, r, sr, iso = R["params"]
    prm = _abi.make_sr_params(list(R["dims"]), [0, 0, 0], vs, r, sr, iso)

    def rel(a, b):
        return np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30)

    G, xb = S.prepass(prm, R["pos"])
    assert rel(G, R["G"]) < 1e-6 and rel(xb, R["xbar"]) < 1e-6
    f, act = S.splat(prm, R["pos"], G, xb)
    nb = [-(-int(d) // _abi.NN_SR_BLOCK) for d in R["dims"]]
    assert np.array_equal(np.argwhere(act.reshape(nb[2], nb[1], nb[0]))[:, ::-1], R["blocks"])
    assert rel(f, R["field_splat"]) < 3e-4
    fs, sd = S.smooth(prm, f, act)
    assert abs(sd - R["sd"]) < 1e-4 * R["sd"]
    assert rel(fs, R["field_smooth"]) < 2e-4
