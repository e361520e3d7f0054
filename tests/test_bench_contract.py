"""bench.py's frozen roofline constants (no GPU): the per-kernel algorithmic bytes per
particle of the kernel table, the whole-step formula 324 + 88 I_div + 88 I_p +
[40 + 120 I_cg] + 600 f_el, and the ncu traffic of each profiled kernel, which must
cover its algorithmic bytes on the 2.4M-particle scene."""
import pytest


def test_kernel_bytes_per_particle():
    import bench

    assert bench.ALG_BYTES["pressure_update"] == 56 and bench.ALG_BYTES["divergence_update"] == 56
    assert bench.ALG_BYTES["density_adv"] == 52 and bench.ALG_BYTES["density_change"] == 48
    # the density/factor pass that also takes the divergence solve's first density change
    assert bench.ALG_BYTES["density_factor"] == 52 and bench.ALG_BYTES["cg_matvec"] == 64
    assert bench.ALG_BYTES["cg_setup"] == 156 and bench.ALG_BYTES["density_change_np"] == 88


@pytest.mark.parametrize("iv,ip,icg,fel,implicit", [(0, 1, 0, 0.0, False), (2, 3, 4, 0.0, True), (1, 1, 1, 0.36, True)])
def test_step_bytes_formula(iv, ip, icg, fel, implicit):
    import bench

    want = 324 + 88 * iv + 88 * ip + (40 + 120 * icg if implicit else 0) + 600 * fel
    assert bench.step_bytes(iv, ip, icg, fel, implicit) == pytest.approx(want)


def test_ncu_traffic_covers_the_algorithmic_bytes():
    import bench

    n, entries = 2_400_002, bench.NCU_ENTRIES_2M  # the 2.4M scene and its list entries at the captured step
    assert bench.NCU_TRAFFIC_2M["build_lists"] >= bench.ALG_BYTES["build_lists"] * n + 4 * entries
    assert bench.NCU_TRAFFIC_2M["density_adv"] >= bench.ALG_BYTES["density_adv"] * n


def test_kernel_ids_follow_the_abi():
    """bench.py names nn_time_kernel's ids itself; they must be the header's NN_K_* values,
    each timed kernel with a byte count."""
    import bench
    from nonnewton_b200 import _abi

    assert bench.KERNEL_IDS == {
        "pressure_update": _abi.NN_K_PRESSURE_UPDATE, "density_adv": _abi.NN_K_DENSITY_ADV,
        "divergence_update": _abi.NN_K_DIVERGENCE_UPDATE, "density_change": _abi.NN_K_DENSITY_CHANGE,
        "density_factor": _abi.NN_K_DENSITY_FACTOR, "build_lists": _abi.NN_K_BUILD_LISTS,
        "cg_matvec": _abi.NN_K_CG_MATVEC, "nonpressure": _abi.NN_K_NONPRESSURE,
        "density_change_np": _abi.NN_K_DENSITY_CHANGE_NP, "cg_setup": _abi.NN_K_CG_SETUP}
    assert set(bench.KERNEL_IDS) <= set(bench.ALG_BYTES)
    assert max(bench.KERNEL_IDS.values()) == _abi.NN_K_COUNT - 1
