"""End-to-end FP64 parity of the optimisation loop against the golden oracle
histories (tests/golden/make_golden.py), through the C ABI.

Bar: identical PCG iteration counts (or within the oracle's own count spread under rounding
noise, `its_var`, where it has one); per-iteration compliance within 1e-9
relative while the reference algorithm's own rounding sensitivity allows it
(the golden files hold `env_c`, the spread of the oracle against itself with
1e-15 and 1e-12 relative noise in its coarse solve), and within 10x that envelope after;
final density within max(1e-6, 10*env_x) in the max norm.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _run(vox, cons, V0, nLoop, rMin, rHat, steps, precision="fp64", **settings):
    from top3d_xl_b200 import Context
    with Context(precision, **settings) as ctx:
        if isinstance(vox, str):
            ctx.load_topvoxel(vox)
        else:
            ctx.load_voxels(vox)
        cs = ctx.begin(cons, V0, nLoop, rMin, rHat)
        hist = []
        for _ in range(steps):
            r = ctx.step()
            if r is None:
                break
            hist.append(r)
        return cs, hist, ctx.density()


def _check(g, cs, hist, x):
    # cSolid is the compliance of iteration 0 (the fully solid design): the 1e-9 per-iteration bar
    assert abs(cs - g["cSolid"]) / g["cSolid"] < 1e-9
    c = np.array([h["c"] for h in hist])
    its = np.array([k for h in hist for k in h["its"]])
    assert len(c) == len(g["c"])
    # counts agree exactly, except where the oracle's own counts move under rounding noise
    var = g["its_var"] if "its_var" in g else np.zeros(len(g["its"]), np.int32)
    assert np.all(np.abs(its - g["its"]) <= var), (its, g["its"], var)
    rel = np.abs(c - g["c"]) / np.abs(g["c"])
    env = g["env_c"]
    bar = np.where(env < 1e-10, 1e-9, np.maximum(1e-9, 10 * env))
    assert np.all(rel < bar), (rel, bar)
    xbar = max(1e-6, 10 * float(g["env_x"]))
    if "x_idx" in g:  # large designs: a seeded sample of the density and the sum of all of it
        assert x.size == int(g["x_size"])
        assert np.max(np.abs(x[g["x_idx"]] - g["xPhys"])) < xbar
        assert abs(np.sum(x) - float(g["x_sum"])) < xbar * x.size
    else:
        assert np.max(np.abs(x - g["xPhys"])) < xbar


def test_config1_global_10_iterations():
    g = np.load(os.path.join(GOLD, "config1_global_10.npz"))
    cs, hist, x = _run(np.ones((25, 50, 25), bool), "GLOBAL", 0.12, 50, np.sqrt(3), 0.0, 10)
    _check(g, cs, hist, x)


def test_irregular_global_6_iterations():
    g = np.load(os.path.join(GOLD, "irregular_global_6.npz"))
    cs, hist, x = _run(g["vox"], "GLOBAL", 0.3, 50, np.sqrt(3), 0.0, 6)
    _check(g, cs, hist, x)


def test_small_local_6_iterations():
    g = np.load(os.path.join(GOLD, "small_local_6.npz"))
    cs, hist, x = _run(np.ones((12, 24, 12), bool), "LOCAL", 0.5, 300, np.sqrt(3), 6.0, 6)
    _check(g, cs, hist, x)


def test_generated_irregular_topvoxel_local_4_iterations(tmp_path):
    """The irregular-workload generator at reduced size, written as .TopVoxel and read back."""
    from top3d_xl_b200.workloads import IRREGULAR_SMALL, irregular_domain, write_topvoxel
    path = str(tmp_path / "irregular_small.TopVoxel")
    write_topvoxel(path, *irregular_domain(**IRREGULAR_SMALL))
    g = np.load(os.path.join(GOLD, "irregular_topvoxel_local_4.npz"))
    cs, hist, x = _run(path, "LOCAL", 0.5, 300, np.sqrt(3), 6.0, 4)
    _check(g, cs, hist, x)


def test_mixed_precision_error_vs_fp64():
    g = np.load(os.path.join(GOLD, "config1_global_10.npz"))
    cs, hist, x = _run(np.ones((25, 50, 25), bool), "GLOBAL", 0.12, 50, np.sqrt(3), 0.0, 10, "mixed")
    c = np.array([h["c"] for h in hist])
    rel = np.abs(c - g["c"]) / np.abs(g["c"])
    assert rel.max() < 1e-5, rel


def _two_case_file(tmp_path):
    from top3d_xl_b200.workloads import two_load_case_model, write_topvoxel
    vox, fixed, loads, passive = two_load_case_model()
    path = str(tmp_path / "two_case_passive.TopVoxel")
    write_topvoxel(path, vox, fixed, loads[0], passive=passive, additional_loads=loads[1:])
    return path


# specifyPassiveRegions_ of the two-load-case fixtures (tests/golden/make_golden.py)
TWO_CASE_PASSIVE_REGIONS = (0, 0, 1)


def test_two_load_cases_and_passive_elements_global_10_iterations(tmp_path):
    """Two load cases (one PCG per case and the weighted compliance, TX:121, 585-597) and passive
    elements from the file and from a layer around the fixations, held at 1 by OC (TX:151, 159)."""
    g = np.load(os.path.join(GOLD, "two_case_passive_global_10.npz"))
    cs, hist, x = _run(_two_case_file(tmp_path), "GLOBAL", 0.3, 50, np.sqrt(3), 0.0, 10,
                       specifyPassiveRegions=TWO_CASE_PASSIVE_REGIONS)
    assert all(len(h["its"]) == 2 for h in hist)
    _check(g, cs, hist, x)


def test_two_load_cases_and_passive_elements_local_10_iterations(tmp_path):
    """The same model under LOCAL: passive elements outside the MMA variables and at 1 after the
    Heaviside projection (TX:352-369, 381)."""
    g = np.load(os.path.join(GOLD, "two_case_passive_local_10.npz"))
    cs, hist, x = _run(_two_case_file(tmp_path), "LOCAL", 0.5, 300, np.sqrt(3), 4.0, 10,
                       specifyPassiveRegions=TWO_CASE_PASSIVE_REGIONS)
    _check(g, cs, hist, x)


def test_local_past_the_beta_doubling_44_iterations():
    """LOCAL on a small cuboid for 44 iterations: beta doubles at loopbeta = 40 (TX:375-379), so
    iterations 40-44 run the Heaviside projection and MMA at beta = 2."""
    g = np.load(os.path.join(GOLD, "small_local_beta_44.npz"))
    assert g["beta"][38] == 1.0 and g["beta"][39] == 2.0
    cs, hist, x = _run(np.ones((12, 24, 12), bool), "LOCAL", 0.5, 300, np.sqrt(3), 6.0, 44)
    _check(g, cs, hist, x)


def test_config2a_demo_cuboid_global_10_iterations():
    """The reference's demo size, TOP3D_XL(true(50,100,50),'GLOBAL',0.12,50,sqrt(3)): 250,000
    elements, 10 iterations; the final density is compared at a seeded sample of 20,000 elements."""
    g = np.load(os.path.join(GOLD, "config2a_global_10.npz"))
    cs, hist, x = _run(np.ones((50, 100, 50), bool), "GLOBAL", 0.12, 50, np.sqrt(3), 0.0, 10)
    _check(g, cs, hist, x)


def test_config2b_demo_cuboid_local_42_iterations():
    """The demo size under LOCAL with rHat 6 (TOP3D_XL(true(50,100,50),'LOCAL',0.5,300,sqrt(3),6)):
    42 iterations, past the beta doubling at loopbeta = 40 (TX:375-379)."""
    g = np.load(os.path.join(GOLD, "config2b_local_42.npz"))
    cs, hist, x = _run(np.ones((50, 100, 50), bool), "LOCAL", 0.5, 300, np.sqrt(3), 6.0, 42)
    _check(g, cs, hist, x)


def test_config3_large_cuboid_global_2_iterations():
    """The benchmarked cuboid, TOP3D_XL(true(128,256,128),'GLOBAL',0.12,50,sqrt(3)): 4,194,304
    elements, cSolid and 2 iterations against the oracle (an oracle iteration takes minutes)."""
    g = np.load(os.path.join(GOLD, "config3_global_2.npz"))
    cs, hist, x = _run(np.ones((128, 256, 128), bool), "GLOBAL", 0.12, 50, np.sqrt(3), 0.0, 2)
    _check(g, cs, hist, x)
