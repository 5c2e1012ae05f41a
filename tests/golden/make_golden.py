"""Generate the golden fixtures of tests/golden/ from the FP64 oracle.

    python tests/golden/make_golden.py [case ...]     (no case: the small cases; "all": every case)

Cases: config1, small_local, irregular_global, irregular_topvoxel_local (the small set);
two_case_passive_global, two_case_passive_local, small_local_beta; config2a, config2b,
config3 (the reference's demo and large cuboids: minutes to an hour of CPU each).

The reference (TOP3D_XL.m, MATLAB) cannot run in this build environment, so
these vectors are outputs of the oracle restatement (oracle/top3dxl_oracle.py);
they freeze its per-iteration history so that GPU parity tests on any machine
compare against the same numbers.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import top3dxl_oracle as O  # noqa: E402
from top3d_xl_b200.workloads import (IRREGULAR_SMALL, irregular_domain, two_load_case_model,  # noqa: E402
                                     write_topvoxel)

# Large designs keep a seeded sample of their final density (the bar is a max norm, so a
# sample of 20,000 elements tests it at those elements) plus its sum.
X_SAMPLE = 20000


def noise_envelope(run, ref, seeds=(1, 2, 3, 4, 5, 6), eps=(1e-15, 1e-12)):
    """Per-iteration spread of the oracle against itself when its coarse solve carries
    random relative noise of each level in `eps`: a few ulps, and the ~1e-12 by which two
    exact factorisations of the coarsest matrix (condition ~1e4) differ in FP64.  This is
    the rounding sensitivity of the reference algorithm, which bounds how closely any
    re-implementation can track it; past the first iterations it saturates near 1e-6 on
    irregular domains, whatever the noise level.  `its_var` is the largest change of each PCG
    iteration count under the same noise (a count can move once the design has)."""
    orig = O.Solver.coarse_solve
    env_c = np.zeros(len(ref["c"]))
    env_x = 0.0
    ref_its = np.asarray(ref["its"])
    its_var = np.zeros(ref_its.size, dtype=np.int32)
    try:
        for sd, ep in [(s, e) for e in eps for s in seeds]:
            rng = np.random.default_rng(sd)

            def noisy(self, r, _o=orig, _rng=rng, _ep=ep):
                z = _o(self, r)
                return z * (1 + _ep * _rng.standard_normal(z.shape))

            O.Solver.coarse_solve = noisy
            h = run()
            n = min(len(h["c"]), len(ref["c"]))
            env_c[:n] = np.maximum(env_c[:n], np.abs(np.array(h["c"][:n]) - ref["c"][:n]) / np.abs(ref["c"][:n]))
            env_x = max(env_x, float(np.max(np.abs(h["xPhys"] - ref["xPhys"]))))
            its = np.asarray(h["its"])
            k = min(its.size, ref_its.size)
            its_var[:k] = np.maximum(its_var[:k], np.abs(its[:k] - ref_its[:k]))
    finally:
        O.Solver.coarse_solve = orig
    return dict(env_c=env_c, env_x=env_x, its_var=its_var)


def save(name, hist, extra=None, sample=False):
    d = dict(cSolid=hist["cSolid"], c=np.array(hist["c"]), its=np.array(hist["its"], dtype=np.int32),
             sharp=np.array(hist["sharp"]), vol=np.array(hist["vol"]), cons=np.array(hist["cons"]),
             change=np.array(hist["change"]), xPhys=hist["xPhys"], loops=hist["loops"])
    if "beta" in hist:
        d["beta"] = np.array(hist["beta"])
    if sample:
        x = hist["xPhys"]
        idx = np.sort(np.random.default_rng(0).choice(x.size, size=min(X_SAMPLE, x.size), replace=False))
        d.update(xPhys=x[idx], x_idx=idx.astype(np.int64), x_sum=float(np.sum(x)), x_size=x.size)
    if extra:
        d.update(extra)
    np.savez_compressed(os.path.join(HERE, name), **d)
    print(name, "c:", d["c"][:3], "its:", d["its"][:5], "env_c:", d.get("env_c"), "env_x:", d.get("env_x"))


def _golden(name, run, seeds=(1, 2, 3, 4, 5, 6), eps=(1e-15, 1e-12), sample=False, extra=None):
    h = run()
    h["c"] = np.array(h["c"])
    env = noise_envelope(run, h, seeds=seeds, eps=eps)
    if extra:
        env.update(extra)
    save(name, h, env, sample=sample)


def two_case_passive_file():
    """The two-load-case model with passive elements (top3d_xl_b200.workloads.two_load_case_model)
    as a .TopVoxel file in a temporary folder."""
    vox, fixed, loads, passive = two_load_case_model()
    path = os.path.join(tempfile.mkdtemp(), "two_case_passive.TopVoxel")
    write_topvoxel(path, vox, fixed, loads[0], passive=passive, additional_loads=loads[1:])
    return path


# specifyPassiveRegions_ of the two-load-case fixtures: one layer of passive elements around
# the fixed nodes, besides the file's own passive block
TWO_CASE_PASSIVE_REGIONS = (0, 0, 1)


def case_config1():
    # the small cuboid case: TOP3D_XL(true(25,50,25),'GLOBAL',0.12,50,sqrt(3)), first 10 iterations
    _golden("config1_global_10.npz",
            lambda: O.run_global(np.ones((25, 50, 25), bool), 0.12, 50, np.sqrt(3), max_loops=10))


def case_small_local():
    # LOCAL porous infill on a small cuboid, first 6 iterations (MMA + Heaviside + two PDE filters)
    _golden("small_local_6.npz",
            lambda: O.run_local(np.ones((12, 24, 12), bool), 0.5, 300, np.sqrt(3), 6.0, max_loops=6))


def case_irregular_global():
    # GLOBAL on a seeded irregular domain (solid x-faces carry the built-in BCs)
    rng = np.random.default_rng(11)
    vox = rng.random((14, 30, 12)) < 0.85
    vox[:, 0, :] = True
    vox[:, -1, :] = True
    _golden("irregular_global_6.npz", lambda: O.run_global(vox, 0.3, 50, np.sqrt(3), max_loops=6),
            extra=dict(vox=vox))


def case_irregular_topvoxel_local():
    # LOCAL on a small generated irregular domain read from a .TopVoxel file (random surface
    # loads, fixed lowest layer): the irregular-workload generator at reduced size
    path = os.path.join(tempfile.mkdtemp(), "irregular_small.TopVoxel")
    write_topvoxel(path, *irregular_domain(**IRREGULAR_SMALL))
    _golden("irregular_topvoxel_local_4.npz", lambda: O.run_local(path, 0.5, 300, np.sqrt(3), 6.0, max_loops=4))


def _two_case_settings():
    S = O.Settings()
    S.specifyPassiveRegions = TWO_CASE_PASSIVE_REGIONS
    return S


def case_two_case_passive_global():
    # two load cases (the PCG loop over F's columns, TX:121, and the weighted compliance, TX:597)
    # and passive elements pinned to 1 in the OC update (TX:151, 159)
    path = two_case_passive_file()
    _golden("two_case_passive_global_10.npz",
            lambda: O.run_global(path, 0.3, 50, np.sqrt(3), S=_two_case_settings(), max_loops=10))


def case_two_case_passive_local():
    # the same model under LOCAL: passive elements outside the MMA variables and set to 1 after
    # the Heaviside projection (TX:352-369, 381)
    path = two_case_passive_file()
    _golden("two_case_passive_local_10.npz",
            lambda: O.run_local(path, 0.5, 300, np.sqrt(3), 4.0, S=_two_case_settings(), max_loops=10))


def case_small_local_beta():
    # LOCAL past the first beta doubling (loopbeta >= 40 doubles beta, TX:375-379): 44 iterations,
    # beta 2 from iteration 40 on
    _golden("small_local_beta_44.npz",
            lambda: O.run_local(np.ones((12, 24, 12), bool), 0.5, 300, np.sqrt(3), 6.0, max_loops=44))


def case_config2a():
    # the reference's demo size, GLOBAL: TOP3D_XL(true(50,100,50),'GLOBAL',0.12,50,sqrt(3)), 10 iterations
    _golden("config2a_global_10.npz",
            lambda: O.run_global(np.ones((50, 100, 50), bool), 0.12, 50, np.sqrt(3), max_loops=10),
            seeds=(1, 2), sample=True)


def case_config2b():
    # the demo size, LOCAL with rHat 6: 42 iterations, past the beta doubling at iteration 40
    _golden("config2b_local_42.npz",
            lambda: O.run_local(np.ones((50, 100, 50), bool), 0.5, 300, np.sqrt(3), 6.0, max_loops=42),
            seeds=(1, 2), sample=True)


def case_config3():
    # the large cuboid: TOP3D_XL(true(128,256,128),'GLOBAL',0.12,50,sqrt(3)), cSolid and 2 iterations
    _golden("config3_global_2.npz",
            lambda: O.run_global(np.ones((128, 256, 128), bool), 0.12, 50, np.sqrt(3), max_loops=2),
            seeds=(1, 2), eps=(1e-12,), sample=True)


SMALL = ["config1", "small_local", "irregular_global", "irregular_topvoxel_local"]
ALL = SMALL + ["two_case_passive_global", "two_case_passive_local", "small_local_beta", "config2a", "config2b",
               "config3"]


def main(argv):
    cases = argv or SMALL
    if cases == ["all"]:
        cases = ALL
    for c in cases:
        if c not in ALL:
            raise SystemExit("unknown case %r; cases: %s" % (c, ", ".join(ALL)))
    for c in cases:
        globals()["case_" + c]()


if __name__ == "__main__":
    main(sys.argv[1:])
