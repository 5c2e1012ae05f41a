"""Give-up path of the bounded wait in the kernels, on the GPU, through the C ABI.

The coarsest-level solve of an engine alone on the GPU runs as one persistent dataflow launch:
a task waits for the tasks of the fronts it reads.  The wait has a poll limit (about a second),
after which it sets an error word and the CTAs waiting after it return; the host reads the word
after the stream synchronises, clears it (with the solve's counters) and raises
TOPX_ERR_TIMEOUT.  topx_selftest_wait has one CTA wait for a counter that nothing raises (no
kernel faults, traps or spins without a limit), so the limit must run out.  The test then checks
the status and message, and that the same context still computes the V-cycle and the PCG solve
exactly as before and as the oracle does.
"""
import numpy as np
import pytest

from oracle import top3dxl_oracle as O

pytestmark = pytest.mark.gpu

TOPX_ERR_TIMEOUT = -7


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.fixture(scope="module")
def setup():
    from top3d_xl_b200 import Context
    vox = np.ones((12, 24, 12), bool)
    m = O.build_model(vox)
    ctx = Context("fp64")
    ctx.load_voxels(vox)
    x = np.random.default_rng(1).uniform(0.05, 1.0, m.levels[0].numElements)
    E = m.S.modulusMin + x ** m.S.SIMPpenalty * (m.S.modulus - m.S.modulusMin)
    ctx.set_moduli(E)
    ctx.assemble()
    sol = O.Solver(m)
    sol.assemble(E)
    r = np.random.default_rng(3).standard_normal(m.levels[0].numDOFs)
    yield dict(ctx=ctx, m=m, sol=sol, r=r, z0=ctx.vcycle(r), u0=ctx.pcg())
    ctx.close()


def test_wait_gives_up_and_context_stays_usable(setup):
    ctx = setup["ctx"]
    st = ctx.lib.topx_selftest_wait(ctx._h, 0)
    assert st == TOPX_ERR_TIMEOUT, (st, ctx.lib.topx_last_error(ctx._h))
    assert b"dependency wait" in ctx.lib.topx_last_error(ctx._h)
    # the error word was cleared: the factorisation, the persistent solve and the PCG run as before
    ctx.assemble()
    z = ctx.vcycle(setup["r"])
    assert _rel(z, setup["z0"]) < 1e-14
    assert _rel(z, setup["sol"].vcycle(setup["r"])) < 1e-11
    u, its = ctx.pcg()
    assert its == setup["u0"][1]
    assert _rel(u, setup["u0"][0]) < 1e-12


def test_other_selftest_cases_are_refused(setup):
    ctx = setup["ctx"]
    for which in (1, 7, -1):
        assert ctx.lib.topx_selftest_wait(ctx._h, which) == -1  # TOPX_ERR_ARG
