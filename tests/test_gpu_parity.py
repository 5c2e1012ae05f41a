"""GPU-vs-oracle parity of the solver building blocks, called through the C ABI.

Sizes are chosen so the FP64 oracle finishes in seconds.  Tolerances: the
native path computes the same FP64 arithmetic in a different summation order
(node-centric gathers instead of accumarray scatters, a nested-dissection
factorisation instead of a permuted sparse Cholesky), so single operators agree
to ~1e-13 relative and iterative solves to ~1e-9.
"""
import numpy as np
import pytest

from oracle import top3dxl_oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.fixture(scope="module", params=["cuboid", "irregular", "u_shape"])
def setup(request):
    # u_shape: most (x, z) columns are void, so the level-1 passes run over the domain's tiles
    # and chunks only: K*u tiles with part of their z-chunk present, the last-row kernel's row
    # tiles (ny = 32), the filter's tiles, the restriction's column mask
    from top3d_xl_b200 import Context
    if request.param == "cuboid":
        vox = np.ones((12, 24, 12), bool)
    elif request.param == "u_shape":
        vox = np.zeros((32, 64, 32), bool)
        vox[:, :4, :] = True
        vox[:, -4:, :] = True
        vox[:, :, :4] = True
    else:
        rng = np.random.default_rng(5)
        vox = rng.random((13, 27, 11)) < 0.75
        vox[:, 0, :] = True
        vox[:, -1, :] = True
    m = O.build_model(vox)
    ctx = Context("fp64")
    ctx.load_voxels(vox)
    rng = np.random.default_rng(1)
    x = rng.uniform(0.05, 1.0, m.levels[0].numElements)
    S = m.S
    E = S.modulusMin + x ** S.SIMPpenalty * (S.modulus - S.modulusMin)
    sol = O.Solver(m)
    sol.assemble(E)
    ctx.set_moduli(E)
    ctx.assemble()
    yield dict(m=m, ctx=ctx, sol=sol, E=E, x=x, vox=vox, kind=request.param)
    ctx.close()


def test_ku(setup):
    m, ctx, sol = setup["m"], setup["ctx"], setup["sol"]
    u = np.random.default_rng(2).standard_normal(m.levels[0].numDOFs)
    y = ctx.ku(u)
    assert _rel(y, sol.ku(u)) < 1e-13


def test_diagonals(setup):
    m, ctx = setup["m"], setup["ctx"]
    for l in range(1, m.numLevels):
        assert _rel(ctx.diag(l), m.levels[l - 1].diagK) < 1e-13, l


def test_vcycle(setup):
    m, ctx, sol = setup["m"], setup["ctx"], setup["sol"]
    r = np.random.default_rng(3).standard_normal(m.levels[0].numDOFs)
    # the U's prongs are cantilevers: its coarsest matrix is ill-conditioned (the V-cycle of a unit
    # residual reaches 1e4), and the two factorisations' rounding differs by that much more
    bar = 1e-10 if setup["kind"] == "u_shape" else 1e-11
    assert _rel(ctx.vcycle(r), sol.vcycle(r)) < bar


def test_pcg(setup):
    # the tol-1e-3 PCG amplifies rounding ~1e8 (tests/test_oracle.py): on this
    # high-contrast random design the solution agrees to ~1e-8 and f'u to ~1e-9
    m, ctx, sol = setup["m"], setup["ctx"], setup["sol"]
    u, its = ctx.pcg()
    uo, itso, _ = O.pcg(sol.ku, sol.vcycle, m.F[:, 0], m.S.tol, m.S.maxIT)
    f = m.F[:, 0]
    if setup["kind"] == "u_shape":
        # 88 iterations of a tol-1e-3 PCG on the ill-conditioned U: the stopping test may fall one
        # iteration apart, and the solutions then differ by that last step
        assert abs(its - itso) <= 1
        assert abs(f @ u - f @ uo) / abs(f @ uo) < 1e-5
        return
    assert its == itso
    assert _rel(u, uo) < 1e-6
    assert abs(f @ u - f @ uo) / abs(f @ uo) < 1e-8


def test_compliance(setup):
    m, ctx, sol = setup["m"], setup["ctx"], setup["sol"]
    U = np.random.default_rng(4).standard_normal((m.levels[0].numDOFs, 1))
    assert _rel(ctx.unit_compliance(U), O.unit_compliance(m, U)) < 1e-13


@pytest.mark.parametrize("rmin", [np.sqrt(3), 6.0])
def test_filter(setup, rmin):
    m, ctx = setup["m"], setup["ctx"]
    src = np.random.default_rng(6).uniform(0, 1, m.levels[0].numElements)
    out, its = ctx.filter(rmin, src)
    flt = O.PDEFilter(m, rmin, m.S)
    ref = flt(src)
    assert its == flt.last_its
    assert _rel(out, ref) < 1e-10


@pytest.fixture(scope="module")
def mixed_setup():
    from top3d_xl_b200 import Context
    vox = np.ones((12, 24, 12), bool)
    m = O.build_model(vox)
    ctx = Context("mixed")
    ctx.load_voxels(vox)
    x = np.random.default_rng(1).uniform(0.05, 1.0, m.levels[0].numElements)
    S = m.S
    E = S.modulusMin + x ** S.SIMPpenalty * (S.modulus - S.modulusMin)
    sol = O.Solver(m)
    sol.assemble(E)
    ctx.set_moduli(E)
    ctx.assemble()
    yield dict(m=m, ctx=ctx, sol=sol)
    ctx.close()


def test_mixed_vcycle_is_fp32_accurate(mixed_setup):
    m, ctx, sol = mixed_setup["m"], mixed_setup["ctx"], mixed_setup["sol"]
    r = np.random.default_rng(3).standard_normal(m.levels[0].numDOFs)
    assert _rel(ctx.vcycle(r), sol.vcycle(r)) < 1e-5


def test_mixed_pcg_keeps_fp64_compliance(mixed_setup):
    # FP32 noise confined to the preconditioner keeps CG's Galerkin property
    m, ctx, sol = mixed_setup["m"], mixed_setup["ctx"], mixed_setup["sol"]
    u, its = ctx.pcg()
    uo, itso, _ = O.pcg(sol.ku, sol.vcycle, m.F[:, 0], m.S.tol, m.S.maxIT)
    f = m.F[:, 0]
    assert abs(its - itso) <= 1
    assert abs(f @ u - f @ uo) / abs(f @ uo) < 1e-6
    assert np.linalg.norm(f - ctx.ku(u)) / np.linalg.norm(f) < m.S.tol


def test_filter_preserves_constants(setup):
    m, ctx = setup["m"], setup["ctx"]
    out, _ = ctx.filter(np.sqrt(3), np.ones(m.levels[0].numElements))
    assert np.max(np.abs(out - 1.0)) < 1e-3


@pytest.mark.parametrize("shape", [(64, 96, 64), (112, 136, 112)])
def test_vcycle_with_large_coarsest_slabs(shape):
    # coarsest grids of 9 x 13 x 9 and 15 x 18 x 15 nodes: elimination trees of several levels,
    # fronts of several 64-wide tiles (Gauss-Jordan steps over many tile tasks)
    from top3d_xl_b200 import Context
    vox = np.ones(shape, bool)
    m = O.build_model(vox)
    x = np.random.default_rng(4).uniform(0.3, 1.0, m.levels[0].numElements)
    S = m.S
    E = S.modulusMin + x ** S.SIMPpenalty * (S.modulus - S.modulusMin)
    sol = O.Solver(m)
    sol.assemble(E)
    with Context("fp64") as ctx:
        ctx.load_voxels(vox)
        ctx.set_moduli(E)
        ctx.assemble()
        for seed in (3, 5):  # two solves with the same factors
            r = np.random.default_rng(seed).standard_normal(m.levels[0].numDOFs)
            assert _rel(ctx.vcycle(r), sol.vcycle(r)) < 1e-10
        ctx.assemble()  # a second factorisation through the same scratch and control words
        r = np.random.default_rng(6).standard_normal(m.levels[0].numDOFs)
        assert _rel(ctx.vcycle(r), sol.vcycle(r)) < 1e-10


@pytest.mark.parametrize("kind", ["cuboid", "irregular", "u_shape"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_persistent_coarse_solve_matches_level_launches(kind, precision):
    # the coarsest solve as one dataflow launch (tasks wait for their children's or an ancestor's
    # counters) and as one launch per tree level run the same tasks with the same summation
    # order: the V-cycles agree bit for bit, over repeated solves (the counters are re-armed by
    # each launch) and after a second factorisation.  The U-shaped domain's tree has fronts whose
    # separator holds no present node (nothing eliminated, update DOFs around it): their
    # children's solves up and down must wait past them, for the nearest eliminating ancestor.
    from top3d_xl_b200 import Context
    if kind == "cuboid":
        vox = np.ones((64, 128, 64), bool)
    elif kind == "irregular":
        vox = np.random.default_rng(12).random((64, 128, 64)) < 0.8
        vox[:, 0, :] = True
        vox[:, -1, :] = True
    else:
        vox = np.zeros((64, 160, 64), bool)
        vox[:, :8, :] = True
        vox[:, -8:, :] = True
        vox[:, :, :8] = True
    E = 1.0 + np.random.default_rng(11).uniform(0.0, 1.0, int(vox.sum())) ** 3
    outs = []
    for coop in (1, 0):
        with Context(precision, coarse_coop=coop) as ctx:
            ctx.load_voxels(vox)
            ctx.set_moduli(E)
            ctx.assemble()
            res = []
            for k, seed in enumerate((21, 22, 23)):
                if k == 2:
                    ctx.assemble()
                res.append(ctx.vcycle(np.random.default_rng(seed).standard_normal(ctx.numDOFs)))
            outs.append(res)
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("kind", ["cuboid", "irregular"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ku_and_pcg_with_last_row_kernel(kind, precision):
    # y extent a multiple of the K*u tile height (32 nodes): the tile kernel stops one node row
    # short and the grid's last row y = ny runs in its own kernel, in both the plain operator and
    # the PCG step (direction update, stored direction, p'q); fixed DOFs lie on that row too
    from top3d_xl_b200 import Context
    if kind == "cuboid":
        vox = np.ones((32, 20, 12), bool)
    else:
        rng = np.random.default_rng(7)
        vox = rng.random((64, 18, 10)) < 0.8
        vox[:, 0, :] = True
        vox[:, -1, :] = True
    m = O.build_model(vox)
    assert m.levels[0].resY % 32 == 0
    x = np.random.default_rng(8).uniform(0.05, 1.0, m.levels[0].numElements)
    S = m.S
    E = S.modulusMin + x ** S.SIMPpenalty * (S.modulus - S.modulusMin)
    sol = O.Solver(m)
    sol.assemble(E)
    with Context(precision) as ctx:
        ctx.load_voxels(vox)
        ctx.set_moduli(E)
        ctx.assemble()
        u = np.random.default_rng(9).standard_normal(m.levels[0].numDOFs)
        assert _rel(ctx.ku(u), sol.ku(u)) < 1e-13
        up, its = ctx.pcg()
    uo, itso, _ = O.pcg(sol.ku, sol.vcycle, m.F[:, 0], m.S.tol, m.S.maxIT)
    f = m.F[:, 0]
    if precision == "fp64":
        assert its == itso
        assert abs(f @ up - f @ uo) / abs(f @ uo) < 1e-8
    else:
        assert abs(its - itso) <= 1
        assert abs(f @ up - f @ uo) / abs(f @ uo) < 1e-6


@pytest.mark.parametrize("kind", ["cuboid", "irregular"])
def test_standard_vcycle(kind):
    # typeVcycle 'Standard' (TX:758-763, 772-777): level-1 and coarse-level K*u inside the
    # V-cycle.  The operator matches at the default omega; PCG runs at omega 0.4, where the cycle
    # is positive definite (at 0.6 it is indefinite and PCG stalls, in the oracle as well)
    from top3d_xl_b200 import Context
    if kind == "cuboid":
        vox = np.ones((12, 24, 12), bool)
    else:
        rng = np.random.default_rng(5)
        vox = rng.random((13, 27, 11)) < 0.75
        vox[:, 0, :] = True
        vox[:, -1, :] = True
    m = O.build_model(vox)
    x = np.random.default_rng(1).uniform(0.05, 1.0, m.levels[0].numElements)
    S = m.S
    E = S.modulusMin + x ** S.SIMPpenalty * (S.modulus - S.modulusMin)
    sol = O.Solver(m)
    sol.assemble(E)
    m.S.typeVcycle = "Standard"
    r = np.random.default_rng(3).standard_normal(m.levels[0].numDOFs)
    with Context("fp64", typeVcycle="Standard") as ctx:
        ctx.load_voxels(vox)
        ctx.set_moduli(E)
        ctx.assemble()
        assert _rel(ctx.vcycle(r), sol.vcycle(r)) < 1e-10
    m.S.weightFactorJacobi = 0.4
    with Context("fp64", typeVcycle="Standard", weightFactorJacobi=0.4) as ctx:
        ctx.load_voxels(vox)
        ctx.set_moduli(E)
        ctx.assemble()
        assert _rel(ctx.vcycle(r), sol.vcycle(r)) < 1e-10
        u, its = ctx.pcg()
    uo, itso, _ = O.pcg(sol.ku, sol.vcycle, m.F[:, 0], m.S.tol, m.S.maxIT)
    f = m.F[:, 0]
    assert abs(its - itso) <= 1
    assert abs(f @ u - f @ uo) / abs(f @ uo) < 1e-8
