"""C ABI of libtopx.so on CPU: every symbol of include/topx.h is exported, the
host-side model (discretisation, hierarchy, BCs) is bit-exact with the oracle's
1-based reference numbering, and errors come back as status codes."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import top3dxl_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    txt = open(os.path.join(ROOT, "include", "topx.h")).read()
    return sorted(set(re.findall(r"\b(?:topx_status|const char\*)\s+(topx_\w+)\s*\(", txt)))


def test_library_exports_every_header_symbol():
    from top3d_xl_b200 import _lib
    lib = _lib.load()
    syms = _header_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(lib, s), s
        assert s in _lib.SIGNATURES, s


def _compare(vox):
    from top3d_xl_b200 import Context
    m = O.build_model(vox)
    ctx = Context()
    info = ctx.load_voxels(vox)
    assert info.numLevels == m.numLevels
    for l in range(1, m.numLevels + 1):
        lv = m.levels[l - 1]
        checks = [("ENODMAT", lv.eNodMat.ravel()), ("ELEMAPBACK", lv.eleMapBack), ("NODMAPBACK", lv.nodMapBack),
                  ("NODESONBOUNDARY", lv.nodesOnBoundary)]
        if l == 1:
            checks += [("ELEMENTSONBOUNDARY", lv.elementsOnBoundary), ("FIXEDDOFS", m.fixedDOFs.astype(np.int32)),
                       ("MAPUNIQUEKES", m.mapUniqueKes)]
        else:
            checks += [("ELEMENTUPWARDMAP", lv.elementUpwardMap.ravel()), ("TRANSFERMAT", lv.transferMat.T.ravel()),
                       ("SOLIDNODEMAP", lv.solidNodeMapCoarser2Finer)]
            assert np.array_equal(ctx.transfer_coeffi(l), lv.transferMatCoeffi)
        if l == 2:
            checks.append(("ISTHISELE2NDLEVEL", m.isThisEle2ndLevel))
        for name, ref in checks:
            got = ctx.index_array(l, name)
            assert got.dtype == np.int32 and np.array_equal(got, ref.astype(np.int32)), (l, name)
    assert np.max(np.abs(ctx.ke() - m.levels[0].Ke)) < 1e-15
    assert np.array_equal(ctx.load_vector(0), m.F[:, 0])
    ctx.close()


def test_indexing_bit_exact_config1():
    _compare(np.ones((25, 50, 25), bool))


def test_indexing_bit_exact_odd_cuboid():
    _compare(np.ones((13, 29, 11), bool))


def test_indexing_bit_exact_irregular():
    rng = np.random.default_rng(4)
    vox = rng.random((18, 37, 15)) < 0.7
    vox[:, 0, :] = True
    vox[:, -1, :] = True
    _compare(vox)


def _write_topvoxel(path, vox, fixed, loads, passive=(), density=False):
    ny, nx, nz = vox.shape
    solid = np.flatnonzero(vox.ravel(order="F")) + 1
    with open(path, "w") as fh:
        fh.write("# TOP3D_XL voxel model\nVersion: 1.0\nResolution: %d %d %d\n" % (nx, ny, nz))
        fh.write("Density included: %d\nSolid voxels: %d\n" % (1 if density else 0, solid.size))
        for s in solid:
            fh.write("%d 1.0\n" % s if density else "%d\n" % s)
        fh.write("Passive elements: %d\n" % len(passive))
        for p in passive:
            fh.write("%d\n" % p)
        fh.write("Fixations: %d\n" % len(fixed))
        for n, a, b, c in fixed:
            fh.write("%d %d %d %d\n" % (n, a, b, c))
        fh.write("Loads: %d\n" % len(loads[0]))
        for n, a, b, c in loads[0]:
            fh.write("%d %.17g %.17g %.17g\n" % (n, a, b, c))
        fh.write("Additional Loads: %d\n" % (len(loads) - 1))
        for k, ld in enumerate(loads[1:], start=2):
            fh.write("Loads: %d %d\n" % (len(ld), k))
            for n, a, b, c in ld:
                fh.write("%d %.17g %.17g %.17g\n" % (n, a, b, c))


def test_topvoxel_reader_matches_oracle(tmp_path):
    from top3d_xl_b200 import Context
    rng = np.random.default_rng(9)
    ny, nx, nz = 10, 21, 9
    vox = np.ones((ny, nx, nz), bool)
    vox[rng.random(vox.shape) < 0.15] = False
    vox[:, :2, :] = True
    nny, nnx = ny + 1, nx + 1
    fixed = [(iy + 1 + nny * nnx * iz, 1, 1, 1) for iz in range(nz + 1) for iy in range(nny)]
    loads = [[(1 + iy + nny * nx + nny * nnx * nz, 0.0, 0.0, -1.0 / 3) for iy in range(3)]]
    vox[:, -1, -1] = True
    path = str(tmp_path / "m.TopVoxel")
    _write_topvoxel(path, vox, fixed, loads, passive=[5, 17], density=True)
    m = O.Model()
    m.load_topvoxel(path)
    m.apply_boundary_condition()
    m.setup()
    ctx = Context()
    info = ctx.load_topvoxel(path)
    assert info.numPassive == len(m.passiveElements)
    assert np.array_equal(ctx.index_array(1, "ENODMAT"), m.levels[0].eNodMat.ravel())
    assert np.array_equal(ctx.index_array(1, "FIXEDDOFS"), m.fixedDOFs.astype(np.int32))
    assert np.array_equal(ctx.load_vector(0), m.F[:, 0])
    ctx.close()


def test_set_bc_matches_the_same_topvoxel_file(tmp_path):
    # topx_set_bc on a voxel array gives the model that a .TopVoxel file with the same voxels and
    # boundary conditions gives: fixings with partial directions, repeated nodes (first row
    # counts), two load cases
    from top3d_xl_b200 import Context, TopxError
    rng = np.random.default_rng(4)
    ny, nx, nz = 9, 18, 8
    vox = np.ones((ny, nx, nz), bool)
    vox[rng.random(vox.shape) < 0.1] = False
    vox[:, :2, :] = True
    vox[:, -1, :] = True
    vox[0:3, 5:8, 0:3] = False  # node (y 1, x 6, z 1) touches void voxels only
    nny, nnx = ny + 1, nx + 1
    fixed = [(iy + 1 + nny * nnx * iz, 1, 1, int(iz % 2 == 0)) for iz in range(nz + 1) for iy in range(nny)]
    fixed.append((1, 0, 0, 0))  # repeated node: ignored
    case1 = [(1 + iy + nny * nx + nny * nnx * 4, 0.0, 0.0, -0.25) for iy in range(4)]
    case2 = [(1 + iy + nny * nx + nny * nnx * 6, 0.0, 0.3, 0.0) for iy in range(3)]
    path = str(tmp_path / "bc.TopVoxel")
    _write_topvoxel(path, vox, fixed, [case1, case2])
    a = Context()
    a.load_topvoxel(path)
    b = Context()
    b.load_voxels(vox)
    info = b.set_bc(fixed, [r + (1,) for r in case1] + [r + (2,) for r in case2])
    assert info.numLoadCases == 2
    for name in ("ENODMAT", "FIXEDDOFS", "MAPUNIQUEKES"):
        assert np.array_equal(a.index_array(1, name), b.index_array(1, name)), name
    for lc in (0, 1):
        assert np.array_equal(a.load_vector(lc), b.load_vector(lc))
    m = O.Model()
    m.load_topvoxel(path)
    m.apply_boundary_condition()
    m.setup()
    assert np.array_equal(b.index_array(1, "FIXEDDOFS"), m.fixedDOFs.astype(np.int32))
    assert np.array_equal(b.load_vector(1), m.F[:, 1])
    with pytest.raises(TopxError) as e:  # node id outside the grid
        b.set_bc([(0, 1, 1, 1)], case1)
    assert "TOPX_ERR_ARG" in str(e.value)
    with pytest.raises(TopxError) as e:  # a node outside the solid model
        b.set_bc(fixed + [(1 + 1 + nny * (6 + nnx * 1), 1, 1, 1)], case1)
    assert "TOPX_ERR_MODEL" in str(e.value)
    with pytest.raises(TopxError) as e:  # no loads
        b.set_bc(fixed, np.empty((0, 5)))
    assert "TOPX_ERR_MODEL" in str(e.value)
    # more load cases than a history row holds (TOPX_MAX_LOAD_CASES = 8) are refused, not truncated
    many = [(1 + iy + nny * nx + nny * nnx * 4, 0.0, 0.0, -0.25, lc) for lc in range(1, 10) for iy in range(2)]
    assert b.set_bc(fixed, many[:16]).numLoadCases == 8
    with pytest.raises(TopxError) as e:
        b.set_bc(fixed, many)
    assert "TOPX_ERR_MODEL" in str(e.value) and "load cases" in str(e.value)
    path9 = str(tmp_path / "bc9.TopVoxel")
    _write_topvoxel(path9, vox, fixed, [[r[:4] for r in many if r[4] == lc] for lc in range(1, 10)])
    with pytest.raises(TopxError) as e:
        a.load_topvoxel(path9)
    assert "TOPX_ERR_MODEL" in str(e.value) and "load cases" in str(e.value)
    a.close()
    b.close()


def test_passive_layers_match_oracle(tmp_path):
    # specifyPassiveRegions_ (TopOpti_SetPassiveElements, TX:1511-1574): boundary layers on a cuboid;
    # layers near loads and fixations on a model whose BC node ids lie within the boundary-node
    # list (the reference indexes that list with them); the built-in cuboid's fixed node ids run
    # past it, which is the reference's index error
    from top3d_xl_b200 import Context, TopxError
    vox = np.ones((8, 16, 8), bool)
    S = O.Settings()
    S.specifyPassiveRegions = (2, 0, 0)
    m = O.build_model(vox, S)
    with Context(specifyPassiveRegions=(2, 0, 0)) as ctx:
        info = ctx.load_voxels(vox)
        assert info.numPassive == len(m.passiveElements) > 0
        assert np.array_equal(ctx.index_array(1, "PASSIVEELEMENTS"), m.passiveElements.astype(np.int32))
    ny, nx, nz = 6, 12, 6
    v2 = np.ones((ny, nx, nz), bool)
    nny = ny + 1
    fixed = [(iy + 1, 1, 1, 1) for iy in range(nny)]            # x = 0, z = 0 column
    loads = [[(nny + iy + 1, 0.0, 0.0, -0.5) for iy in range(2)],  # x = 1, z = 0
             [(2 * nny + iy + 1, 0.2, 0.0, 0.0) for iy in range(3)]]
    path = str(tmp_path / "p.TopVoxel")
    _write_topvoxel(path, v2, fixed, loads, passive=[3])
    for reg in ((0, 2, 1), (1, 1, 2)):
        S = O.Settings()
        S.specifyPassiveRegions = reg
        mo = O.build_model(path, S)
        with Context(specifyPassiveRegions=reg) as ctx:
            ctx.load_topvoxel(path)
            assert np.array_equal(ctx.index_array(1, "PASSIVEELEMENTS"), mo.passiveElements.astype(np.int32)), reg
    S = O.Settings()
    S.specifyPassiveRegions = (0, 0, 1)
    with pytest.raises(IndexError):
        O.build_model(vox, S)
    with Context(specifyPassiveRegions=(0, 0, 1)) as ctx:
        with pytest.raises(TopxError) as e:
            ctx.load_voxels(vox)
        assert "TOPX_ERR_MODEL" in str(e.value)


def test_errors_are_status_codes():
    from top3d_xl_b200 import Context, TopxError
    ctx = Context()
    with pytest.raises(TopxError) as e:
        ctx.load_voxels(np.ones((2, 5, 5), bool))
    assert "TOPX_ERR_ARG" in str(e.value)
    with pytest.raises(TopxError) as e:
        ctx.index_array(1, "ENODMAT")
    assert "TOPX_ERR_STATE" in str(e.value)
    with pytest.raises(TopxError):
        ctx.load_topvoxel("/nonexistent.TopVoxel")
    ctx.close()


def test_standard_vcycle_is_an_fp64_setting():
    from top3d_xl_b200 import Context, TopxError
    Context("fp64", typeVcycle="Standard").close()
    Context("fp64", typeVcycle="Adapted").close()
    with pytest.raises(TopxError) as e:
        Context("mixed", typeVcycle="Standard")
    assert "TOPX_ERR_ARG" in str(e.value)
    with pytest.raises(TopxError):
        Context("fp64", typeVcycle=2)
    with pytest.raises(ValueError):
        Context("fp64", typeVcycle="W")


def test_local_requires_rhat():
    from top3d_xl_b200 import TOP3D_XL
    with pytest.raises(ValueError, match="Wrong Input!"):
        TOP3D_XL(np.ones((4, 8, 4), bool), "LOCAL", 0.5, 3, 1.5, out_dir="/tmp/_topx_unused")


def _have_gpu():
    from tests.conftest import _have_gpu as h
    return h()


@pytest.mark.skipif(_have_gpu(), reason="checks the no-GPU error path")
def test_gpu_call_without_device_fails_loudly():
    from top3d_xl_b200 import Context, TopxError
    ctx = Context()
    ctx.load_voxels(np.ones((4, 8, 4), bool))
    with pytest.raises(TopxError) as e:
        ctx.assemble()
    assert "TOPX_ERR_CUDA" in str(e.value)
    ctx.close()


def test_ke_value_classes_header_is_current_and_matches_ke():
    """The level-1 operator reads Ke through topx_ke_classes.h: the committed header must
    be what its generator writes, and every entry of the element stiffness must equal
    sign * value of its class to rounding."""
    import importlib.util
    csrc = os.path.join(ROOT, "top3d_xl_b200", "csrc")
    spec = importlib.util.spec_from_file_location("gen_ke_classes", os.path.join(csrc, "gen_ke_classes.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    with open(os.path.join(csrc, "topx_ke_classes.h")) as fh:
        assert fh.read() == gen.header()
    table, n = gen.classes()
    Ke = O.element_stiffness(0.3, 1.0).ravel()
    first = {}
    for idx, code in enumerate(table):
        c = abs(code) - 1
        first.setdefault(c, Ke[idx] * np.sign(code))
        assert abs(Ke[idx] - np.sign(code) * first[c]) <= 1e-15 * abs(first[c])
    assert n == 10


def test_mex_gateway_compiles_against_the_c_abi():
    """top3d_xl_b200/matlab/topx_mex.c is compile-checked (no mex.h here: a declaration stub)."""
    import subprocess
    src = os.path.join(ROOT, "top3d_xl_b200", "matlab", "topx_mex.c")
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                        "-I", os.path.join(ROOT, "tests", "mex_stub"), "-I", os.path.join(ROOT, "include"), src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
