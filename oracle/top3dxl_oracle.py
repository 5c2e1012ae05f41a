"""FP64 CPU restatement of TOP3D_XL.m -- TEST INFRASTRUCTURE ONLY.

This module is the correctness oracle for the B200 build.  It is imported only
by ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py``; the product path (``top3d_xl_b200`` + ``libtopx.so``) never
imports, links or calls it.

It restates, function by function, the MATLAB reference ``TOP3D_XL.m`` (one
file; line numbers below are "TX:<line>").  MATLAB and GNU Octave are not
available anywhere this build runs, and the reference ships no tests, fixtures
or golden vectors, so **parity is unpinned**: the restatement is pinned by
self-consistency properties instead (Ke symmetry / rigid-body modes / entries
derived by hand from the closed form at TX:1257-1291, matrix-free K*u equal to
an assembled sparse K, R = P^T, Galerkin coarse operators equal P^T K P, the
filter preserving constants, OC/MMA optimality) -- see tests/test_oracle.py.

Index conventions: every integer array that the reference keeps 1-based
(eNodMat, eleMapBack, nodMapBack, transferMat, ...) is kept 1-based here with
the reference's int32 dtype, so that the native library's arrays can be
compared with them bit for bit.  All voxel/node grids are MATLAB column-major
(y fastest, then x, then z).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

# ----------------------------------------------------------------------------
# Settings (TX:21-38)
# ----------------------------------------------------------------------------


@dataclass
class Settings:
    """Material, solver and optimiser constants of ``InitialSettings`` (TX:21-38)."""

    modulus: float = 1.0
    poissonRatio: float = 0.3
    modulusMin: float = 1.0e-6
    SIMPpenalty: float = 3.0
    cellSize: float = 1.0
    tol: float = 1.0e-3
    maxIT: int = 800
    weightFactorJacobi: float = 0.6
    coarsestResolutionControl: int = 50000
    typeVcycle: str = "Adapted"
    nonDyadic: int = 1
    specifyPassiveRegions: tuple = (0, 0, 0)


def mround(x):
    """MATLAB ``round``: halves away from zero."""
    x = np.asarray(x, dtype=np.float64)
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


# ----------------------------------------------------------------------------
# Element matrices (TX:1254-1292, TX:1785-1798, TX:1768-1783, TX:1617-1627)
# ----------------------------------------------------------------------------

# natural coordinates (s, t, p) of the 8 local nodes of the hex (TX:1785-1797)
HEX_NODES = np.array(
    [[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
     [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)


def trilinear(s, t, p):
    """Trilinear shape functions N (len(s) x 8), TX:1785-1798."""
    s = np.asarray(s, dtype=np.float64)[:, None]
    t = np.asarray(t, dtype=np.float64)[:, None]
    p = np.asarray(p, dtype=np.float64)[:, None]
    sa, ta, pa = HEX_NODES[:, 0], HEX_NODES[:, 1], HEX_NODES[:, 2]
    return 0.125 * (1 + sa * s) * (1 + ta * t) * (1 + pa * p)


def element_stiffness(nu: float, cell: float) -> np.ndarray:
    """24x24 hex8 stiffness for E=1 (TX:1254-1292).

    The reference writes Ke in closed form; here it is integrated exactly with
    2x2x2 Gauss quadrature of B^T D B over a cube of edge ``cell`` (the
    trilinear-hex integrand is of degree <= 2 per direction, so the rule is
    exact).  DOFs are interleaved (node a, component c) -> 3a+c, with local
    node a at HEX_NODES[a] and displacement components along (s, t, p).
    Entries agree with the closed form to rounding (tests/test_oracle.py).
    """
    lam = nu / ((1 + nu) * (1 - 2 * nu))
    mu = 1.0 / (2 * (1 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] = lam + 2 * mu
    D[3, 3] = D[4, 4] = D[5, 5] = mu
    g = 1.0 / math.sqrt(3.0)
    Ke = np.zeros((24, 24))
    jac = 2.0 / cell
    detJ = (cell / 2.0) ** 3
    for gs in (-g, g):
        for gt in (-g, g):
            for gp in (-g, g):
                sa, ta, pa = HEX_NODES[:, 0], HEX_NODES[:, 1], HEX_NODES[:, 2]
                dNs = 0.125 * sa * (1 + ta * gt) * (1 + pa * gp) * jac
                dNt = 0.125 * ta * (1 + sa * gs) * (1 + pa * gp) * jac
                dNp = 0.125 * pa * (1 + sa * gs) * (1 + ta * gt) * jac
                B = np.zeros((6, 24))
                B[0, 0::3] = dNs
                B[1, 1::3] = dNt
                B[2, 2::3] = dNp
                B[3, 0::3] = dNt
                B[3, 1::3] = dNs
                B[4, 1::3] = dNp
                B[4, 2::3] = dNt
                B[5, 0::3] = dNp
                B[5, 2::3] = dNs
                Ke += B.T @ D @ B * detJ
    return 0.5 * (Ke + Ke.T)


def ri_operator(span: int, in_dof: bool = False) -> np.ndarray:
    """Trilinear restriction/interpolation operator, TX:1768-1783.

    Rows = the (span+1)^3 fine nodes of one coarse element in column-major
    order (y fastest); the y sample runs from +1 to -1 (TX:1772)."""
    if span not in (2, 4):
        raise ValueError("Wrong Span Width!")
    n = span + 1
    sy = np.linspace(1, -1, n)
    sx = np.linspace(-1, 1, n)
    sz = np.linspace(-1, 1, n)
    ky, kx, kz = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ky, kx, kz = ky.ravel(order="F"), kx.ravel(order="F"), kz.ravel(order="F")
    N = trilinear(sx[kx], sy[ky], sz[kz])
    if in_dof:
        N = np.kron(N, np.eye(3))
    return N


def grid_enod_offsets(ny: int, nx: int) -> np.ndarray:
    """Local-node offsets of a hex in a column-major node grid (TX:1697)."""
    P = (ny + 1) * (nx + 1)
    return np.array([0, ny + 1, ny, -1, P, P + ny + 1, P + ny, P - 1], dtype=np.int64)


def sub_ele_nod_mat(span: int) -> np.ndarray:
    """1-based node matrix of the span^3 sub-elements of a coarse element (TX:1617-1627)."""
    if span not in (2, 4):
        raise ValueError("Wrong Span Width!")
    n = span
    iy, ix, iz = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    iy, ix, iz = iy.ravel(order="F"), ix.ravel(order="F"), iz.ravel(order="F")
    enodvec = (iy + (n + 1) * ix + (n + 1) ** 2 * iz) + 2  # nodenrs(...)+1, 1-based
    return enodvec[:, None] + grid_enod_offsets(n, n)[None, :]


# ----------------------------------------------------------------------------
# Mesh hierarchy (TX:1629-1730, TX:1076-1236)
# ----------------------------------------------------------------------------


@dataclass
class Level:
    """One entry of ``meshHierarchy_`` (TX:1732-1766)."""

    resX: int
    resY: int
    resZ: int
    spanWidth: int = 0
    eleSize: tuple = (1.0, 1.0, 1.0)
    numElements: int = 0
    numNodes: int = 0
    numDOFs: int = 0
    eNodMat: np.ndarray = None  # int32 (numElements, 8), 1-based compact node ids
    eleMapBack: np.ndarray = None  # int32, 1-based padded-grid element ids
    eleMapForward: np.ndarray = None  # int32 over the padded grid, 0 = void
    nodMapBack: np.ndarray = None  # int32, 1-based padded-grid node ids of this level
    nodMapForward: np.ndarray = None
    nodesOnBoundary: np.ndarray = None
    elementsOnBoundary: np.ndarray = None
    numNod2ElesVec: np.ndarray = None
    elementUpwardMap: np.ndarray = None  # int32 (numElements, span^3), compact finer ids, 0 = void
    transferMat: np.ndarray = None  # int32 ((span+1)^3, numElements), 1-based intermediate ids
    transferMatCoeffi: np.ndarray = None
    solidNodeMapCoarser2Finer: np.ndarray = None
    intermediateNumNodes: int = 0
    multiGridOperatorRI: np.ndarray = None
    Ke: np.ndarray = None
    diagK: np.ndarray = None
    eleModulus: np.ndarray = None
    enod_half_full: np.ndarray = None  # eNodMatHalfTemp_ of this level (all grid elements)


def _discretize_grid(vox_padded: np.ndarray, lvl: Level):
    """Element/node maps of one padded grid (TX:1680-1729, TX:1192-1221)."""
    ny, nx, nz = lvl.resY, lvl.resX, lvl.resZ
    flat = vox_padded.ravel(order="F")
    eleMapBack0 = np.flatnonzero(flat)
    lvl.eleMapBack = (eleMapBack0 + 1).astype(np.int32)
    lvl.numElements = int(eleMapBack0.size)
    lvl.eleMapForward = np.zeros(nx * ny * nz, dtype=np.int32)
    lvl.eleMapForward[eleMapBack0] = np.arange(1, lvl.numElements + 1, dtype=np.int32)
    iy, ix, iz = np.unravel_index(np.arange(nx * ny * nz), (ny, nx, nz), order="F")
    enodvec_all = (iy + 1) + (ny + 1) * ix + (ny + 1) * (nx + 1) * iz + 1  # 1-based
    offs = grid_enod_offsets(ny, nx)
    full = enodvec_all[eleMapBack0][:, None] + offs[None, :]
    lvl.enod_half_full = (enodvec_all[:, None] + offs[None, :])[:, [2, 3, 6, 7]]
    lvl.nodMapBack = np.unique(full).astype(np.int32)
    lvl.numNodes = int(lvl.nodMapBack.size)
    lvl.numDOFs = 3 * lvl.numNodes
    lvl.nodMapForward = np.zeros((nx + 1) * (ny + 1) * (nz + 1), dtype=np.int32)
    lvl.nodMapForward[lvl.nodMapBack - 1] = np.arange(1, lvl.numNodes + 1, dtype=np.int32)
    lvl.eNodMat = lvl.nodMapForward[full - 1].astype(np.int32)
    cnt = np.bincount(lvl.eNodMat.ravel() - 1, minlength=lvl.numNodes)
    lvl.numNod2ElesVec = cnt.astype(np.float64)
    lvl.nodesOnBoundary = (np.flatnonzero(cnt < 8) + 1).astype(np.int32)


def recover_half_enod(half: np.ndarray) -> np.ndarray:
    """Common_RecoverHalfeNodMat (TX:1230-1236)."""
    out = np.zeros((half.shape[0], 8), dtype=np.int64)
    out[:, [2, 3, 6, 7]] = half
    out[:, [1, 0, 5, 4]] = half + 1
    return out


def discretize(vox: np.ndarray, S: Settings):
    """FEA_VoxelBasedDiscretization (TX:1629-1730).  Returns (level1, numLevels)."""
    vox = np.asarray(vox, dtype=bool)
    nely, nelx, nelz = vox.shape
    numVoxels = int(np.count_nonzero(vox))
    L = 0
    while numVoxels >= S.coarsestResolutionControl:
        L += 1
        numVoxels = int(mround(numVoxels / 8))
    L = max(3, L)
    f = 2 ** L
    ax = int(math.ceil(nelx / f) * f)
    ay = int(math.ceil(nely / f) * f)
    az = int(math.ceil(nelz / f) * f)
    numLevels = L + 1
    V = np.zeros((ay, ax, az), dtype=bool)
    V[:nely, :nelx, :nelz] = vox
    lvl = Level(resX=ax, resY=ay, resZ=az, eleSize=(1.0, 1.0, 1.0))
    _discretize_grid(V, lvl)
    isb = np.zeros(lvl.numNodes + 1, dtype=bool)
    isb[lvl.nodesOnBoundary] = True
    lvl.elementsOnBoundary = (np.flatnonzero(isb[lvl.eNodMat].any(axis=1)) + 1).astype(np.int32)
    return lvl, numLevels


def build_hierarchy(levels: list, numLevels: int, S: Settings):
    """Solving_BuildingMeshHierarchy (TX:1076-1228).  Appends coarse levels; returns numLevels."""
    nonDyadic = S.nonDyadic
    if nonDyadic == 1 and numLevels >= 4:
        numLevels -= 1
    else:
        nonDyadic = 0
    for ii in range(2, numLevels + 1):
        prev = levels[-1]
        s = 4 if (ii == 2 and nonDyadic == 1) else 2
        nx, ny, nz = prev.resX // s, prev.resY // s, prev.resZ // s
        lvl = Level(resX=nx, resY=ny, resZ=nz, spanWidth=s,
                    eleSize=tuple(e * s for e in prev.eleSize))
        # coarse element (gy, kx, jz), column-major id; children c = cy + s*cx + s^2*cz
        gy, kx, jz = np.unravel_index(np.arange(nx * ny * nz), (ny, nx, nz), order="F")
        cy, cx, cz = np.unravel_index(np.arange(s ** 3), (s, s, s), order="F")
        fy = s * gy[:, None] + cy[None, :]
        fx = s * kx[:, None] + cx[None, :]
        fz = s * jz[:, None] + cz[None, :]
        fine_full0 = fy + (s * ny) * fx + (s * ny) * (s * nx) * fz
        upward = prev.eleMapForward[fine_full0]
        upward_temp = fine_full0 + 1
        ky, kx2, kz = np.unravel_index(np.arange((s + 1) ** 3), (s + 1, s + 1, s + 1), order="F")
        nfy = s * gy[None, :] + ky[:, None]
        nfx = s * kx[None, :] + kx2[:, None]
        nfz = s * jz[None, :] + kz[:, None]
        tmat_temp = nfy + (s * ny + 1) * nfx + (s * ny + 1) * (s * nx + 1) * nfz + 1  # 1-based
        unempty = np.flatnonzero((upward > 0).any(axis=1))
        inc_void_eles = upward_temp[unempty].ravel(order="F")
        nodes_inc_void = np.unique(recover_half_enod(prev.enod_half_full[inc_void_eles - 1]))
        lvl.intermediateNumNodes = int(nodes_inc_void.size)
        temp = np.zeros((s * nx + 1) * (s * ny + 1) * (s * nz + 1), dtype=np.int32)
        temp[nodes_inc_void - 1] = np.arange(1, lvl.intermediateNumNodes + 1, dtype=np.int32)
        lvl.transferMat = temp[tmat_temp[:, unempty] - 1]
        lvl.transferMatCoeffi = np.bincount(
            lvl.transferMat.ravel() - 1, minlength=lvl.intermediateNumNodes).astype(np.float64)
        last_nodes = np.unique(recover_half_enod(prev.enod_half_full[prev.eleMapBack - 1]))
        idx = np.searchsorted(nodes_inc_void, last_nodes)
        assert np.array_equal(nodes_inc_void[idx], last_nodes)
        lvl.solidNodeMapCoarser2Finer = (idx + 1).astype(np.int32)
        lvl.eleMapForward = np.zeros(nx * ny * nz, dtype=np.int32)
        lvl.eleMapBack = (unempty + 1).astype(np.int32)
        lvl.numElements = int(unempty.size)
        lvl.eleMapForward[unempty] = np.arange(1, lvl.numElements + 1, dtype=np.int32)
        lvl.elementUpwardMap = upward[unempty].astype(np.int32)
        # discretise the coarse grid (TX:1192-1221)
        Vc = np.zeros(nx * ny * nz, dtype=bool)
        Vc[unempty] = True
        lvl2 = Level(resX=nx, resY=ny, resZ=nz)
        _discretize_grid(Vc.reshape((ny, nx, nz), order="F"), lvl2)
        lvl.eNodMat = lvl2.eNodMat
        lvl.nodMapBack = lvl2.nodMapBack
        lvl.nodMapForward = lvl2.nodMapForward
        lvl.numNodes, lvl.numDOFs = lvl2.numNodes, lvl2.numDOFs
        lvl.enod_half_full = lvl2.enod_half_full
        lvl.nodesOnBoundary = lvl2.nodesOnBoundary
        lvl.multiGridOperatorRI = ri_operator(s)
        levels.append(lvl)
    return numLevels


# ----------------------------------------------------------------------------
# Model set-up: BCs (TX:529-560, TX:1294-1336, TX:1338-1437), .TopVoxel (TX:448-528)
# ----------------------------------------------------------------------------


class Model:
    """The reference's global state (``meshHierarchy_``, ``F_``, ``fixingCond_`` ...)."""

    def __init__(self, S: Settings | None = None):
        self.S = S or Settings()
        self.levels: list[Level] = []
        self.numLevels = 0
        self.fixingCond = None  # (k, 4) float: compact node id (1-based), fixX, fixY, fixZ
        self.loadingCond = []  # list of (k, 4): node, fx, fy, fz
        self.objWeightingList = np.array([1.0])
        self.passiveElements = np.zeros(0, dtype=np.int64)
        self.F = None  # (numDOFs, nLoads) dense
        self.fixedDOFs = None  # bool numDOFs
        self.nely = self.nelx = self.nelz = 0

    # -- input models -----------------------------------------------------
    def load_cuboid(self, vox):
        """Built-in cuboid design domain and BCs (TX:529-560)."""
        vox = np.asarray(vox, dtype=bool)
        nely, nelx, nelz = vox.shape
        if nelx < 3 or nely < 3 or nelz < 3:
            raise ValueError("Inappropriate Input Model!")
        self.nely, self.nelx, self.nelz = nely, nelx, nelz
        l1, self.numLevels = discretize(vox, self.S)
        self.levels = [l1]
        NY, NX, NZ = l1.resY + 1, l1.resX + 1, l1.resZ + 1
        vol = np.zeros((NY, NX, NZ))
        vol[0:nely + 1, 0, 0:nelz + 1] = 1
        fixed = l1.nodMapForward[np.flatnonzero(vol.ravel(order="F") == 1)].astype(np.float64)
        self.fixingCond = np.column_stack([fixed, np.ones((fixed.size, 3))])
        vol = np.zeros((NY, NX, NZ))
        zt = int(mround(nelz / 6 + 1))
        vol[0:nely + 1, nelx, 0:zt] = 1
        load = l1.nodMapForward[np.flatnonzero(vol.ravel(order="F") == 1)].astype(np.float64)
        f = np.array([0.0, 0.0, -1.0]) / load.size
        self.loadingCond = [np.column_stack([load, np.tile(f, (load.size, 1))])]
        self.objWeightingList = np.array([1.0])
        self.passiveElements = np.zeros(0, dtype=np.int64)

    def load_topvoxel(self, path: str):
        """``.TopVoxel`` v1.0 reader and BC adaptation (TX:448-528, TX:1439-1509)."""
        with open(path) as fh:
            tok = fh.read().split()
        pos = 0

        def take(k=1):
            nonlocal pos
            v = tok[pos:pos + k]
            pos += k
            return v

        take(4)
        take(1)
        version = float(take(1)[0])
        if version != 1.0:
            raise ValueError("Unsupported Data!")
        if take(1)[0] != "Resolution:":
            raise ValueError("Incompatible Mesh Data Format!")
        nelx, nely, nelz = (int(v) for v in take(3))
        take(2)
        with_density = int(take(1)[0])
        take(2)
        nsolid = int(take(1)[0])
        if with_density:
            arr = np.array(take(2 * nsolid), dtype=np.float64).reshape(nsolid, 2)
            solid = arr[:, 0].astype(np.int64)
        else:
            solid = np.array(take(nsolid), dtype=np.int64)
        if take(1)[0] != "Passive" or take(1)[0] != "elements:":
            raise ValueError("Incompatible Mesh Data Format!")
        npas = int(take(1)[0])
        passive = np.array(take(npas), dtype=np.int64)
        if take(1)[0] != "Fixations:":
            raise ValueError("Incompatible Mesh Data Format!")
        nfix = int(take(1)[0])
        fixing = np.array(take(4 * nfix), dtype=np.float64).reshape(nfix, 4) if nfix > 0 else None
        if take(1)[0] != "Loads:":
            raise ValueError("Incompatible Mesh Data Format!")
        nload = int(take(1)[0])
        loads = {1: np.array(take(4 * nload), dtype=np.float64).reshape(nload, 4) if nload > 0 else None}
        take(2)
        nadd = int(take(1)[0])
        for _ in range(nadd):
            if take(1)[0] != "Loads:":
                raise ValueError("Incompatible Mesh Data Format!")
            k = int(take(1)[0])
            idx = int(take(1)[0])
            loads[idx] = np.array(take(4 * k), dtype=np.float64).reshape(k, 4)
        nL = max(loads.keys())
        self.nely, self.nelx, self.nelz = nely, nelx, nelz
        vox = np.zeros(nelx * nely * nelz, dtype=bool)
        vox[solid - 1] = True
        vox = vox.reshape((nely, nelx, nelz), order="F")
        l1, self.numLevels = discretize(vox, self.S)
        self.levels = [l1]
        adj = (l1.resX + 1, l1.resY + 1, l1.resZ + 1)
        if fixing is not None and fixing.size:
            _, u = np.unique(fixing[:, 0], return_index=True)
            fixing = fixing[u]
            fixing = fixing[np.argsort(fixing[:, 0], kind="stable")]
            fixing = self._adapt_bc(fixing, adj)
            fixing[:, 0] = l1.nodMapForward[fixing[:, 0].astype(np.int64) - 1]
        self.fixingCond = fixing
        self.loadingCond = []
        for i in range(1, nL + 1):
            iL = loads.get(i)
            if iL is not None and iL.size:
                _, u = np.unique(iL[:, 0], return_index=True)
                iL = iL[u]
                iL = iL[np.argsort(iL[:, 0], kind="stable")]
                iL = self._adapt_bc(iL, adj)
                iL[:, 0] = l1.nodMapForward[iL[:, 0].astype(np.int64) - 1]
            self.loadingCond.append(iL)
        self.objWeightingList = np.ones(nL) / nL
        if passive.size:
            passive = np.sort(passive)
            pv = np.zeros(nelx * nely * nelz)
            pv[passive - 1] = 1
            pv = pv.reshape((nely, nelx, nelz), order="F")
            big = np.zeros((l1.resY, l1.resX, l1.resZ))
            big[:nely, :nelx, :nelz] = pv
            adj_idx = np.flatnonzero(big.ravel(order="F"))
            self.passiveElements = np.unique(l1.eleMapForward[adj_idx]).astype(np.int64)
        else:
            self.passiveElements = np.zeros(0, dtype=np.int64)

    def _adapt_bc(self, src, adj):
        """AdaptBCExternalMdl (TX:1439-1490): re-index nodes into the padded grid."""
        nnx, nny, nnz = self.nelx + 1, self.nely + 1, self.nelz + 1
        ax, ay, az = adj
        src = src[np.argsort(src[:, 0], kind="stable")]
        out = np.zeros_like(src)
        cols = []
        for c in range(4):
            vol = np.zeros(nnx * nny * nnz)
            vol[src[:, 0].astype(np.int64) - 1] = 1 if c == 0 else src[:, c]
            vol = vol.reshape((nny, nnx, nnz), order="F")
            big = np.zeros((ay, ax, az))
            big[:nny, :nnx, :nnz] = vol
            cols.append(big.ravel(order="F"))
        new = np.flatnonzero(cols[0])
        out[:, 0] = new + 1
        for c in range(1, 4):
            out[:, c] = cols[c][new]
        return out

    # -- FEA set-up ---------------------------------------------------------
    def apply_boundary_condition(self):
        """FEA_ApplyBoundaryCondition (TX:1294-1336)."""
        l1 = self.levels[0]
        fix = self.fixingCond
        for ii, iL in enumerate(self.loadingCond):
            keep = ~np.isin(fix[:, 0], iL[:, 0])
            fix = fix[keep]
            _, u = np.unique(fix[:, 0], return_index=True)
            fix = fix[u]
            _, u = np.unique(iL[:, 0], return_index=True)
            iL = iL[u]
            if iL.size == 0 or fix.size == 0:
                raise ValueError("No Loads!" if iL.size == 0 else "No Fixations!")
            self.loadingCond[ii] = iL
        self.fixingCond = fix
        if np.any(fix[:, 0] <= 0) or any(np.any(iL[:, 0] <= 0) for iL in self.loadingCond):
            # nodMapForward is 0 for a BC node that is not a solid node; MATLAB then fails on index 0
            raise ValueError("boundary-condition node is not a solid node")
        nL = len(self.loadingCond)
        self.F = np.zeros((l1.numDOFs, nL))
        for ii, iL in enumerate(self.loadingCond):
            Farr = np.zeros((l1.numNodes, 3))
            Farr[iL[:, 0].astype(np.int64) - 1, :] = iL[:, 1:]
            self.F[:, ii] = Farr.ravel()
        nodes = fix[:, 0].astype(np.int64)
        dofs = (3 * nodes[:, None] - np.array([2, 1, 0])[None, :]).ravel()
        state = fix[:, 1:].ravel()
        fixed = dofs[state == 1]
        self.fixedDOFs = np.zeros(l1.numDOFs, dtype=bool)
        self.fixedDOFs[fixed - 1] = True

    def include_adjacent_elements(self, eles):
        """Common_IncludeAdjacentElements (TX:1578-1606): the elements of the 3x3x3 block of padded
        grid cells around each listed element, compact ids, sorted unique."""
        l1 = self.levels[0]
        ny, nx, nz = l1.resY, l1.resX, l1.resZ
        g = l1.eleMapBack[np.asarray(eles, dtype=np.int64) - 1].astype(np.int64) - 1
        iy, ix, iz = g % ny, (g // ny) % nx, g // (ny * nx)
        out = []
        for dz in (-1, 0, 1):
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    y, x, z = iy + dy, ix + dx, iz + dz
                    ok = (y >= 0) & (y < ny) & (x >= 0) & (x < nx) & (z >= 0) & (z < nz)
                    out.append(l1.eleMapForward[(y + ny * (x + nx * z))[ok]])
        out = np.concatenate(out) if out else np.zeros(0, dtype=np.int64)
        return np.unique(out[out > 0]).astype(np.int64)

    def set_passive_elements(self):
        """TopOpti_SetPassiveElements (TX:1511-1574) for S.specifyPassiveRegions = (layers on the
        boundary, near loads, near fixations).  As written, the loaded and fixed node ids (compact)
        index the list of boundary nodes (TX:1557, 1569); an id past its end is MATLAB's index
        error."""
        l1 = self.levels[0]
        nb, nl, nf = (int(mround(v)) for v in self.S.specifyPassiveRegions)
        existing = self.passiveElements
        on_b = np.zeros(0, dtype=np.int64)
        if nb > 0:
            on_b = l1.elementsOnBoundary.astype(np.int64)
            for _ in range(2, nb + 1):
                on_b = self.include_adjacent_elements(on_b)
        near_l = np.zeros(0, dtype=np.int64)
        near_f = np.zeros(0, dtype=np.int64)
        if nl > 0 or nf > 0:
            # node -> boundary elements containing it (TX:1536-1548)
            node_eles = {}
            for e in np.sort(l1.elementsOnBoundary.astype(np.int64)):
                for n in l1.eNodMat[e - 1]:
                    node_eles.setdefault(int(n), []).append(int(e))
            nob = l1.nodesOnBoundary.astype(np.int64)

            def around(ids):
                ids = np.asarray(ids, dtype=np.int64)
                if ids.size and (ids.min() < 1 or ids.max() > nob.size):
                    raise IndexError("Index exceeds the number of array elements (nodesOnBoundary)")
                es = [e for n in nob[ids - 1] for e in node_eles.get(int(n), [])]
                return np.unique(np.array(es, dtype=np.int64))

            if nl > 0:
                near_l = np.concatenate([around(iL[:, 0]) for iL in self.loadingCond])
                for _ in range(2, nl + 1):
                    near_l = self.include_adjacent_elements(near_l)
            if nf > 0:
                near_f = around(self.fixingCond[:, 0])
                for _ in range(2, nf + 1):
                    near_f = self.include_adjacent_elements(near_f)
        self.passiveElements = np.unique(np.concatenate([existing, on_b, near_l, near_f])).astype(np.int64)

    def setup(self):
        """FEA_SetupVoxelBased (TX:1238-1252) + BCs on Ke (TX:1338-1437)."""
        S = self.S
        l1 = self.levels[0]
        l1.Ke = element_stiffness(S.poissonRatio, S.cellSize)
        self.numLevels = build_hierarchy(self.levels, self.numLevels, S)
        self._setup_ke_fixed()

    def _setup_ke_fixed(self):
        """Solving_SetupKeWithFixedDOFs + Solving_ApplyBConEleStiffMat_B (TX:1338-1437)."""
        S = self.S
        l1, l2 = self.levels[0], self.levels[1]
        nob = l1.nodesOnBoundary
        isb = np.zeros(l1.numElements + 1, dtype=bool)
        isb[l1.elementsOnBoundary] = True
        slot = np.zeros(l1.numNodes + 1, dtype=np.int64)
        slot[nob] = np.arange(1, nob.size + 1)
        # node -> ascending list of boundary elements around it
        eles = np.repeat(np.arange(1, l1.numElements + 1), 8)
        nods = l1.eNodMat.ravel()
        m = isb[eles] & (slot[nods] > 0)
        eles, nods = eles[m], nods[m]
        order = np.lexsort((eles, nods))
        eles, nods = eles[order], nods[order]
        starts = np.searchsorted(nods, nob)
        ends = np.searchsorted(nods, nob, side="right")
        fixnodes = self.fixingCond[:, 0].astype(np.int64)
        _, fni, _ = np.intersect1d(nob, fixnodes, return_indices=True)
        lists = [eles[starts[i]:ends[i]] for i in fni]
        allfix = np.unique(np.concatenate(lists)) if lists else np.zeros(0, dtype=np.int64)
        self.allElementsWithFixedDOFs = allfix
        self.mapUniqueKes = np.zeros(l1.numElements, dtype=np.int32)
        self.mapUniqueKes[allfix - 1] = np.arange(1, allfix.size + 1)
        nfix = allfix.size
        self.uniqueKesFree = np.repeat(l1.Ke[None, :, :], nfix, axis=0)
        self.uniqueKesFixed = np.zeros((nfix, 24, 24))
        for ii, ilist in enumerate(lists):
            iFix = self.fixingCond[ii]
            iNode = int(iFix[0])
            state = iFix[1:]
            nAdj = ilist.size
            for e in ilist:
                loc = np.flatnonzero(l1.eNodMat[e - 1] == iNode)
                k = self.mapUniqueKes[e - 1] - 1
                dofs = (3 * (loc[:, None] + 1) - np.array([2, 1, 0])[None, :]).ravel()
                dofs = dofs[np.tile(state, loc.size) == 1] - 1
                self.uniqueKesFree[k][dofs, :] = 0
                self.uniqueKesFree[k][:, dofs] = 0
                self.uniqueKesFixed[k][dofs, dofs] = 1.0 / nAdj
        self.uniqueKesFixed *= S.modulus * S.cellSize
        flag = np.zeros(l1.numElements + 1, dtype=bool)
        flag[allfix] = True
        up = l2.elementUpwardMap
        has = flag[up].any(axis=1) & True
        has &= (up > 0).any(axis=1)
        self.isThisEle2ndLevel = np.zeros(l2.numElements, dtype=np.int32)
        idx = np.flatnonzero(has)
        self.isThisEle2ndLevel[idx] = np.arange(1, idx.size + 1)
        self.sonElesWithFixedDOFs = []
        for j in idx:
            son = up[j]
            _, ia, _ = np.intersect1d(son, allfix, return_indices=True)
            self.sonElesWithFixedDOFs.append(ia)  # 0-based child slots


# ----------------------------------------------------------------------------
# Solver: K*u, V-cycle, PCG, stencil assembly (TX:600-814, TX:919-1066)
# ----------------------------------------------------------------------------


def _gather_u(U, enod):
    """U interleaved (3N,) -> (Ne, 24) element DOF matrix (TX:697-699)."""
    Um = U.reshape(-1, 3)
    e0 = enod - 1
    out = np.empty((enod.shape[0], 24))
    out[:, 0::3] = Um[e0, 0]
    out[:, 1::3] = Um[e0, 1]
    out[:, 2::3] = Um[e0, 2]
    return out


def _scatter(vals, enod, nnodes):
    """accumarray of (Ne, 24) element DOF values onto interleaved nodes (TX:716-721)."""
    Y = np.zeros((nnodes, 3))
    e0 = (enod - 1).ravel(order="F")
    for c in range(3):
        Y[:, c] = np.bincount(e0, weights=vals[:, c::3].ravel(order="F"), minlength=nnodes)
    return Y.ravel()


class Solver:
    """Multigrid-preconditioned PCG of the reference ('Adapted' or 'Standard' V-cycle, per
    ``model.S.typeVcycle``)."""

    def __init__(self, model: Model):
        self.m = model
        S = model.S
        self.S = S
        L = model.levels
        self.Ke = L[0].Ke
        self.fix_idx = np.flatnonzero(model.mapUniqueKes > 0)
        self.fix_slot = model.mapUniqueKes[self.fix_idx] - 1
        # Galerkin templates (TX:926-954)
        self.interp = {}
        self.subdof = {}
        for ii in range(2, model.numLevels + 1):
            s = L[ii - 1].spanWidth
            if s in self.interp:
                continue
            self.interp[s] = ri_operator(s, in_dof=True)
            en = sub_ele_nod_mat(s)
            edof = np.empty((s ** 3, 24), dtype=np.int64)
            for a in range(8):
                for c in range(3):
                    edof[:, 3 * a + c] = 3 * (en[:, a] - 1) + c
            self.subdof[s] = edof
        s2 = L[1].spanWidth
        I2, ed = self.interp[s2], self.subdof[s2]
        self.templates = np.stack([I2[ed[c]].T @ self.Ke @ I2[ed[c]] for c in range(s2 ** 3)])
        self.E = None

    # -- operator -------------------------------------------------------------
    def ku(self, u):
        """Solving_KbyU_MatrixFree, level 1 (TX:684-723)."""
        l1 = self.m.levels[0]
        E = self.E
        Ue = _gather_u(u, l1.eNodMat)
        Ye = (Ue @ self.Ke) * E[:, None]
        if self.fix_idx.size:
            Mf = self.m.uniqueKesFree[self.fix_slot] * E[self.fix_idx][:, None, None] + \
                self.m.uniqueKesFixed[self.fix_slot]
            Ye[self.fix_idx] = np.einsum("ki,kij->kj", Ue[self.fix_idx], Mf)
        return _scatter(Ye, l1.eNodMat, l1.numNodes)

    def ku_level(self, u, ii):
        """Solving_KbyU_MatrixFree on level ii (1-based, TX:684-744): level 1 matrix-free; coarser
        levels the row-vector products u_e' Ks(:,:,e) with the stored Galerkin matrices
        (TX:727-743), scattered in the same element-node order."""
        if ii == 1:
            return self.ku(u)
        lv = self.m.levels[ii - 1]
        Ue = _gather_u(u, lv.eNodMat)
        Ye = np.einsum("ei,eij->ej", Ue, self.Ks_levels[ii])
        return _scatter(Ye, lv.eNodMat, lv.numNodes)

    def element_mats_level1(self):
        """Per-element 24x24 matrices of level 1 as used by ku (for assembled-K tests)."""
        l1 = self.m.levels[0]
        K = np.repeat(self.Ke[None], l1.numElements, axis=0) * self.E[:, None, None]
        if self.fix_idx.size:
            K[self.fix_idx] = self.m.uniqueKesFree[self.fix_slot] * self.E[self.fix_idx][:, None, None] + \
                self.m.uniqueKesFixed[self.fix_slot]
        return K

    # -- transfers ------------------------------------------------------------
    def restrict(self, r, ii):
        """Solving_RestrictResidual (TX:783-798); ii = coarse level (1-based)."""
        L = self.m.levels
        fine, lv = L[ii - 2], L[ii - 1]
        rf = r.reshape(fine.numNodes, 3)
        r1 = np.zeros((lv.intermediateNumNodes, 3))
        r1[lv.solidNodeMapCoarser2Finer - 1] = rf
        r1 = r1 / lv.transferMatCoeffi[:, None]
        out = np.zeros((lv.numNodes, 3))
        for c in range(3):
            t = r1[:, c][lv.transferMat - 1]  # (s+1)^3 x nce
            t = t.T @ lv.multiGridOperatorRI  # nce x 8
            out[:, c] = np.bincount(lv.eNodMat.ravel(order="F") - 1, weights=t.ravel(order="F"),
                                    minlength=lv.numNodes)
        return out.ravel()

    def prolong(self, x, ii):
        """Solving_InterpolationDeviation (TX:800-814); ii = coarse level (1-based)."""
        L = self.m.levels
        lv = L[ii - 1]
        xc = x.reshape(lv.numNodes, 3)
        xf = np.zeros((lv.intermediateNumNodes, 3))
        tm = lv.transferMat.ravel(order="F") - 1
        for c in range(3):
            t = xc[:, c][lv.eNodMat - 1]  # nce x 8
            t1 = lv.multiGridOperatorRI @ t.T  # (s+1)^3 x nce
            xf[:, c] = np.bincount(tm, weights=t1.ravel(order="F"), minlength=lv.intermediateNumNodes)
        xf = xf / lv.transferMatCoeffi[:, None]
        xf = xf[lv.solidNodeMapCoarser2Finer - 1]
        return xf.ravel()

    def vcycle(self, r):
        """Solving_Vcycle (TX:747-781), 'Adapted' or 'Standard' (TX:758-763, 772-777)."""
        L = self.m.levels
        nl = self.m.numLevels
        w = self.S.weightFactorJacobi
        std = self.S.typeVcycle == "Standard"
        if not std and self.S.typeVcycle != "Adapted":
            raise ValueError("typeVcycle must be 'Adapted' or 'Standard'")
        xs = [None] * nl
        rs = [None] * nl
        rs[0] = r
        for ii in range(nl - 1):
            xs[ii] = w * (rs[ii] / L[ii].diagK)
            if std:
                d = rs[ii] - self.ku_level(xs[ii], ii + 1)
                rs[ii + 1] = self.restrict(d, ii + 2)
            else:
                rs[ii + 1] = self.restrict(rs[ii], ii + 2)
        xs[-1] = self.coarse_solve(rs[-1])
        for ii in range(nl - 2, -1, -1):
            xs[ii] = xs[ii] + self.prolong(xs[ii + 1], ii + 2)
            if std:
                xs[ii] = xs[ii] + w * (rs[ii] - self.ku_level(xs[ii], ii + 1)) / L[ii].diagK
            else:
                xs[ii] = xs[ii] + w * rs[ii] / L[ii].diagK
        return xs[0]

    def coarse_solve(self, r):
        """x = P (L^T \\ (L \\ (P^T r))) with the coarsest Cholesky (TX:767)."""
        if self._chol_kind == "dense":
            return sla.cho_solve(self._chol, r)
        return sla.cho_solve_banded(self._chol, r[self._perm])[self._iperm]

    # -- stencil assembly (TX:919-1066) --------------------------------------
    def assemble(self, E):
        """Solving_AssembleFEAstencil for element moduli E (row of numElements)."""
        m = self.m
        L = m.levels
        nl = m.numLevels
        self.E = np.asarray(E, dtype=np.float64).ravel()
        Ks = None
        self.Ks_levels = {}
        for ii in range(2, nl + 1):
            lv = L[ii - 1]
            s = lv.spanWidth
            I, ed = self.interp[s], self.subdof[s]
            up = lv.elementUpwardMap
            nce = lv.numElements
            if ii == 2:
                Ech = np.where(up > 0, self.E[np.maximum(up, 1) - 1], 0.0)
                Ks = np.einsum("jc,cab->jab", Ech, self.templates)
                flagged = np.flatnonzero(m.isThisEle2ndLevel > 0)
                for j in flagged:
                    idx = m.isThisEle2ndLevel[j] - 1
                    son = up[j]
                    nd = (s + 1) ** 3 * 3
                    Kf = np.zeros((nd, nd))
                    fixed_local = set(m.sonElesWithFixedDOFs[idx].tolist())
                    for c in range(s ** 3):
                        if son[c] == 0:
                            continue
                        e = son[c] - 1
                        if c in fixed_local:
                            k = m.mapUniqueKes[e] - 1
                            Kc = m.uniqueKesFree[k] * self.E[e] + m.uniqueKesFixed[k]
                        else:
                            Kc = self.Ke * self.E[e]
                        Kf[np.ix_(ed[c], ed[c])] += Kc
                    Ks[j] = I.T @ Kf @ I
            else:
                prevKs = Ks
                Ks = np.zeros((nce, 24, 24))
                nd = (s + 1) ** 3 * 3
                for j in range(nce):
                    Kf = np.zeros((nd, nd))
                    for c in range(s ** 3):
                        if up[j, c] == 0:
                            continue
                        Kf[np.ix_(ed[c], ed[c])] += prevKs[up[j, c] - 1]
                    Ks[j] = I.T @ Kf @ I
            self.Ks_levels[ii] = Ks
            if ii < nl:
                dg = np.zeros((lv.numNodes, 3))
                e0 = (lv.eNodMat - 1).ravel(order="F")
                d = np.diagonal(Ks, axis1=1, axis2=2)  # nce x 24
                for c in range(3):
                    dg[:, c] = np.bincount(e0, weights=d[:, c::3].ravel(order="F"), minlength=lv.numNodes)
                lv.diagK = dg.ravel()
        # finest diagonal (TX:1020-1050)
        l1 = L[0]
        dKe = np.diag(self.Ke)
        d = self.E[:, None] * dKe[None, :]
        if self.fix_idx.size:
            d[self.fix_idx] = np.diagonal(m.uniqueKesFree[self.fix_slot], axis1=1, axis2=2) * \
                self.E[self.fix_idx][:, None] + np.diagonal(m.uniqueKesFixed[self.fix_slot], axis1=1, axis2=2)
        dg = np.zeros((l1.numNodes, 3))
        e0 = (l1.eNodMat - 1).ravel(order="F")
        for c in range(3):
            dg[:, c] = np.bincount(e0, weights=d[:, c::3].ravel(order="F"), minlength=l1.numNodes)
        l1.diagK = dg.ravel()
        # coarsest assembly and Cholesky (TX:1052-1065)
        lc = L[nl - 1]
        self.Ks_coarsest = Ks
        en = lc.eNodMat - 1
        edof = np.empty((lc.numElements, 24), dtype=np.int64)
        for a in range(8):
            for c in range(3):
                edof[:, 3 * a + c] = 3 * en[:, a] + c
        rows = np.repeat(edof, 24, axis=1).ravel()
        cols = np.tile(edof, (1, 24)).ravel()
        K = sp.csr_matrix((Ks.reshape(lc.numElements, -1).ravel(), (rows, cols)),
                          shape=(lc.numDOFs, lc.numDOFs))
        self.K_coarsest = K
        n = lc.numDOFs
        if n <= 6000:
            self._chol_kind = "dense"
            self._chol = sla.cho_factor(K.toarray(), lower=True)
        else:
            self._chol_kind = "banded"
            perm = np.arange(n)
            Kp = K[perm][:, perm].tocoo()
            bw = int(np.max(np.abs(Kp.row - Kp.col)))
            ab = np.zeros((bw + 1, n))
            mlow = Kp.row >= Kp.col
            ab[Kp.row[mlow] - Kp.col[mlow], Kp.col[mlow]] = Kp.data[mlow]
            self._perm = perm
            self._iperm = np.argsort(perm)
            self._chol = (sla.cholesky_banded(ab, lower=True), True)


def pcg(Atx, Ptv, b, tol, maxIT, y0=None):
    """Solving_PCG (TX:600-639); returns (y, its, resnorm)."""
    normB = np.linalg.norm(b)
    y = np.zeros_like(b) if y0 is None else np.array(y0, dtype=np.float64, copy=True)
    r = b - Atx(y)
    z = Ptv(r)
    p = z.copy()
    x1 = z @ r
    its = 0
    resnorm = np.inf
    for its in range(1, maxIT + 1):
        z = Atx(p)
        lam = x1 / (p @ z)
        y = y + lam * p
        r = r - lam * z
        resnorm = np.linalg.norm(r) / normB
        if resnorm < tol:
            break
        z = Ptv(r)
        x2 = z @ r
        p = z + x2 / x1 * p
        x1 = x2
    return y, its, resnorm


# ----------------------------------------------------------------------------
# PDE filter (TX:816-917), compliance (TX:579-598)
# ----------------------------------------------------------------------------


def pde_filter_kernel(rmin: float, ele_size: float = 1.0):
    """8x8 Helmholtz kernel of TopOpti_SetupPDEfilter_matrixFree (TX:816-853).

    KEF0 uses natural-coordinate derivatives with unit weights (TX:848), as
    the reference writes it."""
    g = 1.0 / math.sqrt(3.0)
    s = np.array([-1, 1, 1, -1, -1, 1, 1, -1]) * g
    t = np.array([-1, -1, 1, 1, -1, -1, 1, 1]) * g
    p = np.array([-1, -1, -1, -1, 1, 1, 1, 1]) * g
    w = np.ones(8)
    N = trilinear(s, t, p)
    sa, ta, pa = HEX_NODES[:, 0], HEX_NODES[:, 1], HEX_NODES[:, 2]
    dS = np.zeros((24, 8))
    dS[0::3] = 0.125 * sa[None, :] * (1 + ta[None, :] * t[:, None]) * (1 + pa[None, :] * p[:, None])
    dS[1::3] = 0.125 * ta[None, :] * (1 + sa[None, :] * s[:, None]) * (1 + pa[None, :] * p[:, None])
    dS[2::3] = 0.125 * pa[None, :] * (1 + sa[None, :] * s[:, None]) * (1 + ta[None, :] * t[:, None])
    detJ = 1.0 / 8 * np.ones(8)
    wgt = w * detJ
    KEF0 = dS.T @ dS
    KEF1 = N.T @ np.diag(wgt) @ N
    iR = (rmin * ele_size) / 2 / math.sqrt(3)
    return iR ** 2 * KEF0 + KEF1


class PDEFilter:
    """TopOpti_SetupPDEfilter_matrixFree + TopOpti_ConductPDEFiltering_matrixFree (TX:816-917)."""

    def __init__(self, model: Model, rmin: float, S: Settings):
        l1 = model.levels[0]
        self.l1 = l1
        self.S = S
        self.KF = pde_filter_kernel(rmin, l1.eleSize[0])
        e0 = (l1.eNodMat - 1).ravel(order="F")
        dg = np.bincount(e0, weights=np.repeat(np.diag(self.KF)[None, :], l1.numElements, 0).ravel(order="F"),
                         minlength=l1.numNodes)
        self.diagPrecond = dg ** -1.0
        self.last_its = 0

    def matvec(self, u):
        """MatTimesVec_matrixFree_B (TX:904-917)."""
        l1 = self.l1
        Ue = u[l1.eNodMat - 1]
        return np.bincount((l1.eNodMat - 1).ravel(order="F"), weights=(Ue @ self.KF).ravel(order="F"),
                           minlength=l1.numNodes)

    def __call__(self, src):
        l1 = self.l1
        vals = np.asarray(src, dtype=np.float64).ravel() * (1 / 8)
        node = np.zeros(l1.numNodes)
        for j in range(8):
            node = node + np.bincount(l1.eNodMat[:, j] - 1, weights=vals, minlength=l1.numNodes)
        tar, its, _ = pcg(self.matvec, lambda x: self.diagPrecond * x, node, self.S.tol / 10, self.S.maxIT)
        self.last_its = its
        return tar[l1.eNodMat - 1].sum(axis=1) * (1 / 8)


def unit_compliance(model: Model, U: np.ndarray) -> np.ndarray:
    """TopOpti_ComputeUnitCompliance (TX:579-598): ce_e = u_e^T Ke u_e, load-weighted."""
    l1 = model.levels[0]
    ce = np.zeros((l1.numElements, U.shape[1]))
    for j in range(U.shape[1]):
        Ue = _gather_u(U[:, j], l1.eNodMat)
        ce[:, j] = np.sum((Ue @ l1.Ke) * Ue, axis=1)
    return ce @ model.objWeightingList.ravel()


# ----------------------------------------------------------------------------
# MMA (TX:1804-2049), m constraints (m=1 used)
# ----------------------------------------------------------------------------


def mma_seq(m, n, it, xval, xmin, xmax, xold1, xold2, dfdx, gx, dgdx, low, upp):
    """MMAseq/Update/GenSub/SolveDIP (TX:1806-2049).  Returns xnew, xold1, xold2, low, upp."""
    asyminit, asymdec, asyminc = 0.5, 0.7, 1.2
    a = np.zeros(m)
    c = 1000.0 * np.ones(m)
    xval = np.asarray(xval, dtype=np.float64).ravel().copy()
    xmin = np.asarray(xmin, dtype=np.float64).ravel()
    xmax = np.asarray(xmax, dtype=np.float64).ravel()
    xold1 = np.asarray(xold1, dtype=np.float64).ravel().copy()
    xold2 = np.asarray(xold2, dtype=np.float64).ravel().copy()
    low = np.asarray(low, dtype=np.float64).ravel().copy()
    upp = np.asarray(upp, dtype=np.float64).ravel().copy()
    dfdx = np.asarray(dfdx, dtype=np.float64).ravel()
    dgdx = np.asarray(dgdx, dtype=np.float64).reshape(m, n)
    gx = np.asarray(gx, dtype=np.float64).ravel()
    # GenSub (TX:1873-1928)
    if it < 3 or low.size < n or upp.size < n:
        low = xval - asyminit * (xmax - xmin)
        upp = xval + asyminit * (xmax - xmin)
    else:
        zzz = (xval - xold1) * (xold1 - xold2)
        gamma = np.ones(n)
        gamma[zzz > 0] = asyminc
        gamma[zzz < 0] = asymdec
        low = xval - gamma * (xold1 - low)
        upp = xval + gamma * (upp - xold1)
        lowmin = xval - 10.0 * (xmax - xmin)
        lowmax = xval - 0.01 * (xmax - xmin)
        uppmin = xval + 0.01 * (xmax - xmin)
        uppmax = xval + 10.0 * (xmax - xmin)
        low = np.maximum(low, lowmin)
        low = np.minimum(low, lowmax)
        upp = np.minimum(upp, uppmax)
        upp = np.maximum(upp, uppmin)
    feps = 1.0e-6
    alpha = 0.9 * low + 0.1 * xval
    tb = alpha - xmin < 0
    alpha[tb] = xmin[tb]
    beta = 0.9 * upp + 0.1 * xval
    tb = beta - xmax > 0
    beta[tb] = xmax[tb]
    dp = np.where(dfdx < 0.0, 0.0, dfdx)
    dm = -1.0 * dfdx
    dm = np.where(dm < 0.0, 0.0, dm)
    p0 = (upp - xval) ** 2.0 * (dp + 0.001 * np.abs(dfdx) + 0.5 * feps / (upp - low))
    q0 = (xval - low) ** 2.0 * (dm + 0.001 * np.abs(dfdx) + 0.5 * feps / (upp - low))
    gp = np.where(dgdx < 0.0, 0.0, dgdx)
    gm = -1.0 * dgdx
    gm = np.where(gm < 0.0, 0.0, gm)
    extra = 0.001 * np.abs(dgdx) + 0.5 * feps / (upp - low)
    pij = (upp - xval) ** 2 * (gp + extra)
    qij = (xval - low) ** 2 * (gm + extra)
    b = -gx + np.sum(pij / (upp - xval) + qij / (xval - low), axis=1)
    # Update (TX:1862-1871)
    xold2 = xold1
    xold1 = xval.copy()
    # SolveDIP (TX:1930-1965)
    lam = c / 2.0
    mu = np.ones(m)
    tol = 1.0e-9 * math.sqrt(m + n)
    epsi = 1.0
    x = xval.copy()
    y = np.zeros(m)
    z = 0.0

    def xyz(lam):
        lam = np.where(lam < 0.0, 0.0, lam)
        y = lam - c
        y = np.where(y < 0.0, 0.0, y)
        lamai = lam @ a
        z = max(0.0, 10.0 * (lamai - 1.0))
        pj = p0 + np.sum(pij * lam[:, None], axis=0)
        qj = q0 + np.sum(qij * lam[:, None], axis=0)
        x = (np.sqrt(pj) * low + np.sqrt(qj) * upp) / (np.sqrt(pj) + np.sqrt(qj))
        tb = x - alpha < 0
        x[tb] = alpha[tb]
        tb = x - beta > 0
        x[tb] = beta[tb]
        return lam, x, y, z

    while epsi > tol:
        loop = 0
        err = np.inf
        while err > 0.9 * epsi and loop < 100:
            loop += 1
            lam, x, y, z = xyz(lam)
            grad = -b - a * z - y
            grad = grad + np.sum(pij / (upp - x) + qij / (x - low), axis=1)
            grad = -1.0 * grad - epsi / lam
            # DualHess (TX:1986-2018)
            pj = p0 + np.sum(pij * lam[:, None], axis=0)
            qj = q0 + np.sum(qij * lam[:, None], axis=0)
            PQ = pij / (upp - x) ** 2.0 - qij / (x - low) ** 2.0
            df2 = -1.0 / (2.0 * pj / (upp - x) ** 3.0 + 2.0 * qj / (x - low) ** 3.0)
            xp = (np.sqrt(pj) * low + np.sqrt(qj) * upp) / (np.sqrt(pj) + np.sqrt(qj))
            df2[xp - alpha < 0] = 0.0
            df2[xp - beta > 0] = 0.0
            H = (PQ * df2) @ PQ.T
            lamai = 0.0
            for jj in range(m):
                if lam[jj] < 0.0:
                    lam[jj] = 0.0
                lamai += lam[jj] * a[jj]
                if lam[jj] > c[jj]:
                    H[jj, jj] -= 1.0
                H[jj, jj] -= mu[jj] / lam[jj]
            if lamai > 1.0:
                H -= 10.0 * np.outer(a, a)
            corr = 1e-4 * np.trace(H) / m
            if -1.0 * corr < 1.0e-7:
                corr = -1.0e-7
            H = H + np.diag(np.full(m, corr))
            s1 = np.linalg.solve(H, grad)
            s2 = -mu + epsi / lam - s1 * mu / lam
            # DualLineSearch (TX:2020-2031)
            theta = 1.005
            for jj in range(m):
                if theta < -1.01 * s1[jj] / lam[jj]:
                    theta = -1.01 * s1[jj] / lam[jj]
                if theta < -1.01 * s2[jj] / mu[jj]:
                    theta = -1.01 * s2[jj] / mu[jj]
            theta = 1.0 / theta
            lam = lam + theta * s1
            mu = mu + theta * s2
            lam, x, y, z = xyz(lam)
            # DualResidual (TX:2033-2049)
            res1 = -b - a * z - y + mu
            res2 = mu * lam - epsi
            res1 = res1 + np.sum(pij / (upp - x), axis=1) + np.sum(qij / (x - low), axis=1)
            err = max(np.max(np.abs(res1)), np.max(np.abs(res2)))
        epsi = epsi * 0.1
    return x, xold1, xold2, low, upp


# ----------------------------------------------------------------------------
# Optimisation drivers (TX:40-223 GLOBAL, TX:225-440 LOCAL)
# ----------------------------------------------------------------------------


def build_model(input_model, S: Settings | None = None) -> Model:
    """CreateVoxelFEAmodel + FEA_ApplyBoundaryCondition + FEA_SetupVoxelBased (TX:68-73)."""
    m = Model(S)
    if isinstance(input_model, str):
        m.load_topvoxel(input_model)
    else:
        m.load_cuboid(input_model)
    m.apply_boundary_condition()
    m.setup()
    m.set_passive_elements()  # TX:79 / 272
    return m


def _solve_all(solver: Solver, model: Model, U, its_list=None):
    S = model.S
    for ii in range(model.F.shape[1]):
        U[:, ii], its, _ = pcg(solver.ku, solver.vcycle, model.F[:, ii], S.tol, S.maxIT, U[:, ii])
        if its_list is not None:
            its_list.append(its)
    return U


def oc_update(x, dc, dv, fval, passive, move=0.2):
    """The OC bisection of TOP3D_XL_TO (TX:145-156): the volume multiplier is bisected from
    (0, 1e9) until (l2 - l1)/(l1 + l2) <= 1e-6; gt is fval plus the SUM of the density change
    (as written in the reference).  Returns the new densities and the last midpoint."""
    l1_, l2_ = 0.0, 1e9
    while (l2_ - l1_) / (l1_ + l2_) > 1e-6:
        lmid = 0.5 * (l2_ + l1_)
        xnew = np.maximum(0, np.maximum(x - move, np.minimum(1, np.minimum(x + move, x * np.sqrt(-dc / dv / lmid)))))
        xnew[passive] = 1.0
        gt = fval + np.sum(dv * (xnew - x))
        if gt > 0:
            l1_ = lmid
        else:
            l2_ = lmid
    return xnew, lmid


def run_global(input_model, V0, nLoop, rMin, S: Settings | None = None, model: Model | None = None,
               max_loops=None, keep_U=False, hook=None):
    """TOP3D_XL_TO (TX:40-223) without file/graphics output.  Returns a history dict.
    `hook(loop)`, if given, is called once cSolid is known (loop 0) and after each iteration;
    a true return value ends the loop there (used to time a bounded number of iterations)."""
    model = model or build_model(input_model, S)
    S = model.S
    l1 = model.levels[0]
    flt = PDEFilter(model, rMin, S)
    Ne = l1.numElements
    passive = model.passiveElements - 1
    x = np.full(Ne, V0, dtype=np.float64)
    xPhys = x.copy()
    loop, change, sharpness = 0, 1.0, 1.0
    solver = Solver(model)
    U = np.zeros_like(model.F)
    solver.assemble(np.full(Ne, S.modulus))
    _solve_all(solver, model, U)
    ce = unit_compliance(model, U)
    cSolid = np.full(Ne, S.modulus) @ ce
    hist = dict(cSolid=cSolid, c=[], vol=[], sharp=[], cons=[], change=[], its=[], filter_its=[])
    E0, Emin, p = S.modulus, S.modulusMin, S.SIMPpenalty
    stop = nLoop if max_loops is None else min(nLoop, max_loops)
    if hook is not None and hook(0):
        stop = 0
    while loop < stop and change > 0.0001 and sharpness > 0.01:
        loop += 1
        E = Emin + xPhys ** p * (E0 - Emin)
        solver.assemble(E)
        _solve_all(solver, model, U, hist["its"])
        ce = unit_compliance(model, U)
        ceNorm = ce / cSolid
        cObj = E @ ceNorm
        cDesign = cObj * cSolid
        V = float(np.sum(xPhys) / Ne)
        dc = -(p * (E0 - Emin) * xPhys ** (p - 1)) * ceNorm
        dv = np.ones(Ne)
        dc = flt(x * dc) / np.maximum(1e-3, x)
        hist["filter_its"].append(flt.last_its)
        fval = np.mean(xPhys) - V0
        xnew, lmid = oc_update(x, dc, dv, fval, passive)
        change = float(np.max(np.abs(xnew - x)))
        x = xnew
        xPhys = xnew.copy()
        xPhys[passive] = 1
        sharpness = 4 * np.sum(xPhys * (1 - xPhys)) / Ne
        hist["c"].append(cDesign)
        hist["vol"].append(V)
        hist["cons"].append(fval)
        hist["sharp"].append(sharpness)
        hist["change"].append(change)
        hist.setdefault("lmid", []).append(lmid)
        if hook is not None and hook(loop):
            break
    hist["xPhys"] = xPhys
    hist["loops"] = loop
    if keep_U:
        hist["U"] = U
    return hist


def run_local(input_model, Ve0, nLoop, rMin, rHat, S: Settings | None = None, model: Model | None = None,
              max_loops=None, hook=None):
    """TOP3D_XL_PIO (TX:225-440) without file/graphics output.  Returns a history dict.
    `hook` as in run_global."""
    model = model or build_model(input_model, S)
    S = model.S
    l1 = model.levels[0]
    betaPIO, etaPIO, pPIO, pMaxPIO = 1.0, 0.5, 16, 128
    fltR = PDEFilter(model, rMin, S)
    fltH = PDEFilter(model, rHat, S)
    Ne = l1.numElements
    passive = model.passiveElements - 1
    active = np.setdiff1d(np.arange(Ne), passive)
    x = np.full(Ne, Ve0, dtype=np.float64)
    volMax = x.copy()
    xTilde = x.copy()
    xPhys = x.copy()
    loopbeta = loop = 0
    change, sharpness = 1.0, 1.0
    solver = Solver(model)
    U = np.zeros_like(model.F)
    solver.assemble(np.full(Ne, S.modulus))
    _solve_all(solver, model, U)
    ce = unit_compliance(model, U)
    cSolid = np.full(Ne, S.modulus) @ ce
    hist = dict(cSolid=cSolid, c=[], vol=[], sharp=[], cons=[], change=[], its=[], beta=[])
    E0, Emin, p = S.modulus, S.modulusMin, S.SIMPpenalty
    stop = nLoop if max_loops is None else min(nLoop, max_loops)
    if hook is not None and hook(0):
        stop = 0
    xold1 = xold2 = low = upp = None
    while loop < stop and change > 0.0001 and sharpness > 0.01:
        loopbeta += 1
        loop += 1
        E = Emin + xPhys ** p * (E0 - Emin)
        solver.assemble(E)
        _solve_all(solver, model, U, hist["its"])
        ce = unit_compliance(model, U)
        ceNorm = ce / cSolid
        cObj = E @ ceNorm
        cDesign = cObj * cSolid
        V = float(np.sum(xPhys) / Ne)
        dc = -(p * (E0 - Emin) * xPhys ** (p - 1)) * ceNorm
        xhat = fltH(xPhys)
        pn = np.sum(xhat ** pPIO / volMax ** pPIO) / Ne
        dfdx_pde = pn ** (1 / pPIO - 1) * (xhat ** (pPIO - 1) / volMax ** pPIO) / Ne
        th = np.tanh(betaPIO * (xTilde - etaPIO))
        dx = betaPIO * (1 - th * th) / (np.tanh(betaPIO * etaPIO) + np.tanh(betaPIO * (1 - etaPIO)))
        dc = fltR(dc * dx)
        dfdx = fltH(dfdx_pde)
        dfdx = fltR(dfdx * dx)
        if loop == 1:
            xold1 = x[active].copy()
            xold2 = xold1.copy()
            low = np.zeros(active.size)
            upp = low.copy()
        move = 0.1
        fval = (np.sum(xhat ** pPIO / volMax ** pPIO) / Ne) ** (1 / pPIO) - 1
        xval = x[active]
        xmin = np.maximum(0.0, xval - move)
        xmax = np.minimum(1, xval + move)
        xmma, xold1, xold2, low, upp = mma_seq(1, active.size, loop, xval, xmin, xmax, xold1, xold2,
                                               dc[active], np.array([fval]), dfdx[active][None, :], low, upp)
        change = float(np.max(np.abs(xmma - xval)))
        x = np.ones(Ne)
        x[active] = xmma
        xTilde = fltR(x)
        if loopbeta >= 40:
            betaPIO = min(2 * betaPIO, pMaxPIO)
            loopbeta = 0
        xPhys = (np.tanh(betaPIO * etaPIO) + np.tanh(betaPIO * (xTilde - etaPIO))) / \
            (np.tanh(betaPIO * etaPIO) + np.tanh(betaPIO * (1 - etaPIO)))
        xPhys[passive] = 1
        sharpness = 4 * np.sum(xPhys * (1 - xPhys)) / Ne
        hist["c"].append(cDesign)
        hist["vol"].append(V)
        hist["cons"].append(fval)
        hist["sharp"].append(sharpness)
        hist["change"].append(change)
        hist["beta"].append(betaPIO)
        if hook is not None and hook(loop):
            break
    hist["xPhys"] = xPhys
    hist["loops"] = loop
    return hist


def write_history_files(out_dir: str, hist: dict):
    """c_Target.dat / iters_Target.dat / sharp_Target.dat in the reference's formats (TX:193-201)."""
    import os
    os.makedirs(out_dir, exist_ok=True)
    with open(os.path.join(out_dir, "iters_Target.dat"), "w") as fh:
        fh.writelines("%d\n" % v for v in hist["its"])
    with open(os.path.join(out_dir, "c_Target.dat"), "w") as fh:
        fh.writelines("%30.16e\n" % v for v in hist["c"])
    with open(os.path.join(out_dir, "sharp_Target.dat"), "w") as fh:
        fh.writelines("%30.16e\n" % v for v in hist["sharp"])
