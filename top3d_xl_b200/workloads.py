"""Synthetic design domains for the benchmarks and tests.

``irregular_domain`` builds the irregular LOCAL workload: a seeded union of randomly rotated
ellipsoids and finite cylinders in a voxel box, reduced to its largest 26-connected
component, fixed at the lowest solid z-layer and loaded at random surface nodes.
``write_topvoxel`` emits it as a ``.TopVoxel`` v1.0 file (the format TOP3D_XL.m:448-497
reads), so it enters through the same reader as any external domain.

Node ids follow the reference's unpadded numbering: 1-based, column-major over the
(nely+1, nelx+1, nelz+1) node grid (y fastest).  Force components are (x, y, z).
"""
from __future__ import annotations

import numpy as np


# The irregular workload at full size (192x384x192 box; seed 8 gives a 33 % fill, 4.66M
# elements) and a reduced copy small enough for the oracle (the parity fixture's domain).
IRREGULAR_FULL = dict(seed=8)
IRREGULAR_SMALL = dict(seed=7, box=(20, 40, 20), n_ellipsoids=3, n_cylinders=2, semi=(4, 10), radius=(2, 4),
                       half_length=(5, 12), n_loads=8)


def _rotation(rng):
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def irregular_domain(seed=8, box=(192, 384, 192), n_ellipsoids=12, n_cylinders=6, semi=(20, 90), radius=(10, 30),
                     half_length=(50, 150), n_loads=64):
    """Voxel mask (nely, nelx, nelz), fixed node ids and loads [(node, fx, fy, fz)].

    Ellipsoids: centre uniform in the box, semi-axes uniform in `semi`, random rotation.
    Cylinders: centre uniform in the box, radius uniform in `radius`, axis a uniform random
    direction, half-length uniform in `half_length` (a finite, flat-ended cylinder).
    The largest 26-connected component is kept.  Fixed: every node of the bottom faces of the
    solid voxels in the lowest solid z-layer.  Loads: `n_loads` distinct surface nodes (nodes
    with fewer than 8 solid voxels around them), not fixed, each with a unit force in a
    uniformly random direction.  Everything is drawn from numpy.random.default_rng(seed).
    """
    from scipy import ndimage

    rng = np.random.default_rng(seed)
    ny, nx, nz = box
    vox = np.zeros((ny, nx, nz), bool)
    centre_of = lambda: rng.uniform(0, 1, 3) * np.array([ny, nx, nz])  # noqa: E731

    def fill(c, reach, inside):
        lo = np.maximum(np.floor(c - reach).astype(int), 0)
        hi = np.minimum(np.ceil(c + reach).astype(int) + 1, [ny, nx, nz])
        if np.any(hi <= lo):
            return
        g = np.stack(np.meshgrid(*[np.arange(lo[k], hi[k]) + 0.5 for k in range(3)], indexing="ij"), -1)
        vox[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] |= inside(g - c)

    for _ in range(n_ellipsoids):
        c, ax, R = centre_of(), rng.uniform(*semi, 3), _rotation(rng)
        fill(c, ax.max(), lambda d, ax=ax, R=R: np.sum(((d @ R) / ax) ** 2, -1) <= 1.0)
    for _ in range(n_cylinders):
        c, r, h = centre_of(), rng.uniform(*radius), rng.uniform(*half_length)
        u = rng.standard_normal(3)
        u /= np.linalg.norm(u)

        def inside(d, u=u, r=r, h=h):
            t = d @ u
            return (np.abs(t) <= h) & (np.sum(d * d, -1) - t * t <= r * r)
        fill(c, np.hypot(r, h), inside)
    lab, n = ndimage.label(vox, structure=np.ones((3, 3, 3), int))
    if n == 0:
        raise ValueError("empty domain")
    sizes = np.bincount(lab.ravel())
    sizes[0] = 0
    vox = lab == np.argmax(sizes)

    nny, nnx = ny + 1, nx + 1
    node = lambda y, x, z: 1 + y + nny * (x + nnx * z)  # noqa: E731
    zs = np.flatnonzero(vox.any(axis=(0, 1)))
    z0 = int(zs[0])
    yy, xx = np.nonzero(vox[:, :, z0])
    fixed = set()
    for dy in (0, 1):
        for dx in (0, 1):
            fixed.update(node(yy + dy, xx + dx, z0).tolist())
    # count solid voxels around every node
    cnt = np.zeros((ny + 1, nx + 1, nz + 1), np.int8)
    for dy in (0, 1):
        for dx in (0, 1):
            for dz in (0, 1):
                cnt[dy:dy + ny, dx:dx + nx, dz:dz + nz] += vox
    sy, sx, sz = np.nonzero((cnt > 0) & (cnt < 8))
    surf = node(sy, sx, sz)
    surf = surf[~np.isin(surf, np.fromiter(fixed, np.int64))]
    pick = rng.choice(surf, size=min(n_loads, surf.size), replace=False)
    dirs = rng.standard_normal((pick.size, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    loads = [(int(p), *map(float, d)) for p, d in zip(np.sort(pick), dirs)]
    return vox, sorted(fixed), loads


def two_load_case_model(ny=10, nx=20, nz=10):
    """A cuboid with two load cases and passive elements, as a ``.TopVoxel`` file gives them.

    Fixed: every node of the bottom face (z = 0), all three directions.  Load case 1: the four
    nodes of the top face's centre with force (0, 0, -1/4) each.  Load case 2: the nodes of the
    top face's edge at x = nx, force (0.5/(ny+1), 0, 0) each.  Passive: a 2 x 2 x 2 block of
    elements under the centre of the top face (compact ids of the full cuboid, 1-based).  The
    bottom-face node ids are all smaller than the boundary-node count, so passive layers near
    the fixations (specifyPassiveRegions_(3), TOP3D_XL.m:1563-1574) index that list as the
    reference does.  Returns vox, fixed, [case1, case2], passive.
    """
    vox = np.ones((ny, nx, nz), bool)
    nny, nnx = ny + 1, nx + 1
    node = lambda y, x, z: 1 + y + nny * (x + nnx * z)  # noqa: E731
    fixed = [node(y, x, 0) for x in range(nnx) for y in range(nny)]
    cy, cx = ny // 2, nx // 2
    case1 = [(node(cy + dy, cx + dx, nz), 0.0, 0.0, -0.25) for dx in (0, 1) for dy in (0, 1)]
    case2 = [(node(y, nx, nz), 0.5 / nny, 0.0, 0.0) for y in range(nny)]
    elem = lambda y, x, z: 1 + y + ny * (x + nx * z)  # noqa: E731
    passive = sorted(elem(cy - 1 + dy, cx - 1 + dx, nz - 2 + dz) for dx in (0, 1) for dy in (0, 1) for dz in (0, 1))
    return vox, fixed, [case1, case2], passive


def write_topvoxel(path, vox, fixed, loads, passive=(), additional_loads=()):
    """Write a ``.TopVoxel`` v1.0 file (TOP3D_XL.m:448-497): fixed nodes get all three DOFs."""
    ny, nx, nz = vox.shape
    solid = np.flatnonzero(np.asarray(vox).ravel(order="F")) + 1
    with open(path, "w") as fh:
        fh.write("# TOP3D_XL voxel model\nVersion: 1.0\nResolution: %d %d %d\n" % (nx, ny, nz))
        fh.write("Density included: 0\nSolid voxels: %d\n" % solid.size)
        fh.write("\n".join(map(str, solid.tolist())) + "\n")
        fh.write("Passive elements: %d\n" % len(passive))
        for p in passive:
            fh.write("%d\n" % p)
        fh.write("Fixations: %d\n" % len(fixed))
        fh.write("".join("%d 1 1 1\n" % n for n in fixed))
        fh.write("Loads: %d\n" % len(loads))
        fh.write("".join("%d %.17g %.17g %.17g\n" % ld for ld in loads))
        fh.write("Additional Loads: %d\n" % len(additional_loads))
        for k, ld in enumerate(additional_loads, start=2):
            fh.write("Loads: %d %d\n" % (len(ld), k))
            fh.write("".join("%d %.17g %.17g %.17g\n" % l for l in ld))
