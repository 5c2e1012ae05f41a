"""The synthetic irregular domain generator (top3d_xl_b200/workloads.py) and its .TopVoxel
file: the properties the workload is defined by, and the file read back identically by the
oracle's and the library's readers."""
import numpy as np

from oracle import top3dxl_oracle as O
from top3d_xl_b200.workloads import IRREGULAR_SMALL, irregular_domain, write_topvoxel


def test_generated_domain_has_the_stated_properties():
    vox, fixed, loads = irregular_domain(**IRREGULAR_SMALL)
    from scipy import ndimage
    _, n = ndimage.label(vox, structure=np.ones((3, 3, 3), int))
    assert n == 1  # one 26-connected component
    ny, nx, nz = vox.shape
    z0 = np.flatnonzero(vox.any(axis=(0, 1)))[0]
    fz = (np.array(fixed) - 1) // ((ny + 1) * (nx + 1))
    assert np.all(fz == z0)  # all on the lowest solid layer
    assert len(loads) == IRREGULAR_SMALL["n_loads"] and len({ld[0] for ld in loads}) == len(loads)
    assert np.allclose([np.linalg.norm(ld[1:]) for ld in loads], 1.0)
    assert not set(fixed) & {ld[0] for ld in loads}
    a, b, c = irregular_domain(**IRREGULAR_SMALL)  # seeded: the same domain again
    assert np.array_equal(a, vox) and b == fixed and c == loads


def test_topvoxel_file_reads_the_same_in_oracle_and_library(tmp_path):
    from top3d_xl_b200 import Context
    path = str(tmp_path / "d.TopVoxel")
    vox, fixed, loads = irregular_domain(**IRREGULAR_SMALL)
    write_topvoxel(path, vox, fixed, loads)
    m = O.build_model(path)
    with Context() as ctx:
        info = ctx.load_topvoxel(path)
        assert info.numElements == m.levels[0].numElements == int(vox.sum())
        assert np.array_equal(ctx.index_array(1, "FIXEDDOFS"), m.fixedDOFs.astype(np.int32))  # DOF mask
        assert np.allclose(ctx.load_vector(0), m.F[:, 0], rtol=0, atol=0)
