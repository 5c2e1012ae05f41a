"""Host mirror of the reference entry point ``TOP3D_XL(inputModel, consType, V0, nLoop, rMin, ...)``
(TOP3D_XL.m:4-19) over the C ABI of libtopx.so.

``Context`` wraps one ``topx_ctx`` (one design job on one GPU); ``TOP3D_XL`` keeps
the reference's signature, argument checks, console lines and ``./out/`` files
(RunLog.log, c_Target.dat, iters_Target.dat, sharp_Target.dat,
timing_Target.dat, TOP3D_XL.m:186-204) and the design files DesignVolume.nii (the padded
density volume, TOP3D_XL.m:564-570) and DesignVolume.stl (its 0.5 isosurface with caps,
TOP3D_XL.m:206-222, 572-577); the volume is also saved as DesignVolume.npy.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import _lib as L

# topx_params.precision: "mixed" runs the multigrid preconditioner in FP32 inside the FP64 Krylov
# iteration; "mixed32" also the PDE filter's CG in FP32
PRECISIONS = {"fp64": 0, "mixed": 1, "mixed32": 2}


class TopxError(RuntimeError):
    """A libtopx call returned an error status."""

    def __init__(self, code, msg):
        super().__init__(f"{L.ERRORS.get(code, code)}: {msg}")
        self.code = code


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Context:
    """One design job: model (host) + device engine (created on first GPU call)."""

    def __init__(self, precision: str = "fp64", device: int = 0, **settings):
        self.lib = L.load()
        p = L.Params()
        self.lib.topx_default_params(C.byref(p))
        if precision not in PRECISIONS:
            raise ValueError("precision must be one of %s" % ", ".join(PRECISIONS))
        p.precision = PRECISIONS[precision]
        p.device = device
        for k, v in settings.items():
            if not hasattr(p, k):
                raise ValueError(f"unknown setting {k}")
            if k == "typeVcycle" and isinstance(v, str):  # the reference's spelling (TX:34)
                if v not in ("Adapted", "Standard"):
                    raise ValueError("typeVcycle must be 'Adapted' or 'Standard'")
                v = 0 if v == "Adapted" else 1
            if k == "specifyPassiveRegions":
                v = (C.c_int * 3)(*[int(round(t)) for t in v])
            setattr(p, k, v)
        self.params = p
        self._h = C.c_void_p()
        self._check(self.lib.topx_create(C.byref(self._h), C.byref(p)))
        self.info = None

    def close(self):
        if self._h:
            self.lib.topx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st, allow=(L.TOPX_OK,)):
        if st in allow:
            return st
        msg = self.lib.topx_last_error(self._h) if self._h else b""
        raise TopxError(st, (msg or b"").decode())

    # ---- model --------------------------------------------------------------
    def load_voxels(self, vox):
        vox = np.asfortranarray(np.asarray(vox, dtype=bool)).astype(np.uint8, order="F")
        if vox.ndim != 3:
            raise ValueError("Inappropriate Input Model!")
        ny, nx, nz = vox.shape
        self._check(self.lib.topx_load_voxels(self._h, vox.ctypes.data_as(C.POINTER(C.c_uint8)), ny, nx, nz))
        return self._load_info()

    def load_topvoxel(self, path):
        self._check(self.lib.topx_load_topvoxel(self._h, os.fsencode(path)))
        return self._load_info()

    def set_bc(self, fixing, loads):
        """Boundary conditions as a .TopVoxel file gives them (topx_set_bc): ``fixing`` rows
        (node, fixX, fixY, fixZ), ``loads`` rows (node, Fx, Fy, Fz[, loadCase]) with 1-based node
        ids of the input model's (nely+1, nelx+1, nelz+1) node grid, y fastest."""
        fx = np.ascontiguousarray(np.asarray(fixing, dtype=np.float64).reshape(-1, 4))
        ld = np.asarray(loads, dtype=np.float64)
        ld = ld.reshape(-1, ld.shape[-1] if ld.ndim > 1 else 5)
        if ld.shape[1] == 4:
            ld = np.column_stack([ld, np.ones(len(ld))])
        ld = np.ascontiguousarray(ld)
        self._check(self.lib.topx_set_bc(self._h, _dptr(fx), len(fx), _dptr(ld), len(ld)))
        return self._load_info()

    def _load_info(self):
        inf = L.Info()
        self._check(self.lib.topx_get_info(self._h, C.byref(inf)))
        self.info = inf
        return inf

    @property
    def numElements(self):
        return int(self.info.numElements)

    @property
    def numDOFs(self):
        return int(self.info.numDOFs)

    def ke(self):
        out = np.empty(576)
        self._check(self.lib.topx_get_ke(self._h, _dptr(out)))
        return out.reshape(24, 24)

    def index_array(self, level: int, which: str):
        n = C.c_size_t()
        self._check(self.lib.topx_get_index_array(self._h, level, L.ARR[which], None, 0, C.byref(n)))
        out = np.empty(n.value, dtype=np.int32)
        self._check(self.lib.topx_get_index_array(self._h, level, L.ARR[which],
                                                  out.ctypes.data_as(C.POINTER(C.c_int32)), n.value, None))
        return out

    def transfer_coeffi(self, level: int):
        n = C.c_size_t()
        self._check(self.lib.topx_get_transfer_coeffi(self._h, level, None, 0, C.byref(n)))
        out = np.empty(n.value)
        self._check(self.lib.topx_get_transfer_coeffi(self._h, level, _dptr(out), n.value, None))
        return out

    def load_vector(self, lc: int = 0):
        out = np.empty(self.numDOFs)
        self._check(self.lib.topx_get_load(self._h, lc, _dptr(out), out.size))
        return out

    # ---- solver building blocks (GPU) -----------------------------------------
    def set_moduli(self, E):
        E = np.ascontiguousarray(E, dtype=np.float64)
        self._check(self.lib.topx_set_moduli(self._h, _dptr(E), E.size))

    def ku(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        y = np.empty_like(u)
        self._check(self.lib.topx_ku(self._h, _dptr(u), _dptr(y), u.size))
        return y

    def assemble(self):
        self._check(self.lib.topx_assemble(self._h))

    def vcycle(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty_like(r)
        self._check(self.lib.topx_vcycle(self._h, _dptr(r), _dptr(z), r.size))
        return z

    def diag(self, level: int):
        n = int(self.info.levelNodes[level - 1]) * 3
        out = np.empty(n)
        self._check(self.lib.topx_get_diag(self._h, level, _dptr(out), n))
        return out

    def pcg(self, u0=None, lc: int = 0):
        u = np.zeros(self.numDOFs) if u0 is None else np.array(u0, dtype=np.float64, copy=True)
        its = C.c_int()
        self._check(self.lib.topx_pcg(self._h, lc, _dptr(u), u.size, C.byref(its)))
        return u, its.value

    def filter(self, rmin, src):
        src = np.ascontiguousarray(src, dtype=np.float64)
        out = np.empty_like(src)
        its = C.c_int()
        self._check(self.lib.topx_filter(self._h, float(rmin), _dptr(src), _dptr(out), src.size, C.byref(its)))
        return out, its.value

    def unit_compliance(self, U):
        U = np.asfortranarray(np.asarray(U, dtype=np.float64).reshape(self.numDOFs, -1))
        ce = np.empty(self.numElements)
        self._check(self.lib.topx_unit_compliance(self._h, _dptr(U), _dptr(ce), ce.size))
        return ce

    # ---- optimisation --------------------------------------------------------
    def begin(self, consType, V0, nLoop, rMin, rHat=0.0):
        ct = {"GLOBAL": 0, "LOCAL": 1}[consType]
        cs = C.c_double()
        self._check(self.lib.topx_begin(self._h, ct, float(V0), int(nLoop), float(rMin), float(rHat), C.byref(cs)))
        return cs.value

    def step(self):
        it = L.Iter()
        st = self._check(self.lib.topx_step(self._h, C.byref(it)), allow=(L.TOPX_OK, L.TOPX_STOP))
        if st == L.TOPX_STOP:
            return None
        return dict(loop=it.loop, c=it.c, vol=it.vol, sharp=it.sharp, cons=it.cons, change=it.change,
                    its=[it.its[i] for i in range(max(1, self.info.numLoadCases))], filter_its=it.filter_its,
                    t_assemble=it.t_assemble, t_cg=it.t_cg, t_opt=it.t_opt, t_filter=it.t_filter,
                    t_total=it.t_total)

    # ---- measurement --------------------------------------------------------
    def timer_start(self):
        self._check(self.lib.topx_timer_start(self._h))

    def timer_stop(self):
        ms = C.c_double()
        self._check(self.lib.topx_timer_stop(self._h, C.byref(ms)))
        return ms.value

    def set_profiling(self, on=True):
        self._check(self.lib.topx_set_profiling(self._h, 1 if on else 0))

    def profile(self):
        p = L.Profile()
        self._check(self.lib.topx_get_profile(self._h, C.byref(p)))
        sections = {self.lib.topx_profile_section_name(i).decode(): (p.section_ms[i], p.section_count[i])
                    for i in range(L.NSECTIONS)}
        return dict(ku_ms=p.ku_ms, ku_launches=p.ku_launches, pcg_iterations=p.pcg_iterations, sections=sections)

    def launch_count(self):
        """Kernels launched by the library in this process so far (graph replays included)."""
        return int(self.lib.topx_launch_count())

    def density(self, out=None):
        """The physical density (compact element order).  out: an optional contiguous float64
        array of numElements entries to write into (e.g. page-locked host memory)."""
        if out is None:
            out = np.empty(self.numElements)
        elif out.dtype != np.float64 or out.size != self.numElements or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous float64 array of numElements entries")
        self._check(self.lib.topx_get_density(self._h, _dptr(out), out.size))
        return out

    def set_density(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        self._check(self.lib.topx_set_density(self._h, _dptr(x), x.size))

    def displacement(self, lc: int = 0):
        out = np.empty(self.numDOFs)
        self._check(self.lib.topx_get_displacement(self._h, lc, _dptr(out), out.size))
        return out


def write_design_files(vol, ny, nx, nz, out_dir, iso=0.5):
    """DesignVolume.nii and DesignVolume.stl from the padded density volume (column-major
    ny x nx x nz, void = 0) through topx_write_design_nii / topx_write_design_stl; returns the
    STL's triangle count."""
    lib = L.load()
    v = np.ascontiguousarray(np.asarray(vol, dtype=np.float64).reshape(-1, order="F") if np.ndim(vol) == 3
                             else np.asarray(vol, dtype=np.float64))
    if v.size != ny * nx * nz:
        raise ValueError("volume size does not match ny x nx x nz")
    st = lib.topx_write_design_nii(_dptr(v), ny, nx, nz, os.path.join(out_dir, "DesignVolume.nii").encode())
    if st != L.TOPX_OK:
        raise TopxError(st, "writing DesignVolume.nii")
    n = C.c_int64(0)
    st = lib.topx_write_design_stl(_dptr(v), ny, nx, nz, float(iso), os.path.join(out_dir, "DesignVolume.stl").encode(),
                                   C.byref(n))
    if st != L.TOPX_OK:
        raise TopxError(st, "writing DesignVolume.stl")
    return int(n.value)


def TOP3D_XL(inputModel, consType, V0, nLoop, rMin, *varargin, precision="fp64", out_dir="./out", verbose=True,
             device=0):
    """Drop-in for ``TOP3D_XL(inputModel, consType, V0, nLoop, rMin, [rHat])`` (TOP3D_XL.m:4-19).

    inputModel: boolean (nely, nelx, nelz) array (built-in cuboid BCs) or a
    ``.TopVoxel`` path.  consType: 'GLOBAL' or 'LOCAL' ('LOCAL' needs rHat).
    Returns a dict with the history and the final density (densityLayout_).
    """
    if consType not in ("GLOBAL", "LOCAL"):
        return None  # the reference's switch has no otherwise branch (TOP3D_XL.m:12-18)
    if consType == "LOCAL":
        if len(varargin) != 1:
            raise ValueError("Wrong Input!")
        rHat = float(varargin[0])
    else:
        rHat = 0.0
    t_all = time.perf_counter()
    os.makedirs(out_dir, exist_ok=True)
    log = open(os.path.join(out_dir, "RunLog.log"), "w")

    def say(s):
        log.write(s + "\n")
        if verbose:
            print(s)

    ctx = Context(precision=precision, device=device)
    try:
        say("==========================Displaying Inputs==========================")
        if consType == "GLOBAL":
            say("..............................................Volume Fraction: %6.4f" % V0)
        else:
            say("........................................Local Volume Fraction: %6.4f" % V0)
            say(".......................................Effecting Radius: %6.4f Cells" % rHat)
        say("..........................................Filter Radius: %6.4f Cells" % rMin)
        t0 = time.perf_counter()
        if isinstance(inputModel, (str, os.PathLike)):
            info = ctx.load_topvoxel(inputModel)
        else:
            info = ctx.load_voxels(inputModel)
        say("Preparing Voxel-based FEA Model Costs %10.1fs" % (time.perf_counter() - t0))
        say("Mesh Hierarchy...")
        say("             #Resolutions         #Elements   #DOFs")
        for l in range(info.numLevels):
            say("...Level %i: %4i x %4i x %4i %11i %11i" % (l + 1, info.resX[l], info.resY[l], info.resZ[l],
                                                           info.levelElements[l], 3 * info.levelNodes[l]))
        cSolid = ctx.begin(consType, V0, nLoop, rMin, rHat)
        say("Compliance of Fully Solid Domain: %16.6e" % cSolid)
        hist = []
        while True:
            r = ctx.step()
            if r is None:
                break
            hist.append(r)
            if consType == "GLOBAL":
                say(" It.:%4i Obj.:%16.8e Vol.:%6.4e Sharp.:%6.4e Cons.:%4.2e Ch.:%4.2e" %
                    (r["loop"], r["c"], r["vol"], r["sharp"], r["cons"], r["change"]))
            else:
                say(" It.:%4i Obj.:%16.8e Vol.:%6.4e Sharp.:%6.4e Cons.:%4.2e  Ch.:%4.2e " %
                    (r["loop"], r["c"], r["vol"], r["sharp"], r["cons"], r["change"]))
            say(" It.: %i (Time)... Total per-It.: %8.2es; Assemb.: %8.2es; CG: %8.2es; Opti.: %8.2es; "
                "Filtering: %8.2es." % (r["loop"], r["t_total"], r["t_assemble"], r["t_cg"], r["t_opt"],
                                        r["t_filter"]))
        xPhys = ctx.density()
        with open(os.path.join(out_dir, "iters_Target.dat"), "w") as fh:
            fh.writelines("%d\n" % k for r in hist for k in r["its"])
        with open(os.path.join(out_dir, "c_Target.dat"), "w") as fh:
            fh.writelines("%30.16e\n" % r["c"] for r in hist)
        with open(os.path.join(out_dir, "sharp_Target.dat"), "w") as fh:
            fh.writelines("%30.16e\n" % r["sharp"] for r in hist)
        with open(os.path.join(out_dir, "timing_Target.dat"), "w") as fh:
            fh.writelines("%16.6e\n" % r["t_total"] for r in hist)
        emb = ctx.index_array(1, "ELEMAPBACK")
        vol = np.zeros(info.resX[0] * info.resY[0] * info.resZ[0])
        vol[emb - 1] = xPhys
        np.save(os.path.join(out_dir, "DesignVolume.npy"),
                vol.reshape((info.resY[0], info.resX[0], info.resZ[0]), order="F"))
        write_design_files(vol, info.resY[0], info.resX[0], info.resZ[0], out_dir)
        say("..........Performing Topology Optimization Costs (in total): %10.4es." % (time.perf_counter() - t_all))
        return dict(cSolid=cSolid, history=hist, xPhys=xPhys, info=info)
    finally:
        ctx.close()
        log.close()


class Server:
    """Continuous-batching job server (topx_server_* in include/topx.h).

    Jobs are solid cuboids (or voxel masks) run through the same optimisation loop as
    ``TOP3D_XL``; up to ``slots`` of them are on the GPU at once, admitted by device-memory
    footprint against ``hbm_budget_bytes``.
    """

    def __init__(self, slots=6, precision="fp64", hbm_budget_bytes=0.0, device=0):
        self.lib = L.load()
        p = L.ServerParams()
        self.lib.topx_server_default_params(C.byref(p))
        p.slots = int(slots)
        p.precision = PRECISIONS[precision]
        p.hbm_budget_bytes = float(hbm_budget_bytes)
        p.device = int(device)
        self._h = C.c_void_p()
        st = self.lib.topx_server_create(C.byref(self._h), C.byref(p))
        if st != 0:
            raise TopxError(st, "topx_server_create failed")
        self._keep = {}

    def close(self):
        if self._h:
            self.lib.topx_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, shape=None, consType="GLOBAL", V0=0.12, nLoop=50, rMin=np.sqrt(3), rHat=0.0, voxels=None,
               keep_density=False):
        """Enqueue one job; returns its id at once."""
        j = L.Job()
        if voxels is not None:
            v = np.asfortranarray(np.asarray(voxels, dtype=np.uint8))
            j.nely, j.nelx, j.nelz = v.shape
            buf = np.ascontiguousarray(v.ravel(order="F"))
            j.voxels = buf.ctypes.data_as(C.POINTER(C.c_uint8))
        else:
            j.nely, j.nelx, j.nelz = shape
            j.voxels = None
        j.consType = {"GLOBAL": 0, "LOCAL": 1}.get(consType, -1)  # the C side rejects anything else
        j.V0, j.nLoop, j.rMin, j.rHat = float(V0), int(nLoop), float(rMin), float(rHat)
        j.keep_density = 1 if keep_density else 0
        jid = C.c_int64()
        st = self.lib.topx_server_submit(self._h, C.byref(j), C.byref(jid))
        if st != 0:
            raise TopxError(st, "topx_server_submit failed")
        return int(jid.value)

    @staticmethod
    def _res(r):
        return {k: getattr(r, k) for k, _ in L.JobResult._fields_}

    def poll(self, jid):
        r = L.JobResult()
        st = self.lib.topx_server_poll(self._h, jid, C.byref(r))
        return None if st == 1 else self._res(r)

    def wait(self, jid):
        r = L.JobResult()
        st = self.lib.topx_server_wait(self._h, jid, C.byref(r))
        if st != 0:
            raise TopxError(st, "topx_server_wait failed")
        return self._res(r)

    def history(self, jid):
        n = C.c_int()
        self.lib.topx_server_get_history(self._h, jid, None, 0, C.byref(n))
        arr = (L.Iter * max(1, n.value))()
        st = self.lib.topx_server_get_history(self._h, jid, arr, n.value, C.byref(n))
        if st != 0:
            raise TopxError(st, "topx_server_get_history failed")
        return [dict(loop=it.loop, c=it.c, vol=it.vol, sharp=it.sharp, cons=it.cons, change=it.change,
                     its=it.its[0]) for it in arr[:n.value]]

    def density(self, jid, numElements):
        out = np.empty(int(numElements))
        st = self.lib.topx_server_get_density(self._h, jid, _dptr(out), out.size)
        if st != 0:
            raise TopxError(st, "topx_server_get_density failed")
        return out

    def stats(self):
        s = L.ServerStats()
        self.lib.topx_server_get_stats(self._h, C.byref(s))
        return {k: getattr(s, k) for k, _ in L.ServerStats._fields_}

    def last_error(self):
        return self.lib.topx_server_last_error(self._h).decode()
