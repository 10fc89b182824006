"""Python mirror of the reference's host interfaces over the C ABI.

Names follow the reference: ``Config`` (Config.h:4-48), ``AngularData``
(AngularData.h:8-18), ``MeshData`` (MeshData.h:13-32) and ``CudaContext``
(CudaContext.h:9-50, methods computeLhs / computeLhsDiag / computeRhs /
scale / addProd / mulAdd / mulAddProd / norm / dot / allocVector / N).
Device vectors are torch CUDA tensors (or raw device addresses); torch is
only the allocator here, every computation runs in libtransfer_b200.so.
"""
import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import check, lib

TET_DTYPE = np.dtype([("p", "<u4", (4,)), ("kappa_volume", "<f8"), ("I_p", "<f8"), ("s", "<f8", (4, 3))])
FACE_DTYPE = np.dtype([("p", "<u4", (4,)), ("s", "<f8", (3,)), ("_pad", "<f8", (3,))])
assert TET_DTYPE.itemsize == 128 and FACE_DTYPE.itemsize == 64


def _ptr(a):
    """Address of a numpy array, a torch tensor or an int."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError(f"cannot take the address of {type(a)}")


def _carr(p, dtype, n):
    if not p or n == 0:
        return np.zeros(0, dtype=dtype)
    buf = (C.c_char * (n * np.dtype(dtype).itemsize)).from_address(p)
    return np.frombuffer(buf, dtype=dtype, count=n).copy()


class AngularData:
    """AngularData(maxk): slm, omega[3][slm][slm], omega_pos, Ox, Oy, Oz."""

    def __init__(self, maxk=None, *, tables=None):
        self._h = None
        if tables is not None:   # arbitrary (e.g. the reference's) tables
            self.slm = int(tables["slm"])
            n = self.slm
            self.omega = np.ascontiguousarray(tables["omega"], dtype=np.float64).reshape(3, n, n)
            self.omega_pos = np.ascontiguousarray(tables["omega_pos"], dtype=np.uint32).reshape(3, n, n)
            self.Ox = np.ascontiguousarray(tables["Ox"], dtype=np.float64).reshape(n, n)
            self.Oy = np.ascontiguousarray(tables["Oy"], dtype=np.float64).reshape(n, n)
            self.Oz = np.ascontiguousarray(tables["Oz"], dtype=np.float64).reshape(n, n)
            self.maxk = None
            return
        h = C.c_void_p()
        check(lib.tr_angular_create(int(maxk), C.byref(h)))
        self._h = h
        v = L.tr_angular_view()
        check(lib.tr_angular_view_get(h, C.byref(v)))
        n = self.slm = v.slm
        self.maxk = int(maxk)
        self.omega = _carr(v.omega, np.float64, 3 * n * n).reshape(3, n, n)
        self.omega_pos = _carr(v.omega_pos, np.uint32, 3 * n * n).reshape(3, n, n)
        self.Ox = _carr(v.Ox, np.float64, n * n).reshape(n, n)
        self.Oy = _carr(v.Oy, np.float64, n * n).reshape(n, n)
        self.Oz = _carr(v.Oz, np.float64, n * n).reshape(n, n)

    def view(self):
        v = L.tr_angular_view()
        v.slm = self.slm
        v.omega, v.omega_pos = _ptr(self.omega), _ptr(self.omega_pos)
        v.Ox, v.Oy, v.Oz = _ptr(self.Ox), _ptr(self.Oy), _ptr(self.Oz)
        return v

    def __del__(self):
        if getattr(self, "_h", None):
            lib.tr_angular_destroy(self._h)
            self._h = None


class Config:
    """Config(path): the radiation.cfg grammar (Config.cpp:8-131)."""

    def __init__(self, path):
        h = C.c_void_p()
        check(lib.tr_config_load(str(path).encode(), C.byref(h)))
        self._h = h

    def _int(self, key):
        ok = C.c_int()
        v = lib.tr_config_get_int(self._h, key.encode(), C.byref(ok))
        return v if ok.value else None

    def getMaxK(self):
        return self._int("angorder")

    def getDevice(self):
        return self._int("device")

    def doDump(self):
        return bool(self._int("dump"))

    def usePrec(self):
        return bool(self._int("precondition"))

    def solType(self):
        return self._int("soltype")

    def numRegions(self):
        return lib.tr_config_num_regions(self._h)

    def getMeshFilename(self):
        return lib.tr_config_get_string(self._h, b"meshfile").decode()

    def getOutFilename(self):
        return lib.tr_config_get_string(self._h, b"outfile").decode()

    def _region(self, r, key):
        ok = C.c_int()
        v = lib.tr_config_region_double(self._h, int(r), key.encode(), C.byref(ok))
        return v if ok.value else None

    def getKappa(self, r):
        return self._region(r, "kappa")

    def getIp(self, r):
        return self._region(r, "Ip")

    def region(self, r, key, default=None):
        v = self._region(r, key)
        return default if v is None else v

    def get(self, key, default=None):
        s = lib.tr_config_get_string(self._h, key.encode())
        return default if s is None else s.decode()

    def __del__(self):
        if getattr(self, "_h", None):
            lib.tr_config_destroy(self._h)
            self._h = None


class MeshData:
    """The reference's MeshData arrays (MeshData.h:13-32) as numpy arrays.

    Build with MeshData.kuhn(...), MeshData.from_tets(...) or
    MeshData.from_arrays(...) (arrays from any producer, e.g. the reference's
    own MeshData)."""

    def __init__(self):
        self._h = None

    @staticmethod
    def _rp(kappa, Ip, albedo):
        kappa = np.ascontiguousarray(kappa, dtype=np.float64)
        Ip = np.ascontiguousarray(Ip, dtype=np.float64)
        alb = None if albedo is None else np.ascontiguousarray(albedo, dtype=np.float64)
        rp = L.tr_region_params()
        rp.nreg = len(kappa) - 1
        rp.kappa, rp.Ip = _ptr(kappa), _ptr(Ip)
        rp.albedo = _ptr(alb)
        return rp, (kappa, Ip, alb)

    @classmethod
    def kuhn(cls, n, box=(0, 1, 0, 1, 0, 1), jitter=0.0, seed=20261203, kappa=(0.0, 1.0), Ip=(0.0, 1.0),
             albedo=None, region_kind=0, region_arg=(0, 0, 0, 0), ball=None):
        """Kuhn-split box of n=(nx,ny,nz) hexahedra (6 tets each).  kappa / Ip /
        albedo are per region, index 0 unused.  region_kind: 0 uniform,
        1 sphere (region_arg = cx, cy, cz, r -> region 1 inside, 2 outside),
        2 half space x < region_arg[0].  ball=(cx, cy, cz, R) keeps only tets
        whose centroid lies in the ball."""
        kp = L.tr_kuhn_params()
        for i in range(3):
            kp.n[i] = int(n[i])
        for i in range(6):
            kp.box[i] = float(box[i])
        kp.jitter, kp.seed, kp.region_kind = float(jitter), int(seed), int(region_kind)
        for i in range(4):
            kp.region_arg[i] = float(region_arg[i])
        if ball is not None:
            kp.ball = 1
            for i in range(3):
                kp.ball_center[i] = float(ball[i])
            kp.ball_radius = float(ball[3])
        rp, keep = cls._rp(kappa, Ip, albedo)
        h = C.c_void_p()
        check(lib.tr_meshdata_kuhn(C.byref(kp), C.byref(rp), C.byref(h)))
        return cls._from_handle(h)

    @classmethod
    def from_tets(cls, xyz, tets, region, kappa, Ip, albedo=None):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        tets = np.ascontiguousarray(tets, dtype=np.uint32)
        region = np.ascontiguousarray(region, dtype=np.int32)
        rp, keep = cls._rp(kappa, Ip, albedo)
        h = C.c_void_p()
        check(lib.tr_meshdata_from_tets(len(xyz), _ptr(xyz), len(tets), _ptr(tets), _ptr(region),
                                        C.byref(rp), C.byref(h)))
        return cls._from_handle(h)

    @classmethod
    def read_vol(cls, path, kappa, Ip, albedo=None):
        """Netgen .vol mesh (the reference's meshfile format); region of a
        tetrahedron = its matnr; face_bcnr = the bc number of each boundary
        face's surface element (-1 if none)."""
        rp, keep = cls._rp(kappa, Ip, albedo)
        h = C.c_void_p()
        check(lib.tr_meshdata_read_vol(str(path).encode(), C.byref(rp), C.byref(h)))
        md = cls._from_handle(h)
        fb = lib.tr_meshdata_face_bcnr(h)
        md.face_bcnr = _carr(fb, np.int32, md.nF) if fb else None
        return md

    def write_vtk(self, path, point_fields=None, cell_fields=None, real_bytes=8):
        """Legacy VTK of the mesh with fields, as the reference's saveVtk
        (main.cpp:209-216): each field is an array [n] (scalar), [3, n]
        (vector) or [6, n] (symmetric tensor xx xy xz yy yz zz)."""
        if not getattr(self, "_h", None):
            raise ValueError("write_vtk needs a MeshData built by this library (kuhn, from_tets, read_vol)")
        fields, keep = [], []
        for loc, group in ((L.TR_VTK_POINT, point_fields or {}), (L.TR_VTK_CELL, cell_fields or {})):
            for name, arr in group.items():
                a = np.ascontiguousarray(arr, dtype=np.float64)
                ncomp = 1 if a.ndim == 1 else a.shape[0]
                kind = {1: L.TR_VTK_SCALAR, 3: L.TR_VTK_VECTOR, 6: L.TR_VTK_TENSOR}[ncomp]
                keep.append(a)
                fields.append(L.tr_vtk_field(name.encode(), loc, kind, a.ctypes.data))
        arr_t = (L.tr_vtk_field * max(len(fields), 1))(*fields)
        check(lib.tr_vtk_write(str(path).encode(), self._h, int(real_bytes), len(fields), arr_t))

    @classmethod
    def _from_handle(cls, h):
        md = cls()
        md._h = h
        v = L.tr_mesh_view()
        check(lib.tr_meshdata_view_get(h, C.byref(v)))
        md.nP, md.nF, md.nT = v.nP, v.nF, v.nT
        md.tetstart = _carr(v.tetstart, np.uint32, v.nP + 1)
        nt = int(md.tetstart[-1])
        md.tetidx = _carr(v.tetidx, np.uint32, nt)
        md.tetpos = _carr(v.tetpos, np.uint32, nt)
        md.mesh = _carr(v.mesh, TET_DTYPE, v.nT)
        md.facestart = _carr(v.facestart, np.uint32, v.nP + 1)
        nf = int(md.facestart[-1])
        md.faceidx = _carr(v.faceidx, np.uint32, nf)
        md.facepos = _carr(v.facepos, np.uint32, nf)
        md.bnd = _carr(v.bnd, FACE_DTYPE, v.nF)
        md.coords = _carr(lib.tr_meshdata_coords(h), np.float64, 3 * v.nP).reshape(-1, 3)
        md.regions = _carr(lib.tr_meshdata_regions(h), np.int32, v.nT)
        kav = lib.tr_meshdata_kappa_abs_volume(h)
        md.kappa_abs_volume = _carr(kav, np.float64, v.nT) if kav else None
        fs = lib.tr_meshdata_face_side(h)
        md.face_side = _carr(fs, np.int32, v.nF) if fs else None
        return md

    @classmethod
    def from_arrays(cls, **a):
        md = cls()
        for k in ("tetstart", "tetidx", "tetpos", "facestart", "faceidx", "facepos"):
            setattr(md, k, np.ascontiguousarray(a[k], dtype=np.uint32))
        md.mesh = np.ascontiguousarray(a["mesh"]).view(TET_DTYPE).reshape(-1)
        md.bnd = np.ascontiguousarray(a["bnd"]).view(FACE_DTYPE).reshape(-1)
        md.nP = len(md.tetstart) - 1
        md.nT = len(md.mesh)
        md.nF = len(md.bnd)
        md.coords = a.get("coords")
        md.regions = a.get("regions")
        md.kappa_abs_volume = a.get("kappa_abs_volume")
        md.face_side = a.get("face_side")
        return md

    def view(self):
        v = L.tr_mesh_view()
        v.nP, v.nF, v.nT = self.nP, self.nF, self.nT
        v.tetstart, v.tetidx, v.tetpos = _ptr(self.tetstart), _ptr(self.tetidx), _ptr(self.tetpos)
        v.mesh = _ptr(self.mesh)
        v.facestart, v.faceidx, v.facepos = _ptr(self.facestart), _ptr(self.faceidx), _ptr(self.facepos)
        v.bnd = _ptr(self.bnd) if self.nF else None
        return v

    def __del__(self):
        if getattr(self, "_h", None):
            lib.tr_meshdata_destroy(self._h)
            self._h = None


class Physics:
    """Optional physics beyond the reference (tr_physics_view)."""

    def __init__(self, kappa_abs_volume=None, face_bc=None, face_incident=None, surface_mode=0):
        self.kappa_abs_volume = None if kappa_abs_volume is None else np.ascontiguousarray(kappa_abs_volume,
                                                                                           dtype=np.float64)
        self.face_bc = None if face_bc is None else np.ascontiguousarray(face_bc, dtype=np.int32)
        self.face_incident = None if face_incident is None else np.ascontiguousarray(face_incident,
                                                                                     dtype=np.float64)
        self.surface_mode = int(surface_mode)

    def view(self):
        v = L.tr_physics_view()
        v.kappa_abs_volume = _ptr(self.kappa_abs_volume)
        v.face_bc = _ptr(self.face_bc)
        v.face_incident = _ptr(self.face_incident)
        v.surface_mode = self.surface_mode
        return v


class SolveReport(dict):
    __getattr__ = dict.__getitem__


def solve_options(**kw):
    o = L.tr_solve_opts()
    lib.tr_solve_opts_default(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class CudaContext:
    """CudaContext(device, MeshData, AngularData[, Physics])."""

    def __init__(self, device, md, ad, physics=None):
        import torch  # device-memory plumbing only
        self._torch = torch
        self._keep = (md, ad, physics)
        mv, av = md.view(), ad.view()
        h = C.c_void_p()
        if physics is None:
            check(lib.tr_ctx_create(int(device), C.byref(mv), C.byref(av), C.byref(h)))
        else:
            pv = physics.view()
            check(lib.tr_ctx_create_ex(int(device), C.byref(mv), C.byref(av), C.byref(pv), C.byref(h)))
        self._h = h
        info = L.tr_ctx_info()
        check(lib.tr_ctx_info_get(h, C.byref(info)))
        self.nP, self.nT, self.nF = info.nP, info.nT, info.nF
        self.slm, self.aslm, self.aslm_f32 = info.slm, info.aslm, info.aslm_f32
        self.n_edges, self.n_bnd_edges = info.n_edges, info.n_bnd_edges
        self.device_bytes = info.device_bytes
        self.device = device

    # ---- reference interface
    def N(self):
        return self.nP * self.aslm

    def allocVector(self, dtype=None):
        t = self._torch
        dtype = dtype or t.float64
        n = self.nP * (self.aslm if dtype == t.float64 else self.aslm_f32)
        return t.zeros(n, dtype=dtype, device=f"cuda:{self.device}")

    def _c(self, st):
        return check(st, self._h)

    def computeLhs(self, f, Af):
        self._c(lib.tr_compute_lhs(self._h, _ptr(f), _ptr(Af)))

    def computeLhsDiag(self, f, Af):
        self._c(lib.tr_compute_lhs_diag(self._h, _ptr(f), _ptr(Af)))

    def computeRhs(self, b):
        self._c(lib.tr_compute_rhs(self._h, _ptr(b)))

    def computeLhs_f32(self, f, Af):
        self._c(lib.tr_compute_lhs_f32(self._h, _ptr(f), _ptr(Af)))

    def computeLhsDiag_f32(self, f, Af):
        self._c(lib.tr_compute_lhs_diag_f32(self._h, _ptr(f), _ptr(Af)))

    def computeRhs_f32(self, b):
        self._c(lib.tr_compute_rhs_f32(self._h, _ptr(b)))

    def scale(self, x, wx):
        self._c(lib.tr_scale(self._h, _ptr(x), float(wx)))

    def addProd(self, x, y, wy):
        self._c(lib.tr_add_prod(self._h, _ptr(x), _ptr(y), float(wy)))

    def mulAdd(self, x, wx, y):
        self._c(lib.tr_mul_add(self._h, _ptr(x), float(wx), _ptr(y)))

    def mulAddProd(self, x, wx, y, wy):
        self._c(lib.tr_mul_add_prod(self._h, _ptr(x), float(wx), _ptr(y), float(wy)))

    def norm(self, x):
        out = C.c_double()
        self._c(lib.tr_norm(self._h, _ptr(x), C.byref(out)))
        return out.value

    def dot(self, x, y):
        out = C.c_double()
        self._c(lib.tr_dot(self._h, _ptr(x), _ptr(y), C.byref(out)))
        return out.value

    def dot_f32(self, x, y):
        out = C.c_double()
        self._c(lib.tr_dot_f32(self._h, _ptr(x), _ptr(y), C.byref(out)))
        return out.value

    # ---- solver / post-processing
    def solve(self, b=None, f=None, history=0, raise_on_error=True, **opts):
        """tr_solve; returns (f, report[, history])."""
        o = solve_options(**opts)
        hist = None
        if history:
            hist = np.zeros(int(history), dtype=np.float64)
            o.history_len = len(hist)
            o.history = hist.ctypes.data_as(C.POINTER(C.c_double))
        if f is None:
            f = self.allocVector()
        rep = L.tr_solve_report()
        st = lib.tr_solve(self._h, C.byref(o), _ptr(b), _ptr(f), C.byref(rep))
        if raise_on_error and st not in (L.TR_OK, L.TR_ERR_NOT_CONVERGED):
            check(st, self._h)
        report = SolveReport({k: getattr(rep, k) for k, _ in L.tr_solve_report._fields_})
        report["status"] = st
        if history:
            return f, report, hist
        return f, report

    def solve_host(self, b_host=None, f_host=None, **opts):
        o = solve_options(**opts)
        if f_host is None:
            f_host = np.zeros(self.N(), dtype=np.float64)
        bh = None if b_host is None else np.ascontiguousarray(b_host, dtype=np.float64)
        rep = L.tr_solve_report()
        st = lib.tr_solve_host(self._h, C.byref(o), _ptr(bh), _ptr(f_host), C.byref(rep))
        if st not in (L.TR_OK, L.TR_ERR_NOT_CONVERGED):
            check(st, self._h)
        report = SolveReport({k: getattr(rep, k) for k, _ in L.tr_solve_report._fields_})
        report["status"] = st
        return f_host, report

    def computeMoments(self, f):
        t = self._torch
        U = t.zeros(self.nP, dtype=t.float64, device=f.device)
        T = t.zeros(9 * self.nP, dtype=t.float64, device=f.device)
        self._c(lib.tr_compute_moments(self._h, _ptr(f), _ptr(U), _ptr(T)))
        return U, T.view(3, 3, self.nP)

    def computeFlux(self, T):
        t = self._torch
        W = t.zeros(3 * self.nT, dtype=t.float64, device=T.device)
        self._c(lib.tr_compute_flux(self._h, _ptr(T.contiguous()), _ptr(W)))
        return W.view(3, self.nT)

    def eig_lanczos(self, v, max_steps=30):
        v0, w = self.allocVector(), self.allocVector()
        lmax, extra, steps = C.c_double(), C.c_double(), C.c_int()
        self._c(lib.tr_eig_lanczos(self._h, _ptr(v), _ptr(v0), _ptr(w), int(max_steps), C.byref(lmax),
                                   C.byref(extra), C.byref(steps)))
        return lmax.value, extra.value, steps.value

    def set_operator(self, kind):
        """TR_OPERATOR_TENSOR (default) or TR_OPERATOR_SIMT."""
        self._c(lib.tr_ctx_set_operator(self._h, int(kind)))

    def autotune_operator(self, iters=10):
        """tr_ctx_autotune_operator: times `iters` persistent CG iterations
        with each operator family in each precision and keeps the faster per
        precision.  Returns ({"fp64": kind, "fp32": kind},
        {(precision, kind): ms per CG iteration})."""
        ms = (C.c_double * 4)()
        self._c(lib.tr_ctx_autotune_operator(self._h, int(iters), ms))
        simt, tensor = L.TR_OPERATOR_SIMT, L.TR_OPERATOR_TENSOR
        return self.operator_kinds(), {(64, simt): ms[0], (64, tensor): ms[1], (32, simt): ms[2], (32, tensor): ms[3]}

    def operator_kinds(self):
        """tr_ctx_get_operator: {"fp64": kind, "fp32": kind}."""
        k = (C.c_int * 2)()
        self._c(lib.tr_ctx_get_operator(self._h, k))
        return {"fp64": k[0], "fp32": k[1]}

    def set_stream(self, stream):
        self._c(lib.tr_ctx_set_stream(self._h, _ptr(stream) if stream is not None else None))

    def close(self):
        if getattr(self, "_h", None):
            lib.tr_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def trieig(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return lib.tr_trieig(_ptr(a), _ptr(b), len(a))
