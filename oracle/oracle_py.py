"""TEST INFRASTRUCTURE: ctypes binding of the C oracle (oracle/liboracle.so).

The oracle is the FP64 CPU restatement of the reference path that the CUDA
product is checked against.  Built by `make -C oracle`.
"""
import ctypes as C
import os

import numpy as np

ORACLE_SO = os.path.join(os.path.dirname(os.path.abspath(__file__)), "liboracle.so")


class or_mesh(C.Structure):
    _fields_ = [("nP", C.c_uint32), ("nT", C.c_uint32), ("nF", C.c_uint32),
                ("tetstart", C.c_void_p), ("tetidx", C.c_void_p), ("tetpos", C.c_void_p), ("mesh", C.c_void_p),
                ("facestart", C.c_void_p), ("faceidx", C.c_void_p), ("facepos", C.c_void_p), ("bnd", C.c_void_p),
                ("kappa_abs_volume", C.c_void_p), ("face_bc", C.c_void_p), ("face_incident", C.c_void_p)]


class or_ang(C.Structure):
    _fields_ = [("slm", C.c_uint32), ("aslm", C.c_uint32), ("omega", C.c_void_p), ("omega_pos", C.c_void_p),
                ("Ox", C.c_void_p), ("Oy", C.c_void_p), ("Oz", C.c_void_p)]


class or_cg_opts(C.Structure):
    _fields_ = [("precondition", C.c_int), ("max_iter", C.c_int), ("relative", C.c_int), ("tol", C.c_double),
                ("inner_tol", C.c_double), ("inner_max_iter", C.c_int), ("history_len", C.c_int),
                ("history", C.POINTER(C.c_double))]


class or_cg_result(C.Structure):
    _fields_ = [("iterations", C.c_int), ("inner_iterations", C.c_int), ("converged", C.c_int),
                ("final_residual", C.c_double), ("rhs_norm", C.c_double)]


def _load():
    if not os.path.exists(ORACLE_SO):
        raise ImportError(f"{ORACLE_SO} missing: run `make -C oracle`")
    lib = C.CDLL(ORACLE_SO)
    P, D, U32 = C.c_void_p, C.c_double, C.c_uint32
    sig = {
        "oracle_slm": (C.c_int, [C.c_int]),
        "oracle_angular": (None, [C.c_int, P, P, P, P, P]),
        "oracle_align_angular": (None, [U32, U32, P, P, P, P, P, P, P, P, P, P]),
        "oracle_ylm": (D, [C.c_int, C.c_int, D, D, D]),
        "oracle_compute_lhs": (None, [P, P, P, P]),
        "oracle_compute_lhs_diag": (None, [P, P, P, P]),
        "oracle_volume_part": (None, [P, P, P, P]),
        "oracle_surface_part": (None, [P, P, P, P]),
        "oracle_rhs": (None, [P, P, P]),
        "oracle_scale": (None, [C.c_uint64, P, D]),
        "oracle_add_prod": (None, [C.c_uint64, P, P, D]),
        "oracle_mul_add": (None, [C.c_uint64, P, D, P]),
        "oracle_mul_add_prod": (None, [C.c_uint64, P, D, P, D]),
        "oracle_norm": (D, [U32, U32, U32, P]),
        "oracle_dot": (D, [U32, U32, U32, P, P]),
        "oracle_cg": (C.c_int, [P, P, P, P, P, P]),
        "oracle_compute_moments": (None, [U32, U32, U32, P, P, P, P, P]),
        "oracle_compute_flux": (None, [P, P, P]),
        "oracle_trieig": (D, [P, P, U32]),
        "oracle_eigest": (D, [P, P, P, C.c_int, P, P]),
        "oracle_expint_en": (D, [C.c_int, D]),
        "oracle_sweep_create": (P, [P, U32, P, P, P, P, P]),
        "oracle_sweep_destroy": (None, [P]),
        "oracle_sweep_info": (None, [P, P]),
        "oracle_sweep_levels": (None, [P, P]),
        "oracle_sweep_apply": (None, [P, P, P, C.c_int, P, P, P]),
        "oracle_sweep_solve": (C.c_int, [P, C.c_int, D, C.c_int, C.c_int, P, P, P, P]),
        "oracle_sweep_balance": (None, [P, P, P, P, P]),
        "oracle_sweep_moments": (None, [P, P, C.c_int, P]),
        "oracle_ordinates_product": (None, [C.c_int, C.c_int, P, P, P, P]),
        "oracle_sweep_outflow": (D, [P, P, P]),
        "oracle_num_threads": (C.c_int, []),
        "oracle_set_num_threads": (None, [C.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def _p(a):
    return None if a is None else a.ctypes.data


def aslm_of(slm, real=8):
    q = 64 // real
    return (slm + q - 1) // q * q


class Oracle:
    """Binds a MeshData (numpy arrays, reference layout) and angular tables
    (unpadded, reference host layout) for the oracle kernels."""

    def __init__(self, md, ad, kappa_abs_volume=None, face_bc=None, face_incident=None):
        self.md = md
        self.slm = int(ad.slm)
        self.aslm = aslm_of(self.slm)
        n, a = self.slm, self.aslm
        self.omega_h = np.ascontiguousarray(ad.omega, dtype=np.float64).reshape(-1)
        self.omega_pos_h = np.ascontiguousarray(ad.omega_pos, dtype=np.uint32).reshape(-1)
        self.aomega = np.zeros(3 * a * a)
        self.apos = np.zeros(3 * a * a, dtype=np.uint32)
        self.aO = [np.zeros(a * a) for _ in range(3)]
        Os = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1) for x in (ad.Ox, ad.Oy, ad.Oz)]
        lib.oracle_align_angular(n, a, _p(self.omega_h), _p(self.omega_pos_h), _p(Os[0]), _p(Os[1]), _p(Os[2]),
                                 _p(self.aomega), _p(self.apos), _p(self.aO[0]), _p(self.aO[1]), _p(self.aO[2]))
        self.ang = or_ang(n, a, _p(self.aomega), _p(self.apos), _p(self.aO[0]), _p(self.aO[1]), _p(self.aO[2]))
        self.kav = None if kappa_abs_volume is None else np.ascontiguousarray(kappa_abs_volume, dtype=np.float64)
        self.fbc = None if face_bc is None else np.ascontiguousarray(face_bc, dtype=np.int32)
        self.finc = None if face_incident is None else np.ascontiguousarray(face_incident, dtype=np.float64)
        m = or_mesh()
        m.nP, m.nT, m.nF = md.nP, md.nT, md.nF
        m.tetstart, m.tetidx, m.tetpos = _p(md.tetstart), _p(md.tetidx), _p(md.tetpos)
        m.mesh = _p(md.mesh)
        m.facestart, m.faceidx, m.facepos = _p(md.facestart), _p(md.faceidx), _p(md.facepos)
        m.bnd = _p(md.bnd) if md.nF else None
        m.kappa_abs_volume, m.face_bc, m.face_incident = _p(self.kav), _p(self.fbc), _p(self.finc)
        self.mesh = m
        self.N = md.nP * self.aslm

    def vec(self):
        return np.zeros(self.N)

    def lhs(self, f):
        r = self.vec()
        lib.oracle_compute_lhs(C.byref(self.mesh), C.byref(self.ang), _p(np.ascontiguousarray(f)), _p(r))
        return r

    def lhs_diag(self, f):
        r = self.vec()
        lib.oracle_compute_lhs_diag(C.byref(self.mesh), C.byref(self.ang), _p(np.ascontiguousarray(f)), _p(r))
        return r

    def rhs(self):
        b = self.vec()
        lib.oracle_rhs(C.byref(self.mesh), C.byref(self.ang), _p(b))
        return b

    def norm(self, x):
        return lib.oracle_norm(self.md.nP, self.aslm, self.slm, _p(np.ascontiguousarray(x)))

    def dot(self, x, y):
        return lib.oracle_dot(self.md.nP, self.aslm, self.slm, _p(np.ascontiguousarray(x)),
                              _p(np.ascontiguousarray(y)))

    def cg(self, b=None, precondition=0, max_iter=1000, relative=0, tol=1e-4, inner_tol=1e-8, inner_max_iter=1000,
           history=0):
        o = or_cg_opts(precondition, max_iter, relative, tol, inner_tol, inner_max_iter, 0, None)
        hist = None
        if history:
            hist = np.zeros(history)
            o.history_len = history
            o.history = hist.ctypes.data_as(C.POINTER(C.c_double))
        f = self.vec()
        res = or_cg_result()
        bb = None if b is None else np.ascontiguousarray(b, dtype=np.float64)
        lib.oracle_cg(C.byref(self.mesh), C.byref(self.ang), C.byref(o), _p(bb), _p(f), C.byref(res))
        out = dict(iterations=res.iterations, inner_iterations=res.inner_iterations, converged=res.converged,
                   final_residual=res.final_residual, rhs_norm=res.rhs_norm)
        return (f, out, hist) if history else (f, out)

    def moments(self, f):
        nP = self.md.nP
        U, T = np.zeros(nP), np.zeros(9 * nP)
        lib.oracle_compute_moments(nP, self.slm, self.aslm, _p(self.omega_h), _p(self.omega_pos_h),
                                   _p(np.ascontiguousarray(f)), _p(U), _p(T))
        return U, T.reshape(3, 3, nP)

    def flux(self, T):
        W = np.zeros(3 * self.md.nT)
        lib.oracle_compute_flux(C.byref(self.mesh), _p(np.ascontiguousarray(T, dtype=np.float64).reshape(-1)),
                                _p(W))
        return W.reshape(3, self.md.nT)

    def eigest(self, v, max_steps=30):
        v = np.ascontiguousarray(v, dtype=np.float64).copy()
        extra, steps = C.c_double(), C.c_int()
        lmax = lib.oracle_eigest(C.byref(self.mesh), C.byref(self.ang), _p(v), max_steps, C.byref(extra),
                                 C.byref(steps))
        return lmax, extra.value, steps.value, v


def angular(maxk):
    """The oracle's own angular tables (unpadded), as a dict."""
    n = lib.oracle_slm(maxk)
    om, pos = np.zeros(3 * n * n), np.zeros(3 * n * n, dtype=np.uint32)
    Ox, Oy, Oz = np.zeros(n * n), np.zeros(n * n), np.zeros(n * n)
    lib.oracle_angular(maxk, _p(om), _p(pos), _p(Ox), _p(Oy), _p(Oz))
    return dict(slm=n, omega=om.reshape(3, n, n), omega_pos=pos.reshape(3, n, n), Ox=Ox.reshape(n, n),
                Oy=Oy.reshape(n, n), Oz=Oz.reshape(n, n))


def expint(n, x):
    return lib.oracle_expint_en(n, x)


def trieig(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return lib.oracle_trieig(_p(a), _p(b), len(a))


class or_sweep_mesh(C.Structure):
    _fields_ = [("nT", C.c_uint32), ("nF", C.c_uint32), ("mesh", C.c_void_p), ("bnd", C.c_void_p),
                ("kappa_abs_volume", C.c_void_p), ("face_bc", C.c_void_p), ("face_incident", C.c_void_p)]


def ordinates_product(n_polar, n_azim):
    """Gauss-Legendre (mu) x uniform azimuth ordinates; returns (x, y, z, w)."""
    n = n_polar * n_azim
    x, y, z, w = (np.zeros(n) for _ in range(4))
    lib.oracle_ordinates_product(n_polar, n_azim, _p(x), _p(y), _p(z), _p(w))
    return x, y, z, w


class SweepOracle:
    """FP64 CPU restatement of the linear-discontinuous discrete-ordinates
    sweep (oracle/sweep_oracle.h) bound to a MeshData and an ordinate set."""

    def __init__(self, md, ordinates, kappa_abs_volume=None, face_bc=None, face_incident=None):
        self.md = md
        self.ox, self.oy, self.oz, self.w = (np.ascontiguousarray(a, dtype=np.float64) for a in ordinates)
        self.nq, self.nT = len(self.w), int(md.nT)
        self.kav = None if kappa_abs_volume is None else np.ascontiguousarray(kappa_abs_volume, dtype=np.float64)
        self.fbc = None if face_bc is None else np.ascontiguousarray(face_bc, dtype=np.int32)
        self.finc = None if face_incident is None else np.ascontiguousarray(face_incident, dtype=np.float64)
        m = or_sweep_mesh(md.nT, md.nF, _p(md.mesh), _p(md.bnd) if md.nF else None, _p(self.kav), _p(self.fbc),
                          _p(self.finc))
        err = C.c_char_p()
        self.h = lib.oracle_sweep_create(C.byref(m), self.nq, _p(self.ox), _p(self.oy), _p(self.oz), _p(self.w),
                                         C.byref(err))
        if not self.h:
            raise ValueError(err.value.decode())
        info = np.zeros(6, dtype=np.int64)
        lib.oracle_sweep_info(self.h, _p(info))
        self.nB, self.n_reflective, self.n_lag, self.max_levels, self.forced, self.n_interior = (int(v) for v in info)

    def levels(self):
        lv = np.zeros(self.nq * self.nT, dtype=np.int32)
        lib.oracle_sweep_levels(self.h, _p(lv))
        return lv.reshape(self.nq, self.nT)

    def apply(self, J=None, B=None, with_ext=1, want_psi=False):
        Jo, Bo = np.zeros(4 * self.nT), np.zeros(max(self.nB, 1))
        psi = np.zeros(4 * self.nq * self.nT) if want_psi else None
        Ji = None if J is None else np.ascontiguousarray(J, dtype=np.float64).reshape(-1)
        Bi = None if B is None else np.ascontiguousarray(B, dtype=np.float64).reshape(-1)
        lib.oracle_sweep_apply(self.h, _p(Ji), _p(Bi), int(with_ext), _p(Jo), _p(Bo), _p(psi))
        out = (Jo.reshape(self.nT, 4), Bo[:self.nB])
        return out + ((psi.reshape(self.nq, self.nT, 4),) if want_psi else ())

    def solve(self, method=1, tol=1e-10, max_iter=500, restart=30):
        J, B = np.zeros(4 * self.nT), np.zeros(max(self.nB, 1))
        it, res = C.c_int(), C.c_double()
        rc = lib.oracle_sweep_solve(self.h, int(method), float(tol), int(max_iter), int(restart), _p(J), _p(B),
                                    C.byref(it), C.byref(res))
        return J.reshape(self.nT, 4), B[:self.nB], dict(converged=rc == 0, iterations=it.value, residual=res.value)

    def balance(self, J_in, B_in, psi):
        out = np.zeros(5)
        Ji = None if J_in is None else np.ascontiguousarray(J_in, dtype=np.float64).reshape(-1)
        Bi = None if B_in is None else np.ascontiguousarray(B_in, dtype=np.float64).reshape(-1)
        lib.oracle_sweep_balance(self.h, _p(Ji), _p(Bi), _p(np.ascontiguousarray(psi, dtype=np.float64).reshape(-1)),
                                 _p(out))
        return dict(emitted=out[0], absorbed=out[1], escaped=out[2], incoming=out[3], reflective_net=out[4])

    def outflow(self, psi, face_mask):
        m = np.ascontiguousarray(face_mask, dtype=np.int32)
        return lib.oracle_sweep_outflow(self.h, _p(np.ascontiguousarray(psi, dtype=np.float64).reshape(-1)), _p(m))

    def moments(self, psi, nmom=16):
        mom = np.zeros(nmom * 4 * self.nT)
        lib.oracle_sweep_moments(self.h, _p(np.ascontiguousarray(psi, dtype=np.float64).reshape(-1)), int(nmom),
                                 _p(mom))
        return mom.reshape(nmom, self.nT, 4)

    def __del__(self):
        if getattr(self, "h", None):
            lib.oracle_sweep_destroy(self.h)
            self.h = None


def tet_volumes(md):
    """V from the face area normals: |det(s_1, s_2, s_3)| = 9 V^2 / 2."""
    s = md.mesh["s"]
    return np.sqrt(np.abs(np.linalg.det(s[:, 1:4, :])) / 4.5)


def sweep_adjoint_gradient(md, ordinates, kappa_abs_volume, face_bc, face_incident, face_mask, tol=1e-13):
    """FP64 reference for the adjoint gradient of the outflow F through
    face_mask's faces with respect to each cell's sigma_a and sigma_s:
    forward and adjoint (reversed ordinates, unit inflow on the functional's
    faces, no emission) solves by the oracle, then per cell
      G = sum_q w_q mu_q^T M psi_q,  M = (1 + d_ij)/20,
      dF/dsigma_a = V (B/4) sum_i Phi_i - V G,  dF/dsigma_s = V Phi^T M J - V G.
    Returns (F, dsa, dss)."""
    x, y, z, w = (np.asarray(a, dtype=np.float64) for a in ordinates)
    Of = SweepOracle(md, (x, y, z, w), kappa_abs_volume=kappa_abs_volume, face_bc=face_bc,
                     face_incident=face_incident)
    J, B, info = Of.solve(method=1, tol=tol)
    _, _, psi = Of.apply(J, B, want_psi=True)
    F = Of.outflow(psi, face_mask)
    mesh = md.mesh.copy()
    mesh["I_p"] = 0.0

    class _Adj:  # the adjoint problem's mesh: same arrays, no emission
        pass
    ma = _Adj()
    ma.nT, ma.nF, ma.mesh, ma.bnd = md.nT, md.nF, mesh, md.bnd
    mask = np.asarray(face_mask) != 0
    Oa = SweepOracle(ma, (-x, -y, -z, w), kappa_abs_volume=kappa_abs_volume,
                     face_bc=np.where(mask, 2, 0).astype(np.int32), face_incident=mask.astype(np.float64))
    Ja, _, _ = Oa.solve(method=1, tol=tol)
    _, _, mu = Oa.apply(Ja, None, want_psi=True)
    G = np.einsum("q,qcj,qcj->c", w, mu, psi) + np.einsum("q,qc,qc->c", w, mu.sum(axis=2), psi.sum(axis=2))
    G /= 20.0
    V = tet_volumes(md)
    Bp = md.mesh["I_p"]
    PJ = ((Ja * J).sum(axis=1) + Ja.sum(axis=1) * J.sum(axis=1)) / 20.0
    dsa = V * (Bp / 4.0 * Ja.sum(axis=1) - G)
    dss = V * (PJ - G)
    return F, dsa, dss
