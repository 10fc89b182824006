"""Discrete-ordinates transport sweep over the reference's problem data.

``Sweep(device, MeshData, ordinates, physics)`` binds the C ABI's tr_sweep
(include/transfer_b200.h): the linear-discontinuous upwind sweep over the
`tetrahedron` / `face` records of MeshData (MeshData.h:13-32), with isotropic
scattering (``Physics.kappa_abs_volume``), vacuum / reflective / incident
faces (``Physics.face_bc``, ``face_incident``), GMRES or source iteration
over the scattering source, FP64 or FP32-in-FP64 defect correction.  The
reference has no sweep of its own.  Device vectors are torch CUDA tensors
(torch is only the allocator); every computation runs in libtransfer_b200.so.
"""
import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import check, lib
from .core import _ptr


def ordinates_product(n_polar, n_azim):
    """Gauss-Legendre (cos theta) x uniform azimuth ordinates: (x, y, z, w)."""
    n = int(n_polar) * int(n_azim)
    x, y, z, w = (np.zeros(n) for _ in range(4))
    check(lib.tr_ordinates_product(int(n_polar), int(n_azim), _ptr(x), _ptr(y), _ptr(z), _ptr(w)))
    return x, y, z, w


def lebedev(mindegree):
    """LebedevQuad(mindegree) as an ordinate set (x, y, z, w), weights summing
    to 1 (rules up to 350 points are generated)."""
    n = lib.tr_lebedev(int(mindegree), None, None, None, None, 0)
    if n < 0:
        raise ValueError(f"no Lebedev rule of degree {mindegree} is generated")
    x, y, z, w = (np.zeros(n) for _ in range(4))
    lib.tr_lebedev(int(mindegree), _ptr(x), _ptr(y), _ptr(z), _ptr(w), n)
    return x, y, z, w


class SweepReport(dict):
    __getattr__ = dict.__getitem__


class Sweep:
    """Sweep(device, md, ordinates=(x, y, z, w), physics=None, dsa=False).

    dsa=True prepares the diffusion operator for solve(precondition=
    TR_SWEEP_PREC_DSA) (tr_sweep_enable_dsa)."""

    def __init__(self, device, md, ordinates, physics=None, dsa=False):
        import torch  # device-memory plumbing only
        self._torch = torch
        self.ordinates = tuple(np.ascontiguousarray(a, dtype=np.float64) for a in ordinates)
        self._keep = (md, physics, self.ordinates)
        ov = L.tr_ordinates_view()
        ov.nq = len(self.ordinates[3])
        ov.x, ov.y, ov.z, ov.w = (_ptr(a) for a in self.ordinates)
        mv = md.view()
        pv = physics.view() if physics is not None else None
        h = C.c_void_p()
        check(lib.tr_sweep_create(int(device), C.byref(mv), C.byref(pv) if pv is not None else None, C.byref(ov),
                                  C.byref(h)))
        self._h = h
        info = L.tr_sweep_info()
        check(lib.tr_sweep_info_get(h, C.byref(info)))
        self.nT, self.nF, self.nq = info.nT, info.nF, info.nq
        self.n_extra, self.n_reflective, self.n_lag = info.n_extra, info.n_reflective, info.n_lag
        self.max_levels, self.forced_levels, self.device_bytes = info.max_levels, info.forced_levels, info.device_bytes
        self.device = device
        if dsa:
            self._c(lib.tr_sweep_enable_dsa(h, C.byref(mv), C.byref(pv) if pv is not None else None))

    def _c(self, st):
        if st != L.TR_OK:
            msg = lib.tr_sweep_last_error(self._h)
            raise L.TransferError(st, msg.decode() if msg else lib.tr_status_string(st).decode())
        return st

    def _dev(self, n, dtype=None):
        t = self._torch
        return t.zeros(max(int(n), 1), dtype=dtype or t.float64, device=f"cuda:{self.device}")

    def vector_J(self):
        return self._dev(4 * self.nT)

    def vector_B(self):
        return self._dev(self.n_extra)

    def levels(self):
        lv = np.zeros(self.nq * self.nT, dtype=np.int32)
        self._c(lib.tr_sweep_levels(self._h, _ptr(lv)))
        return lv.reshape(self.nq, self.nT)

    def apply(self, J=None, B=None, with_ext=True, precision=64):
        """One sweep; returns (J_out [nT,4], B_out [n_extra]) as device tensors."""
        Jo, Bo = self.vector_J(), self.vector_B()
        self._c(lib.tr_sweep_apply(self._h, int(precision), _ptr(J), _ptr(B), int(bool(with_ext)), _ptr(Jo),
                                   _ptr(Bo)))
        return Jo.view(self.nT, 4), Bo[:self.n_extra]

    def psi(self):
        out = self._dev(4 * self.nq * self.nT)
        self._c(lib.tr_sweep_psi(self._h, _ptr(out)))
        return out.view(self.nq, self.nT, 4)

    def set_moments_kernel(self, kind):
        """tr_sweep_set_moments_kernel: TR_MOMENTS_TCGEN05 (default), TR_MOMENTS_MMA_SYNC or
        TR_MOMENTS_TMA_FFMA2."""
        self._c(lib.tr_sweep_set_moments_kernel(self._h, int(kind)))

    def moments(self, nmom=16):
        out = self._dev(nmom * 4 * self.nT)
        self._c(lib.tr_sweep_moments(self._h, int(nmom), _ptr(out)))
        return out.view(nmom, self.nT, 4)

    def balance(self, J_in, B_in, J_out):
        out = (C.c_double * 5)()
        self._c(lib.tr_sweep_balance(self._h, _ptr(J_in), _ptr(B_in), _ptr(J_out), out))
        return dict(emitted=out[0], absorbed=out[1], escaped=out[2], incoming=out[3], reflective_net=out[4])

    def solve(self, raise_on_error=True, **kw):
        """Returns (J [nT,4], B [n_extra], report)."""
        o = L.tr_sweep_opts()
        lib.tr_sweep_opts_default(C.byref(o))
        for k, v in kw.items():
            if not hasattr(o, k):
                raise KeyError(k)
            setattr(o, k, v)
        J, B = self.vector_J(), self.vector_B()
        rep = L.tr_sweep_report()
        st = lib.tr_sweep_solve(self._h, C.byref(o), _ptr(J), _ptr(B), C.byref(rep))
        report = SweepReport({f: getattr(rep, f) for f, _ in L.tr_sweep_report._fields_})
        if st != L.TR_OK and (raise_on_error or st != L.TR_ERR_NOT_CONVERGED):
            self._c(st)
        return J.view(self.nT, 4), B[:self.n_extra], report

    def autotune(self):
        """tr_sweep_autotune: (shape kept, ms of one FP32 sweep full, small)."""
        shape = C.c_int()
        ms = (C.c_double * 2)()
        self._c(lib.tr_sweep_autotune(self._h, C.byref(shape), ms))
        return shape.value, ms[0], ms[1]

    def set_coefficients(self, kappa_volume, kappa_abs_volume=None, I_p=None):
        """Per-cell sigma_t V, sigma_a V (None: no scattering) and Planck
        intensity (None: kept), host arrays [nT]; geometry and schedule stay."""
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                for a in (kappa_volume, kappa_abs_volume, I_p)]
        self._c(lib.tr_sweep_set_coefficients(self._h, *(_ptr(a) for a in arrs)))

    def create_group(self, kappa_volume, kappa_abs_volume=None, I_p=None):
        """tr_sweep_create_group: a frequency group with its own per-cell
        sigma_t V, sigma_a V and Planck intensity, sharing this sweep's mesh,
        ordinates and schedule.  The group keeps this sweep alive."""
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                for a in (kappa_volume, kappa_abs_volume, I_p)]
        h = C.c_void_p()
        self._c(lib.tr_sweep_create_group(self._h, *(_ptr(a) for a in arrs), C.byref(h)))
        g = Sweep.__new__(Sweep)
        g._torch, g.ordinates, g._keep, g._h, g.device = self._torch, self.ordinates, (self,), h, self.device
        for k in ("nT", "nF", "nq", "n_extra", "n_reflective", "n_lag", "max_levels", "forced_levels"):
            setattr(g, k, getattr(self, k))
        info = L.tr_sweep_info()
        check(lib.tr_sweep_info_get(h, C.byref(info)))
        g.device_bytes = info.device_bytes
        return g

    def release_work(self):
        """tr_sweep_release_work: frees the angular flux and Krylov work space."""
        self._c(lib.tr_sweep_release_work(self._h))

    def set_batch_form(self, form):
        """tr_sweep_set_batch_form (TR_BATCH_*)."""
        self._c(lib.tr_sweep_set_batch_form(self._h, int(form)))

    def outflow(self, face_mask):
        """Outflow of the last sweep through the faces with face_mask != 0."""
        m = np.ascontiguousarray(face_mask, dtype=np.int32)
        F = C.c_double()
        self._c(lib.tr_sweep_outflow(self._h, _ptr(m), C.byref(F)))
        return F.value

    def bench(self, precision=32, iters=20):
        ms = C.c_double()
        self._c(lib.tr_sweep_bench(self._h, int(precision), int(iters), C.byref(ms)))
        return ms.value

    def __del__(self):
        if getattr(self, "_h", None):
            lib.tr_sweep_destroy(self._h)
            self._h = None


def sweep_apply_batch(sweeps, precision=64, J=None, B=None, with_ext=True):
    """One sweep of every problem in `sweeps` (distinct Sweep objects on one
    device) in a single kernel launch (tr_sweep_apply_batch).  J, B: lists of
    device inputs per problem (None = zero).  Returns [(J_out, B_out)]."""
    n = len(sweeps)
    arr = C.c_void_p * n

    def ptrs(lst):
        return None if lst is None else arr(*(_ptr(x) for x in lst))
    outs = [(S.vector_J(), S.vector_B()) for S in sweeps]
    hs = arr(*(S._h for S in sweeps))
    st = lib.tr_sweep_apply_batch(n, hs, int(precision), ptrs(J), ptrs(B), int(bool(with_ext)),
                                  arr(*(_ptr(o[0]) for o in outs)), arr(*(_ptr(o[1]) for o in outs)))
    if st != L.TR_OK:
        sweeps[0]._c(st)
    return [(Jo.view(S.nT, 4), Bo[:S.n_extra]) for S, (Jo, Bo) in zip(sweeps, outs)]


def sweep_autotune_batch(sweeps, precision=32):
    """tr_sweep_autotune_batch: times one batched sweep in each launch form,
    keeps the fastest on all the sweeps; returns (form, {form: ms})."""
    arr = (C.c_void_p * len(sweeps))(*[s._h for s in sweeps])
    form = C.c_int()
    ms = (C.c_double * 4)()
    st = lib.tr_sweep_autotune_batch(len(sweeps), arr, int(precision), C.byref(form), ms)
    if st != L.TR_OK:
        sweeps[0]._c(st)
    return form.value, {f: ms[f] for f in range(4) if ms[f] >= 0}


def sweep_solve_batch(sweeps, precision=64, tol=1e-10, max_iter=1000, raise_on_error=True):
    """Source iteration of every problem in `sweeps` at once, one batched
    sweep launch per iteration replayed from a CUDA graph
    (tr_sweep_solve_batch).  Returns ([(J, B)], iterations, residuals)."""
    n = len(sweeps)
    arr = C.c_void_p * n
    outs = [(S.vector_J(), S.vector_B()) for S in sweeps]
    its = np.zeros(n, dtype=np.int32)
    res = np.zeros(n)
    st = lib.tr_sweep_solve_batch(n, arr(*(S._h for S in sweeps)), int(precision), float(tol), int(max_iter),
                                  arr(*(_ptr(o[0]) for o in outs)), arr(*(_ptr(o[1]) for o in outs)), _ptr(its),
                                  _ptr(res))
    if st != L.TR_OK and (raise_on_error or st != L.TR_ERR_NOT_CONVERGED):
        sweeps[0]._c(st)
    return [(Jo.view(S.nT, 4), Bo[:S.n_extra]) for S, (Jo, Bo) in zip(sweeps, outs)], its, res


def adjoint_problem(md, physics, face_mask):
    """The adjoint of the outflow functional through face_mask's faces: the
    same mesh and coefficients without emission, unit isotropic inflow on
    those faces, vacuum elsewhere (the sweep runs in reversed ordinates)."""
    from .core import MeshData, Physics
    mesh = md.mesh.copy()
    mesh["I_p"] = 0.0
    md_adj = MeshData.from_arrays(tetstart=md.tetstart, tetidx=md.tetidx, tetpos=md.tetpos, facestart=md.facestart,
                                  faceidx=md.faceidx, facepos=md.facepos, mesh=mesh, bnd=md.bnd, coords=md.coords,
                                  regions=md.regions, kappa_abs_volume=md.kappa_abs_volume, face_side=md.face_side)
    mask = np.asarray(face_mask) != 0
    bc = np.where(mask, L.TR_BC_INCIDENT, L.TR_BC_VACUUM).astype(np.int32)
    kav = None if physics is None else physics.kappa_abs_volume
    return md_adj, Physics(kappa_abs_volume=kav, face_bc=bc, face_incident=mask.astype(np.float64))


def adjoint_gradient(device, md, ordinates, physics, face_mask, precision=64, mode=L.TR_MODE_FP64, tol=1e-10,
                     restart=30, fwd=None):
    """Outflow F through face_mask's faces and its gradient with respect to
    every cell's sigma_a and sigma_s.  Returns (F, dF/dsigma_a, dF/dsigma_s,
    forward report, adjoint report); the gradients are device tensors [nT]."""
    x, y, z, w = (np.ascontiguousarray(a, dtype=np.float64) for a in ordinates)
    fwd = fwd or Sweep(device, md, (x, y, z, w), physics)
    md_adj, ph_adj = adjoint_problem(md, physics, face_mask)
    adj = Sweep(device, md_adj, (-x, -y, -z, w), ph_adj)
    J, B, rep = fwd.solve(mode=mode, tol=tol, restart=restart)
    Ja, _, rep_a = adj.solve(mode=mode, tol=tol, restart=restart)
    fwd.apply(J, B, precision=64)
    F = fwd.outflow(face_mask)
    dsa, dss = fwd._dev(fwd.nT), fwd._dev(fwd.nT)
    fwd._c(lib.tr_sweep_gradient(fwd._h, adj._h, int(precision), _ptr(J), _ptr(B), _ptr(Ja), _ptr(dsa), _ptr(dss)))
    return F, dsa[:fwd.nT], dss[:fwd.nT], rep, rep_a

