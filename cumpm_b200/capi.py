"""ctypes binding of the C ABI (include/cumpm_b200.h) with PyTorch at the edge.

``Field`` wraps the batched field operator on device buffers: moments and
fields are complex128 CUDA tensors of shape (rows, M), rows = 3N (+5Nq), the
same [row][M] layout the kernels use; self coefficients are (N, M).
``batch_solve`` runs the batched device Krylov solve on such tensors.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _load

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

MPM_OK, MPM_ERR_INVALID, MPM_ERR_RUNTIME, MPM_ERR_CUDA = 0, 1, 2, 3
FIELD_DIRECT, FIELD_MONO, FIELD_POLY = 0, 1, 2
MODE_SOLVER_AX, MODE_INTERACTION = 0, 1
METHOD_GMRES, METHOD_BICGSTAB = 0, 1

# every symbol the header declares (checked by the CPU test suite)
EXPORTS = [
    "mpm_last_error", "mpm_version",
    "mpm_solver_create", "mpm_solver_destroy", "mpm_solver_compute", "mpm_solver_dims",
    "mpm_solver_get_dipoles", "mpm_solver_get_quadrupoles", "mpm_solver_get_eff_polarizability",
    "mpm_solver_set_jacobi", "mpm_solver_get_jacobi", "mpm_solver_set_options", "mpm_solver_iterations",
    "mpm_near_create", "mpm_near_destroy", "mpm_near_set_dipoles", "mpm_near_set_dipole_positions",
    "mpm_near_set_field_points", "mpm_near_calculate",
    "mpm_field_create", "mpm_field_destroy", "mpm_field_set_positions", "mpm_field_set_field_points",
    "mpm_field_apply", "mpm_field_apply_part", "mpm_field_info_get", "mpm_batch_solve",
    "mpm_mono_tables", "mpm_ewald_geometry", "mpm_poly_geometry", "mpm_poly_pair_functions",
    "mpm_poly_quad_tables", "mpm_poly_quad_self",
    "mpm_profile_enable", "mpm_profile_reset", "mpm_profile_read", "mpm_kernel_launches",
    "mpm_field_apply_noalloc", "mpm_noalloc_scratch_bytes", "mpm_field_grad", "mpm_line_fft",
    "mpm_field_create_tuned", "mpm_field_autotune", "mpm_tune_xi_candidates", "mpm_tune_next_size",
    "mpm_solver_set_tuning", "mpm_solver_autotune", "mpm_field_set_bloch",
]

STAGES = ["spread", "fft_fwd", "kspace", "fft_inv", "contract", "real", "direct", "krylov", "precalc"]


class SolveOptions(C.Structure):
    _fields_ = [("method", C.c_int), ("restart", C.c_int), ("maxiter", C.c_int), ("tol", C.c_double),
                ("jacobi", C.c_int), ("recip_fp32", C.c_int), ("real_fp32", C.c_int), ("refine", C.c_int),
                ("inner_tol", C.c_double), ("compact", C.c_int), ("shifted", C.c_int)]


class SolveReport(C.Structure):
    _fields_ = [("matvecs", C.c_int), ("refine_steps", C.c_int), ("total_iterations", C.c_int),
                ("max_iterations", C.c_int), ("num_converged", C.c_int), ("max_rel_resid", C.c_double),
                ("column_matvecs", C.c_longlong), ("reorth_steps", C.c_int), ("shift_seeds", C.c_int),
                ("fp64_matvecs", C.c_int)]


class FieldInfo(C.Structure):
    _fields_ = [("kind", C.c_int), ("mode", C.c_int), ("num_particles", C.c_int), ("num_targets", C.c_int),
                ("num_quads", C.c_int), ("grid", C.c_int * 3), ("stencil", C.c_int), ("pruned", C.c_int),
                ("z_slots", C.c_int), ("num_pairs", C.c_longlong), ("rc", C.c_double), ("h", C.c_double * 3),
                ("eta", C.c_double * 3), ("selfo", C.c_double), ("slab_fused", C.c_int),
                ("single_layer", C.c_int)]


class FieldTuning(C.Structure):
    _fields_ = [("xi", C.c_double), ("grid", C.c_int * 3), ("support", C.c_int), ("tile", C.c_int * 2)]

    def as_dict(self):
        return {"xi": self.xi, "grid": tuple(self.grid), "support": self.support, "tile": tuple(self.tile)}


class TuneReport(C.Structure):
    _fields_ = [("apply_ms", C.c_double), ("apply_ms_rule", C.c_double), ("error", C.c_double),
                ("error_rule", C.c_double), ("error_bound", C.c_double), ("candidates", C.c_int),
                ("accepted", C.c_int)]


def make_tuning(xi, grid=(0, 0, 0), support=0, tile=(0, 0)):
    t = FieldTuning()
    t.xi = float(xi)
    for d in range(3):
        t.grid[d] = int(grid[d])
    t.support = int(support)
    t.tile[0], t.tile[1] = int(tile[0]), int(tile[1])
    return t


def lib():
    L = _load.library()
    if not getattr(L, "_mpm_typed", False):
        L.mpm_last_error.restype = C.c_char_p
        L.mpm_version.restype = C.c_char_p
        L.mpm_field_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, _dp, C.c_double, C.c_double, _dp,
                                       C.c_int, C.c_int, _ip, C.c_int]
        L.mpm_field_destroy.argtypes = [C.c_void_p]
        L.mpm_field_set_positions.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_int, C.c_void_p]
        L.mpm_field_set_field_points.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_int, C.c_void_p]
        L.mpm_field_apply.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                      C.c_int, C.c_void_p]
        L.mpm_field_apply_part.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                           C.c_int, C.c_int, C.c_void_p]
        L.mpm_field_info_get.argtypes = [C.c_void_p, C.POINTER(FieldInfo)]
        L.mpm_batch_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                      C.POINTER(SolveOptions), C.POINTER(SolveReport), C.c_void_p]
        L.mpm_mono_tables.argtypes = [C.c_double, _dp, _dp, _dp]
        L.mpm_ewald_geometry.argtypes = [_dp, C.c_double, C.c_double, _ip, _ip, _dp, _dp, _dp]
        L.mpm_poly_geometry.argtypes = [_dp, C.c_double, C.c_double, _dp, C.c_int, _ip, _ip, _dp, _dp, _ip, _ip]
        L.mpm_poly_pair_functions.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _dp, C.c_int,
                                              _dp, _dp, _dp]
        L.mpm_poly_quad_tables.argtypes = [C.c_double, C.c_double, _dp, C.c_size_t, _ip]
        L.mpm_poly_quad_self.argtypes = [C.c_double, _dp, C.c_int, _dp]
        L.mpm_profile_read.argtypes = [_dp, C.POINTER(C.c_longlong), C.c_int]
        L.mpm_field_apply_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                              C.c_int, C.c_int, C.c_void_p]
        L.mpm_noalloc_scratch_bytes.restype = C.c_size_t
        L.mpm_field_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                     C.c_void_p]
        L.mpm_kernel_launches.restype = C.c_longlong
        L.mpm_line_fft.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_size_t, C.c_int, C.c_size_t, C.c_int, C.c_int,
                                   C.c_void_p, C.c_int, C.c_int, C.c_int, _ip, C.c_void_p]
        L.mpm_field_create_tuned.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, _dp, C.c_double,
                                             C.POINTER(FieldTuning), _dp, C.c_int, C.c_int, _ip, C.c_int]
        L.mpm_field_autotune.argtypes = [C.c_int, _dp, C.c_double, C.c_double, _dp, C.c_int, C.c_int, _ip, C.c_int,
                                         _dp, _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(FieldTuning),
                                         C.POINTER(TuneReport), C.c_void_p]
        L.mpm_tune_xi_candidates.argtypes = [C.c_int, _dp, C.c_double, C.c_double, _dp, C.c_int, _dp, _ip, _ip, _dp,
                                             C.c_int, _ip]
        L.mpm_tune_next_size.argtypes = [C.c_int, C.c_int]
        L.mpm_field_set_bloch.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.mpm_solver_set_tuning.argtypes = [C.c_void_p, C.POINTER(FieldTuning)]
        L.mpm_solver_autotune.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_int, C.POINTER(FieldTuning),
                                          C.POINTER(TuneReport)]
        L._mpm_typed = True
    return L


def check(status):
    if status != MPM_OK:
        msg = lib().mpm_last_error().decode()
        if status == MPM_ERR_INVALID:
            raise ValueError(msg)
        raise RuntimeError(msg)


def _arr(a, dtype=np.float64):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a, a.ctypes.data_as(_dp if dtype == np.float64 else _ip)


def mono_tables(xi):
    """Host-side real-space tables: (r, {name: values}, selfo, self_grad)."""
    out = np.zeros(10 * 9001)
    so, sg = C.c_double(), C.c_double()
    check(lib().mpm_mono_tables(float(xi), out.ctypes.data_as(_dp), C.byref(so), C.byref(sg)))
    out = out.reshape(10, 9001)
    names = ["fd1", "fd2", "fq1", "fq2", "fq3", "gq1", "gq2", "gq3", "gq4"]
    return out[0], {n: out[i + 1] for i, n in enumerate(names)}, so.value, sg.value


def poly_quad_tables(xi, rc):
    """Radius-1 quadrupole tables of the polydisperse field for cutoff rc:
    (r, {name: values}) with names fq1, fq2, fq3, gq1, gq2, gq3, gq4."""
    n = C.c_int()
    check(lib().mpm_poly_quad_tables(float(xi), float(rc), None, 0, C.byref(n)))
    out = np.zeros(8 * n.value)
    check(lib().mpm_poly_quad_tables(float(xi), float(rc), out.ctypes.data_as(_dp), out.size, C.byref(n)))
    out = out.reshape(8, n.value)
    names = ["fq1", "fq2", "fq3", "gq1", "gq2", "gq3", "gq4"]
    return out[0], {k: out[i + 1] for i, k in enumerate(names)}


def poly_quad_self(xi, radii):
    """Quadrupole self value of each radius."""
    rr, rp = _arr(np.atleast_1d(radii))
    out = np.zeros(len(rr))
    check(lib().mpm_poly_quad_self(float(xi), rp, len(rr), out.ctypes.data_as(_dp)))
    return out


def poly_geometry(box, errortol, xi, radii):
    """Polydisperse grid, support, eta, cutoff and radius classes."""
    b, bp = _arr(box)
    rr, rp = _arr(radii)
    grid = (C.c_int * 3)()
    P, nc = C.c_int(), C.c_int()
    eta, rc = C.c_double(), C.c_double()
    cls = np.zeros(len(rr), dtype=np.int32)
    check(lib().mpm_poly_geometry(bp, float(errortol), float(xi), rp, len(rr), grid, C.byref(P), C.byref(eta),
                                  C.byref(rc), C.byref(nc), cls.ctypes.data_as(C.POINTER(C.c_int))))
    return dict(grid=list(grid), P=P.value, eta=eta.value, rc=rc.value, n_classes=nc.value, cls=cls)


def line_fft(data, n, es, ncols, os, nouter, mode=0, scale=None, sz=1, sb=1, general=False):
    """In-place batched line DFT of a complex64/complex128 CUDA tensor (the
    grid transform of the spectral-Ewald fields): element e of line o,
    column c at flat index o*os + e*es + c.  mode 0 forward, 1 inverse,
    2 forward * scale[(e*nouter + o)*sz + c//sb] then inverse (scale a real
    CUDA tensor of the matching precision).  Returns the two-pass split
    (r1, r2), (0, 0) when the multi-pass kernel ran."""
    import torch

    if not data.is_cuda or not data.is_contiguous() or data.dtype not in (torch.complex64, torch.complex128):
        raise ValueError("data must be a contiguous complex64/complex128 CUDA tensor")
    fp64 = data.dtype == torch.complex128
    sp = None
    if mode == 2:
        if scale is None or not scale.is_cuda or not scale.is_contiguous():
            raise ValueError("mode 2 needs a contiguous CUDA scale tensor")
        if scale.dtype != (torch.float64 if fp64 else torch.float32):
            raise ValueError("scale precision must match data")
        sp = C.c_void_p(scale.data_ptr())
    split = (C.c_int * 2)()
    stream = torch.cuda.current_stream(data.device).cuda_stream
    check(lib().mpm_line_fft(C.c_void_p(data.data_ptr()), int(fp64), int(n), int(es), int(ncols), int(os),
                             int(nouter), int(mode), sp, int(sz), int(sb), int(bool(general)), split,
                             C.c_void_p(stream)))
    return split[0], split[1]


def poly_pair_functions(a, b, xi, r, rc=None, lookup=False):
    """(fd1, fd2, self) of the polydisperse pair functions at distances r
    (the table lookup at r when lookup=True, for a cutoff rc)."""
    rr, rp = _arr(np.atleast_1d(r))
    f1 = np.zeros(len(rr))
    f2 = np.zeros(len(rr))
    sv = C.c_double()
    check(lib().mpm_poly_pair_functions(float(a), float(b), float(xi), float(rc or 0.0), int(lookup), rp, len(rr),
                                        f1.ctypes.data_as(_dp), f2.ctypes.data_as(_dp), C.byref(sv)))
    return f1, f2, sv.value


def ewald_geometry(box, errortol, xi):
    b, bp = _arr(box)
    grid = (C.c_int * 3)()
    st = C.c_int()
    rc = C.c_double()
    h = (C.c_double * 3)()
    eta = (C.c_double * 3)()
    check(lib().mpm_ewald_geometry(bp, float(errortol), float(xi), grid, C.byref(st), C.byref(rc), h, eta))
    return dict(grid=list(grid), stencil=st.value, rc=rc.value, h=list(h), eta=list(eta))


def profile_enable(on=True):
    check(lib().mpm_profile_enable(int(on)))


def profile_reset():
    check(lib().mpm_profile_reset())


def profile_read():
    """{stage: (milliseconds, intervals)} accumulated since the last reset."""
    ms = (C.c_double * 9)()
    cnt = (C.c_longlong * 9)()
    check(lib().mpm_profile_read(ms, cnt, 9))
    return {n: (ms[i], cnt[i]) for i, n in enumerate(STAGES)}


def kernel_launches():
    return int(lib().mpm_kernel_launches())


def _stream_ptr(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class Field:
    """Batched field operator A(omega) on CUDA tensors (see module docstring)."""

    def __init__(self, kind, box=None, errortol=1e-3, xi=0.5, mode=MODE_SOLVER_AX, radius=None, quad_idxs=None,
                 solve_quads=False, tuning=None):
        """tuning: a dict as ``autotune`` returns (xi, grid, support, tile;
        zeros keep the rule); its xi replaces ``xi``."""
        L = lib()
        self._h = C.c_void_p()
        bx, bp = _arr(box if box is not None else [0.0, 0.0, 0.0])
        rad = None if radius is None else np.ascontiguousarray(radius, dtype=np.float64)
        qi = None if quad_idxs is None else np.ascontiguousarray(quad_idxs, dtype=np.int32)
        tail = (None if rad is None else rad.ctypes.data_as(_dp), 0 if rad is None else len(rad),
                int(bool(solve_quads) or qi is not None),
                None if qi is None else qi.ctypes.data_as(_ip), 0 if qi is None else len(qi))
        if tuning is None:
            check(L.mpm_field_create(C.byref(self._h), int(kind), int(mode), bp, float(errortol), float(xi), *tail))
        else:
            t = make_tuning(tuning["xi"], tuning.get("grid", (0, 0, 0)), tuning.get("support", 0),
                            tuning.get("tile", (0, 0)))
            check(L.mpm_field_create_tuned(C.byref(self._h), int(kind), int(mode), bp, float(errortol),
                                           C.byref(t), *tail))
        self.kind = kind

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().mpm_field_destroy(h)
            except Exception:  # interpreter shutdown: module globals already cleared
                pass
            self._h = None

    def set_positions(self, pos, stream=None):
        p = np.ascontiguousarray(np.asarray(pos, dtype=np.float64))
        x, y, z = (np.ascontiguousarray(p[:, d]) for d in range(3))
        check(lib().mpm_field_set_positions(self._h, x.ctypes.data_as(_dp), y.ctypes.data_as(_dp),
                                            z.ctypes.data_as(_dp), len(p), _stream_ptr(stream)))

    def set_bloch(self, kx, ky):
        """Bloch wavevector (non-dimensional) of the periodic images: k-space
        at k - (kx, ky, 0), a phase on every real-space pair (dipoles only;
        (0, 0) is the plain operator)."""
        check(lib().mpm_field_set_bloch(self._h, float(kx), float(ky)))

    def set_field_points(self, pts, stream=None):
        p = np.ascontiguousarray(np.asarray(pts, dtype=np.float64))
        x, y, z = (np.ascontiguousarray(p[:, d]) for d in range(3))
        check(lib().mpm_field_set_field_points(self._h, x.ctypes.data_as(_dp), y.ctypes.data_as(_dp),
                                               z.ctypes.data_as(_dp), len(p), _stream_ptr(stream)))

    def info(self):
        fi = FieldInfo()
        check(lib().mpm_field_info_get(self._h, C.byref(fi)))
        return {k: (list(getattr(fi, k)) if k in ("grid", "h", "eta") else getattr(fi, k)) for k, _ in fi._fields_}

    def apply(self, X, Y=None, self_coef=None, jacobi=False, recip_fp32=False, real_fp32=False, stream=None):
        import torch
        assert X.is_cuda and X.dtype == torch.complex128 and X.is_contiguous() and X.dim() == 2
        info = self.info()
        rows_out = 3 * info["num_targets"] + 5 * info["num_quads"]
        if Y is None:
            Y = torch.empty((rows_out, X.shape[1]), dtype=torch.complex128, device=X.device)
        sc = None if self_coef is None else self_coef.contiguous()
        check(lib().mpm_field_apply(self._h, C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()), X.shape[1],
                                    None if sc is None else C.c_void_p(sc.data_ptr()), int(jacobi),
                                    int(recip_fp32), int(real_fp32), _stream_ptr(stream)))
        return Y

    def apply_part(self, X, part, self_coef=None, recip_fp32=False, real_fp32=False, stream=None):
        import torch
        info = self.info()
        rows_out = 3 * info["num_targets"] + 5 * info["num_quads"]
        if not (X.is_cuda and X.dtype == torch.complex128 and X.dim() == 2):
            raise ValueError("X must be a 2-D complex128 CUDA tensor")
        X = X.contiguous()
        Y = torch.zeros((rows_out, X.shape[1]), dtype=torch.complex128, device=X.device)
        sc = None if self_coef is None else self_coef.contiguous()
        check(lib().mpm_field_apply_part(self._h, C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()), X.shape[1],
                                         None if sc is None else C.c_void_p(sc.data_ptr()), int(recip_fp32),
                                         int(real_fp32), int(part), _stream_ptr(stream)))
        return Y

    def grad(self, lam, p, stream=None):
        """(gx [N,3], ga [N]) complex128: d/dx and d/d(radius) of sum_m lam_m^T G p_m."""
        import torch
        assert lam.is_cuda and p.is_cuda and lam.shape == p.shape and lam.dtype == torch.complex128
        N = self.info()["num_particles"]
        gx = torch.empty((N, 3), dtype=torch.complex128, device=p.device)
        ga = torch.empty((N,), dtype=torch.complex128, device=p.device)
        check(lib().mpm_field_grad(self._h, C.c_void_p(lam.contiguous().data_ptr()), C.c_void_p(p.contiguous().data_ptr()),
                                   p.shape[1], C.c_void_p(gx.data_ptr()), C.c_void_p(ga.data_ptr()),
                                   _stream_ptr(stream)))
        return gx, ga

    def batch_solve(self, B, X, self_coef, tol, method=METHOD_GMRES, restart=50, maxiter=1000, jacobi=True,
                    recip_fp32=True, real_fp32=False, refine=False, inner_tol=1e-4, compact=True, shifted=True,
                    stream=None):
        import torch
        for name, t in (("B", B), ("X", X), ("self_coef", self_coef)):
            if not (t.is_cuda and t.dtype == torch.complex128 and t.dim() == 2):
                raise ValueError(f"{name} must be a 2-D complex128 CUDA tensor")
        if not X.is_contiguous():
            raise ValueError("X is updated in place and must be contiguous")
        if X.shape != B.shape or self_coef.shape[1] != B.shape[1]:
            raise ValueError("B, X and self_coef must have the same number of columns")
        B = B.contiguous()
        self_coef = self_coef.contiguous()
        o = SolveOptions(int(method), int(restart), int(maxiter), float(tol), int(jacobi), int(recip_fp32),
                         int(real_fp32), int(refine), float(inner_tol), int(compact), int(shifted))
        r = SolveReport()
        check(lib().mpm_batch_solve(self._h, C.c_void_p(B.data_ptr()), C.c_void_p(X.data_ptr()), B.shape[1],
                                    C.c_void_p(self_coef.data_ptr()), C.byref(o), C.byref(r), _stream_ptr(stream)))
        return {k: getattr(r, k) for k, _ in r._fields_}


def autotune(kind, box, errortol, xi, pos, M, radius=None, quad_idxs=None, solve_quads=False, recip_fp32=True,
             real_fp32=False, stream=None):
    """Tune a SOLVER_AX field (xi, grid, support, spread tile) for the
    positions pos (N, 3, non-dimensional) and a batch of M columns; returns
    the pick and the report as one dict (see mpm_field_autotune)."""
    L = lib()
    bx, bp = _arr(box)
    p = np.ascontiguousarray(np.asarray(pos, dtype=np.float64))
    x, y, z = (np.ascontiguousarray(p[:, d]) for d in range(3))
    rad = None if radius is None else np.ascontiguousarray(radius, dtype=np.float64)
    qi = None if quad_idxs is None else np.ascontiguousarray(quad_idxs, dtype=np.int32)
    t, r = FieldTuning(), TuneReport()
    check(L.mpm_field_autotune(int(kind), bp, float(errortol), float(xi),
                               None if rad is None else rad.ctypes.data_as(_dp), 0 if rad is None else len(rad),
                               int(bool(solve_quads) or qi is not None),
                               None if qi is None else qi.ctypes.data_as(_ip), 0 if qi is None else len(qi),
                               x.ctypes.data_as(_dp), y.ctypes.data_as(_dp), z.ctypes.data_as(_dp), len(p), int(M),
                               int(bool(recip_fp32)), int(bool(real_fp32)), C.byref(t), C.byref(r),
                               _stream_ptr(stream)))
    out = t.as_dict()
    out.update({k: getattr(r, k) for k, _ in r._fields_})
    return out


def tune_xi_candidates(kind, box, errortol, xi, radius=None):
    """Host only: the tuner's first-stage xi candidates as a list of dicts
    (xi, grid, support, rc)."""
    L = lib()
    bx, bp = _arr(box)
    rad = None if radius is None else np.ascontiguousarray(radius, dtype=np.float64)
    n = C.c_int()
    args = (int(kind), bp, float(errortol), float(xi), None if rad is None else rad.ctypes.data_as(_dp),
            0 if rad is None else len(rad))
    check(L.mpm_tune_xi_candidates(*args, None, None, None, None, 0, C.byref(n)))
    k = n.value
    xs, gs, ps, rs = np.zeros(k), np.zeros(3 * k, np.int32), np.zeros(k, np.int32), np.zeros(k)
    check(L.mpm_tune_xi_candidates(*args, xs.ctypes.data_as(_dp), gs.ctypes.data_as(_ip), ps.ctypes.data_as(_ip),
                                   rs.ctypes.data_as(_dp), k, C.byref(n)))
    return [{"xi": xs[i], "grid": tuple(int(g) for g in gs[3 * i:3 * i + 3]), "support": int(ps[i]), "rc": rs[i]}
            for i in range(k)]


def tune_next_size(n, smooth23=False):
    """Host only: smallest length >= n with prime factors 2, 3, 5, 7 (or
    2, 3 with smooth23)."""
    return lib().mpm_tune_next_size(int(n), int(bool(smooth23)))
