"""ctypes bindings for the CPU oracle (test infrastructure only).

The oracle restates the reference CPU backend (crates/backend-cpu/src/ops.rs)
and runtime solver loops of DenisChpt/fluxion in C (``fx_oracle.c``).  Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module; it is the checker, never the thing measured or shipped.

All arrays are C-contiguous float64 numpy arrays laid out row-major with the
boundary ring included.  Functions operate in place on their output arrays,
as the reference's ``&mut Buffer`` arguments do.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libfxoracle.so")

BC_DIRICHLET, BC_NEUMANN, BC_ROBIN, BC_PERIODIC = 0, 1, 2, 3

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_sz = C.c_size_t


class Bc(C.Structure):
    _fields_ = [("kind", C.c_int), ("a", C.c_double), ("b", C.c_double), ("g", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_size_t), ("residual", C.c_double), ("reason", C.c_int)]


class Op(C.Structure):
    _fields_ = [
        ("rows", C.c_size_t), ("cols", C.c_size_t), ("coeff", C.c_double), ("ne", C.c_int),
        ("dr", _ip), ("dc", _ip), ("w", _dp), ("bcs", C.POINTER(Bc)),
        ("cd", C.c_int), ("sigma", C.c_double), ("kappa_s", C.c_double), ("dx", C.c_double), ("dy", C.c_double),
        ("kappa", _dp), ("vx", _dp), ("vy", _dp),
    ]


PC_FN = C.CFUNCTYPE(None, C.c_void_p, _dp, _dp)

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            import importlib.util
            spec = importlib.util.spec_from_file_location("_fxo_build", os.path.join(HERE, "build.py"))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build()
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    def d(name, res, *args):
        f = getattr(L, name)
        f.restype = res
        f.argtypes = list(args)

    d("fxo_set_threads", None, C.c_int)
    d("fxo_get_threads", C.c_int)
    d("fxo_fill", None, _dp, _sz, C.c_double)
    d("fxo_copy", None, _dp, _dp, _sz)
    d("fxo_axpy", None, C.c_double, _dp, _dp, _sz)
    d("fxo_scale", None, _dp, _sz, C.c_double)
    d("fxo_waxpy", None, C.c_double, _dp, C.c_double, _dp, _dp, _sz)
    d("fxo_aypx", None, C.c_double, _dp, _dp, _sz)
    for n in ("mult", "div", "max", "min"):
        d("fxo_pointwise_" + n, None, _dp, _dp, _dp, _sz)
    d("fxo_reciprocal", None, _dp, _sz)
    d("fxo_abs_val", None, _dp, _sz)
    for n in ("fxo_norm_l2", "fxo_reduce_sum", "fxo_reduce_max", "fxo_reduce_min"):
        d(n, C.c_double, _dp, _sz)
    d("fxo_dot", C.c_double, _dp, _dp, _sz)
    d("fxo_dot2", None, _dp, _dp, _dp, _dp, _sz, _dp, _dp)
    bcp = C.POINTER(Bc)
    d("fxo_apply_stencil", C.c_int, _dp, _dp, _sz, _sz, C.c_double, C.c_double, C.c_int, _ip, _ip, _dp, bcp)
    d("fxo_apply_stencil_var", C.c_int, _dp, _dp, _dp, _sz, _sz, C.c_double, C.c_double, C.c_int, _ip, _ip, _dp, bcp)
    d("fxo_stencil_axpy", C.c_int, C.c_double, _dp, _dp, _sz, _sz, C.c_int, _ip, _ip, _dp, bcp)
    d("fxo_zero_boundaries", None, _dp, _sz, _sz)
    d("fxo_apply_conv_diff", None, _dp, _dp, _dp, _dp, _dp, _sz, _sz, C.c_double, C.c_double)
    d("fxo_conv_diff_axpy", None, C.c_double, _dp, _dp, _dp, _dp, _dp, _sz, _sz, C.c_double, C.c_double)
    d("fxo_restrict", C.c_int, _dp, _dp, _sz, _sz, _sz, _sz)
    d("fxo_prolong", C.c_int, _dp, _dp, _sz, _sz, _sz, _sz)
    d("fxo_weighted_jacobi", C.c_int, _dp, _dp, C.c_double, _sz, _sz, C.c_int, _ip, _ip, _dp)
    d("fxo_pcg_fused_update", None, C.c_double, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _sz)
    d("fxo_jacobi_sweep", None, _dp, _dp, _dp, C.c_double, _sz, _sz, _dp)
    d("fxo_residual", None, _dp, _dp, _dp, _sz, _sz, _dp)
    d("fxo_restrict_fw", C.c_int, _dp, _dp, _sz, _sz, _sz, _sz)
    d("fxo_prolong_bilinear", C.c_int, _dp, _dp, _sz, _sz, _sz, _sz)
    opp = C.POINTER(Op)
    stp = C.POINTER(Stats)
    d("fxo_cg_solve", C.c_int, opp, _dp, _dp, C.c_double, _sz, PC_FN, C.c_void_p, stp)
    d("fxo_pipelined_cg_solve", C.c_int, opp, _dp, _dp, C.c_double, _sz, stp)
    d("fxo_pipelined_pcg_solve", C.c_int, opp, _dp, _dp, C.c_double, _sz, PC_FN, C.c_void_p, stp)
    d("fxo_bicgstab_solve", C.c_int, opp, _dp, _dp, C.c_double, _sz, PC_FN, C.c_void_p, stp)
    d("fxo_gmres_solve", C.c_int, opp, _dp, _dp, _sz, C.c_double, _sz, PC_FN, C.c_void_p, stp)
    d("fxo_fcg_solve", C.c_int, opp, _dp, _dp, C.c_double, _sz, PC_FN, C.c_void_p, stp)
    d("fxo_fgmres_solve", C.c_int, opp, _dp, _dp, _sz, C.c_double, _sz, PC_FN, C.c_void_p, stp)
    d("fxo_inner_cg_pc_apply", None, C.c_void_p, _dp, _dp)
    d("fxo_op_apply", C.c_int, opp, _dp, _dp)
    d("fxo_cd_jacobi_apply", None, C.c_void_p, _dp, _dp)
    d("fxo_cdmg_create", C.c_void_p, opp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int)
    d("fxo_cdmg_destroy", None, C.c_void_p)
    d("fxo_cdmg_depth", C.c_int, C.c_void_p)
    d("fxo_cdmg_pc_apply", None, C.c_void_p, _dp, _dp)
    d("fxo_mg_create", C.c_void_p, _sz, _sz, C.c_double, C.c_double, bcp, C.c_int, C.c_int,
      C.c_double, C.c_int, C.c_double, C.c_int, _ip, _ip, _dp, C.c_int, C.c_int)
    d("fxo_mg_destroy", None, C.c_void_p)
    d("fxo_mg_set_smoother", C.c_int, C.c_void_p, C.c_int)
    d("fxo_mg_depth", C.c_int, C.c_void_p)
    d("fxo_mg_level_dims", None, C.c_void_p, C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t))
    d("fxo_mg_v_cycle", None, C.c_void_p, _dp, _dp)
    d("fxo_mg_v_cycle_f32", C.c_int, C.c_void_p, _dp, _dp)
    d("fxo_mg_coarse_op", None, _dp, C.c_double, _dp)


# ---------------------------------------------------------------- helpers

def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous, "oracle arrays must be contiguous f64"
    return a.ctypes.data_as(_dp)


def _stencil_arrays(entries):
    """entries: sequence of (dr, dc, w)."""
    n = len(entries)
    dr = (C.c_int * max(n, 1))(*[int(e[0]) for e in entries])
    dc = (C.c_int * max(n, 1))(*[int(e[1]) for e in entries])
    w = (C.c_double * max(n, 1))(*[float(e[2]) for e in entries])
    return n, dr, dc, w


def bcs_array(bcs):
    """bcs: 4 tuples (kind, a, b, g) for top, bottom, left, right."""
    arr = (Bc * 4)()
    for i, b in enumerate(bcs):
        arr[i].kind, arr[i].a, arr[i].b, arr[i].g = int(b[0]), float(b[1]), float(b[2]), float(b[3])
    return arr


ZERO_DIRICHLET = [(BC_DIRICHLET, 0.0, 0.0, 0.0)] * 4


def laplacian_5pt(dx, dy):
    """crates/core/src/stencil.rs:152-168, as (dr, dc, w) triples."""
    inv_dx2 = 1.0 / (dx * dx)
    inv_dy2 = 1.0 / (dy * dy)
    return [(0, 0, -2.0 * (inv_dx2 + inv_dy2)), (-1, 0, inv_dy2), (1, 0, inv_dy2),
            (0, -1, inv_dx2), (0, 1, inv_dx2)]


def set_threads(n: int) -> None:
    lib().fxo_set_threads(int(n))


def get_threads() -> int:
    return lib().fxo_get_threads()


class OracleError(RuntimeError):
    def __init__(self, code, what=""):
        super().__init__(f"oracle status {code} {what}")
        self.code = code


def _chk(code, what=""):
    if code != 0:
        raise OracleError(code, what)


# ---------------------------------------------------------------- ops

def fill(x, v): lib().fxo_fill(_p(x), x.size, v)
def copy(src, dst): lib().fxo_copy(_p(src), _p(dst), src.size)
def axpy(alpha, x, y): lib().fxo_axpy(alpha, _p(x), _p(y), x.size)
def scale(x, alpha): lib().fxo_scale(_p(x), x.size, alpha)
def waxpy(alpha, x, beta, y, w): lib().fxo_waxpy(alpha, _p(x), beta, _p(y), _p(w), x.size)
def aypx(alpha, x, y): lib().fxo_aypx(alpha, _p(x), _p(y), x.size)
def pointwise_mult(x, y, z): lib().fxo_pointwise_mult(_p(x), _p(y), _p(z), x.size)
def pointwise_div(x, y, z): lib().fxo_pointwise_div(_p(x), _p(y), _p(z), x.size)
def pointwise_max(x, y, z): lib().fxo_pointwise_max(_p(x), _p(y), _p(z), x.size)
def pointwise_min(x, y, z): lib().fxo_pointwise_min(_p(x), _p(y), _p(z), x.size)
def reciprocal(x): lib().fxo_reciprocal(_p(x), x.size)
def abs_val(x): lib().fxo_abs_val(_p(x), x.size)
def norm_l2(x): return lib().fxo_norm_l2(_p(x), x.size)
def reduce_sum(x): return lib().fxo_reduce_sum(_p(x), x.size)
def reduce_max(x): return lib().fxo_reduce_max(_p(x), x.size)
def reduce_min(x): return lib().fxo_reduce_min(_p(x), x.size)
def dot(x, y): return lib().fxo_dot(_p(x), _p(y), x.size)


def dot2(a, b, c, d):
    ab, cd = C.c_double(), C.c_double()
    lib().fxo_dot2(_p(a), _p(b), _p(c), _p(d), a.size, C.byref(ab), C.byref(cd))
    return ab.value, cd.value


def apply_stencil(inp, out, rows, cols, dx, dy, entries, bcs=ZERO_DIRICHLET):
    n, dr, dc, w = _stencil_arrays(entries)
    _chk(lib().fxo_apply_stencil(_p(inp), _p(out), rows, cols, dx, dy, n, dr, dc, w, bcs_array(bcs)),
         "apply_stencil")


def apply_stencil_var(inp, out, coeff, rows, cols, dx, dy, entries, bcs=ZERO_DIRICHLET):
    n, dr, dc, w = _stencil_arrays(entries)
    _chk(lib().fxo_apply_stencil_var(_p(inp), _p(out), _p(coeff), rows, cols, dx, dy, n, dr, dc, w,
                                     bcs_array(bcs)), "apply_stencil_var")


def stencil_axpy(alpha, x, y, rows, cols, entries, bcs=ZERO_DIRICHLET):
    n, dr, dc, w = _stencil_arrays(entries)
    _chk(lib().fxo_stencil_axpy(alpha, _p(x), _p(y), rows, cols, n, dr, dc, w, bcs_array(bcs)),
         "stencil_axpy")


def zero_boundaries(x, rows, cols): lib().fxo_zero_boundaries(_p(x), rows, cols)


def apply_conv_diff(u, out, kappa, vx, vy, rows, cols, dx, dy):
    lib().fxo_apply_conv_diff(_p(u), _p(out), _p(kappa), _p(vx), _p(vy), rows, cols, dx, dy)


def conv_diff_axpy(alpha, u, out, kappa, vx, vy, rows, cols, dx, dy):
    lib().fxo_conv_diff_axpy(alpha, _p(u), _p(out), _p(kappa), _p(vx), _p(vy), rows, cols, dx, dy)


def restrict(fine, coarse, fg, cg):
    _chk(lib().fxo_restrict(_p(fine), _p(coarse), fg[0], fg[1], cg[0], cg[1]), "restrict")


def prolong(coarse, fine, cg, fg):
    _chk(lib().fxo_prolong(_p(coarse), _p(fine), cg[0], cg[1], fg[0], fg[1]), "prolong")


def weighted_jacobi(x, b, omega, rows, cols, entries):
    n, dr, dc, w = _stencil_arrays(entries)
    _chk(lib().fxo_weighted_jacobi(_p(x), _p(b), omega, rows, cols, n, dr, dc, w), "weighted_jacobi")


def pcg_fused_update(alpha, beta, z, t, p, x, r, w, q):
    lib().fxo_pcg_fused_update(alpha, beta, _p(z), _p(t), _p(p), _p(x), _p(r), _p(w), _p(q), z.size)


def _a5(a5):
    arr = (C.c_double * 5)(*[float(v) for v in a5])
    return arr


def jacobi_sweep(x_in, x_out, b, omega, rows, cols, a5):
    lib().fxo_jacobi_sweep(_p(x_in), _p(x_out), _p(b), omega, rows, cols, _a5(a5))


def residual(x, b, r, rows, cols, a5):
    lib().fxo_residual(_p(x), _p(b), _p(r), rows, cols, _a5(a5))


def restrict_fw(fine, coarse, fg, cg):
    _chk(lib().fxo_restrict_fw(_p(fine), _p(coarse), fg[0], fg[1], cg[0], cg[1]), "restrict_fw")


def prolong_bilinear(coarse, fine, cg, fg):
    _chk(lib().fxo_prolong_bilinear(_p(coarse), _p(fine), cg[0], cg[1], fg[0], fg[1]),
         "prolong_bilinear")


def coarse_op(fine_a5, sigma):
    out = (C.c_double * 5)()
    lib().fxo_mg_coarse_op(_a5(fine_a5), sigma, out)
    return list(out)


# ---------------------------------------------------------------- solvers

def _op(rows, cols, coeff, entries, bcs):
    n, dr, dc, w = _stencil_arrays(entries)
    b = bcs_array(bcs)
    op = Op(rows, cols, coeff, n, dr, dc, w, b)
    op._keep = (dr, dc, w, b)
    return op


_NULL_PC = C.cast(None, PC_FN)


class Multigrid:
    """Oracle multigrid.  mode 0 = reference semantics (multigrid.rs), mode 1 = vertex-centred
    full-weighting / bilinear / true weighted Jacobi on the operator being solved."""

    def __init__(self, rows, cols, dx, dy, n_pre=2, n_post=2, omega=2.0 / 3.0, mode=0,
                 op_coeff=1.0, entries=None, bcs=ZERO_DIRICHLET, coarse_max=15, coarse_sweeps=200,
                 smoother=0, f32=False):
        entries = entries or laplacian_5pt(dx, dy)
        n, dr, dc, w = _stencil_arrays(entries)
        self._bcs = bcs_array(bcs)
        self.h = lib().fxo_mg_create(rows, cols, dx, dy, self._bcs, n_pre, n_post, omega, mode,
                                     op_coeff, n, dr, dc, w, coarse_max, coarse_sweeps)
        if not self.h:
            raise OracleError(6, "mg_create")
        if smoother:
            _chk(lib().fxo_mg_set_smoother(self.h, int(smoother)), "mg_set_smoother")
        if f32:  # the single-precision cycle on FP64 vectors (vertex mode only), from zero
            if mode != 1:
                raise OracleError(5, "the FP32 cycle exists for the vertex hierarchy only")
            self._cb = PC_FN(lambda ctx, z, r: lib().fxo_mg_v_cycle_f32(self.h, z, r))
        else:
            self._cb = PC_FN(lambda ctx, z, r: lib().fxo_mg_v_cycle(self.h, z, r))

    def depth(self):
        return lib().fxo_mg_depth(self.h)

    def level_dims(self, lvl):
        r, c = C.c_size_t(), C.c_size_t()
        lib().fxo_mg_level_dims(self.h, lvl, C.byref(r), C.byref(c))
        return r.value, c.value

    def v_cycle(self, x, b):
        lib().fxo_mg_v_cycle(self.h, _p(x), _p(b))

    def v_cycle_f32(self, z, r):
        """z = the FP32 cycle of r from zero (vertex mode), widened to FP64."""
        _chk(lib().fxo_mg_v_cycle_f32(self.h, _p(z), _p(r)), "mg_v_cycle_f32")

    def __del__(self):
        try:
            if self.h:
                lib().fxo_mg_destroy(self.h)
        except Exception:
            pass


class IdentityPC:
    """Identity preconditioner (preconditioner.rs:31-37): z = r."""

    def __init__(self, n):
        self.n = n
        self._cb = PC_FN(lambda ctx, z, r: lib().fxo_copy(r, z, n))


class InnerCg(C.Structure):
    _fields_ = [("op", C.c_void_p), ("steps", C.POINTER(C.c_size_t)), ("nsteps", C.c_size_t),
                ("calls", C.c_size_t), ("pc", PC_FN), ("pc_ctx", C.c_void_p)]


class InnerCgPC:
    """Nonlinear preconditioner (fxo_inner_cg_pc_apply): the k-th application runs
    steps[k % len(steps)] CG steps (preconditioned by `pc` when given) on A z = r from z = 0
    with tolerance 0.  A z = r is the operator v + coeff*S v on the same grid and rings."""

    def __init__(self, rows, cols, coeff, entries, steps, pc=None, bcs=ZERO_DIRICHLET):
        self._op = _op(rows, cols, coeff, entries, bcs)
        self._steps = (C.c_size_t * len(steps))(*[int(k) for k in steps])
        self._pc = pc  # kept alive with its callback
        fn, ctx = _pc_args(pc)
        self._ic = InnerCg(C.cast(C.pointer(self._op), C.c_void_p), self._steps, len(steps), 0, fn, ctx)
        self._cb = C.cast(lib().fxo_inner_cg_pc_apply, PC_FN)
        self._ctx = C.cast(C.pointer(self._ic), C.c_void_p)

    @property
    def calls(self):
        return self._ic.calls


def _pc_args(pc):
    if pc is None:
        return _NULL_PC, None
    return pc._cb, getattr(pc, "_ctx", None)


def cg_solve(x, b, rows, cols, coeff, entries, tol, max_iter, bcs=ZERO_DIRICHLET, pc=None):
    st = Stats()
    fn, ctx = _pc_args(pc)
    _chk(lib().fxo_cg_solve(C.byref(_op(rows, cols, coeff, entries, bcs)), _p(x), _p(b), tol,
                            max_iter, fn, ctx, C.byref(st)), "cg")
    return st.iterations, st.residual, st.reason


def pipelined_cg_solve(x, b, rows, cols, coeff, entries, tol, max_iter, bcs=ZERO_DIRICHLET):
    st = Stats()
    _chk(lib().fxo_pipelined_cg_solve(C.byref(_op(rows, cols, coeff, entries, bcs)), _p(x), _p(b),
                                      tol, max_iter, C.byref(st)), "pipelined_cg")
    return st.iterations, st.residual, st.reason


def pipelined_pcg_solve(x, b, rows, cols, coeff, entries, tol, max_iter, pc, bcs=ZERO_DIRICHLET):
    st = Stats()
    fn, ctx = _pc_args(pc)
    _chk(lib().fxo_pipelined_pcg_solve(C.byref(_op(rows, cols, coeff, entries, bcs)), _p(x), _p(b), tol,
                                       max_iter, fn, ctx, C.byref(st)), "pipelined_pcg")
    return st.iterations, st.residual, st.reason


def bicgstab_solve(x, b, rows, cols, coeff, entries, tol, max_iter, bcs=ZERO_DIRICHLET, pc=None):
    st = Stats()
    fn, ctx = _pc_args(pc)
    _chk(lib().fxo_bicgstab_solve(C.byref(_op(rows, cols, coeff, entries, bcs)), _p(x), _p(b), tol,
                                  max_iter, fn, ctx, C.byref(st)), "bicgstab")
    return st.iterations, st.residual, st.reason


def cd_op(rows, cols, dx, dy, vx, vy, kappa=None, kappa_s=0.0, sigma=1.0, coeff=1.0):
    """Conv-diff operator A v = sigma v + coeff (kappa Lap v + v.grad v) inside, v on the ring
    (fxo_op with cd = 1).  kappa: a field, or None for the scalar kappa_s.  The arrays must be
    contiguous float64 and are kept alive by the returned object."""
    vx = np.ascontiguousarray(vx, dtype=np.float64)
    vy = np.ascontiguousarray(vy, dtype=np.float64)
    k = None if kappa is None else np.ascontiguousarray(kappa, dtype=np.float64)
    op = Op()
    op.rows, op.cols, op.coeff = rows, cols, coeff
    op.cd, op.sigma, op.kappa_s, op.dx, op.dy = 1, sigma, kappa_s, dx, dy
    op.vx, op.vy = _p(vx), _p(vy)
    op.kappa = _p(k) if k is not None else C.cast(None, _dp)
    op._keep = (vx, vy, k)
    return op


def op_apply(op, v):
    """A v for an Op (stencil or conv-diff)."""
    out = np.empty_like(v)
    _chk(lib().fxo_op_apply(C.byref(op), _p(out), _p(np.ascontiguousarray(v))), "op_apply")
    return out


class CdJacobiPC:
    """z = r / diag(A) for a conv-diff Op (fxo_cd_jacobi_apply)."""

    def __init__(self, op):
        self._op = op
        self._cb = C.cast(lib().fxo_cd_jacobi_apply, PC_FN)
        self._ctx = C.cast(C.pointer(op), C.c_void_p)


class CdMultigrid:
    """V-cycle preconditioner for a conv-diff Op (fxo_cdmg_*): rediscretised coarse operators
    with injected fields, weighted Jacobi with the operator's diagonal, one cycle from z = 0."""

    def __init__(self, op, n_pre=2, n_post=2, omega=0.8, coarse_max=15, coarse_sweeps=200):
        self._op = op
        self.h = lib().fxo_cdmg_create(C.byref(op), n_pre, n_post, omega, coarse_max, coarse_sweeps)
        if not self.h:
            raise OracleError(6, "cdmg_create")
        self._cb = C.cast(lib().fxo_cdmg_pc_apply, PC_FN)
        self._ctx = C.c_void_p(self.h)

    def depth(self):
        return lib().fxo_cdmg_depth(self.h)

    def apply(self, r):
        z = np.zeros_like(r)
        lib().fxo_cdmg_pc_apply(self.h, _p(z), _p(np.ascontiguousarray(r)))
        return z

    def __del__(self):
        try:
            if self.h:
                lib().fxo_cdmg_destroy(self.h)
        except Exception:
            pass


def bicgstab_solve_op(x, b, op, tol, max_iter, pc=None):
    st = Stats()
    fn, ctx = _pc_args(pc)
    _chk(lib().fxo_bicgstab_solve(C.byref(op), _p(x), _p(b), tol, max_iter, fn, ctx, C.byref(st)), "bicgstab")
    return st.iterations, st.residual, st.reason


def gmres_solve_op(x, b, op, restart, tol, max_iter, pc=None):
    st = Stats()
    fn, ctx = _pc_args(pc)
    _chk(lib().fxo_gmres_solve(C.byref(op), _p(x), _p(b), restart, tol, max_iter, fn, ctx, C.byref(st)), "gmres")
    return st.iterations, st.residual, st.reason


def fgmres_solve_op(x, b, op, restart, tol, max_iter, pc=None):
    st = Stats()
    fn, ctx = _pc_args(pc)
    _chk(lib().fxo_fgmres_solve(C.byref(op), _p(x), _p(b), restart, tol, max_iter, fn, ctx, C.byref(st)), "fgmres")
    return st.iterations, st.residual, st.reason


def fcg_solve(x, b, rows, cols, coeff, entries, tol, max_iter, pc, bcs=ZERO_DIRICHLET):
    """Flexible CG (fxo_fcg_solve): PCG with the Polak-Ribiere beta."""
    st = Stats()
    fn, ctx = _pc_args(pc)
    _chk(lib().fxo_fcg_solve(C.byref(_op(rows, cols, coeff, entries, bcs)), _p(x), _p(b), tol,
                             max_iter, fn, ctx, C.byref(st)), "fcg")
    return st.iterations, st.residual, st.reason


def fgmres_solve(x, b, rows, cols, coeff, entries, restart, tol, max_iter, bcs=ZERO_DIRICHLET,
                 pc=None):
    """Flexible GMRES(m) (fxo_fgmres_solve): right preconditioning, z_k kept."""
    st = Stats()
    fn, ctx = _pc_args(pc)
    _chk(lib().fxo_fgmres_solve(C.byref(_op(rows, cols, coeff, entries, bcs)), _p(x), _p(b),
                                restart, tol, max_iter, fn, ctx, C.byref(st)), "fgmres")
    return st.iterations, st.residual, st.reason


def gmres_solve(x, b, rows, cols, coeff, entries, restart, tol, max_iter, bcs=ZERO_DIRICHLET,
                pc=None):
    st = Stats()
    fn, ctx = _pc_args(pc)
    _chk(lib().fxo_gmres_solve(C.byref(_op(rows, cols, coeff, entries, bcs)), _p(x), _p(b),
                               restart, tol, max_iter, fn, ctx, C.byref(st)), "gmres")
    return st.iterations, st.residual, st.reason
