"""B200 (sm_100a) compact Helmholtz direct solver -- Python host mirror of the C ABI.

The product is the in-tree shared library `libhh.so` (CUDA kernels for sm_100a behind the
C ABI of include/hh.h) and the drop-in libraries `libhh2d.so` / `libhh3d.so` that export the
reference's own entry points (solver(System), forwardDST, reverseDST, DST).  This module only
loads `libhh.so` with ctypes and wraps its calls; it has no numerical code of its own and no
CPU fallback -- if the library or a GPU is missing, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhh.so")
DROPIN2D_PATH = os.path.join(HERE, "libhh2d.so")
DROPIN3D_PATH = os.path.join(HERE, "libhh3d.so")

HH_OK = 0
STATUS = {0: "HH_OK", 1: "HH_ERR_INVALID", 2: "HH_ERR_CUDA", 3: "HH_ERR_NOMEM", 4: "HH_ERR_UNSUPPORTED",
          5: "HH_ERR_DEVICE"}

# every symbol include/hh.h declares, with its ctypes signature
_vp, _i, _l, _d, _sz = C.c_void_p, C.c_int, C.c_long, C.c_double, C.c_size_t
_dp = C.POINTER(C.c_double)


class Request(C.Structure):
    """include/hh.h hh_request"""
    _fields_ = [("dim", C.c_int), ("n", C.c_int), ("order", C.c_int), ("k_re", C.c_double), ("k_im", C.c_double),
                ("nrhs", C.c_int), ("on_device", C.c_int), ("f", C.c_void_p), ("u", C.c_void_p)]


class RequestInfo(C.Structure):
    """include/hh.h hh_request_info"""
    _fields_ = [("status", C.c_int), ("t_submit", C.c_double), ("t_start", C.c_double), ("t_done", C.c_double),
                ("batch_rhs", C.c_int)]


class Rhs2DData(C.Structure):
    """include/hh.h hh_rhs2d_data"""
    _fields_ = [("order", C.c_int), ("hx", C.c_double), ("hy", C.c_double)] + \
               [(nm, C.c_void_p) for nm in ("f_ext", "k_ext", "k2y_bc", "fxx_xb", "fxx_yb", "fyy_xb", "fyy_yb",
                                            "fy_yb", "u_xb", "u_yb")]


class Rhs3DData(C.Structure):
    """include/hh.h hh_rhs3d_data"""
    _fields_ = [("order", C.c_int), ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double)] + \
               [(nm, C.c_void_p) for nm in ("f_ext", "k2_ext", "kz_bc", "fxx_b", "fyy_b", "fzz_b", "ue_ext")]


SIGNATURES = {
    "hh_last_error": (C.c_char_p, []),
    "hh_version": (_i, []),
    "hh_ctx_create": (_i, [_i, _vp, C.POINTER(_vp)]),
    "hh_ctx_destroy": (_i, [_vp]),
    "hh_ctx_set_stream": (_i, [_vp, _vp]),
    "hh_ctx_synchronize": (_i, [_vp]),
    "hh_ctx_launch_count": (C.c_longlong, [_vp]),
    "hh_ctx_inject_wait_expiry": (_i, [_vp]),
    "hh_malloc": (_i, [_vp, _sz, C.POINTER(_vp)]),
    "hh_free": (_i, [_vp, _vp]),
    "hh_memcpy_h2d": (_i, [_vp, _vp, _vp, _sz]),
    "hh_memcpy_d2h": (_i, [_vp, _vp, _vp, _sz]),
    "hh_dst1_rows": (_i, [_vp, _i, _l, _vp, _l, _vp, _l]),
    "hh_dst1_cols": (_i, [_vp, _i, _l, _l, _vp, _l, _l, _vp]),
    "hh_dst2_planes": (_i, [_vp, _i, _i, _l, _vp, _vp]),
    "hh_lines_pack": (_i, [_vp, _vp, _vp, _l, _l, _l, _i, _i]),
    "hh_plan2d_create": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, C.POINTER(_vp)]),
    "hh_plan3d_create": (_i, [_vp, _i, _i, _i, C.POINTER(_vp), C.POINTER(_vp)]),
    "hh_plan2d_create_helmholtz": (_i, [_vp, _i, _i, _d, _d, C.POINTER(_vp)]),
    "hh_plan3d_create_helmholtz": (_i, [_vp, _i, _i, _d, _d, C.POINTER(_vp)]),
    "hh_plan3d_create_helmholtz_lines": (_i, [_vp, _i, _i, _d, _d, _l, _l, C.POINTER(_vp)]),
    "hh_plan_destroy": (_i, [_vp]),
    "hh_plan_field_size": (_l, [_vp]),
    "hh_plan_tune": (_i, [_vp, _i]),
    "hh_plan_set_variant": (_i, [_vp, _i]),
    "hh_plan_variant": (_i, [_vp]),
    "hh_plan_apply_tuning": (_i, [_vp, C.POINTER(_i)]),
    "hh_tune_cache_stats": (_i, [C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "hh_tune_cache_clear": (_i, []),
    "hh_tune_cache_save": (_i, [C.c_char_p]),
    "hh_tune_cache_load": (_i, [C.c_char_p, C.POINTER(C.c_longlong)]),
    "hh_plan_set_slab": (_i, [_vp, _l]),
    "hh_plan_slab": (_l, [_vp]),
    "hh_plan_set_dst_variant": (_i, [_vp, _i]),
    "hh_plan_dst_variant": (_i, [_vp]),
    "hh_plan_set_rows_variant": (_i, [_vp, _i]),
    "hh_plan_rows_variant": (_i, [_vp]),
    "hh_solve": (_i, [_vp, _vp, _vp, _i]),
    "hh_solve_host": (_i, [_vp, _vp, _vp, _i]),
    "hh_solve_source": (_i, [_vp, _vp, _vp, _i]),
    "hh_solve_source_host": (_i, [_vp, _vp, _vp, _i]),
    "hh_solve_lines": (_i, [_vp, _vp, _vp, _i, _i]),
    "hh_solve_lines_strided": (_i, [_vp, _vp, _vp, _i, _i, _l, _l]),
    "hh_solve_source_host_noalloc": (_i, [_vp, _vp, _vp, _i]),
    "hh_solve_source_multi": (_i, [C.POINTER(_vp), C.POINTER(_i), _i, _vp, _vp]),
    "hh_rhs2d": (_i, [_vp, C.POINTER(Rhs2DData), _vp]),
    "hh_rhs3d": (_i, [_vp, C.POINTER(Rhs3DData), _vp]),
    "hh_residual": (_i, [_vp, _vp, _vp, _vp, _i, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "hh_solve_refined": (_i, [_vp, _vp, _vp, _i, C.c_double, _i, C.POINTER(_i), C.POINTER(C.c_double)]),
    "hh_coefficients2d": (_i, [_i, _i, _d, _d, C.POINTER(_vp)]),
    "hh_coefficients3d": (_i, [_i, _i, _d, _d, C.POINTER(_vp)]),
    "hh_ctx_set_stage_timing": (_i, [_vp, _i]),
    "hh_ctx_stage_times": (_i, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
    "hh_server_create": (_i, [_i, _sz, _i, C.POINTER(_vp)]),
    "hh_server_submit": (_i, [_vp, C.POINTER(Request), C.POINTER(C.c_longlong)]),
    "hh_server_wait": (_i, [_vp, C.c_longlong, C.POINTER(RequestInfo)]),
    "hh_server_stats": (_i, [_vp, C.POINTER(C.c_longlong), C.POINTER(_sz), C.POINTER(_i)]),
    "hh_server_clock": (_d, [_vp]),
    "hh_server_destroy": (_i, [_vp]),
    "hh_server_inject_error": (_i, [_vp, _i]),
    "hh_server_inject_wait_expiry": (_i, [_vp]),
}

_lib = None


class HHError(RuntimeError):
    pass


def lib() -> C.CDLL:
    """Load libhh.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HHError(f"{LIB_PATH} is missing; build it with `python -m hackathon_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str = "") -> None:
    if rc != HH_OK:
        msg = lib().hh_last_error().decode(errors="replace")
        raise HHError(f"{what}: {STATUS.get(rc, rc)}: {msg}")


def _addr(buf) -> int:
    """Device or host address of a torch tensor, a numpy array or an integer."""
    if isinstance(buf, int):
        return buf
    if isinstance(buf, np.ndarray):
        assert buf.flags["C_CONTIGUOUS"]
        return buf.ctypes.data
    if hasattr(buf, "data_ptr"):
        return buf.data_ptr()
    raise TypeError(type(buf))


class Context:
    """One device + one CUDA stream (include/hh.h hh_ctx)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        import weakref
        p = _vp()
        check(lib().hh_ctx_create(device, stream, C.byref(p)), "hh_ctx_create")
        self.h = p
        self.device = device
        self.plans = weakref.WeakSet()

    def close(self):
        if self.h:
            for plan in list(self.plans):  # the C context releases them with itself
                plan.h = None
            lib().hh_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream: int | None):
        check(lib().hh_ctx_set_stream(self.h, stream), "hh_ctx_set_stream")

    def synchronize(self):
        check(lib().hh_ctx_synchronize(self.h), "hh_ctx_synchronize")

    def inject_wait_expiry(self):
        """Arm one expired bounded wait in the next rows-transform launch (hh_ctx_inject_wait_expiry)."""
        check(lib().hh_ctx_inject_wait_expiry(self.h), "hh_ctx_inject_wait_expiry")

    def set_stage_timing(self, on: bool):
        check(lib().hh_ctx_set_stage_timing(self.h, 1 if on else 0), "hh_ctx_set_stage_timing")

    def stage_times(self):
        """(ms per stage [forward, lines, inverse], solves timed) since the last call."""
        ms = (C.c_double * 3)()
        n = C.c_longlong()
        check(lib().hh_ctx_stage_times(self.h, ms, C.byref(n)), "hh_ctx_stage_times")
        return list(ms), int(n.value)

    @property
    def launches(self) -> int:
        return int(lib().hh_ctx_launch_count(self.h))

    # -- transforms on device buffers (complex128)
    def dst1_rows(self, n: int, rows: int, src, dst, in_ld: int | None = None, out_ld: int | None = None):
        check(lib().hh_dst1_rows(self.h, n, rows, _addr(src), in_ld or n, _addr(dst), out_ld or n), "hh_dst1_rows")

    def dst1_cols(self, n: int, ncols: int, planes: int, src, ld: int, plane_stride: int, dst):
        check(lib().hh_dst1_cols(self.h, n, ncols, planes, _addr(src), ld, plane_stride, _addr(dst)), "hh_dst1_cols")

    def lines_pack(self, src, dst, batch: int, planes: int, nlines: int, world: int, unpack: bool = False):
        """hh_lines_pack: a slab [batch][planes][nlines] into the ranks' line parts, or back."""
        check(lib().hh_lines_pack(self.h, _addr(src), _addr(dst), batch, planes, nlines, world, 1 if unpack else 0),
              "hh_lines_pack")

    def dst2_planes(self, nx: int, ny: int, planes: int, src, dst):
        check(lib().hh_dst2_planes(self.h, nx, ny, planes, _addr(src), _addr(dst)), "hh_dst2_planes")


def _coef_ptrs(arrs):
    keep = [np.ascontiguousarray(a, dtype=np.complex128) for a in arrs]
    return keep, (_vp * len(keep))(*[k.ctypes.data for k in keep])


class Plan:
    """A device-resident problem (include/hh.h hh_plan)."""

    def __init__(self, ctx: Context, handle, dim: int, shape: tuple):
        self.ctx, self.h, self.dim, self.shape = ctx, handle, dim, shape
        self.field = int(lib().hh_plan_field_size(handle))
        ctx.plans.add(self)

    @classmethod
    def from_coefficients_2d(cls, ctx: Context, nx: int, ny: int, coef: dict):
        keep = [np.ascontiguousarray(coef[k], dtype=np.complex128) for k in ("bp", "ap", "b", "a", "bm", "am")]
        p = _vp()
        check(lib().hh_plan2d_create(ctx.h, nx, ny, *[k.ctypes.data for k in keep], C.byref(p)), "hh_plan2d_create")
        return cls(ctx, p, 2, (ny, nx))

    @classmethod
    def from_coefficients_3d(cls, ctx: Context, nx: int, ny: int, nz: int, coef: dict):
        names = ("a", "b", "c", "d", "ap", "bp", "cp", "dp", "am", "bm", "cm", "dm")
        keep, arr = _coef_ptrs([coef[k] for k in names])
        p = _vp()
        check(lib().hh_plan3d_create(ctx.h, nx, ny, nz, arr, C.byref(p)), "hh_plan3d_create")
        return cls(ctx, p, 3, (nz, ny, nx))

    @classmethod
    def helmholtz(cls, ctx: Context, dim: int, n: int, order: int, k: complex):
        p = _vp()
        k = complex(k)
        if dim == 2:
            check(lib().hh_plan2d_create_helmholtz(ctx.h, n, order, k.real, k.imag, C.byref(p)), "helmholtz2d")
            return cls(ctx, p, 2, (n, n))
        check(lib().hh_plan3d_create_helmholtz(ctx.h, n, order, k.real, k.imag, C.byref(p)), "helmholtz3d")
        return cls(ctx, p, 3, (n, n, n))

    @classmethod
    def helmholtz_lines(cls, ctx: Context, n: int, order: int, k: complex, q0: int, q1: int):
        """The z line solves of lines [q0, q1) of a 3D Helmholtz plan (a rank's pencil,
        hh_plan3d_create_helmholtz_lines); fields are laid out [z][q - q0]."""
        p = _vp()
        k = complex(k)
        check(lib().hh_plan3d_create_helmholtz_lines(ctx.h, n, order, k.real, k.imag, q0, q1, C.byref(p)),
              "hh_plan3d_create_helmholtz_lines")
        return cls(ctx, p, 3, (n, q1 - q0))

    def close(self):
        if self.h and self.ctx.h:
            lib().hh_plan_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tune(self, batch: int) -> int:
        """Time the line-solve variants on `batch` right-hand sides, keep the fastest (or apply the
        tuning cache's entry for this shape)."""
        check(lib().hh_plan_tune(self.h, batch), "hh_plan_tune")
        return self.variant

    def apply_tuning(self) -> bool:
        """Apply the tuning cache's entry for this plan's shape, if any (never measures)."""
        found = C.c_int()
        check(lib().hh_plan_apply_tuning(self.h, C.byref(found)), "hh_plan_apply_tuning")
        return bool(found.value)

    @property
    def variant(self) -> int:
        return int(lib().hh_plan_variant(self.h))

    @variant.setter
    def variant(self, v: int):
        check(lib().hh_plan_set_variant(self.h, v), "hh_plan_set_variant")

    @property
    def slab(self) -> int:
        """3D: planes per slab of the transform passes (0: the whole batch)."""
        return int(lib().hh_plan_slab(self.h))

    @slab.setter
    def slab(self, planes: int):
        check(lib().hh_plan_set_slab(self.h, planes), "hh_plan_set_slab")

    @property
    def dst_variant(self) -> int:
        """3D: the column-transform kernel (0: CTA tiles of 8 swizzled columns, 1: per-warp tiles)."""
        return int(lib().hh_plan_dst_variant(self.h))

    @dst_variant.setter
    def dst_variant(self, v: int):
        check(lib().hh_plan_set_dst_variant(self.h, v), "hh_plan_set_dst_variant")

    @property
    def rows_variant(self) -> int:
        """The rows-transform kernel (0: the length's default, 1: CTA ring, 2: per-warp buffers)."""
        return int(lib().hh_plan_rows_variant(self.h))

    @rows_variant.setter
    def rows_variant(self, v: int):
        check(lib().hh_plan_set_rows_variant(self.h, v), "hh_plan_set_rows_variant")

    # -- device buffers (torch tensors / raw addresses)
    def solve(self, rhs, sol, batch: int = 1):
        check(lib().hh_solve(self.h, _addr(rhs), _addr(sol), batch), "hh_solve")

    def solve_source(self, f, u, batch: int = 1):
        check(lib().hh_solve_source(self.h, _addr(f), _addr(u), batch), "hh_solve_source")

    def solve_lines(self, src, dst, batch: int = 1, fused: bool = True):
        """The line solve alone on transformed fields (hh_solve_lines): fused = True for transformed
        sources (the Helmholtz plans' compact operator), False for assembled right-hand sides."""
        check(lib().hh_solve_lines(self.h, _addr(src), _addr(dst), batch, 1 if fused else 0), "hh_solve_lines")

    def solve_lines_strided(self, src, dst, batch: int, fused: bool, row_stride: int, field: int):
        """hh_solve_lines_strided: the line solve over fields at b field + r row_stride + q."""
        check(lib().hh_solve_lines_strided(self.h, _addr(src), _addr(dst), batch, 1 if fused else 0, row_stride,
                                           field), "hh_solve_lines_strided")

    def solve_refined(self, rhs, sol, batch: int = 1, tol: float = 1e-10, max_iter: int = 10):
        """hh_solve_refined on device buffers; returns (corrections, relative residual)."""
        it, rr = C.c_int(), C.c_double()
        check(lib().hh_solve_refined(self.h, _addr(rhs), _addr(sol), batch, tol, max_iter, C.byref(it), C.byref(rr)),
              "hh_solve_refined")
        return it.value, rr.value

    def assemble_rhs(self, rhs, order: int, h, **data):
        """hh_rhs2d / hh_rhs3d: the reference's rhs() on the device into the device buffer rhs.
        h: (hx, hy) or (hx, hy, hz).  data: the hh_rhs{2,3}d_data arrays by name -- device buffers
        (torch tensors or addresses), except k_ext / k2y_bc / k2_ext / kz_bc, which are host numpy
        arrays; missing boundary arrays are zero."""
        keep = []

        def ptr(name, v):
            if v is None:
                return None
            if name in ("k_ext", "k2y_bc", "k2_ext", "kz_bc"):
                a = np.ascontiguousarray(v, dtype=np.complex128)
                keep.append(a)
                return a.ctypes.data
            return _addr(v)

        if self.dim == 2:
            d = Rhs2DData(order, *h)
            for nm, _ in Rhs2DData._fields_[3:]:
                setattr(d, nm, ptr(nm, data.get(nm)))
            check(lib().hh_rhs2d(self.h, C.byref(d), _addr(rhs)), "hh_rhs2d")
        else:
            d = Rhs3DData(order, *h)
            for nm, _ in Rhs3DData._fields_[4:]:
                setattr(d, nm, ptr(nm, data.get(nm)))
            check(lib().hh_rhs3d(self.h, C.byref(d), _addr(rhs)), "hh_rhs3d")

    def residual(self, sol, rhs, res, batch: int = 1, norms: bool = False):
        """hh_residual on device buffers: res = A_h sol - rhs; with norms, (max|res|, max|rhs|)."""
        if not norms:
            check(lib().hh_residual(self.h, _addr(sol), _addr(rhs), _addr(res), batch, None, None), "hh_residual")
            return None
        mr, mf = C.c_double(), C.c_double()
        check(lib().hh_residual(self.h, _addr(sol), _addr(rhs), _addr(res), batch, C.byref(mr), C.byref(mf)),
              "hh_residual")
        return mr.value, mf.value

    # -- host numpy arrays
    def _batch_of(self, a: np.ndarray) -> int:
        """Right-hand sides in `a`: a whole, non-zero number of fields, or HHError."""
        if a.size == 0 or a.size % self.field:
            raise HHError(f"array of {a.size} values is not a whole number of {self.field}-value fields")
        return a.size // self.field

    def solve_host(self, rhs: np.ndarray) -> np.ndarray:
        rhs = np.ascontiguousarray(rhs, dtype=np.complex128)
        batch = self._batch_of(rhs)
        out = np.empty_like(rhs)
        check(lib().hh_solve_host(self.h, rhs.ctypes.data, out.ctypes.data, batch), "hh_solve_host")
        return out

    def solve_source_host_noalloc(self, f: np.ndarray) -> np.ndarray:
        """hh_solve_source_host_noalloc: staging in the library's fixed 32 MiB device array."""
        f = np.ascontiguousarray(f, dtype=np.complex128)
        batch = self._batch_of(f)
        out = np.empty_like(f)
        check(lib().hh_solve_source_host_noalloc(self.h, f.ctypes.data, out.ctypes.data, batch),
              "hh_solve_source_host_noalloc")
        return out

    def solve_source_host(self, f: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(f, dtype=np.complex128)
        batch = self._batch_of(f)
        out = np.empty_like(f)
        check(lib().hh_solve_source_host(self.h, f.ctypes.data, out.ctypes.data, batch), "hh_solve_source_host")
        return out


def solve_source_multi(plans, nrhs, f, u):
    """hh_solve_source_multi: plans of one shape, plan i taking nrhs[i] consecutive fields of the
    device buffers f and u."""
    hs = (_vp * len(plans))(*[p.h for p in plans])
    ns = (_i * len(plans))(*nrhs)
    check(lib().hh_solve_source_multi(hs, ns, len(plans), _addr(f), _addr(u)), "hh_solve_source_multi")


def tune_cache_stats() -> dict:
    h, m, e = C.c_longlong(), C.c_longlong(), C.c_longlong()
    check(lib().hh_tune_cache_stats(C.byref(h), C.byref(m), C.byref(e)), "hh_tune_cache_stats")
    return {"hits": h.value, "misses": m.value, "entries": e.value}


def tune_cache_clear():
    check(lib().hh_tune_cache_clear(), "hh_tune_cache_clear")


def tune_cache_save(path: str):
    check(lib().hh_tune_cache_save(os.fsencode(path)), "hh_tune_cache_save")


def tune_cache_load(path: str) -> int:
    n = C.c_longlong()
    check(lib().hh_tune_cache_load(os.fsencode(path), C.byref(n)), "hh_tune_cache_load")
    return n.value


def coefficients(dim: int, n: int, order: int, k: complex) -> dict:
    """Stencil coefficients of the constant-k schemes (hh_coefficients2d/3d)."""
    k = complex(k)
    names = ("bp", "ap", "b", "a", "bm", "am") if dim == 2 else \
        ("a", "b", "c", "d", "ap", "bp", "cp", "dp", "am", "bm", "cm", "dm")
    arrs = [np.zeros(n, dtype=np.complex128) for _ in names]
    ptrs = (_vp * len(arrs))(*[a.ctypes.data for a in arrs])
    f = lib().hh_coefficients2d if dim == 2 else lib().hh_coefficients3d
    check(f(n, order, k.real, k.imag, ptrs), "hh_coefficients")
    return dict(zip(names, arrs))


class Server:
    """Request loop over one device (include/hh.h hh_server_*): submit returns at once, wait
    blocks for one request.  Buffers (numpy arrays, torch tensors or raw addresses) must stay
    alive until the request's wait returns."""

    def __init__(self, device: int = 0, hbm_budget: int = 150 << 30, streams: int = 4):
        self.h = _vp()
        check(lib().hh_server_create(device, hbm_budget, streams, C.byref(self.h)), "hh_server_create")
        self._keep = {}

    def submit(self, dim: int, n: int, order: int, k: complex, nrhs: int, f, u, on_device: bool = False) -> int:
        k = complex(k)
        r = Request(dim, n, order, k.real, k.imag, nrhs, int(on_device), _addr(f), _addr(u))
        rid = C.c_longlong()
        check(lib().hh_server_submit(self.h, C.byref(r), C.byref(rid)), "hh_server_submit")
        self._keep[rid.value] = (f, u)
        return rid.value

    def wait(self, rid: int) -> dict:
        info = RequestInfo()
        rc = lib().hh_server_wait(self.h, rid, C.byref(info))
        self._keep.pop(rid, None)
        check(rc, "hh_server_wait")
        return {"t_submit": info.t_submit, "t_start": info.t_start, "t_done": info.t_done,
                "batch_rhs": info.batch_rhs}

    def stats(self) -> dict:
        done, used, plans = C.c_longlong(), C.c_size_t(), C.c_int()
        check(lib().hh_server_stats(self.h, C.byref(done), C.byref(used), C.byref(plans)), "hh_server_stats")
        return {"completed": done.value, "bytes_in_use": used.value, "plans": plans.value}

    def clock(self) -> float:
        return float(lib().hh_server_clock(self.h))

    def inject_wait_expiry(self):
        """Arm one expired bounded wait on the loop's device (hh_server_inject_wait_expiry)."""
        check(lib().hh_server_inject_wait_expiry(self.h), "hh_server_inject_wait_expiry")

    def inject_error(self, batches: int = 1):
        """The next `batches` batches complete with HH_ERR_DEVICE (hh_server_inject_error)."""
        check(lib().hh_server_inject_error(self.h, batches), "hh_server_inject_error")

    def close(self):
        if self.h:
            lib().hh_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
