"""ctypes bindings to the oracle (TEST INFRASTRUCTURE ONLY).

Two CPU implementations of gonzrona/hackathon's solver path are reachable from here:

* `liboracle.so` -- this project's plain-C restatement (oracle/hh_oracle.c);
* `_ref/libref2d.so`, `_ref/libref2d_orig.so`, `_ref/libref3d.so` -- the reference's own
  C sources compiled unchanged against the FFTW-API shim (oracle/Makefile `ref`).

Only tests/, the smoke check and bench.py's CPU-baseline leg import this module; the
product never does.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_cd = C.POINTER(C.c_double)


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_cd)


def _lib(name: str) -> C.CDLL:
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle all ref`")
    return C.CDLL(path)


# ----------------------------------------------------------------- restatement ----

class _Coef2D(C.Structure):
    _fields_ = [(n, _cd) for n in ("bp", "ap", "b", "a", "bm", "am")]


class _Problem2D(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("order", C.c_int),
                ("x0", C.c_double), ("x1", C.c_double), ("y0", C.c_double), ("y1", C.c_double),
                ("hx", C.c_double), ("hy", C.c_double)] + \
               [(n, _cd) for n in ("k_ext", "k2y_ext", "k2yy", "f_ext", "fxx_xb", "fxx_yb",
                                   "fyy_xb", "fyy_yb", "fy_yb", "u_xb", "u_yb")]


class _Coef3D(C.Structure):
    _fields_ = [(n, _cd) for n in ("a", "b", "c", "d", "ap", "bp", "cp", "dp", "am", "bm", "cm", "dm")]


class _Problem3D(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("order", C.c_int),
                ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double)] + \
               [(n, _cd) for n in ("k2_ext", "kz_bc", "kzz_bc", "rhs_ext", "ue_ext", "fxx_b", "fyy_b", "fzz_b")]


COEF2D_NAMES = ("bp", "ap", "b", "a", "bm", "am")
COEF3D_NAMES = ("a", "b", "c", "d", "ap", "bp", "cp", "dp", "am", "bm", "cm", "dm")


class Oracle:
    """The restatement in liboracle.so."""

    def __init__(self):
        self.lib = _lib("liboracle.so")

    # -- transforms
    def dst1_rows(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.complex128)
        n = x.shape[-1]
        rows = x.size // n
        out = np.empty_like(x)
        rc = self.lib.ora_dst1_rows(C.c_int(n), C.c_long(rows), _ptr(x), C.c_long(n), _ptr(out), C.c_long(n))
        assert rc == 0
        return out

    # -- 2D
    def problem2d(self, n: int, order: int, k, f_ext: np.ndarray, x0=0.0, x1=1.0, **bnd):
        """k: a constant, or the n+2 samples k(y0 + j h) of a variable wavenumber."""
        h = (x1 - x0) / (n + 1)
        keep = {}
        k_ext = (np.ascontiguousarray(k, dtype=np.complex128) if np.ndim(k) else
                 np.full(n + 2, complex(k), dtype=np.complex128))
        keep["k_ext"] = k_ext
        keep["f_ext"] = np.ascontiguousarray(f_ext, dtype=np.complex128)
        pb = _Problem2D(nx=n, ny=n, order=order, x0=x0, x1=x1, y0=x0, y1=x1, hx=h, hy=h)
        pb.k_ext = _ptr(k_ext)
        pb.f_ext = _ptr(keep["f_ext"])
        for name, arr in bnd.items():
            dt = np.float64 if name in ("u_xb", "u_yb") else np.complex128
            keep[name] = np.ascontiguousarray(arr, dtype=dt)
            setattr(pb, name, _ptr(keep[name]))
        return pb, keep

    def coefficients_2d(self, pb) -> dict:
        co = {nm: np.zeros(pb.ny, dtype=np.complex128) for nm in COEF2D_NAMES}
        cs = _Coef2D(**{nm: _ptr(co[nm]) for nm in COEF2D_NAMES})
        self.lib.ora_coefficients_2d(C.byref(pb), C.byref(cs))
        return co

    def _cs2(self, co):
        return _Coef2D(**{nm: _ptr(co[nm]) for nm in COEF2D_NAMES})

    def rhs_2d(self, pb, co) -> np.ndarray:
        rhs = np.zeros((pb.ny, pb.nx), dtype=np.complex128)
        cs = self._cs2(co)
        self.lib.ora_rhs_2d(C.byref(pb), C.byref(cs), _ptr(rhs))
        return rhs

    def lu_2d(self, nx, ny, co):
        L, U, Up = (np.zeros(nx * ny, dtype=np.complex128) for _ in range(3))
        cs = self._cs2(co)
        self.lib.ora_lu_2d(C.c_int(nx), C.c_int(ny), C.byref(cs), _ptr(L), _ptr(U), _ptr(Up))
        return L, U, Up

    def solver_2d(self, rhs, L, U, Up) -> np.ndarray:
        ny, nx = rhs.shape
        rhs = np.ascontiguousarray(rhs)
        sol = np.zeros_like(rhs)
        rc = self.lib.ora_solver_2d(C.c_int(nx), C.c_int(ny), _ptr(rhs), _ptr(L), _ptr(U), _ptr(Up), _ptr(sol))
        assert rc == 0
        return sol

    def solver_2d_ld(self, co, rhs) -> np.ndarray:
        """Extended-precision solve of the same discrete system (see ora_solver_2d_ld)."""
        ny, nx = rhs.shape
        rhs = np.ascontiguousarray(rhs)
        sol = np.zeros_like(rhs)
        cs = self._cs2(co)
        rc = self.lib.ora_solver_2d_ld(C.c_int(nx), C.c_int(ny), C.byref(cs), _ptr(rhs), _ptr(sol))
        assert rc == 0
        return sol

    def residual_2d(self, co, sol, rhs) -> np.ndarray:
        ny, nx = sol.shape
        res = np.zeros_like(sol)
        cs = self._cs2(co)
        self.lib.ora_residual_2d(C.c_int(nx), C.c_int(ny), C.byref(cs), _ptr(np.ascontiguousarray(sol)),
                                 _ptr(np.ascontiguousarray(rhs)), _ptr(res))
        return res

    def pipeline_2d(self, n: int, order: int, k: complex, f_ext: np.ndarray):
        """coefficients -> rhs -> LU -> solver, as the reference's main() does."""
        pb, keep = self.problem2d(n, order, k, f_ext)
        co = self.coefficients_2d(pb)
        rhs = self.rhs_2d(pb, co)
        L, U, Up = self.lu_2d(n, n, co)
        sol = self.solver_2d(rhs, L, U, Up)
        return dict(coef=co, rhs=rhs, sol=sol)

    # -- 3D
    def set_3d_real_sums(self, on: bool):
        self.lib.ora_set_3d_real_sums(C.c_int(1 if on else 0))

    def problem3d(self, n: int, order: int, k2_ext: np.ndarray, rhs_ext: np.ndarray, h: float,
                  nxyz=None, **extra):
        nx, ny, nz = nxyz if nxyz else (n, n, n)
        keep = {"k2_ext": np.ascontiguousarray(k2_ext, dtype=np.complex128),
                "rhs_ext": np.ascontiguousarray(rhs_ext, dtype=np.complex128)}
        pb = _Problem3D(nx=nx, ny=ny, nz=nz, order=order, hx=h, hy=h, hz=h)
        pb.k2_ext = _ptr(keep["k2_ext"])
        pb.rhs_ext = _ptr(keep["rhs_ext"])
        for name, arr in extra.items():
            keep[name] = np.ascontiguousarray(arr, dtype=np.complex128)
            setattr(pb, name, _ptr(keep[name]))
        return pb, keep

    def coefficients_3d(self, pb) -> dict:
        co = {nm: np.zeros(pb.nz, dtype=np.complex128) for nm in COEF3D_NAMES}
        cs = _Coef3D(**{nm: _ptr(co[nm]) for nm in COEF3D_NAMES})
        self.lib.ora_coefficients_3d(C.byref(pb), C.byref(cs))
        return co

    def _cs3(self, co):
        return _Coef3D(**{nm: _ptr(co[nm]) for nm in COEF3D_NAMES})

    def rhs_3d(self, pb, co) -> np.ndarray:
        rhs = np.zeros((pb.nz, pb.ny, pb.nx), dtype=np.complex128)
        cs = self._cs3(co)
        self.lib.ora_rhs_3d(C.byref(pb), C.byref(cs), _ptr(rhs))
        return rhs

    def lu_3d(self, nx, ny, nz, co):
        L, U, Up = (np.zeros(nx * ny * nz, dtype=np.complex128) for _ in range(3))
        cs = self._cs3(co)
        self.lib.ora_lu_3d(C.c_int(nx), C.c_int(ny), C.c_int(nz), C.byref(cs), _ptr(L), _ptr(U), _ptr(Up))
        return L, U, Up

    def solver_3d(self, rhs, L, U, Up) -> np.ndarray:
        nz, ny, nx = rhs.shape
        rhs = np.ascontiguousarray(rhs)
        sol = np.zeros_like(rhs)
        rc = self.lib.ora_solver_3d(C.c_int(nx), C.c_int(ny), C.c_int(nz), _ptr(rhs), _ptr(L), _ptr(U),
                                    _ptr(Up), _ptr(sol))
        assert rc == 0
        return sol

    def residual_3d(self, co, sol, rhs) -> np.ndarray:
        nz, ny, nx = sol.shape
        res = np.zeros_like(sol)
        cs = self._cs3(co)
        self.lib.ora_residual_3d(C.c_int(nx), C.c_int(ny), C.c_int(nz), C.byref(cs),
                                 _ptr(np.ascontiguousarray(sol)), _ptr(np.ascontiguousarray(rhs)), _ptr(res))
        return res

    def pipeline_3d(self, n: int, order: int, k: complex, f_ext: np.ndarray):
        """Config problem (constant k, zero boundary data): the source is scaled by h^2 as
        3D rhs.c:249 does before the assembly."""
        h = 1.0 / (n + 1)
        k2_ext = np.full(n + 2, complex(k) ** 2, dtype=np.complex128)
        pb, keep = self.problem3d(n, order, k2_ext, (h * h) * np.asarray(f_ext), h)
        co = self.coefficients_3d(pb)
        rhs = self.rhs_3d(pb, co)
        L, U, Up = self.lu_3d(n, n, n, co)
        sol = self.solver_3d(rhs, L, U, Up)
        return dict(coef=co, rhs=rhs, sol=sol)


# ---------------------------------------------------- the reference (oracle/_ref) ----

class Lattice2D(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("Nxy", C.c_int),
                ("hx", C.c_double), ("hy", C.c_double), ("x0", C.c_double), ("x1", C.c_double),
                ("y0", C.c_double), ("y1", C.c_double)]


class System2D(C.Structure):
    """2D_Program/headers/structs.h:20-30 (192 bytes)."""
    _fields_ = [("lat", Lattice2D), ("threadCount", C.c_int), ("order", C.c_int)] + \
               [(n, _cd) for n in ("k", "rhs", "L", "U", "Up", "sol", "sol_analytic", "res", "error",
                                   "bp", "ap", "b", "a", "bm", "am")]


class Lattice3D(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int), ("Nxyz", C.c_int)] + \
               [(n, C.c_double) for n in ("hx", "hy", "hz", "x0", "x1", "y0", "y1", "z0", "z1")]


class System3D(C.Structure):
    """3D_Program/headers/structs.h:46-58 (312 bytes)."""
    _fields_ = [("lat", Lattice3D), ("order", C.c_int)] + \
               [(n, _cd) for n in ("a", "b", "c", "d", "ap", "bp", "cp", "dp", "am", "bm", "cm", "dm",
                                   "k_bg_ext", "k2_bg_ext")] + \
               [(n, C.c_double) for n in ("A", "B", "C", "beta", "gamma")] + \
               [(n, _cd) for n in ("sol_analytic", "rhs", "L", "U", "Up", "sol", "res", "error")]


ORDER_ENUM = {2: 0, 4: 1, 6: 2}  # enum Order{second, fourth, sixth}


@dataclass
class RefRun:
    sys: C.Structure
    arrays: dict


class Reference2D:
    """The reference's own 2D C code (oracle/_ref/libref2d*.so)."""

    def __init__(self, original_problem: bool = False):
        self.lib = _lib(os.path.join("_ref", "libref2d_orig.so" if original_problem else "libref2d.so"))
        self.original = original_problem

    def make_system(self, n: int, order: int, threads: int = 1, x0=0.0, x1=1.0) -> RefRun:
        nxy = n * n
        arrs = {nm: np.zeros(nxy, dtype=np.complex128) for nm in
                ("rhs", "L", "U", "Up", "sol", "sol_analytic", "res", "error")}
        arrs["k"] = np.zeros(n, dtype=np.complex128)
        for nm in COEF2D_NAMES:
            arrs[nm] = np.zeros(n, dtype=np.complex128)
        h = (x1 - x0) / (n + 1)
        lat = Lattice2D(Nx=n, Ny=n, Nxy=nxy, hx=h, hy=h, x0=x0, x1=x1, y0=x0, y1=x1)
        s = System2D(lat=lat, threadCount=threads, order=ORDER_ENUM[order])
        for nm, a in arrs.items():
            setattr(s, nm, _ptr(a))
        return RefRun(s, arrs)

    def set_problem(self, n: int, k: complex, f_ext: np.ndarray, x0=0.0, x1=1.0):
        h = (x1 - x0) / (n + 1)
        f = np.ascontiguousarray(f_ext, dtype=np.complex128)
        self.lib.hhref2d_set_problem(C.c_int(n), C.c_double(x0), C.c_double(x0), C.c_double(h),
                                     C.c_double(complex(k).real), C.c_double(complex(k).imag), _ptr(f))

    def pipeline(self, n: int, order: int, k: complex | None, f_ext: np.ndarray | None, threads: int = 1,
                 stages=("coefficients", "rhs", "LU", "solver")):
        if self.original:
            run = self.make_system(n, order, threads, x0=0.5, x1=math.pi - 0.5)
        else:
            self.set_problem(n, k, f_ext)
            run = self.make_system(n, order, threads)
        for st in stages:
            getattr(self.lib, st)(run.sys)
        return run


class Reference3D:
    """The reference's own 3D CPU code (oracle/_ref/libref3d.so)."""

    def __init__(self):
        self.lib = _lib(os.path.join("_ref", "libref3d.so"))

    def make_system(self, n: int, order: int, A: float, B: float, Cc: float, gamma: float,
                    x1: float = math.pi, nxyz=None) -> RefRun:
        nx, ny, nz = nxyz if nxyz else (n, n, n)
        nxyz_ = nx * ny * nz
        arrs = {nm: np.zeros(nz, dtype=np.complex128) for nm in COEF3D_NAMES}
        arrs["k_bg_ext"] = np.zeros(nz + 2, dtype=np.complex128)
        arrs["k2_bg_ext"] = np.zeros(nz + 2, dtype=np.complex128)
        for nm in ("sol_analytic", "rhs", "L", "U", "Up", "sol", "res", "error"):
            arrs[nm] = np.zeros(nxyz_, dtype=np.complex128)
        lat = Lattice3D(Nx=nx, Ny=ny, Nz=nz, Nxyz=nxyz_, hx=x1 / (nx + 1), hy=x1 / (ny + 1), hz=x1 / (nz + 1),
                        x0=0.0, x1=x1, y0=0.0, y1=x1, z0=0.0, z1=x1)
        beta = math.sqrt(A * A + B * B - gamma * gamma)
        s = System3D(lat=lat, order=ORDER_ENUM[order], A=A, B=B, C=Cc, beta=beta, gamma=gamma)
        for nm, a in arrs.items():
            setattr(s, nm, _ptr(a))
        return RefRun(s, arrs)


def reference3d_problem_inputs(n: int, A: float, B: float, Cc: float, gamma: float, x1: float = math.pi,
                               nxyz=None) -> dict:
    """Sampled data of the reference's hard-wired 3D test problem (3D_Program/user_input.c:5-18,
    main_functions/rhs.c:220-252 and 83-109, partial_derivatives/4th_order_partials.c:314-315,
    359-360) in the array form the restatement takes.  Scalar arithmetic follows the
    reference's expression order and uses libm (math.*) so the samples match bit for bit."""
    nx, ny, nz = nxyz if nxyz else (n, n, n)
    hx, hy, hz = x1 / (nx + 1), x1 / (ny + 1), x1 / (nz + 1)
    beta = math.sqrt(A * A + B * B - gamma * gamma)
    k_ext = [A - B * math.sin(Cc * (0.0 + hz * l)) for l in range(nz + 2)]
    k2_ext = np.array([complex(kk) * complex(kk) for kk in k_ext], dtype=np.complex128)
    fix = [math.sin(gamma * (0.0 + l * hx)) for l in range(nx + 2)]
    fiy = [math.sin(beta * (0.0 + l * hy)) for l in range(ny + 2)]
    fiz = [math.exp(-1.0 * k_ext[l] / Cc) for l in range(nz + 2)]
    ue = np.zeros((nz + 2, ny + 2, nx + 2), dtype=np.complex128)
    rhs = np.zeros_like(ue)
    for i in range(nx + 2):
        for j in range(ny + 2):
            bxy = fix[i] * fiy[j]
            for l in range(nz + 2):
                z = 0.0 + l * hz
                u = fiz[l] * bxy
                ue[l, j, i] = u
                rhs[l, j, i] = -1.0 * hz * hz * B * (2.0 * A + Cc) * math.sin(Cc * z) * u
    fxx_b = np.zeros(2 * (ny + 2) * (nz + 2), dtype=np.complex128)
    fyy_b = np.zeros(2 * (nx + 2) * (nz + 2), dtype=np.complex128)
    fzz_b = np.zeros(2 * (nx + 2) * (ny + 2), dtype=np.complex128)
    for l in range(nz + 2):
        for j in range(ny + 2):
            fxx_b[j + l * (ny + 2)] = -1.0 * gamma * gamma * rhs[l, j, 0]
            fxx_b[(ny + 2) * (nz + 2) + j + l * (ny + 2)] = -1.0 * gamma * gamma * rhs[l, j, nx + 1]
        for i in range(nx + 2):
            fyy_b[i + l * (nx + 2)] = -1.0 * beta * beta * rhs[l, 0, i]
            fyy_b[(nx + 2) * (nz + 2) + i + l * (nx + 2)] = -1.0 * beta * beta * rhs[l, ny + 1, i]

    def zterm(zz):
        s, c = math.sin(Cc * zz), math.cos(Cc * zz)
        return B * Cc * s * s + s * (Cc * Cc - B * B * c * c) - 2.0 * B * Cc * c * c

    z0, z1 = 0.0, x1
    for j in range(ny + 2):
        for i in range(nx + 2):
            fzz_b[i + j * (nx + 2)] = hz * hz * B * (2.0 * A + Cc) * ue[0, j, i] * zterm(z0)
            fzz_b[(nx + 2) * (ny + 2) + i + j * (nx + 2)] = hz * hz * B * (2.0 * A + Cc) * ue[nz + 1, j, i] * zterm(z1)
    kz_bc = np.array([2.0 * B * Cc * math.cos(Cc * z0) * (A - B * math.sin(Cc * z0)),
                      2.0 * B * Cc * math.cos(Cc * z1) * (A - B * math.sin(Cc * z1))], dtype=np.complex128)
    kzz_bc = np.array([2.0 * B * Cc * Cc * (B * math.sin(Cc * z0) * math.sin(Cc * z0) - A * math.sin(Cc * z0)
                                            - B * math.cos(Cc * z0) * math.cos(Cc * z0)),
                       2.0 * B * Cc * Cc * (B * math.sin(Cc * z1) * math.sin(Cc * z1) - A * math.sin(Cc * z1)
                                            - B * math.cos(Cc * z1) * math.cos(Cc * z1))], dtype=np.complex128)
    return dict(h=(hx, hy, hz), k2_ext=k2_ext, rhs_ext=rhs, ue_ext=ue, fxx_b=fxx_b, fyy_b=fyy_b, fzz_b=fzz_b,
                kz_bc=kz_bc, kzz_bc=kzz_bc)
