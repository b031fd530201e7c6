"""The drop-in libraries' entry points called through their C ABI, array against array, with
the reference's own functions (its C sources compiled unchanged into oracle/_ref, FFTW replaced
by the oracle's FFTW-API shim) on the same inputs:

* libhh2d.so forwardDST / reverseDST  vs  2D_Program/solver_functions/DST.c:6-44
  (including a transform length dst.Nx below sys.lat.Nx and a non-orthonormal dst.coef);
* libhh3d.so DST                      vs  3D_Program/solver_functions/DST.c:148-204;
* libhh2d.so / libhh3d.so solver()    vs  2D_Program/solver_functions/solver.c:14-117 and
  3D_Program/solver_functions/solver.c:263-413, on a System the reference's own coefficients(),
  rhs() and LU() filled.

Tolerance: 1e-13 relative (max|a - b| / max|b|) for the transforms, which are well conditioned;
1e-12 for solutions, with the extended-precision fallback of conftest.assert_parity_2d for the
near-resonant lines."""
import ctypes as C
import math
import os

import numpy as np
import pytest
from conftest import FACTOR_ASSEMBLED, REF_DIR, assert_parity_2d, golden, rel_err

import hackathon_b200 as hh

pytestmark = pytest.mark.gpu

TOL_DST = 1e-13
TOL_SOL = 1e-12
FFTW_ESTIMATE = 1 << 6


class DSTN(C.Structure):
    """2D_Program/headers/structs.h:14-17"""
    _fields_ = [("Nx", C.c_int), ("N", C.c_int), ("coef", C.c_double)]


def _p(a):
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


@pytest.fixture(scope="module")
def libs():
    from oracle import System2D, System3D  # noqa: F401  (layouts used below)
    path2, path3 = os.path.join(REF_DIR, "libref2d.so"), os.path.join(REF_DIR, "libref3d.so")
    if not (os.path.exists(path2) and os.path.exists(path3)):
        pytest.skip("oracle/_ref not built (make -C oracle ref)")
    ref2, ref3 = C.CDLL(path2), C.CDLL(path3)
    hh2, hh3 = C.CDLL(hh.DROPIN2D_PATH), C.CDLL(hh.DROPIN3D_PATH)
    for lib in (ref2, ref3):
        lib.fftw_plan_dft_r2c_1d.restype = C.c_void_p
        lib.fftw_plan_many_dft_r2c.restype = C.c_void_p
    return ref2, ref3, hh2, hh3


def _sys2d(nx, ny):
    from oracle import Lattice2D, System2D
    return System2D(lat=Lattice2D(Nx=nx, Ny=ny, Nxy=nx * ny))


class _Plans2D:
    """The reference's per-thread FFTW set-up of solver.c:40-62: two r2c plans of length
    N = 2 dst.Nx + 2 over zeroed buffers."""

    def __init__(self, ref2, n):
        self.N = 2 * n + 2
        nc = self.N // 2 + 1
        self.inb, self.in2 = np.zeros(self.N), np.zeros(self.N)
        self.outb, self.out2 = np.zeros(2 * nc), np.zeros(2 * nc)
        self.p1 = ref2.fftw_plan_dft_r2c_1d(C.c_int(self.N), _p(self.inb), _p(self.outb), C.c_uint(FFTW_ESTIMATE))
        self.p2 = ref2.fftw_plan_dft_r2c_1d(C.c_int(self.N), _p(self.in2), _p(self.out2), C.c_uint(FFTW_ESTIMATE))

    def args(self):
        return (C.c_void_p(self.p1), _p(self.inb), _p(self.outb), C.c_void_p(self.p2), _p(self.in2), _p(self.out2))


def _cplx(rng, shape):
    return np.ascontiguousarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


@pytest.mark.parametrize("nx,ny,dnx,coef", [(7, 7, 7, None), (15, 20, 15, None), (63, 63, 63, None),
                                            (100, 100, 100, None), (255, 17, 255, None), (1023, 64, 1023, None),
                                            (64, 9, 63, None), (31, 31, 31, 1.0), (100, 5, 97, 0.25)])
def test_forward_and_reverse_dst_match_reference(libs, nx, ny, dnx, coef):
    ref2, _, hh2, _ = libs
    rng = np.random.default_rng(nx * 1000 + ny)
    sys_ = _sys2d(nx, ny)
    plans = _Plans2D(ref2, dnx)
    dst = DSTN(Nx=dnx, N=plans.N, coef=math.sqrt(2.0 / (dnx + 1)) if coef is None else coef)
    rhs = _cplx(rng, (ny, nx))
    # outputs start from the same values: entries past dst.Nx keep them in both
    start = _cplx(rng, (ny, nx))
    want, got = start.copy(), start.copy()
    ref2.forwardDST(sys_, dst, _p(rhs), _p(want), *plans.args())
    hh2.forwardDST(sys_, dst, _p(rhs), _p(got), None, None, None, None, None, None)
    assert hh2.hh2d_status() == 0
    assert rel_err(got, want) < TOL_DST
    assert np.array_equal(got[:, dnx:], start[:, dnx:])
    # reverseDST reads the transposed layout xhat[j + i*Ny] (the line solve's output)
    xhat = _cplx(rng, (nx, ny))
    want, got = start.copy(), start.copy()
    ref2.reverseDST(sys_, dst, _p(xhat), _p(want), *plans.args())
    hh2.reverseDST(sys_, dst, _p(xhat), _p(got), None, None, None, None, None, None)
    assert hh2.hh2d_status() == 0
    assert rel_err(got, want) < TOL_DST
    assert np.array_equal(got[:, dnx:], start[:, dnx:])


def test_forward_dst_matches_golden_rows(libs):
    """The committed golden rows (the reference's forwardDST on random rows) through the drop-in."""
    _, _, hh2, _ = libs
    g = golden("dst_rows.npz")
    for n in (1, 7, 31, 63, 100):
        x, y = np.ascontiguousarray(g[f"x_{n}"]), g[f"y_{n}"]
        rows = x.shape[0]
        got = np.zeros_like(x)
        hh2.forwardDST(_sys2d(n, rows), DSTN(Nx=n, N=2 * n + 2, coef=math.sqrt(2.0 / (n + 1))), _p(x), _p(got),
                       None, None, None, None, None, None)
        assert hh2.hh2d_status() == 0
        assert rel_err(got, y) < TOL_DST, n


def test_dst_length_out_of_range_is_reported(libs):
    _, _, hh2, _ = libs
    x = np.zeros((4, 8), dtype=np.complex128)
    y = np.zeros_like(x)
    hh2.forwardDST(_sys2d(8, 4), DSTN(Nx=9, N=20, coef=1.0), _p(x), _p(y), None, None, None, None, None, None)
    assert hh2.hh2d_status() == 1  # HH_ERR_INVALID; the output is untouched
    assert not y.any()


@pytest.mark.parametrize("nx,ny", [(15, 15), (31, 63), (100, 100), (255, 255), (127, 40)])
def test_dst3d_plane_matches_reference(libs, nx, ny):
    _, ref3, _, hh3 = libs
    rng = np.random.default_rng(nx + 7 * ny)
    # the reference's plans (3D solver.c:285-329): howmany = Ny rows of length 2Nx+2, then
    # howmany = Nx columns of length 2Ny+2, over zeroed buffers
    nr1, nr2 = 2 * nx + 2, 2 * ny + 2
    in1, in2 = np.zeros(nr1 * ny), np.zeros(nr2 * nx)
    out1, out2 = np.zeros(2 * (nr1 // 2 + 1) * ny), np.zeros(2 * (nr2 // 2 + 1) * nx)
    n1, n2 = (C.c_int * 1)(nr1), (C.c_int * 1)(nr2)
    p1 = ref3.fftw_plan_many_dft_r2c(1, n1, ny, _p(in1), None, 1, nr1, _p(out1), None, 1, nr1 // 2 + 1,
                                     C.c_uint(FFTW_ESTIMATE))
    p2 = ref3.fftw_plan_many_dft_r2c(1, n2, nx, _p(in2), None, 1, nr2, _p(out2), None, 1, nr2 // 2 + 1,
                                     C.c_uint(FFTW_ESTIMATE))
    b = np.ascontiguousarray(rng.standard_normal((ny, nx)))
    want, got = np.zeros_like(b), np.zeros_like(b)
    b_ref = b.copy()  # the reference leaves its x-pass intermediate in its input (DST.c:175-179)
    ref3.DST(nx, ny, _p(b_ref), _p(want), C.c_void_p(p1), _p(in1), _p(out1), C.c_void_p(p2), _p(in2), _p(out2))
    b_hh = b.copy()
    hh3.DST(nx, ny, _p(b_hh), _p(got), None, None, None, None, None, None)
    assert hh3.hh3d_status() == 0
    assert rel_err(got, want) < TOL_DST
    assert np.array_equal(b_hh, b)  # the drop-in does not modify its input


@pytest.mark.parametrize("original,n,order,k", [(True, 15, 6, None), (True, 127, 6, None), (True, 255, 4, None),
                                                (False, 1023, 6, 50.0), (False, 511, 2, 200.0)])
def test_dropin_solver2d_solution_array(libs, oracle, original, n, order, k):
    """solver(System) of libhh2d.so writes sys.sol equal to the reference's solver() on the
    System that the reference's coefficients(), rhs() and LU() filled: its own variable-k problem
    (2D_Program/user_input.c) or the constant-k sine-mode class."""
    from hackathon_b200 import workload as W
    from oracle import Reference2D
    _, _, hh2, _ = libs
    R = Reference2D(original_problem=original)
    f = None if original else W.source_2d(n, W.sine_modes(17, 32, 200), noise_seed=18, noise_var=1e-3, fast=True)
    run = R.pipeline(n, order, k, f, stages=("coefficients", "rhs", "LU", "solver"))
    a = run.arrays
    want = a["sol"].copy().reshape(n, n)
    a["sol"][:] = 0
    hh2.solver(run.sys)
    assert hh2.hh2d_status() == 0
    got = a["sol"].reshape(n, n)
    coef = {nm: a[nm] for nm in ("bp", "ap", "b", "a", "bm", "am")}
    assert_parity_2d(oracle, got, dict(sol=want, coef=coef, rhs=a["rhs"].reshape(n, n)), TOL_SOL, FACTOR_ASSEMBLED)
    hh2.solver(run.sys)  # the same stencil again: the cached plan (bytes compared) is reused
    assert np.array_equal(a["sol"].reshape(n, n), got)


@pytest.mark.parametrize("n,order,B,g", [(31, 6, 9.0, 9.0), (63, 6, 9.0, 9.0), (63, 4, 0.0, 6.0), (127, 2, 9.0, 9.0)])
def test_dropin_solver3d_solution_array(libs, n, order, B, g):
    """solver(System) of libhh3d.so against the reference's 3D CPU solver() on its own problem
    (3D_Program/user_input.c; B = 9, gamma = 9 is the paper's test problem)."""
    from oracle import Reference3D
    _, _, _, hh3 = libs
    R = Reference3D()
    run = R.make_system(n, order, 10.0, B, 10.0, g)
    for st in ("background3D", "coefficients", "rhs", "LU", "solver"):
        getattr(R.lib, st)(run.sys)
    a = run.arrays
    want = a["sol"].copy()
    a["sol"][:] = 0
    hh3.solver(run.sys)
    assert hh3.hh3d_status() == 0
    assert rel_err(a["sol"], want) < TOL_SOL
