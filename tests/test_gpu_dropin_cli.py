"""The reference's own programs (Direct_Solver CLI, main.c, setup, coefficients, rhs, LU,
residual: all unchanged) linked against the drop-in libraries instead of their solver.c and
DST.c, against the same programs linked with their own solver (oracle/_ref, built by
`make -C oracle ref` where the reference sources are available).

They solve the reference's own problems (2D_Program/user_input.c: k(y) = y^2 + iy on
[0.5, pi - 0.5]^2; 3D_Program/user_input.c: k = 10, Dirichlet data on the z faces), so this
also covers the variable-coefficient line solves.  Both print the residual and the error
against the analytic solution (2D_Program/main_functions/main.c:42-43,
3D_Program/main_functions/main.c:30-32)."""
import os
import re
import subprocess

import pytest
from conftest import ROOT

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref")


def _run(exe, *args):
    path = os.path.join(REF, exe)
    if not os.path.exists(path):
        pytest.skip(f"{exe} not built (make -C oracle ref)")
    out = subprocess.run([path, *map(str, args)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "ERROR" not in out.stderr, out.stderr
    norms = dict(re.findall(r"\|\|(\w+)\|\|_(?:inf)\s*=\s*([-+0-9.eE]+)", out.stdout))
    return {k: float(v) for k, v in norms.items()}


@pytest.mark.parametrize("order,n", [(6, 100), (4, 127), (2, 63), (6, 255)])
def test_direct_solver_2d_dropin(order, n):
    ref = _run("Direct_Solver2d", order, n, 4)
    hh = _run("Direct_Solver2d_hh", order, n, 4)
    # same discrete solution: the error against the analytic solution agrees to rounding
    # (|u| ~ 1 on this problem; printed with 8 significant digits)
    assert abs(hh["error"] - ref["error"]) <= 1e-11 + 1e-7 * ref["error"]
    assert hh["res"] < 1e-11


@pytest.mark.parametrize("order,n", [(6, 31), (4, 31), (2, 15), (6, 63)])
def test_direct_solver_3d_dropin(order, n):
    ref = _run("Direct_Solver3d", order, n)
    hh = _run("Direct_Solver3d_hh", order, n)
    assert abs(hh["error"] - ref["error"]) <= 1e-11 + 1e-7 * ref["error"]
    assert hh["res"] < 1e-11
