"""GPU FP64 residual (the reference's residual()) against the oracle's restatement of it."""
import numpy as np
import pytest
from conftest import rel_err

import hackathon_b200 as hh
from hackathon_b200 import workload as W

pytestmark = pytest.mark.gpu

RES_TOL = 1e-13  # max|res - res_ref| / max|A_h u| terms: rounding of a 9/27-point sum only


def _perturbed(sol, seed):
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(sol.shape) + 1j * rng.standard_normal(sol.shape)
    return sol + 1e-3 * np.abs(sol).max() * noise


@pytest.mark.parametrize("n,order,k", [(15, 6, 10.0), (63, 4, 50.0), (100, 6, 10.0), (255, 2, 30.0)])
def test_residual_2d_matches_oracle(ctx, oracle, n, order, k):
    """res = A_h sol - rhs on the reference's own coefficient rows and assembled rhs, for the
    reference's solution and for a perturbed one (so the residual is not just rounding)."""
    torch = pytest.importorskip("torch")
    f = W.source_2d(n, W.sine_modes(n + order, 8, 20), noise_seed=n, noise_var=1e-3)
    ref = oracle.pipeline_2d(n, order, k, f)
    plan = hh.Plan.from_coefficients_2d(ctx, n, n, ref["coef"])
    rhs = torch.from_numpy(np.ascontiguousarray(ref["rhs"])).cuda()
    for sol_h in (ref["sol"], _perturbed(ref["sol"], n)):
        sol = torch.from_numpy(np.ascontiguousarray(sol_h)).cuda()
        res = torch.empty_like(sol)
        mr, mf = plan.residual(sol, rhs, res, 1, norms=True)
        want = oracle.residual_2d(ref["coef"], sol_h, ref["rhs"])
        got = res.cpu().numpy()
        # the size of the summed terms bounds the rounding of either sum
        terms = sum(np.abs(np.asarray(ref["coef"][c])).max() for c in ("bp", "ap", "b", "a", "bm", "am"))
        scale = np.abs(ref["rhs"]).max() + 3 * terms * np.abs(sol_h).max()
        assert np.abs(got - want).max() <= RES_TOL * scale
        assert mr == pytest.approx(np.abs(got).max(), rel=1e-12)
        assert mf == pytest.approx(np.abs(ref["rhs"]).max(), rel=1e-12)
    plan.close()


@pytest.mark.parametrize("n,order,k", [(15, 6, 30.0), (31, 4, 10.0), (100, 6, 20.0), (127, 2, 30.0)])
def test_residual_3d_matches_oracle(ctx, oracle, n, order, k):
    """The tiled residual (32 x 8 tiles of the (x, y) plane marching through 64 layers): partial
    tiles at n = 100 and 15, and more than one chunk of layers at n = 100 and 127."""
    torch = pytest.importorskip("torch")
    m = W.sine_modes(n + order, 16, min(n, 64), dim=3)
    ref = oracle.pipeline_3d(n, order, k, W.source_3d(n, m))
    plan = hh.Plan.from_coefficients_3d(ctx, n, n, n, ref["coef"])
    sol_h = _perturbed(ref["sol"], n)
    sol = torch.from_numpy(np.ascontiguousarray(sol_h)).cuda()
    rhs = torch.from_numpy(np.ascontiguousarray(ref["rhs"])).cuda()
    res = torch.empty_like(sol)
    plan.residual(sol, rhs, res, 1)
    ctx.synchronize()
    want = oracle.residual_3d(ref["coef"], sol_h, ref["rhs"])
    assert rel_err(res.cpu().numpy(), want) < RES_TOL * 10
    plan.close()


def test_residual_batch_and_argument_checks(ctx, oracle):
    """A batch of fields gives each field's own residual; res aliasing sol is refused."""
    torch = pytest.importorskip("torch")
    n, order, k = 63, 6, 20.0
    f = W.source_2d(n, W.sine_modes(5, 8, 20))
    ref = oracle.pipeline_2d(n, order, k, f)
    plan = hh.Plan.from_coefficients_2d(ctx, n, n, ref["coef"])
    sols = np.stack([_perturbed(ref["sol"], s) for s in range(3)])
    rhs = torch.from_numpy(np.stack([ref["rhs"]] * 3)).cuda()
    sol = torch.from_numpy(sols).cuda()
    res = torch.empty_like(sol)
    plan.residual(sol, rhs, res, 3)
    ctx.synchronize()
    for b in range(3):
        want = oracle.residual_2d(ref["coef"], sols[b], ref["rhs"])
        assert rel_err(res[b].cpu().numpy(), want) < RES_TOL * 10
    with pytest.raises(hh.HHError):
        plan.residual(sol, rhs, sol, 3)
    plan.close()


@pytest.mark.parametrize("dim,n,order,k,batch", [(2, 1023, 6, 50.0, 2), (2, 255, 6, 400.0, 3), (2, 511, 4, 100.0, 2),
                                                 (2, 100, 6, 10.0, 1), (3, 63, 6, 30.0, 2), (3, 127, 4, 10.0, 1)])
def test_refined_solve_reaches_tolerance(ctx, oracle, dim, n, order, k, batch):
    """Mixed-precision refined solve (single-precision transforms, FP64 line solves, FP64
    residual): it reaches max|A_h u - rhs| / max|rhs| <= 1e-10, its solution agrees with the
    plain FP64 solve to the accuracy the residual bounds, and the single-precision first solve
    alone is far from it (so the refinement does the work)."""
    torch = pytest.importorskip("torch")
    plan = hh.Plan.helmholtz(ctx, dim, n, order, k)
    g = torch.Generator().manual_seed(7 * n + order)
    shape = (batch,) + (n,) * dim
    rhs = torch.complex(torch.randn(shape, generator=g, dtype=torch.float64),
                        torch.randn(shape, generator=g, dtype=torch.float64)).cuda()
    u = torch.empty_like(rhs)
    iters, rr = plan.solve_refined(rhs, u, batch, tol=1e-10, max_iter=10)
    assert rr <= 1e-10
    res = torch.empty_like(rhs)
    mr, mf = plan.residual(u, rhs, res, batch, norms=True)
    assert mr / mf == pytest.approx(rr, rel=1e-6)
    plain = torch.empty_like(rhs)
    plan.solve(rhs, plain, batch)
    ctx.synchronize()
    assert rel_err(u.cpu().numpy(), plain.cpu().numpy()) < 1e-8
    if n + 1 in (64, 128, 256, 512, 1024, 2048):
        assert iters >= 1  # single-precision transforms alone do not reach 1e-10
    u0 = torch.empty_like(rhs)
    it0, rr0 = plan.solve_refined(rhs, u0, batch, tol=1e-10, max_iter=0)
    assert it0 == 0 and (rr0 > 1e-10 or n + 1 not in (64, 128, 256, 512, 1024, 2048))
    plan.close()


@pytest.mark.parametrize("k", [10.0, 100.0, 400.0])
def test_refined_solve_2047_against_oracle_and_exact(ctx, oracle, k):
    """The refined form at 2D N = 2047, order 6 (the mixed-precision configuration's size and
    wavenumbers; k = 400 makes the lines lose diagonal dominance), on the right-hand side the
    oracle assembles from a seeded 8-mode source: the 2048-point transforms run in
    single-precision arithmetic, so at least one correction is needed; the result reaches the
    1e-10 residual and agrees with the oracle's FP64 solution, and with the manufactured exact
    solution as well as the oracle does (both to 1e-8 relative: the residual bound times the
    lines' conditioning)."""
    torch = pytest.importorskip("torch")
    n, order = 2047, 6
    modes = W.sine_modes(3000, 8, 20)
    f_ext = W.source_2d(n, modes, fast=True)
    ref = oracle.pipeline_2d(n, order, k, f_ext)
    rhs = torch.from_numpy(np.ascontiguousarray(ref["rhs"].reshape(1, n, n))).cuda()
    u = torch.empty_like(rhs)
    plan = hh.Plan.helmholtz(ctx, 2, n, order, k)
    iters, rr = plan.solve_refined(rhs, u, 1, tol=1e-10, max_iter=10)
    plan.close()
    got = u.cpu().numpy()[0]
    assert iters >= 1 and rr <= 1e-10, (iters, rr)
    assert rel_err(got, ref["sol"]) < 1e-8
    exact = W.exact_2d(n, modes, k)
    assert abs(rel_err(got, exact) - rel_err(ref["sol"], exact)) < 1e-8


def test_refined_solve_argument_checks(ctx):
    torch = pytest.importorskip("torch")
    plan = hh.Plan.helmholtz(ctx, 2, 63, 4, 10.0)
    rhs = torch.zeros((1, 63, 63), dtype=torch.complex128, device="cuda")
    with pytest.raises(hh.HHError):
        plan.solve_refined(rhs, rhs, 1)
    with pytest.raises(hh.HHError):
        plan.solve_refined(rhs, torch.empty_like(rhs), 1, tol=0.0)
    it, rr = plan.solve_refined(rhs, torch.empty_like(rhs), 1)  # zero rhs: zero residual at once
    assert it == 0 and rr == 0.0
    plan.close()
