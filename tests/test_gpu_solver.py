"""GPU parity of the full solve (plain FP64) against the oracle restatement, which is itself
bit-exact with the reference's C code (tests/test_oracle.py)."""
import numpy as np
import pytest
from conftest import FACTOR_ASSEMBLED, assert_parity_2d, golden, rel_err

import hackathon_b200 as hh
from hackathon_b200 import workload as W

pytestmark = pytest.mark.gpu

TOL = 1e-12  # plain FP64 form vs the reference path: max|u - u_ref| / max|u_ref|


def _source(n, seed, pmax=20, noise=1e-3):
    return W.source_2d(n, W.sine_modes(seed, 8, pmax), noise_seed=seed + 1 if noise else None, noise_var=noise)


@pytest.mark.parametrize("n,order,k", [(15, 6, 10.0), (16, 4, 50.0), (31, 2, 10.0), (63, 6, 200.0), (100, 6, 10.0),
                                       (127, 4, 50.0), (255, 6, 50.0), (300, 6, 20.0), (511, 2, 30.0),
                                       (1023, 6, 10.0), (1023, 4, 200.0)])
def test_solver2d_assembled_rhs_matches_oracle(ctx, oracle, n, order, k):
    """drop-in path: solver() on the reference's assembled rhs with its coefficient rows."""
    f = _source(n, n + order)
    ref = oracle.pipeline_2d(n, order, k, f)
    plan = hh.Plan.from_coefficients_2d(ctx, n, n, ref["coef"])
    sol = plan.solve_host(ref["rhs"])
    assert_parity_2d(oracle, sol, ref, TOL, FACTOR_ASSEMBLED)
    plan.close()


@pytest.mark.parametrize("n,order,k", [(15, 6, 10.0), (31, 4, 50.0), (31, 2, 10.0), (100, 6, 10.0), (255, 6, 50.0),
                                       (1023, 6, 50.0), (1023, 4, 10.0), (1023, 6, 200.0), (2047, 6, 100.0)])
def test_solver2d_fused_source_matches_oracle(ctx, oracle, n, order, k):
    """Helmholtz plan: RHS assembly fused on the device vs the reference pipeline
    coefficients -> rhs -> LU -> solver."""
    f = _source(n, 3 * n + order)
    ref = oracle.pipeline_2d(n, order, k, f)
    plan = hh.Plan.helmholtz(ctx, 2, n, order, k)
    u = plan.solve_source_host(f[1:-1, 1:-1])
    assert_parity_2d(oracle, u, ref, TOL)
    plan.close()


@pytest.mark.parametrize("dim,n,order,k", [(2, 255, 6, 50 + 5j), (2, 1023, 4, 100 - 20j), (2, 127, 2, 30 + 30j),
                                           (3, 31, 6, 20 + 3j), (3, 63, 4, 10 - 4j)])
def test_complex_k_fused_source_matches_oracle(ctx, oracle, dim, n, order, k):
    """Complex constant k (a damped or absorbing medium; the reference's problem structs carry
    complex k): the fused operator and the shifted lines with complex k^2, for every line-solve
    variant, against the reference pipeline."""
    if dim == 2:
        f = _source(n, 5 * n + order)
        ref = oracle.pipeline_2d(n, order, k, f)
        src = f[1:-1, 1:-1]
    else:
        f = W.source_3d(n, W.sine_modes(n + order, 16, min(n, 64), dim=3))
        ref = oracle.pipeline_3d(n, order, k, f)
        src = f[1:-1, 1:-1, 1:-1]
    plan = hh.Plan.helmholtz(ctx, dim, n, order, k)
    for v in range(7):
        plan.variant = v
        u = plan.solve_source_host(src)
        if dim == 2:
            assert_parity_2d(oracle, u, ref, TOL)
        else:
            assert rel_err(u, ref["sol"]) < TOL
    plan.close()


def test_readme_case_against_golden_and_exact(ctx):
    """./Direct_Solver 6 100 class: the reference's own output (golden) and the manufactured
    exact solution."""
    g = golden("ref2d_o6_n100_k10_readme.npz")
    n = int(g["n"])
    m = W.sine_modes(int(g["seed"]), 8, int(g["pmax"]))
    f = W.source_2d(n, m)
    plan = hh.Plan.helmholtz(ctx, 2, n, 6, 10.0)
    u = plan.solve_source_host(f[1:-1, 1:-1])
    assert rel_err(u, g["sol"]) < TOL
    exact = W.exact_2d(n, m, 10.0)
    # 6th-order discretisation error at h = 1/101 with modes up to p = 20: (20 pi h)^6 / 6! scale
    assert rel_err(u, exact) < 1e-5


def test_batch_equals_single(ctx, oracle):
    n, order, k, B = 255, 6, 50.0, 6
    fs = np.stack([_source(n, 100 + b)[1:-1, 1:-1] for b in range(B)])
    plan = hh.Plan.helmholtz(ctx, 2, n, order, k)
    ub = plan.solve_source_host(fs)
    for b in (0, 3, 5):
        assert np.array_equal(plan.solve_source_host(fs[b]), ub[b])  # bitwise: alone == in batch


@pytest.mark.parametrize("n,order,k", [(15, 6, 10.0), (31, 6, 10.0), (63, 2, 30.0), (255, 4, 50.0), (511, 6, 20.0),
                                       (1023, 6, 50.0), (1023, 4, 10.0), (2047, 6, 100.0)])
def test_every_line_solve_variant_matches_oracle(ctx, oracle, n, order, k):
    """Each line-solve kernel on its own (0/1: general rows, 512 or 256 threads; 2..6: symmetric
    constant rows with the order-6 partial fractions -- 2 or 1 blocks per SM, one or two
    right-hand sides per pass, 8- or 16-row segments, right-hand sides moved as TMA tiles), then
    hh_plan_tune's choice."""
    f = _source(n, 7 * n + order)
    ref = oracle.pipeline_2d(n, order, k, f)
    plan = hh.Plan.helmholtz(ctx, 2, n, order, k)
    assert plan.variant == 2  # constant k: the symmetric kernel by default
    outs = []
    for v in range(7):
        plan.variant = v
        assert plan.variant == v
        outs.append(plan.solve_source_host(f[1:-1, 1:-1]))
        assert_parity_2d(oracle, outs[-1], ref, TOL)
    for v in range(1, 7):
        assert rel_err(outs[v], outs[0]) < TOL  # same system, different rounding only
    assert np.array_equal(outs[6], outs[5])  # tile I/O moves the same values as variant 5
    v = plan.tune(4)
    assert v in range(7)
    assert np.array_equal(plan.solve_source_host(f[1:-1, 1:-1]), outs[v])
    with pytest.raises(hh.HHError):
        plan.variant = 7
    plan.close()


@pytest.mark.parametrize("n,order,k", [(4095, 6, 100.0), (4095, 4, 400.0)])
def test_solver2d_longest_lines_matches_oracle(ctx, oracle, n, order, k):
    """The longest lines the symmetric kernel takes (4095 rows: 16-row segments, one line per
    CTA, per-thread prefetch) beside the general kernel, and variant 2, whose 8-row segments
    stop at 2048 rows and which therefore runs the general kernel here."""
    f = _source(n, 11 * n + order)
    ref = oracle.pipeline_2d(n, order, k, f)
    plan = hh.Plan.helmholtz(ctx, 2, n, order, k)
    assert plan.variant == 5  # the default for lines beyond 2048 rows: the symmetric kernel
    outs = {}
    for v in (0, 2, 5, 6):
        plan.variant = v
        outs[v] = plan.solve_source_host(f[1:-1, 1:-1])
        assert_parity_2d(oracle, outs[v], ref, TOL)
    assert np.array_equal(outs[2], outs[0])  # the same general kernel
    assert np.array_equal(outs[6], outs[5])  # no tile input at one line per CTA
    assert rel_err(outs[5], outs[0]) < TOL
    plan.close()


def test_symmetric_kernel_assembled_rhs(ctx, oracle):
    """Helmholtz plan on an assembled right-hand side (no fused operator) through the symmetric
    kernel, against the reference pipeline."""
    n, order, k = 1023, 6, 50.0
    f = _source(n, 17)
    ref = oracle.pipeline_2d(n, order, k, f)
    plan = hh.Plan.helmholtz(ctx, 2, n, order, k)
    sol = plan.solve_host(ref["rhs"])
    assert_parity_2d(oracle, sol, ref, TOL)
    plan.close()


def test_host_path_chunked_equals_device_path(ctx):
    """Host-buffer solves run in overlapped chunks (copies on their own streams); the result is
    bitwise the device-buffer solve of the whole batch."""
    torch = pytest.importorskip("torch")
    n, B = 1023, 8
    fs = np.stack([_source(n, 300 + b)[1:-1, 1:-1] for b in range(B)])
    plan = hh.Plan.helmholtz(ctx, 2, n, 6, 50.0)
    host = plan.solve_source_host(torch.from_numpy(fs).pin_memory().numpy())
    f = torch.from_numpy(fs).cuda()
    u = torch.empty_like(f)
    plan.solve_source(f, u, B)
    ctx.synchronize()
    assert np.array_equal(host, u.cpu().numpy())
    plan.close()


@pytest.mark.parametrize("dim,n,order,batch", [(2, 1023, 4, 7), (2, 1023, 6, 5), (2, 511, 2, 9), (2, 127, 4, 3),
                                               (3, 63, 6, 3), (3, 127, 4, 2)])
def test_tile_io_variant_equals_prefetch_variant(ctx, dim, n, order, batch):
    """Variant 6 brings each right-hand side in as TMA tiles.  On device buffers of several
    right-hand sides, over every chunk boundary of the grid, its result is bitwise variant 5's,
    whose arithmetic it shares."""
    torch = pytest.importorskip("torch")
    g = torch.Generator().manual_seed(1000 * dim + n + order)
    shape = (batch,) + (n,) * dim
    f = torch.complex(torch.randn(shape, generator=g, dtype=torch.float64),
                      torch.randn(shape, generator=g, dtype=torch.float64)).cuda()
    plan = hh.Plan.helmholtz(ctx, dim, n, order, 40.0)
    outs = []
    for v in (5, 6):
        plan.variant = v
        u = torch.full_like(f, float("nan"))
        plan.solve_source(f, u, batch)
        ctx.synchronize()
        outs.append(u.cpu())
    assert torch.isfinite(outs[1]).all()
    assert torch.equal(outs[0], outs[1])
    plan.close()


@pytest.mark.parametrize("n,order,k", [(15, 6, 30.0), (31, 6, 30.0), (31, 4, 10.0), (63, 2, 20.0), (127, 6, 30.0)])
def test_solver3d_fused_source_matches_oracle(ctx, oracle, n, order, k):
    m = W.sine_modes(n + order, 16, min(n, 64), dim=3)
    f = W.source_3d(n, m)
    ref = oracle.pipeline_3d(n, order, k, f)
    plan = hh.Plan.helmholtz(ctx, 3, n, order, k)
    u = plan.solve_source_host(f[1:-1, 1:-1, 1:-1])
    assert rel_err(u, ref["sol"]) < TOL
    # drop-in path on the assembled rhs
    plan3 = hh.Plan.from_coefficients_3d(ctx, n, n, n, ref["coef"])
    assert rel_err(plan3.solve_host(ref["rhs"]), ref["sol"]) < TOL


@pytest.mark.parametrize("name", ["paper_o6_n11", "paper_o4_n11", "default_o6_n13"])
def test_solver3d_reference_problem_golden(ctx, name):
    """The reference's own 3D problems (variable k(z) for the paper case): our solver on the
    reference's assembled rhs and per-layer stencil vs its own solve."""
    g = golden(f"ref3d_{name}.npz")
    n = int(g["n"])
    coef = {nm: g[f"c_{nm}"] for nm in ("a", "b", "c", "d", "ap", "bp", "cp", "dp", "am", "bm", "cm", "dm")}
    plan = hh.Plan.from_coefficients_3d(ctx, n, n, n, coef)
    assert rel_err(plan.solve_host(g["rhs"]), g["sol"]) < TOL


def test_invalid_arguments(ctx):
    with pytest.raises(hh.HHError):
        hh.Plan.helmholtz(ctx, 2, 31, 5, 10.0)
    plan = hh.Plan.helmholtz(ctx, 2, 31, 6, 10.0)
    with pytest.raises(hh.HHError):
        plan.solve(0, 0, 1)
    plan.solve(0, 0, 0)  # empty batch is a no-op


def test_3d_transform_slabs_give_identical_results(ctx, oracle):
    """The 3D transforms run slab by slab (rows pass then columns pass per slab of planes); the
    slab changes only the order of the launches, never a value: every slab size gives the same
    bits, and they match the oracle."""
    n, order, k, B = 63, 6, 30.0, 3
    f_ext = [W.source_3d(n, W.sine_modes(40 + b, 16, 32, dim=3)) for b in range(B)]
    f = np.stack([x[1:-1, 1:-1, 1:-1] for x in f_ext])
    plan = hh.Plan.helmholtz(ctx, 3, n, order, k)
    outs = []
    for slab in (0, 1, 5, 63, 64, 189):
        plan.slab = slab
        assert plan.slab == slab
        outs.append(plan.solve_source_host(f))
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    assert rel_err(outs[0][1], oracle.pipeline_3d(n, order, k, f_ext[1])["sol"]) < TOL
    plan.tune(B)
    assert 1 <= plan.slab <= n * B
    assert np.array_equal(plan.solve_source_host(f), outs[0])
    with pytest.raises(hh.HHError):
        plan.slab = -1
    plan.close()


@pytest.mark.parametrize("n", [63, 127, 255])
def test_3d_column_dst_variants_give_identical_results(ctx, oracle, n):
    """The two column-transform kernels of the 3D plans (CTA tiles of 8 swizzled columns, or
    per-warp tiles) run the same transform arithmetic on the same values: identical bits."""
    order, k, B = 6, 20.0, 2
    f_ext = [W.source_3d(n, W.sine_modes(70 + b, 16, min(n, 64), dim=3)) for b in range(B)]
    f = np.stack([x[1:-1, 1:-1, 1:-1] for x in f_ext])
    plan = hh.Plan.helmholtz(ctx, 3, n, order, k)
    outs = []
    for v in (0, 1):
        plan.dst_variant = v
        assert plan.dst_variant == v
        outs.append(plan.solve_source_host(f))
    assert np.array_equal(outs[0], outs[1])
    assert rel_err(outs[0][0], oracle.pipeline_3d(n, order, k, f_ext[0])["sol"]) < TOL
    with pytest.raises(hh.HHError):
        plan.dst_variant = 2
    plan.close()


@pytest.mark.parametrize("dim,n,order", [(3, 31, 4), (3, 31, 6), (2, 63, 6), (3, 63, 4), (2, 15, 4)])
def test_tile_io_short_lines_every_variant(ctx, dim, n, order):
    """Short lines (31 or 63 rows) in CTAs of 32 lines with 16-row segments: most segments of
    the TMA-tile variant lie wholly past the end of the line and must read nothing from the tile
    (their halo rows included).  Every line-solve variant on a batch of 8, tuned as the request
    loop's shapes are, gives the same solution as variant 5."""
    torch = pytest.importorskip("torch")
    g = torch.Generator().manual_seed(97 * n + order)
    shape = (8,) + (n,) * dim
    f = torch.complex(torch.randn(shape, generator=g, dtype=torch.float64),
                      torch.randn(shape, generator=g, dtype=torch.float64)).cuda()
    plan = hh.Plan.helmholtz(ctx, dim, n, order, 100.0)
    outs = {}
    for v in range(7):
        plan.variant = v
        u = torch.full_like(f, float("nan"))
        plan.solve_source(f, u, 8)
        ctx.synchronize()
        outs[v] = u.cpu().numpy()
    for v in range(7):
        assert np.isfinite(outs[v]).all()
        assert rel_err(outs[v], outs[5]) < TOL
    assert np.array_equal(outs[6], outs[5])
    plan.close()


@pytest.mark.parametrize("dim,n,order,variant", [(2, 255, 6, 6), (2, 1023, 4, 6), (2, 127, 2, 4), (3, 63, 6, 5),
                                                 (3, 31, 4, 6), (2, 2047, 6, 5), (2, 511, 6, 0)])
def test_several_wavenumbers_in_one_solve(ctx, dim, n, order, variant):
    """hh_solve_source_multi: plans of one shape at different k share the transform launches and
    (same symmetric variant) one line-solve launch; each field is bitwise the solo solve of its own
    plan.  Variant 0 (the general kernel) takes the one-launch-per-plan path."""
    torch = pytest.importorskip("torch")
    ks, counts = [7.0, 33.3 + 1.5j, 120.0], [3, 1, 2]
    g = torch.Generator().manual_seed(n + order)
    shape = (sum(counts),) + (n,) * dim
    f = torch.complex(torch.randn(shape, generator=g, dtype=torch.float64),
                      torch.randn(shape, generator=g, dtype=torch.float64)).cuda()
    plans = [hh.Plan.helmholtz(ctx, dim, n, order, k) for k in ks]
    for p in plans:
        p.variant = variant
    u = torch.full_like(f, float("nan"))
    before = ctx.launches
    hh.solve_source_multi(plans, counts, f, u)
    ctx.synchronize()
    launches = ctx.launches - before
    per_dir = 1 if dim == 2 else 2
    assert launches == 2 * per_dir + (1 if variant >= 2 else len(ks))
    got = u.cpu().numpy()
    off = 0
    for p, c in zip(plans, counts):
        solo = torch.empty_like(f[off:off + c])
        p.solve_source(f[off:off + c], solo, c)
        ctx.synchronize()
        assert np.array_equal(got[off:off + c], solo.cpu().numpy())
        off += c
    with pytest.raises(hh.HHError):
        other = hh.Plan.helmholtz(ctx, dim, n, 2 if order != 2 else 4, 10.0)
        hh.solve_source_multi([plans[0], other], [1, 1], f, u)
    for p in plans:
        p.close()


@pytest.mark.parametrize("dim,n", [(2, 255), (2, 511), (2, 1023), (2, 63), (3, 63), (3, 127)])
def test_rows_dst_variants_give_identical_results(ctx, dim, n):
    """The CTA-ring and the per-warp-buffer rows transforms run the same arithmetic on the same
    values: every rows variant gives the same bits."""
    torch = pytest.importorskip("torch")
    g = torch.Generator().manual_seed(n + dim)
    B = 3
    shape = (B,) + (n,) * dim
    f = torch.complex(torch.randn(shape, generator=g, dtype=torch.float64),
                      torch.randn(shape, generator=g, dtype=torch.float64)).cuda()
    plan = hh.Plan.helmholtz(ctx, dim, n, 6, 25.0)
    outs = []
    for v in (0, 1, 2):
        plan.rows_variant = v
        assert plan.rows_variant == v
        u = torch.empty_like(f)
        plan.solve_source(f, u, B)
        ctx.synchronize()
        outs.append(u.cpu())
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[1], outs[2])
    with pytest.raises(hh.HHError):
        plan.rows_variant = 3
    plan.close()


def test_rows_2047_two_warp_and_stockham_kernels_agree(ctx):
    """At n + 1 = 2048 the rows variants 0 and 1 run the two-warps-per-line transform and variant 2
    the first-design Stockham kernel: different arithmetic, so the solutions agree to rounding
    as the solve amplifies it (relative 1e-12, the solution parity bound; 2e-13 measured at
    k = 100), and 0 and 1 give the same bits."""
    torch = pytest.importorskip("torch")
    g = torch.Generator().manual_seed(2047)
    n, B = 2047, 2
    f = torch.complex(torch.randn((B, n, n), generator=g, dtype=torch.float64),
                      torch.randn((B, n, n), generator=g, dtype=torch.float64)).cuda()
    plan = hh.Plan.helmholtz(ctx, 2, n, 6, 100.0)
    outs = []
    for v in (0, 1, 2):
        plan.rows_variant = v
        u = torch.empty_like(f)
        plan.solve_source(f, u, B)
        ctx.synchronize()
        outs.append(u.cpu())
    assert torch.equal(outs[0], outs[1])
    assert ((outs[2] - outs[0]).abs().max() / outs[0].abs().max()).item() < 1e-12
    plan.close()
