"""GPU parity of the DST-I kernels against the oracle (and the reference's golden rows)."""
import ctypes as C

import numpy as np
import pytest
from conftest import golden, rel_err

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SIZES = [1, 2, 7, 63, 100, 127, 255, 300, 511, 1023, 2047, 4095, 8191]


def _dev(a: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _host(t) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("n", SIZES)
def test_dst_rows_matches_oracle(ctx, oracle, n):
    rows = 37 if n < 4000 else 5
    rng = np.random.default_rng(n)
    x = rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))
    src, dst = _dev(x), torch.empty((rows, n), dtype=torch.complex128, device="cuda")
    ctx.dst1_rows(n, rows, src, dst)
    ctx.synchronize()
    assert rel_err(_host(dst), oracle.dst1_rows(x)) < 1e-13


@pytest.mark.parametrize("rows", [1, 5, 1776, 1777, 2072, 5001])
def test_dst_rows_1023_ring_ticket_counts(ctx, oracle, rows):
    """1023-point rows go through the CTA-ring kernel (four warps sharing six line buffers, at
    most two blocks per SM, so 296 blocks on 148 SMs): fewer tickets per block than buffers,
    exactly as many (1776 rows), one block with one more, one more each, and thousands of rows
    whose tickets fall unevenly on the blocks."""
    n = 1023
    rng = np.random.default_rng(rows)
    x = rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))
    src, dst = _dev(x), torch.empty((rows, n), dtype=torch.complex128, device="cuda")
    ctx.dst1_rows(n, rows, src, dst)
    ctx.synchronize()
    assert rel_err(_host(dst), oracle.dst1_rows(x)) < 1e-13


@pytest.mark.parametrize("rows", [1, 3, 593, 888, 889, 3001])
def test_dst_rows_2047_two_warp_ticket_counts(ctx, oracle, rows):
    """2047-point rows go through the two-warps-per-line kernel (four lines per block, six line
    buffers, one block per SM): fewer lines than teams, one more line than the 592 teams of 148
    blocks, exactly the 888 buffers, one more, and thousands of rows spread unevenly."""
    n = 2047
    rng = np.random.default_rng(rows + 7)
    x = rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))
    src, dst = _dev(x), torch.empty((rows, n), dtype=torch.complex128, device="cuda")
    ctx.dst1_rows(n, rows, src, dst)
    ctx.synchronize()
    assert rel_err(_host(dst), oracle.dst1_rows(x)) < 1e-13
    ctx.dst1_rows(n, rows, dst, dst)  # in place, and the transform is its own inverse
    ctx.synchronize()
    assert rel_err(_host(dst), x) < 1e-13


def test_dst_rows_golden_and_in_place(ctx):
    g = golden("dst_rows.npz")
    for n in (1, 7, 31, 63, 100):
        t = _dev(g[f"x_{n}"])
        ctx.dst1_rows(n, t.shape[0], t, t)  # in place
        ctx.synchronize()
        assert rel_err(_host(t), g[f"y_{n}"]) < 1e-13


def test_dst_is_an_involution(ctx):
    n, rows = 1023, 64
    rng = np.random.default_rng(1)
    x = rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))
    t = _dev(x)
    ctx.dst1_rows(n, rows, t, t)
    ctx.dst1_rows(n, rows, t, t)
    ctx.synchronize()
    assert rel_err(_host(t), x) < 1e-13


@pytest.mark.parametrize("n", [255, 1023, 2047])
def test_dst_rows_pitched(ctx, oracle, n):
    """Rows inside wider pitched buffers (in_ld, out_ld > n), with a line count that leaves the
    last CTA partly empty."""
    rows, ld_in, ld_out = 21, n + 9, n + 3
    rng = np.random.default_rng(7 * n)
    x = rng.standard_normal((rows, ld_in)) + 1j * rng.standard_normal((rows, ld_in))
    out = torch.full((rows, ld_out), 7.0 + 7.0j, dtype=torch.complex128, device="cuda")
    ctx.dst1_rows(n, rows, _dev(x), out, in_ld=ld_in, out_ld=ld_out)
    ctx.synchronize()
    o = _host(out)
    assert rel_err(o[:, :n], oracle.dst1_rows(x[:, :n])) < 1e-13
    assert np.all(o[:, n:] == 7.0 + 7.0j)  # nothing written past the line


@pytest.mark.parametrize("n,ncols,planes", [(255, 255, 3), (63, 100, 2), (100, 37, 2), (1023, 64, 1), (7, 5, 4),
                                              (127, 33, 3), (511, 7, 2), (255, 1, 5), (63, 3, 7), (255, 8, 3),
                                              (255, 16, 2), (511, 24, 2), (127, 9, 4), (63, 255, 1)])
def test_dst_cols_matches_oracle(ctx, oracle, n, ncols, planes):
    """Columns of planes: n + 1 = 64 .. 512 with at least 8 columns take the CTA-tile kernel
    (8 swizzled columns per tensor box; counts that leave the last tile partly outside the plane),
    narrower planes and other lengths the per-warp tiles or the first-design kernels."""
    rng = np.random.default_rng(n + ncols)
    x = rng.standard_normal((planes, n, ncols)) + 1j * rng.standard_normal((planes, n, ncols))
    t = _dev(x)
    ctx.dst1_cols(n, ncols, planes, t, ncols, n * ncols, t)
    ctx.synchronize()
    ref = np.stack([oracle.dst1_rows(np.ascontiguousarray(x[p].T)).T for p in range(planes)])
    assert rel_err(_host(t), ref) < 1e-13


@pytest.mark.parametrize("nx,ny", [(255, 255), (31, 63), (100, 15)])
def test_dst2_planes_matches_reference_plane_transform(ctx, oracle, nx, ny):
    """hh_dst2_planes against the reference's 3D DST() restated (3D DST.c:148-204) on the real
    and imaginary planes."""
    planes = 3
    rng = np.random.default_rng(nx * ny)
    x = rng.standard_normal((planes, ny, nx)) + 1j * rng.standard_normal((planes, ny, nx))
    t = _dev(x)
    ctx.dst2_planes(nx, ny, planes, t, t)
    ctx.synchronize()
    ref = np.empty_like(x)
    for p in range(planes):
        for part, put in ((x[p].real, 1.0), (x[p].imag, 1j)):
            inp = np.ascontiguousarray(part)
            out = np.zeros_like(inp)
            oracle.lib.ora_dst2_plane_real(C.c_int(nx), C.c_int(ny), inp.ctypes.data_as(C.POINTER(C.c_double)),
                                           out.ctypes.data_as(C.POINTER(C.c_double)))
            if put == 1.0:
                ref[p] = out
            else:
                ref[p] += 1j * out
    assert rel_err(_host(t), ref) < 1e-13


@pytest.mark.parametrize("n", [63, 255, 1023])
def test_dst_cols_pitched(ctx, oracle, n):
    """Columns inside pitched planes (ld > ncols, plane stride > n*ld), written in place; values
    outside the columns stay untouched."""
    ncols, ld, planes = 9, 13, 3
    pstride = n * ld + 5
    rng = np.random.default_rng(n)
    buf = rng.standard_normal(planes * pstride) + 1j * rng.standard_normal(planes * pstride)
    t = _dev(buf)
    ctx.dst1_cols(n, ncols, planes, t, ld, pstride, t)
    ctx.synchronize()
    o = _host(t)
    for p in range(planes):
        blk = buf[p * pstride: p * pstride + n * ld].reshape(n, ld)
        got = o[p * pstride: p * pstride + n * ld].reshape(n, ld)
        want = oracle.dst1_rows(np.ascontiguousarray(blk[:, :ncols].T)).T
        assert rel_err(got[:, :ncols], want) < 1e-13
        assert np.array_equal(got[:, ncols:], blk[:, ncols:])
    for p in range(planes - 1):
        assert np.array_equal(o[p * pstride + n * ld:(p + 1) * pstride], buf[p * pstride + n * ld:(p + 1) * pstride])
