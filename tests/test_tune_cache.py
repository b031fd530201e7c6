"""The tuning cache of hh_plan_tune (include/hh.h): file round trip and malformed lines on the
CPU; on the GPU, a second tune of the same shape (also at another wavenumber) is a cache hit that
launches no kernel and applies what the first one measured."""
import numpy as np
import pytest

import hackathon_b200 as hh


def test_cache_file_round_trip_without_a_gpu(tmp_path):
    hh.tune_cache_clear()
    src = tmp_path / "in.txt"
    src.write_text("# comment\n"
                   "NVIDIA B200\t2\t1023\t1023\t1\t6\t2\t6\t0\t0\t1\n"
                   "NVIDIA B200\t3\t255\t255\t255\t6\t2\t6\t0\t1020\t2\n"
                   "garbage line without fields\n")
    assert hh.tune_cache_load(str(src)) == 2
    assert hh.tune_cache_stats()["entries"] == 2
    out = tmp_path / "out.txt"
    hh.tune_cache_save(str(out))
    lines = [x for x in out.read_text().splitlines() if not x.startswith("#")]
    assert sorted(lines) == sorted(["NVIDIA B200\t2\t1023\t1023\t1\t6\t2\t6\t0\t0\t1",
                                    "NVIDIA B200\t3\t255\t255\t255\t6\t2\t6\t0\t1020\t2"])
    hh.tune_cache_clear()
    assert hh.tune_cache_stats() == {"hits": 0, "misses": 0, "entries": 0}
    with pytest.raises(hh.HHError):
        hh.tune_cache_load(str(tmp_path / "missing.txt"))


@pytest.mark.gpu
def test_cache_hit_skips_timing(ctx, tmp_path):
    hh.tune_cache_clear()
    n = 255
    a = hh.Plan.helmholtz(ctx, 2, n, 6, 10.0)
    a.variant = 0
    v = a.tune(8)
    s = hh.tune_cache_stats()
    assert s["misses"] == 1 and s["hits"] == 0 and s["entries"] == 1
    b = hh.Plan.helmholtz(ctx, 2, n, 6, 77.0)  # same shape, another k
    before = ctx.launches
    assert b.tune(8) == v
    assert ctx.launches == before  # the hit measured nothing
    assert hh.tune_cache_stats()["hits"] == 1
    c = hh.Plan.helmholtz(ctx, 2, n, 4, 77.0)  # another fused order: another entry
    assert not c.apply_tuning()
    path = str(tmp_path / "tune.txt")
    hh.tune_cache_save(path)
    hh.tune_cache_clear()
    assert not b.apply_tuning()
    assert hh.tune_cache_load(path) == 1
    b.variant = 0
    assert b.apply_tuning() and b.variant == v
    f = np.random.default_rng(1).standard_normal((n, n)) + 0j
    assert np.array_equal(b.solve_source_host(f), b.solve_source_host(f))
    for p in (a, b, c):
        p.close()
    hh.tune_cache_clear()
