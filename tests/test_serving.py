"""Serving many cases: continuous admission, overlap, HBM budget.

The GPU tests check that every case's result is bit-identical whether it
runs alone or mixed with other cases arriving while it runs, and that the
admitted cases never hold more device bytes than the budget.  The CPU test
checks the stream generator (sizes, parameters, arrivals) the benchmark uses.
"""
import numpy as np
import pytest

from hydraphase import PREC_FP64_PARITY, PREC_MIXED, cases
from hydraphase.engine import estimate_bytes


def test_serving_stream_is_seeded_and_shaped():
    a = cases.serving_stream(n_cases=12, steps=7, cells=(6000, 60000), seed=5)
    b = cases.serving_stream(n_cases=12, steps=7, cells=(6000, 60000), seed=5)
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert all(np.array_equal(x.spec.cu, y.spec.cu) for x, y in zip(a, b))
    arr = np.array([r.arrival for r in a])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    n = np.array([r.spec.mesh.neles for r in a])
    assert n.min() >= 6 * 9 ** 3 and n.max() <= 6 * 22 ** 3
    assert all(r.steps == 7 for r in a)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_FP64_PARITY, PREC_MIXED])
def test_each_result_same_alone_and_in_the_mix(precision):
    from hydraphase.serve import Server, run_alone
    reqs = cases.serving_stream(n_cases=6, rate=400.0, steps=12, cells=(6000, 40000), seed=7)
    rep = Server(hbm_budget=8 << 30, precision=precision, max_active=4, chunk=3).run(reqs)
    assert len(rep.results) == 6 and all(r.error is None for r in rep.results)
    assert rep.peak_active > 1          # cases did overlap
    for r, q in zip(rep.results, reqs):
        t, cu, gp = run_alone(q.spec, q.steps, precision=precision)
        assert t == r.time
        np.testing.assert_array_equal(r.cu, cu)
        np.testing.assert_array_equal(r.ghost_prims, gp)


@pytest.mark.gpu
def test_admission_respects_the_budget():
    from hydraphase.serve import Server
    reqs = cases.serving_stream(n_cases=8, rate=1000.0, steps=6, cells=(20000, 40000), seed=3)
    sizes = [estimate_bytes(q.spec.mesh, q.spec.params(precision=PREC_MIXED)) for q in reqs]
    budget = 2 * max(sizes) + 1          # room for two cases at a time
    rep = Server(hbm_budget=budget, precision=PREC_MIXED, max_active=8, chunk=2, keep_state=False).run(reqs)
    assert len(rep.results) == 8 and all(r.error is None for r in rep.results)
    assert rep.peak_bytes <= budget
    s = rep.summary()
    assert s["p99_s"] >= s["p50_s"] > 0 and s["updates_per_s"] > 0
