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


def test_size_classes_and_tune_cache(tmp_path, monkeypatch):
    from hydraphase import tune
    assert [tune.size_class(n) for n in (6000, 50000, 200000, 5000000)] == ["xs", "s", "m", "l"]
    monkeypatch.setenv("HYDRAPHASE_TUNE_CACHE", str(tmp_path / "t.json"))
    tune._store({"k": {"best": 128}})
    assert tune._load() == {"k": {"best": 128}}


def test_server_groups_small_compatible_cases():
    from hydraphase.serve import Server
    reqs = cases.serving_stream(n_cases=10, steps=5, cells=(6000, 60000), seed=9)
    s = Server(hbm_budget=1 << 40, batch_cells=100000, max_batch=4)
    unit = s._take_unit(list(reqs))
    assert 1 <= len(unit) <= 4
    assert sum(r.spec.mesh.neles for r in unit) <= 100000 or len(unit) == 1
    assert [r.rid for r in unit] == [r.rid for r in reqs[:len(unit)]]
    assert Server(hbm_budget=1 << 40)._take_unit(list(reqs)) == [reqs[0]]


@pytest.mark.gpu
def test_batched_serving_equals_alone():
    from hydraphase.serve import Server, run_alone
    reqs = cases.serving_stream(n_cases=7, rate=1000.0, steps=9, cells=(6000, 30000), seed=11)
    rep = Server(hbm_budget=8 << 30, precision=PREC_MIXED, max_active=3, chunk=4, batch_cells=60000,
                 block_size=128).run(reqs, realtime=False)
    assert len(rep.results) == 7 and all(r.error is None for r in rep.results)
    assert rep.units < 7                 # some cases did share a batch
    for r, q in zip(rep.results, reqs):
        t, cu, gp = run_alone(q.spec, q.steps, precision=PREC_MIXED)
        assert t == r.time
        np.testing.assert_array_equal(r.cu, cu)
        np.testing.assert_array_equal(r.ghost_prims, gp)


@pytest.mark.gpu
def test_block_size_tuner_measures_and_caches(tmp_path, monkeypatch):
    from hydraphase import tune
    monkeypatch.setenv("HYDRAPHASE_TUNE_CACHE", str(tmp_path / "t.json"))
    spec = cases.shock_bubble(n=8, alpha_min=0.1)
    best, ms = tune.tune_block_size(spec, candidates=(128, 256), steps=2)
    assert best in (128, 256) and set(ms) == {128, 256}
    best2, ms2 = tune.tune_block_size(spec, candidates=(128, 256), steps=2)
    assert best2 == best and ms2 == ms


@pytest.mark.gpu
def test_face_mode_tuner_measures_and_caches(tmp_path, monkeypatch):
    from hydraphase import PREC_FP64_PARITY, tune
    monkeypatch.setenv("HYDRAPHASE_TUNE_CACHE", str(tmp_path / "t.json"))
    spec = cases.shock_bubble(n=8, alpha_min=0.1)
    best, ms = tune.tune_face_mode(spec, steps=2)
    assert set(ms) == {0, 1, 2}                     # gather, each side, colouring
    _, ms_a = tune.tune_face_mode(spec, steps=2, deterministic=False)
    assert set(ms_a) == {0, 1, 2, 3}                # and atomics
    assert best in (0, 1, 2)
    assert tune.tune_face_mode(spec, steps=2) == (best, ms)
    assert tune.tune_face_mode(spec, precision=PREC_FP64_PARITY) == (0, {})


@pytest.mark.gpu
def test_step_mode_tuner_measures_and_caches(tmp_path, monkeypatch):
    from hydraphase import PREC_FP64_PARITY, tune
    monkeypatch.setenv("HYDRAPHASE_TUNE_CACHE", str(tmp_path / "t.json"))
    spec = cases.shock_bubble(n=8, alpha_min=0.1)
    best, ms = tune.tune_step_mode(spec, precision=PREC_FP64_PARITY, steps=2)
    assert set(ms) == {1, 2} and best in (1, 2)      # graph, fused step
    assert tune.tune_step_mode(spec, precision=PREC_FP64_PARITY, steps=2) == (best, ms)
    assert tune.tune_step_mode(spec, precision=PREC_MIXED) == (1, {})


@pytest.mark.gpu
def test_served_fused_results_equal_graph_results():
    from hydraphase.serve import Server
    reqs = cases.serving_stream(n_cases=6, rate=1000.0, steps=20, cells=(3000, 30000), seed=5)
    outs = []
    for mode in (1, 2):
        server = Server(hbm_budget=8 << 30, precision=PREC_FP64_PARITY, max_active=3, chunk=10,
                        batch_cells=60000, step_mode=mode)
        rep = server.run(reqs, realtime=False)
        assert all(r.error is None for r in rep.results)
        outs.append({r.rid: r.cu for r in rep.results})
    for rid in outs[0]:
        np.testing.assert_array_equal(outs[1][rid], outs[0][rid])
