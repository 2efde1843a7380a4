"""Serving: requests served with continuous batching give the same results as
the same requests run alone, one after the other (alone vs in the mix)."""
import pytest

pytestmark = pytest.mark.gpu


def test_served_results_equal_alone():
    from multiphase_lbm_b200 import serve
    edges = [32, 48]
    reqs = serve.make_requests(10, rate=200.0, seed=11, budget_scale=0.05,
                               edges=edges)
    mk, done = serve.serve_batched(reqs, hbm_cap=2e9)
    reqs2 = serve.make_requests(10, rate=200.0, seed=11, budget_scale=0.05,
                                edges=edges)
    mk2, alone = serve.serve_fifo(reqs2)
    for a, b in zip(sorted(done, key=lambda r: r.rid),
                    sorted(alone, key=lambda r: r.rid)):
        assert a.steps == b.steps
        assert a.history == b.history       # every saturation sample equal
        assert a.done_at >= a.arrival
    s = serve.summarise(mk, done)
    assert s["requests"] == 10 and s["p99_s"] >= s["p50_s"] > 0


def test_admission_respects_the_memory_cap():
    """With a cap that fits one domain at a time, requests still all finish
    (admitted as memory frees up)."""
    from multiphase_lbm_b200 import capi, serve
    reqs = serve.make_requests(4, rate=1000.0, seed=3, budget_scale=0.03,
                               edges=[32])
    one = capi.lattice_bytes((32, 32, 32), capi.STORE_F32)
    mk, done = serve.serve_batched(reqs, hbm_cap=one * 1.5)
    assert all(r.done_at > 0 for r in done)
