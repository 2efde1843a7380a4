"""Serving: requests served with continuous batching give the same results as
the same requests run alone, one after the other (alone vs in the mix),
also when the server preempts requests (exact checkpoint, resume later)."""
import pytest

pytestmark = pytest.mark.gpu


def test_served_results_equal_alone():
    from multiphase_lbm_b200 import serve
    edges = [32, 48]
    reqs = serve.make_requests(10, rate=200.0, seed=11, budget_scale=0.05,
                               edges=edges)
    mk, done, idle = serve.serve_batched(reqs, hbm_cap=2e9)
    reqs2 = serve.make_requests(10, rate=200.0, seed=11, budget_scale=0.05,
                                edges=edges)
    mk2, alone, _ = serve.serve_fifo(reqs2)
    for a, b in zip(sorted(done, key=lambda r: r.rid),
                    sorted(alone, key=lambda r: r.rid)):
        assert a.steps == b.steps
        assert a.history == b.history       # every saturation sample equal
        assert a.done_at >= a.arrival
    s = serve.summarise(mk, done, idle)
    assert s["requests"] == 10 and s["p99_s"] >= s["p50_s"] > 0


def test_admission_respects_the_memory_cap():
    """With a cap that fits one domain at a time, requests still all finish
    (admitted as memory frees up)."""
    from multiphase_lbm_b200 import capi, serve
    reqs = serve.make_requests(4, rate=1000.0, seed=3, budget_scale=0.03,
                               edges=[32])
    one = capi.lattice_bytes((32, 32, 32), capi.STORE_F32)
    mk, done, _ = serve.serve_batched(reqs, hbm_cap=one * 1.5)
    assert all(r.done_at > 0 for r in done)


def test_preempted_requests_resume_exactly():
    """A long request followed by short ones under a node cap that holds one
    request: the short ones preempt the long one (saved to host memory,
    resumed later), and every result equals the request run alone."""
    from multiphase_lbm_b200 import serve
    def stream():
        reqs = serve.make_requests(4, rate=50.0, seed=5, budget_scale=0.05,
                                   edges=[32, 48])
        reqs[0].shape, reqs[0].budget = (48, 48, 48), 6000
        for r in reqs[1:]:
            r.shape, r.budget = (32, 32, 32), 1000
        return reqs
    reqs = stream()
    mk, done, idle = serve.serve_batched(reqs, node_cap=48 ** 3 + 1,
                                         preempt=True)
    assert sum(r.preemptions for r in done) >= 1
    mk2, alone, _ = serve.serve_fifo(stream())
    for a, b in zip(sorted(done, key=lambda r: r.rid),
                    sorted(alone, key=lambda r: r.rid)):
        assert a.steps == b.steps
        assert a.history == b.history
