"""Serving loop: requests served in a mix (several sizes, overlapping on the
device) give the same results as each request served alone, and every
request completes with its latency recorded."""
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _server(precision, per_size):
    from redondito_b200 import serve, sphp as S
    prec = S.SPH_FP64 if precision == "fp64" else S.SPH_MIXED
    return serve.Server(S, torch, prec, per_size)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mix_equals_alone(precision):
    from redondito_b200 import serve
    reqs = serve.poisson_mix(14, rate=2000.0, seed=5, sizes=(15, 31, 63), weights=(2, 2, 1))
    srv = _server(precision, {15: 2, 31: 2, 63: 1})
    srv.serve(reqs, keep_results=True)
    st = serve.latency_stats(reqs)
    assert st["jobs"] == len(reqs) and st["p99_ms"] >= st["p50_ms"] > 0
    assert all(r.t_done >= r.t_admit >= r.arrival for r in reqs)
    srv.close()
    alone = _server(precision, {15: 1, 31: 1, 63: 1})
    for r in reqs:
        a = serve.Request(r.rid, 0.0, r.lmax, r.kind, r.steps)
        alone.serve([a], keep_results=True)
        for x, y in zip(r.result, a.result):
            assert torch.equal(x, y), (r.rid, r.kind, r.lmax)
    alone.close()
