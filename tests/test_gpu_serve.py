"""Serving loop: requests served in a mix (several sizes and kinds,
overlapping on the device) give the same results as each request served
alone; admission keeps the slots within the HBM budget, releasing idle slots
of other sizes; a served pair matches the CPU oracle; plan clones (the
slots of one size share their tables) compute what their source computes."""
import numpy as np
import pytest

from tests._helpers import check

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _server(precision, budget=60e9, max_slots=None):
    from redondito_b200 import serve, sphp as S
    prec = S.SPH_FP64 if precision == "fp64" else S.SPH_MIXED
    return serve.Server(S, torch, prec, budget, max_slots=max_slots)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mix_equals_alone(precision):
    from redondito_b200 import serve
    reqs = serve.poisson_mix(16, rate=2000.0, seed=5, sizes=(15, 31, 63, 255), weights=(3, 3, 2, 2))
    assert any(r.lmax == 255 and r.kind == "rk3" for r in reqs)
    srv = _server(precision)
    srv.serve(reqs, keep_results=True)
    st = serve.latency_stats(reqs)
    assert st["jobs"] == len(reqs) and st["p99_ms"] >= st["p50_ms"] > 0
    assert all(r.t_done >= r.t_admit >= r.arrival for r in reqs)
    assert srv.peak_bytes <= srv.budget
    srv.close()
    alone = _server(precision)
    for r in reqs:
        a = serve.Request(r.rid, 0.0, r.lmax, r.kind, r.steps)
        alone.serve([a], keep_results=True)
        for x, y in zip(r.result, a.result):
            assert torch.equal(x, y), (r.rid, r.kind, r.lmax)
    alone.close()


def test_budget_releases_idle_slots_and_rejects_oversize():
    """A budget that holds about one large slot: requests of alternating
    sizes force idle slots of the other size out; all complete, the bytes
    held never pass the budget, and a request larger than the budget is an
    error instead of a wait that never ends."""
    from redondito_b200 import serve
    probe = _server("fp64")
    probe.warm([(127, "rk3"), (63, "rk3")])
    measured = dict(probe.measured)
    probe.close()
    b127, b63 = measured[(127, "rk3", True)], measured[(63, "rk3", True)]
    assert b127 > b63 > 0
    srv = _server("fp64", budget=b127 + 0.5 * b63)  # one slot of either size, not both
    srv.measured.update(measured)
    reqs = [serve.Request(i, 0.0005 * i, (127, 63)[i % 2], "rk3", 1) for i in range(6)]
    srv.serve(reqs)
    assert all(r.t_done is not None for r in reqs)
    assert srv.released >= 1 and srv.peak_bytes <= srv.budget
    srv.close()
    tiny = _server("fp64", budget=1e6)
    with pytest.raises(MemoryError):
        tiny.serve([serve.Request(0, 0.0, 31, "pair")])
    tiny.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_served_pair_matches_oracle(precision):
    """One pair request, served: the seeded spectrum taken to (lm, kz), the 3D
    inverse and forward transforms, against the oracle on the same input."""
    from oracle import oracle as O
    from redondito_b200 import serve
    r = serve.Request(7, 0.0, 63, "pair")
    srv = _server(precision)
    srv.serve([r], keep_results=True)
    P = srv.slots[(63, "pair")][0].plan
    x = serve.pair_input(P, torch, r.rid).cpu().numpy()
    srv.close()
    lmax, nz, nlat, nphi = serve.size_of(63)
    Po = O.Plan(lmax, nz, nlat=nlat, nphi=nphi, C=25, d=5, rint=0.5, rext=1.5)
    ref = Po.forward_3d(Po.inverse_3d(Po.z_forward(x)))
    got = r.result[0].cpu().numpy()
    err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    check(err, 1e-12 if precision == "fp64" else 1e-6, f"served pair {precision}")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_clone_shares_tables(precision):
    """A clone computes bit for bit what its source computes, keeps working
    after the source is destroyed (the tables go with the last plan), and
    the MMA rows of shared tables cannot be changed."""
    from redondito_b200 import sphp as S
    prec = S.SPH_FP64 if precision == "fp64" else S.SPH_MIXED
    A = S.Plan(31, 64, nlat=48, nphi=96, Cz=25, oz=5, precision=prec)
    B = A.clone()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(3)
    spec = torch.randn((64, A.nlm), dtype=torch.complex128, device="cuda", generator=gen)
    spec[:, A.emm.cuda() == 0] = spec[:, A.emm.cuda() == 0].real.to(torch.complex128)
    ga, gb = A.new_grid(), B.new_grid()
    S.fftp3d_complex_to_real(A, spec.clone(), ga)
    S.fftp3d_complex_to_real(B, spec.clone(), gb)
    assert torch.equal(ga, gb)
    S.setup_bc(A)
    S.setup_bc(B)  # the boundary matrices A built
    ta, tb = A.new_spec(), B.new_spec()
    S.invDl(A, spec, ta)
    S.invDl(B, spec, tb)
    assert torch.equal(ta, tb)
    if prec == S.SPH_MIXED:
        with pytest.raises(S.SphError):
            S.set_tiles(B, rows=64)
    A.close()
    torch.cuda.synchronize()
    gb2, sb = B.new_grid(), B.new_spec()
    S.fftp3d_complex_to_real(B, spec.clone(), gb2)
    S.fftp3d_real_to_complex(B, gb2, sb)
    assert torch.equal(gb2, ga)
    S.plan_status(B)
    B.close()
