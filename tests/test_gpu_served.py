"""The serving loop: requests of different sizes and kinds arrive over time and
are batched as they come; every result must be the same in the mix as alone
(the plain one-call path, bit for bit) and match the FP64 oracle."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_csr_close

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _host(t):
    return t.cpu().numpy()


@pytest.mark.parametrize("pool", [120e9, 3e6])
def test_served_results_equal_alone_and_oracle(orc, pool):
    from rtt_spgemm import serve

    reqs = serve.poisson_requests(40, rate=2000.0, n_lo=200, n_hi=6000, reuse=0.3, seed=3)
    alone = serve.poisson_requests(40, rate=2000.0, n_lo=200, n_hi=6000, reuse=0.3, seed=3)
    stats = serve.Server(pool_bytes=pool, workers=2).run(reqs)
    serve.serve_plain(alone)
    assert stats["requests"] == 40 and stats["p99_ms"] >= stats["p50_ms"] > 0
    for i, (r, p) in enumerate(zip(reqs, alone)):
        rp, ci, va = (_host(t) for t in r.result)
        prp, pci, pva = (_host(t) for t in p.result)
        assert np.array_equal(rp, prp) and np.array_equal(ci, pci), f"request {i}"
        assert np.array_equal(va.view(np.int64), pva.view(np.int64)), f"request {i}"
        if i % 7 == 0:
            B = r.a if r.op == "A2" else r.a.transpose()
            erp, ecol, evals, eabs = orc.spgemm_csr(r.a, B)
            assert_csr_close(rp, ci, va, erp, ecol, evals, eabs, f"request {i} ({r.op}): ")


def test_served_batches_bounded_by_int32_entries(monkeypatch):
    """A batch's C keeps int32 offsets: with the cap lowered to a few
    thousand products per batch the loop cuts many small batches, and every
    result is still the plain path's, bit for bit."""
    from rtt_spgemm import serve

    monkeypatch.setattr(serve, "INT32_MAX", 5000)
    reqs = serve.poisson_requests(12, rate=2000.0, n_lo=200, n_hi=2000, reuse=0.0, seed=5)
    alone = serve.poisson_requests(12, rate=2000.0, n_lo=200, n_hi=2000, reuse=0.0, seed=5)
    serve.Server(workers=2).run(reqs)
    serve.serve_plain(alone)
    for r, p in zip(reqs, alone):
        assert r.error is None and r.result is not None
        for x, y in zip(r.result, p.result):
            assert np.array_equal(_host(x).view(np.uint8), _host(y).view(np.uint8))


def test_served_failing_request_does_not_stop_the_loop():
    """A request the library rejects (a column index past n) is finished with
    its error; the requests batched with it get their results."""
    from rtt_spgemm import serve
    from rtt_spgemm.generators import CSR

    reqs = serve.poisson_requests(8, rate=1e6, n_lo=300, n_hi=1000, reuse=0.0, seed=6)
    bad = CSR(4, 4, np.array([0, 1, 2, 3, 4], np.int32), np.array([0, 1, 9, 3], np.int32),
              np.ones(4))
    reqs.insert(3, serve.Request(bad, "A2", None, reqs[3].arrival))
    stats = serve.Server(workers=1).run(reqs)
    assert stats["failed"] == 1
    assert reqs[3].error is not None and reqs[3].result is None
    assert all(r.result is not None for i, r in enumerate(reqs) if i != 3)


@pytest.mark.parametrize("max_structures", [16, 1])
def test_served_resident_structures(max_structures):
    """Keys used again keep their tile structure resident (from the third
    use on); later requests run
    the numeric step only (the same A object) or a values-only update (a new
    CSR with the same structure and other values).  Every result equals the
    plain path's, bit for bit; with room for one structure the keys evict
    each other and are rebuilt."""
    from rtt_spgemm import generators as G
    from rtt_spgemm import serve

    bases = [(G.stencil_27(12, 4), "A2"), (G.rmat(10, 8, seed=2), "AAT"),
             (G.banded_scatter(3000, 12, seed=6), "A2")]
    rng = np.random.default_rng(1)

    def stream():
        reqs, t = [], 0.0
        for i in range(18):
            j = i % 3
            a, op = bases[j]
            if i >= 9 and i % 2 == 0:  # same structure, other values
                a = G.CSR(a.m, a.n, a.rowptr, a.col, a.val * (1.0 + 0.5 * (i + 1)))
            t += 0.002
            reqs.append(serve.Request(a, op, ("key", j), t))
        return reqs

    reqs, alone = stream(), stream()
    server = serve.Server(workers=2, max_structures=max_structures)
    server.run(reqs[:6])  # two requests per key: batched, operands now resident
    server.run(reqs[6:])  # resident structures from each key's third use on
    assert 1 <= len(server.structures) <= max_structures
    serve.serve_plain(alone)
    for i, (r, p) in enumerate(zip(reqs, alone)):
        assert r.error is None and p.error is None, (i, r.error, p.error)
        for x, y in zip(r.result, p.result):
            assert np.array_equal(_host(x).view(np.uint8), _host(y).view(np.uint8)), f"request {i}"
    server.close()
