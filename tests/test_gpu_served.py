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
