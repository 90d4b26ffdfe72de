"""The autotuner on the GPU: it times the candidate configurations of a shape
class once, stores the fastest, configures the context with it, and the
products it configures stay within the FP64 bar of the oracle."""
from __future__ import annotations

import json

import numpy as np
import pytest

import rtt_spgemm as R
from rtt_spgemm import autotune as T
from rtt_spgemm import generators as G
from conftest import assert_csr_close

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
DEV = torch.device("cuda:0")


def _dev(A):
    return (A.m, A.n, torch.from_numpy(A.rowptr).to(DEV), torch.from_numpy(A.col).to(DEV),
            torch.from_numpy(A.val).to(DEV))


def test_tuned_plain_product(tmp_path, orc):
    A = G.banded_scatter(3000, 24, seed=3)
    ctx = R.Context(0)
    tuner = T.Tuner(tmp_path / "tune.json", repeats=1)
    cfg = tuner.configure(ctx, _dev(A))
    assert ctx.config["split_target"] == cfg["split_target"]
    stored = json.loads((tmp_path / "tune.json").read_text())
    (entries,) = stored["devices"].values()
    (key,) = entries
    assert key.startswith("AB|") and len(entries[key]["candidates"]) == len(T.CANDIDATES)
    when = entries[key]["tuned_at"]
    # the class is known now: no second tuning
    tuner.configure(ctx, _dev(A))
    again = json.loads((tmp_path / "tune.json").read_text())
    assert list(again["devices"].values())[0][key]["tuned_at"] == when
    a = _dev(A)
    nnz, _ = ctx.symbolic(a)
    rp = torch.empty(A.m + 1, dtype=torch.int32, device=DEV)
    ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=DEV)
    va = torch.empty(max(nnz, 1), dtype=torch.float64, device=DEV)
    ctx.numeric(rp, ci, va)
    erp, ecol, evals, eabs = orc.spgemm_csr(A, A)
    assert_csr_close(rp.cpu().numpy(), ci[:nnz].cpu().numpy(), va[:nnz].cpu().numpy(),
                     erp, ecol, evals, eabs, "tuned: ")
    ctx.close()


def test_tuned_batch(tmp_path, orc):
    As = G.batched_instances(6, 500, 5000, seed=4)
    views = [_dev(A) for A in As]
    ctx = R.Context(0)
    tuner = T.Tuner(tmp_path / "tune.json", repeats=1)
    outs = R.spgemm_batched(ctx, views, tuner=tuner)
    stored = json.loads((tmp_path / "tune.json").read_text())
    (entries,) = stored["devices"].values()
    assert any(k.startswith("batch:") for k in entries)
    for A, (rp, ci, va) in zip(As, outs):
        erp, ecol, evals, eabs = orc.spgemm_csr(A, A)
        assert_csr_close(rp.cpu().numpy(), ci.cpu().numpy(), va.cpu().numpy(),
                         erp, ecol, evals, eabs, "tuned batch: ")
    ctx.close()
