"""CUDA graphs of the numeric phase (rtt_config.cuda_graphs, on by default).
The second numeric call in a row with the same shapes, pointers, configuration
and workspace captures its launches and launches the graph; later calls
replay it.  Every call gives bitwise what the eager path gives: repeated
numeric steps, values-only updates with new values written in place between
replays (A*A, A*A^T with the transpose inside the graph, A*B), tile rows split
into window tasks (the side-stream workers inside the graph), and the batched
form.  A changed key (new output buffers, new configuration) runs eagerly."""
from __future__ import annotations

import numpy as np
import pytest

import rtt_spgemm as R
from rtt_spgemm import generators as G
from conftest import assert_csr_close

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
DEV = torch.device("cuda:0")
INVALID_CSR = 2  # RTT_ERR_INVALID_CSR

CASES = {
    "stencil": (lambda: G.stencil_27(10, 1), {}),
    "banded": (lambda: G.banded_scatter(3000, 40, seed=9), {}),
    "unsorted": (lambda: G.random_csr(300, 300, 0.02, seed=3, sort=False), {}),
    # multi-window tile rows cut into one task per window: workers on the side stream
    "rmat_14_split": (lambda: G.rmat(14, 16, seed=2), {"split_target": 1}),
}


def _dev(A):
    return (A.m, A.n, torch.from_numpy(A.rowptr).to(DEV), torch.from_numpy(A.col).to(DEV),
            torch.from_numpy(A.val).to(DEV))


def _outputs(m, nnz):
    return (torch.empty(m + 1, dtype=torch.int32, device=DEV),
            torch.empty(max(nnz, 1), dtype=torch.int32, device=DEV),
            torch.empty(max(nnz, 1), dtype=torch.float64, device=DEV))


def _host(out, nnz):
    rp, ci, va = out
    return rp.cpu().numpy(), ci[:nnz].cpu().numpy(), va[:nnz].cpu().numpy()


def _eager(A, B=None, op=R.RTT_OP_AB, cfg=None):
    ctx = R.Context(0, dict(cfg or {}, cuda_graphs=0))
    nnz, _ = ctx.symbolic(_dev(A), _dev(B) if B is not None else None, op)
    out = _outputs(A.m, nnz)
    ctx.numeric(*out)
    got = _host(out, nnz)
    assert ctx.stats()["graph_launched"] == 0
    ctx.close()
    return got


def _same(got, want, bitwise_values=True, tag=""):
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), tag
    if bitwise_values:
        assert np.array_equal(got[2].view(np.int64), want[2].view(np.int64)), tag
    else:
        assert np.allclose(got[2], want[2], rtol=1e-12, atol=1e-14), tag


def test_default_config_has_graphs_on():
    ctx = R.Context(0)
    assert ctx.config["cuda_graphs"] == 1
    ctx.close()


@pytest.mark.parametrize("case", list(CASES))
def test_numeric_replay_bitwise(case, orc):
    make, cfg = CASES[case]
    A = make()
    want = _eager(A, cfg=cfg)
    ctx = R.Context(0, cfg)
    a = _dev(A)  # numeric reads B = A's CSR: it stays alive while the context uses it
    nnz, _ = ctx.symbolic(a)
    out = _outputs(A.m, nnz)
    flags = []
    for it in range(4):
        out[1].fill_(-1)
        out[2].fill_(np.nan)
        ctx.numeric(*out)
        st = ctx.stats()
        flags.append(st["graph_launched"])
        if "split" in case:
            assert st["split_windows"] > 0
        assert st["nnz_cub"] > 0
        _same(_host(out, nnz), want, case != "unsorted", f"{case} call {it}")
    assert flags == [0, 1, 1, 1], flags
    erp, ecol, evals, eabs = orc.spgemm_csr(A, A)
    assert_csr_close(*_host(out, nnz), erp, ecol, evals, eabs, f"{case} replay: ")
    ctx.close()


@pytest.mark.parametrize("op", ["A2", "AAT"])
@pytest.mark.parametrize("case", ["stencil", "banded", "rmat_14_split"])
def test_values_update_replay(case, op):
    """New values written into the same device tensor between replays: the
    graph reads them, as a fresh eager product of those values does."""
    make, cfg = CASES[case]
    A = make()
    o = R.RTT_OP_AAT if op == "AAT" else R.RTT_OP_AB
    rng = np.random.default_rng(5)
    ctx = R.Context(0, cfg)
    a = _dev(A)
    nnz, _ = ctx.symbolic(a, None, o)
    out = _outputs(A.m, nnz)
    ctx.numeric(*out)
    vt = torch.empty(A.nnz, dtype=torch.float64, device=DEV)
    flags = []
    for it in range(4):
        vals = rng.uniform(-1, 1, A.nnz)
        vt.copy_(torch.from_numpy(vals))
        out[2].fill_(np.nan)
        ctx.numeric_values(vt, None, *out)
        flags.append(ctx.stats()["graph_launched"])
        A2 = G.CSR(A.m, A.n, A.rowptr, A.col, vals)
        want = _eager(A2, None, o, cfg)
        _same(_host(out, nnz), want, True, f"{case} {op} update {it}")
    assert flags == [0, 1, 1, 1], flags
    ctx.close()


def test_values_update_general_ab_replay():
    A = G.banded_scatter(2000, 24, seed=4)
    B = G.random_csr(2000, 1500, 0.01, seed=6)
    rng = np.random.default_rng(8)
    ctx = R.Context(0)
    a, b = _dev(A), _dev(B)
    nnz, _ = ctx.symbolic(a, b)
    out = _outputs(A.m, nnz)
    ctx.numeric(*out)
    va_t = torch.empty(A.nnz, dtype=torch.float64, device=DEV)
    vb_t = torch.empty(B.nnz, dtype=torch.float64, device=DEV)
    flags = []
    for it in range(3):
        va, vb = rng.uniform(-1, 1, A.nnz), rng.uniform(-1, 1, B.nnz)
        va_t.copy_(torch.from_numpy(va))
        vb_t.copy_(torch.from_numpy(vb))
        ctx.numeric_values(va_t, vb_t, *out)
        flags.append(ctx.stats()["graph_launched"])
        want = _eager(G.CSR(A.m, A.n, A.rowptr, A.col, va), G.CSR(B.m, B.n, B.rowptr, B.col, vb))
        _same(_host(out, nnz), want, True, f"A*B update {it}")
    assert flags == [0, 1, 1], flags
    ctx.close()


def test_changed_key_runs_eagerly():
    A = G.banded_scatter(3000, 40, seed=9)
    want = _eager(A)
    ctx = R.Context(0)
    a = _dev(A)
    nnz, _ = ctx.symbolic(a)
    out = _outputs(A.m, nnz)
    for _ in range(3):
        ctx.numeric(*out)
    assert ctx.stats()["graph_launched"] == 1
    # other output buffers: eager, then captured again
    out2 = _outputs(A.m, nnz)
    flags = []
    for _ in range(3):
        ctx.numeric(*out2)
        flags.append(ctx.stats()["graph_launched"])
        _same(_host(out2, nnz), want)
    assert flags == [0, 1, 1], flags
    # a new configuration: eager again
    ctx.configure({"split_target": -1})
    ctx.numeric(*out2)
    assert ctx.stats()["graph_launched"] == 0
    _same(_host(out2, nnz), want)
    # a new symbolic of the same matrix with the same buffers keeps the key
    nnz2, _ = ctx.symbolic(a)
    assert nnz2 == nnz
    ctx.numeric(*out2)
    ctx.numeric(*out2)
    _same(_host(out2, nnz), want)
    ctx.close()


@pytest.mark.parametrize("cfg", [{"cuda_graphs": 0}, {"stage_timing": 1},
                                 {"fused_csr_output": 0}])
def test_graphs_off(cfg):
    A = G.stencil_27(10, 1)
    want = _eager(A)
    ctx = R.Context(0, cfg)
    a = _dev(A)
    nnz, _ = ctx.symbolic(a)
    out = _outputs(A.m, nnz)
    for _ in range(3):
        ctx.numeric(*out)
        assert ctx.stats()["graph_launched"] == 0
        _same(_host(out, nnz), want)
    ctx.close()


def test_batched_replay(orc):
    """The batched form run three times on the same instances and output
    buffers: the numeric phase and the per-instance split are one graph."""
    rng = np.random.default_rng(3)
    mats = [G.banded_scatter(int(n), int(w), seed=int(s))
            for n, w, s in zip(rng.integers(200, 3000, 7), rng.integers(4, 32, 7), range(7))]
    As = [_dev(M) for M in mats]
    ctx = R.Context(0)
    flags, outs = [], None
    for it in range(3):
        nnz, total = ctx.batched_symbolic(As)
        if outs is None:
            outs = _outputs(sum(M.m + 1 for M in mats) - 1, total)
        outs[2].fill_(np.nan)
        ctx.batched_numeric(*outs)
        flags.append(ctx.stats()["graph_launched"])
        rp, ci, va = (t.cpu().numpy() for t in outs)
        r0 = e0 = 0
        for M, z in zip(mats, nnz):
            got = rp[r0:r0 + M.m + 1] - rp[r0], ci[e0:e0 + z], va[e0:e0 + z]
            want = _eager(M)
            _same(got, want, True, f"batched call {it}")
            r0 += M.m + 1
            e0 += z
    assert flags == [0, 1, 1], flags
    ctx.close()


def test_values_update_checks_the_structure():
    """The structure arrays given to symbolic are checked on the device before
    a values-only update indexes by them: a column out of range, or tile
    columns that now decrease inside a row, is RTT_ERR_INVALID_CSR (nothing
    else runs), and the context works again once the arrays are restored."""
    A = G.banded_scatter(2000, 24, seed=4)
    want = _eager(A)
    ctx = R.Context(0)
    a = _dev(A)
    nnz, _ = ctx.symbolic(a)
    out = _outputs(A.m, nnz)
    ctx.numeric(*out)
    vt = a[4].clone()
    col = a[3]
    keep = col.clone()
    col[5] = A.n + 7  # out of range
    with pytest.raises(R.RttError) as e:
        ctx.numeric_values(vt, None, *out)
    assert e.value.status == INVALID_CSR
    col.copy_(keep)
    r = 0
    lo = int(A.rowptr[r])
    # first and last entry of a row swapped: valid CSR, decreasing tile columns
    row = keep[lo:int(A.rowptr[r + 1])].cpu().numpy()
    if row[0] >> 4 != row[-1] >> 4:
        col[lo] = int(row[-1])
        col[int(A.rowptr[r + 1]) - 1] = int(row[0])
        with pytest.raises(R.RttError) as e:
            ctx.numeric_values(vt, None, *out)
        assert e.value.status == INVALID_CSR
        col.copy_(keep)
    for _ in range(3):
        ctx.numeric_values(vt, None, *out)
        _same(_host(out, nnz), want)
    ctx.close()


@pytest.mark.parametrize("A", [G.CSR(5, 5, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0)),
                               G.CSR(1, 1, np.array([0, 1], np.int32), np.array([0], np.int32),
                                     np.array([3.0]))], ids=["empty_5x5", "one_1x1"])
def test_graphs_on_empty_and_tiny(A):
    """Capture and replay of products with no entry and with one."""
    want = _eager(A)
    ctx = R.Context(0)
    a = _dev(A)
    nnz, _ = ctx.symbolic(a)
    out = _outputs(A.m, nnz)
    for _ in range(3):
        ctx.numeric(*out)
        _same(_host(out, nnz), want)
    vt = torch.from_numpy(np.resize(A.val, max(A.nnz, 1))).to(DEV)  # same values
    for _ in range(3):
        ctx.numeric_values(vt, None, *out)
        _same(_host(out, nnz), want)
    assert ctx.stats()["graph_launched"] == 1
    ctx.close()
