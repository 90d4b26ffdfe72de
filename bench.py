"""Benchmark of the tiled FP64 SpGEMM path on B200.

One step = one full device-resident product C = A*A of the workload:
csr2tile(A) (B = A shares A's tiles) -> tile CSC index -> symbolic steps 1-2
-> allocation of C -> numeric (tile2csr fused) -> device CSR(C).  Inputs are
resident in HBM when the timed region starts; A's CSR (284 MB for the 3-D
workload) is larger than L2, so no explicit flush is needed.

Metric: SpGEMM GFLOP/s = 2 * nnzCub / t (nnzCub = sum over (i,k) in A of
nnz(B row k)), the reference's definition.  Algorithmic bytes follow the
reference's model 4(m_A+1)+12 nnz_A + 4(m_B+1)+12 nnz_B + 4(m_C+1)+12 nnz_C.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
  python bench.py --impl reference ...   # the reference's CPU code, host cores

Multi-GPU (torchrun): the workload is replicated per rank (independent
products, no collective on the data path); value = all ranks' flops / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "rtt-spgemm_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

WORKLOADS = {
    "stencil27_96": "3-D 27-point stencil, 96^3 grid (n=884,736), C = A^2, natural ordering",
    "stencil27_96_brick": "3-D 27-point stencil, 96^3 grid, 2x2x4 brick ordering, C = A^2",
    "laplacian2d_256": "2-D 5-point Laplacian, 256^2 grid (n=65,536), C = A^2",
    "stencil27_80": "3-D 27-point stencil, 80^3 grid (n=512,000), C = A^2 (profiling size)",
    "stencil27_48_brick": "3-D 27-point stencil, 48^3 grid, 2x2x4 brick ordering, C = A^2 "
                          "(profiling size of the DMMA path)",
    "rmat16_aat": "R-MAT 2^16, 16 edges/row, (a,b,c,d)=(.57,.19,.19,.05), C = A*A^T (the R-MAT "
                  "config's generator at the largest scale whose C fits int32 offsets)",
    "rmat20_aat": "R-MAT 2^20, 16 edges/row, (a,b,c,d)=(.57,.19,.19,.05), C = A*A^T: nnz(C) past "
                  "INT32_MAX, through the 64-bit chunked path (int64 row pointer)",
    "served": "Poisson request stream (2,000 req/s) of mixed A^2 / A*A^T products, n log-uniform "
              "in [4,096, n_max], 2-D/3-D stencils, R-MAT, banded+scatter, 30% reuse a resident A; "
              "120 GB pool; served (batched as they arrive) vs plain one-call FIFO",
    "mtx": "a Matrix Market file (--mtx; e.g. a SuiteSparse matrix), C = A^2, read as the "
           "reference's mmio_allinone reads it",
    "mtx_aat": "a Matrix Market file (--mtx), C = A*A^T",
    "batched": "independent A_i^2: n_i log-uniform in [2,000, 200,000], banded (half-bandwidth "
               "8..64, band kept w.p. 0.5) + 0..4 random entries per row; batched form vs one "
               "call per product",
}


MTX = {"path": None, "value_mode": 0}


def make_workload(name: str, seed: int):
    from rtt_spgemm import generators as G
    if name in ("mtx", "mtx_aat"):
        import rtt_spgemm as R
        return R.mmio_read(MTX["path"], MTX["value_mode"])
    if name == "stencil27_96":
        return G.stencil_27(96, seed)
    if name == "stencil27_96_brick":
        return G.stencil_27(96, seed).permute_symmetric(G.brick_permutation(96))
    if name == "laplacian2d_256":
        return G.laplacian_2d(256)
    if name == "stencil27_80":
        return G.stencil_27(80, seed)
    if name == "stencil27_48_brick":
        return G.stencil_27(48, seed).permute_symmetric(G.brick_permutation(48))
    if name == "rmat16_aat":
        return G.rmat(16, 16, seed=seed + 1)
    if name == "rmat20_aat":
        return G.rmat(20, 16, seed=seed + 1)
    raise SystemExit(f"unknown workload {name}")


def workload_aat(name: str) -> bool:
    return name.endswith("_aat")


def nnz_cub(A, aat: bool = False) -> int:
    if aat:  # B = A^T: nnz(B row k) = entries of A's column k
        cc = np.bincount(A.col, minlength=A.n).astype(np.int64)
        return int(cc[A.col].sum())
    return int(np.diff(A.rowptr).astype(np.int64)[A.col].sum())


def alg_bytes(m, nnz_a, nnz_b, nnz_c) -> int:
    return 3 * 4 * (m + 1) + 12 * (nnz_a + nnz_b + nnz_c)


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def load_traffic(workload: str):
    p = ROOT / "profiles" / "numeric_traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        e = d.get(workload)
        if e:
            return e.get("dram_bytes_per_launch")
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.path = Path(tempfile.gettempdir()) / f"rtt_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                   "-lms", "100"]
            if self.uuid:
                cmd += ["-i", self.uuid]
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(cmd, stdout=self.fh, stderr=subprocess.DEVNULL)
            # wait until the sampler has written its first samples: its start-up
            # (driver queries) then lies before the warm-up steps, not in them
            t0 = time.perf_counter()
            while time.perf_counter() - t0 < 5.0:
                time.sleep(0.05)
                if self.path.stat().st_size > 0 and self.path.read_text().count("\n") >= 2:
                    break
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline_port(A, flops: float, B=None) -> dict:
    import oracle
    orc = oracle.Oracle()
    t0 = time.perf_counter()
    orc.spgemm_csr(A, A if B is None else B, with_abs=False)
    dt = time.perf_counter() - t0
    return {"value": flops / dt / 1e9, "unit": "GFLOP/s", "cores": orc.threads(), "kind": "port",
            "sample": "full product, FP64 OpenMP row SPA restating spgemm_serialref "
                      "(src/external/cusparse/spgemm_serialref_spa.h)", "seconds": dt}


VALUE_RTOL = 1e-12  # |dC_ij| <= VALUE_RTOL * (|A||B|)_ij


def oracle_product(A, B):
    """The checker: the oracle's FP64 row SPA with (|A||B|)_ij per entry."""
    import oracle
    return oracle.Oracle().spgemm_csr(A, B, with_abs=True)


def parity(rowptr, col, val, want, what: str) -> dict:
    """Structure bit-exact against the oracle, values within
    VALUE_RTOL * (|A||B|)_ij; the observed maximum errors are reported."""
    erp, ecol, evals, eabs = want
    rowptr = np.asarray(rowptr).astype(np.int64)
    col = np.asarray(col)
    same = (rowptr.shape == erp.shape and np.array_equal(rowptr, erp) and
            col.shape == ecol.shape and np.array_equal(col, ecol))
    out = {"checked": what, "entries": int(ecol.shape[0]), "structure_bit_exact": bool(same),
           "bound": VALUE_RTOL}
    if not same:
        out.update(max_abs_err=None, max_rel_err=None, **{"pass": False})
        return out
    err = np.abs(np.asarray(val, dtype=np.float64) - evals)
    pos = eabs > 0
    rel = float((err[pos] / eabs[pos]).max()) if pos.any() else 0.0
    if (err[~pos] > 0).any():  # an entry whose products are all zero must be exactly zero
        rel = float("inf")
    out.update(max_abs_err=float(err.max()) if err.size else 0.0, max_rel_err=rel,
               **{"pass": bool(rel <= VALUE_RTOL)})
    return out


def run_reference(args) -> None:
    """The reference's own CPU SpGEMM (csr2tile_row_major + spgemm_cpu, compiled
    from its sources), on a bounded sample of the workload's tile rows."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    A = make_workload(args.workload, args.seed)
    aat = workload_aat(args.workload)
    B = A.transpose() if aat else A
    from rtt_spgemm import generators as G
    if oracle.reference_available():
        ref = oracle.Reference()
        b_tiles = ref.csr2tile_col_major(B)  # B prepared once, outside the timed steps
        rows = min(A.m, args.ref_tile_rows * 16)
        rp = A.rowptr[: rows + 1].copy()
        As = G.CSR(rows, A.n, rp, A.col[: rp[-1]].copy(), A.val[: rp[-1]].copy())
        flops = 2.0 * int(np.diff(B.rowptr).astype(np.int64)[As.col].sum())
        times = []
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            a_tiles = ref.csr2tile_row_major(As)
            ref.spgemm_cpu(a_tiles, b_tiles)
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                times.append(dt)
        t = statistics.median(times)
        kind, cores = "reference", 1
        sample = (f"first {rows} rows of A ({rows // 16} tile rows) times all of B per step: "
                  f"csr2tile_row_major(A rows) + spgemm_cpu (src/spgemm-cpu.h:369, serial, with "
                  f"the in-tile column fix at the call site); B's csr2tile_col_major done once "
                  f"before timing")
    else:
        flops = 2.0 * nnz_cub(A, aat)
        cb = cpu_baseline_port(A, flops, B if aat else None)
        t, kind, cores, sample = cb["seconds"], "port", cb["cores"], cb["sample"]
    value = flops / t / 1e9
    line = {"impl": "reference", "metric": "SpGEMM GFLOP/s", "value": value, "unit": "GFLOP/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload]},
            "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_batched(args) -> None:
    """Batched form against the plain one-call-per-product path on the same
    instances: SpGEMMs/s of each, instances processed in memory-bounded waves."""
    import torch
    import rtt_spgemm as R
    from rtt_spgemm import generators as G

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    As = G.batched_instances(args.batch_count, 2000, 200000, seed=args.seed)
    flops = sum(2.0 * nnz_cub(A) for A in As)
    views = [(A.m, A.n, torch.from_numpy(A.rowptr).to(dev), torch.from_numpy(A.col).to(dev),
              torch.from_numpy(A.val).to(dev)) for A in As]
    waves, cur, rows = [], [], 0
    for i, A in enumerate(As):
        if cur and rows + A.m > args.wave_rows:
            waves.append(cur)
            cur, rows = [], 0
        cur.append(i)
        rows += A.m
    if cur:
        waves.append(cur)
    ctx = R.Context(0, {"stage_timing": 0, "dmma_pair_cutoff": args.dmma_cutoff,
                        "b_staging": 1 if args.staging else 0,
                        "persistent_rows": 1 if args.persistent_rows else 0,
                "sym_window_slots": args.sym_window_slots, "leaf_dmma": 1 if args.leaf_dmma else 0, "global_rows": args.global_rows})
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)

    tuner = None
    if args.tune:
        from rtt_spgemm import autotune
        tuner = autotune.Tuner(os.environ.get("RTT_TUNE_CACHE"))  # None: the per-user default

    def batched():
        for w in waves:
            R.spgemm_batched(ctx, [views[i] for i in w], tuner=tuner)

    def plain():
        for v in views:
            nnz, _ = ctx.symbolic(v)
            rp = torch.empty(v[0] + 1, dtype=torch.int32, device=dev)
            ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
            va = torch.empty(max(nnz, 1), dtype=torch.float64, device=dev)
            ctx.numeric(rp, ci, va)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / args.steps

    base_cfg = {"stage_timing": 0, "dmma_pair_cutoff": args.dmma_cutoff,
                "b_staging": 1 if args.staging else 0,
                "persistent_rows": 1 if args.persistent_rows else 0,
                "sym_window_slots": args.sym_window_slots, "leaf_dmma": 1 if args.leaf_dmma else 0, "global_rows": args.global_rows}
    ms_b = timed(batched)
    ctx.configure(base_cfg)  # the plain arm keeps the given configuration
    ms_p = timed(plain)

    # values-only update of the same batch (new values of every instance,
    # structures kept): one context per wave keeps its batch's structure
    upd = None
    if not args.no_update:
        # wave by wave (the waves' C together do not fit the device): each
        # wave's structure on a context of its own, its values-only updates
        # timed, then its memory released; the per-wave times add up
        ms_u, graphs = 0.0, 0
        for w in waves:
            c = R.Context(0, base_cfg)
            c.set_stream(stream.cuda_stream)
            nnz, total = c.batched_symbolic([views[i] for i in w])
            out = (torch.empty(sum(views[i][0] + 1 for i in w), dtype=torch.int32, device=dev),
                   torch.empty(max(total, 1), dtype=torch.int32, device=dev),
                   torch.empty(max(total, 1), dtype=torch.float64, device=dev))
            c.batched_numeric(*out)
            newvals = [views[i][4] * 0.5 for i in w]
            ms_u += timed(lambda: c.batched_numeric_values(newvals, None, *out))
            graphs += c.stats()["graph_launched"]
            c.close()
            del out, newvals
            torch.cuda.empty_cache()
        upd = {"value": len(As) / (ms_u * 1e-3), "unit": "SpGEMMs/s", "ms_per_step": ms_u,
               "graph_launched_waves": graphs,
               "what": "same instances' structures, new values of every A_i: gathered on the "
                       "device, numeric step only (rtt_spgemm_batched_numeric_values), wave by "
                       "wave"}
    # the checker: every instance of the first wave, batched, against the oracle
    checks = None
    if not args.no_parity:
        outs = R.spgemm_batched(ctx, [views[i] for i in waves[0]])
        torch.cuda.synchronize(dev)
        worst = {"structure_bit_exact": True, "max_abs_err": 0.0, "max_rel_err": 0.0}
        for i, (rp_, ci_, va_) in zip(waves[0], outs):
            c = parity(rp_.cpu().numpy(), ci_.cpu().numpy(), va_.cpu().numpy(),
                       oracle_product(As[i], As[i]), "")
            worst["structure_bit_exact"] &= c["structure_bit_exact"]
            if c["structure_bit_exact"]:
                worst["max_abs_err"] = max(worst["max_abs_err"], c["max_abs_err"])
                worst["max_rel_err"] = max(worst["max_rel_err"], c["max_rel_err"])
        del outs
        checks = {"checked": f"the {len(waves[0])} instances of the first wave, batched, vs "
                             f"the oracle's FP64 row SPA", "bound": VALUE_RTOL, **worst,
                  "pass": bool(worst["structure_bit_exact"] and worst["max_rel_err"] <= VALUE_RTOL)}
    n = len(As)
    line = {
        "metric": "SpGEMMs/s (batched)", "value": n / (ms_b * 1e-3), "unit": "SpGEMMs/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_b,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator)",
        "config": {"workload": "batched", "description": WORKLOADS["batched"], "instances": n,
                   "rows_total": int(sum(A.m for A in As)), "nnz_a_total": int(sum(A.nnz for A in As)),
                   "flops": flops, "waves": len(waves), "wave_rows": args.wave_rows,
                   "dmma_pair_cutoff": args.dmma_cutoff},
        "gflops_batched": flops / (ms_b * 1e-3) / 1e9,
        "plain": {"spgemms_per_s": n / (ms_p * 1e-3), "ms_per_step": ms_p,
                  "gflops": flops / (ms_p * 1e-3) / 1e9},
        "batched_over_plain": ms_p / ms_b,
        "parity": checks,
        "values_only_update": upd,
        "tuned": (list(tuner.table.get("devices", {}).values()) or [{}])[0] if tuner else None,
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def run_served(args) -> None:
    """Serving loop against the plain path under the same Poisson arrivals."""
    import gc

    import torch
    import rtt_spgemm as R
    from rtt_spgemm import serve

    torch.cuda.set_device(0)
    mk = lambda: serve.poisson_requests(args.serve_count, 2000.0, 4096, args.serve_nmax,
                                        reuse=0.3, seed=args.seed)

    def settle():
        # results are dropped as they complete in both arms; hand the cached
        # blocks back so that neither arm inherits the other's memory state
        gc.collect()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()

    # steady state: each arm first serves the same stream once, untimed, with
    # the contexts it keeps, so that their buffers have grown to the stream's
    # sizes (a server runs on); resident operands are dropped in between, so
    # only the stream's own 30 % reuse hits them
    t0 = time.perf_counter()
    stream0 = mk()
    gen_s = time.perf_counter() - t0

    def fresh():
        # the same requests (same matrices, arrivals and keys), results cleared
        return [serve.Request(r.a, r.op, r.key, r.arrival) for r in stream0]

    # every run is the stream once: its 30 % of requests that repeat an
    # earlier A reuse that request's operands (and, from a key's third use
    # on, its tile structure); nothing carries over from one run to the next
    server = serve.Server(pool_bytes=120e9, keep_results=False)
    server.run(fresh())
    server.reset_reuse()
    settle()
    served_runs = []
    for _ in range(max(1, args.serve_repeats)):
        served_runs.append(server.run(fresh()))
        server.reset_reuse()
        settle()
    server.close()
    settle()
    pctx = R.Context(0)
    serve.serve_plain(fresh(), keep_results=False, ctx=pctx)
    settle()
    plain_runs = []
    for _ in range(max(1, args.serve_repeats)):
        plain_runs.append(serve.serve_plain(fresh(), keep_results=False, ctx=pctx))
        settle()
    pctx.close()

    def med(runs):
        # the run with the median throughput, plus the spread over the runs
        order = sorted(runs, key=lambda r: r["spgemms_per_s"])
        m = dict(order[len(order) // 2])
        m["runs_spgemms_per_s"] = [r["spgemms_per_s"] for r in runs]
        m["runs_p50_ms"] = [r["p50_ms"] for r in runs]
        m["runs_p99_ms"] = [r["p99_ms"] for r in runs]
        return m

    served, plain = med(served_runs), med(plain_runs)

    # the checker: a sample of the stream's requests served again (in one mix,
    # results kept), each against the oracle
    checks = None
    if not args.no_parity:
        import torch as _t
        cand = [r for r in stream0 if serve.product_cub(r.a, r.op) < 60_000_000]
        rng = np.random.default_rng(args.seed + 5)
        pick = sorted(rng.choice(len(cand), size=min(12, len(cand)), replace=False))
        sample = [serve.Request(cand[i].a, cand[i].op, None, 0.0) for i in pick]
        srv = serve.Server(pool_bytes=120e9, keep_results=True)
        srv.run(sample)
        worst = {"structure_bit_exact": True, "max_abs_err": 0.0, "max_rel_err": 0.0}
        for r in sample:
            if r.error is not None:
                worst["structure_bit_exact"] = False
                continue
            B = r.a.transpose() if r.op == "AAT" else r.a
            rp_, ci_, va_ = (x.cpu().numpy() for x in r.result)
            c = parity(rp_, ci_, va_, oracle_product(r.a, B), "")
            worst["structure_bit_exact"] &= c["structure_bit_exact"]
            if c["structure_bit_exact"]:
                worst["max_abs_err"] = max(worst["max_abs_err"], c["max_abs_err"])
                worst["max_rel_err"] = max(worst["max_rel_err"], c["max_rel_err"])
        srv.close()
        _t.cuda.empty_cache()
        checks = {"checked": f"{len(sample)} requests of the stream (nnzCub < 6e7), served together, "
                             f"vs the oracle's FP64 row SPA", "bound": VALUE_RTOL, **worst,
                  "pass": bool(worst["structure_bit_exact"] and worst["max_rel_err"] <= VALUE_RTOL)}
    ratios = sorted(a["spgemms_per_s"] / max(b["spgemms_per_s"], 1e-9)
                    for a, b in zip(served_runs, plain_runs))
    line = {
        "metric": "SpGEMMs/s (served)", "value": served["spgemms_per_s"], "unit": "SpGEMMs/s",
        "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": served["seconds"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generators, Poisson arrivals)",
        "config": {"workload": "served", "description": WORKLOADS["served"],
                   "requests": args.serve_count, "n_max": args.serve_nmax, "rate_per_s": 2000.0,
                   "arrival_span_s": max(r.arrival for r in stream0),
                   "generator_s": gen_s, "repeats": args.serve_repeats,
                   "warmup": "one untimed run of the same stream per arm"},
        "served": served, "plain": plain,
        "served_over_plain": served["spgemms_per_s"] / max(plain["spgemms_per_s"], 1e-9),
        "served_over_plain_runs": ratios,
        "parity": checks,
    }
    print(json.dumps(line), flush=True)


def cusparse_control(a_view, b_view, steps: int, warmup: int, flops: float, got=None) -> dict:
    """Control: the same product through cuSPARSE's SpGEMM (torch's CSR @ CSR on
    CUDA), timed with CUDA events on the same inputs - a library baseline on
    the same GPU, as the reference's cuSPARSE harness measures beside its own
    kernels.  Its structure is compared with ours."""
    import torch
    try:
        rows, cols, rp, ci, va = a_view
        A = torch.sparse_csr_tensor(rp.long(), ci.long(), va, size=(rows, cols))
        if b_view is None:
            B = A
        else:
            rows_b, cols_b, rpb, cib, vab = b_view
            B = torch.sparse_csr_tensor(rpb.long(), cib.long(), vab, size=(rows_b, cols_b))
        for _ in range(warmup):
            C = A @ B
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            C = A @ B
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out = {"what": "cuSPARSE SpGEMM through torch (CSR @ CSR, float64), device-resident",
               "ms_per_step": ms, "gflops": flops / (ms * 1e-3) / 1e9}
        if got is not None:
            crow = C.crow_indices().cpu().numpy()
            ccol = C.col_indices().cpu().numpy()
            out["same_structure"] = bool(np.array_equal(crow, np.asarray(got[0], np.int64)) and
                                         np.array_equal(ccol, np.asarray(got[1], np.int64)))
        del C
        torch.cuda.empty_cache()
        return out
    except Exception as e:  # the control is optional: report why it did not run
        return {"unavailable": f"{type(e).__name__}: {e}"[:300]}


def run_wide(args) -> None:
    """A product whose C exceeds INT32_MAX entries (R-MAT 2^20 A*A^T) through
    rtt_spgemm_symbolic64 / rtt_spgemm_numeric64, one GPU.  The check samples
    rows: the heaviest rows of A plus random ones, against the oracle's row SPA
    of those rows of A times A^T."""
    import torch
    import rtt_spgemm as R
    from rtt_spgemm import generators as G

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    A = make_workload(args.workload, args.seed)
    gen_s = time.perf_counter() - t0
    cub = nnz_cub(A, True)
    flops = 2.0 * cub
    stream = torch.cuda.current_stream(dev)
    ctx = R.Context(0, {"stage_timing": 0, "sym_window_slots": args.sym_window_slots, "leaf_dmma": 1 if args.leaf_dmma else 0, "global_rows": args.global_rows})
    ctx.set_stream(stream.cuda_stream)
    a_view = (A.m, A.n, torch.from_numpy(A.rowptr).to(dev), torch.from_numpy(A.col).to(dev),
              torch.from_numpy(A.val).to(dev))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    out = None

    def step():
        nonlocal out
        out = None  # C of the previous step goes back to the pool first
        ev[0].record(stream)
        nnz = ctx.symbolic64(a_view, None, R.RTT_OP_AAT)
        ev[1].record(stream)
        rp = torch.empty(A.m + 1, dtype=torch.int64, device=dev)
        ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
        va = torch.empty(max(nnz, 1), dtype=torch.float64, device=dev)
        ctx.numeric64(rp, ci, va)
        ev[2].record(stream)
        out = (rp, ci, va)
        return nnz

    for _ in range(args.warmup):
        nnz_c = step()
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(None)
    sampler.start()
    sym, num = [], []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        nnz_c = step()
        torch.cuda.synchronize(dev)
        sym.append(ev[0].elapsed_time(ev[1]))
        num.append(ev[1].elapsed_time(ev[2]))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    st = ctx.stats()
    peaks = load_peaks()
    abytes = alg_bytes(A.m, A.nnz, A.nnz, nnz_c)

    checks = None
    if not args.no_parity:
        rows_len = np.diff(A.rowptr)
        rng = np.random.default_rng(args.seed + 17)
        heavy = np.argsort(rows_len)[-100:]
        pick = np.unique(np.concatenate([heavy, rng.choice(A.m, size=2900, replace=False)]))
        rp_all = out[0].cpu().numpy()
        lo, hi = rp_all[pick], rp_all[pick + 1]
        idx = np.concatenate([np.arange(a, b, dtype=np.int64) for a, b in zip(lo, hi)])
        it = torch.from_numpy(idx).to(dev)
        got_col = out[1][it].cpu().numpy()
        got_val = out[2][it].cpu().numpy()
        got_rp = np.zeros(pick.size + 1, np.int64)
        np.cumsum(hi - lo, out=got_rp[1:])
        # the sampled rows of A, times A^T
        srp = np.zeros(pick.size + 1, np.int64)
        np.cumsum(rows_len[pick], out=srp[1:])
        scol = np.concatenate([A.col[A.rowptr[i]:A.rowptr[i + 1]] for i in pick])
        sval = np.concatenate([A.val[A.rowptr[i]:A.rowptr[i + 1]] for i in pick])
        As = G.CSR(pick.size, A.n, srp.astype(np.int32), scol, sval)
        checks = parity(got_rp, got_col, got_val, oracle_product(As, A.transpose()),
                        f"{pick.size} rows (the 100 heaviest of A and random ones) vs the oracle's "
                        f"FP64 row SPA")
    line = {
        "metric": "SpGEMM GFLOP/s", "value": flops / (ms * 1e-3) / 1e9, "unit": "GFLOP/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator)",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                   "n": A.m, "nnz_a": A.nnz, "nnz_c": nnz_c, "nnz_cub": cub, "flops": flops,
                   "tiles_a": st["tiles_a"], "tiles_c": st["tiles_c"], "alg_bytes": abytes,
                   "c_gib_on_device": 12 * nnz_c / 2 ** 30, "generator_s": gen_s,
                   "l2": "inputs larger than L2"},
        "roofline": {"bound": "hbm", "kernel": "whole step (chunked symbolic + numeric)",
                     "achieved": abytes / (ms * 1e-3) / 1e9, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": abytes / (ms * 1e-3) / 1e9 / peaks["hbm_gbs"],
                     "traffic": None, "peak_source": peaks["source"]},
        "stages_ms": {"symbolic64_ms (csr2tile, A^T, chunked steps 1-2)": statistics.mean(sym),
                      "numeric64_ms (steps 1-2 again + numeric, per chunk)": statistics.mean(num)},
        "nnz_cub_counted": st["nnz_cub"], "host_syncs_numeric": st["host_syncs"],
        "gpu_launches": st["kernel_launches"],
        "clocks": clocks, "parity": checks,
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def run_ours(args) -> None:
    import torch
    import rtt_spgemm as R
    from rtt_spgemm import shards

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    A = make_workload(args.workload, args.seed)
    aat = workload_aat(args.workload)
    op = R.RTT_OP_AAT if aat else R.RTT_OP_AB
    cub = nnz_cub(A, aat)
    flops = 2.0 * cub
    stream = torch.cuda.current_stream(dev)
    ctx = R.Context(local, {"stage_timing": 1, "dmma_pair_cutoff": args.dmma_cutoff,
                            "fused_csr_output": 0 if args.unfused else 1,
                            "b_staging": 1 if args.staging else 0,
                            "segment_walk": 1 if args.segment_walk else 0,
                            "persistent_rows": 1 if args.persistent_rows else 0,
                "sym_window_slots": args.sym_window_slots, "leaf_dmma": 1 if args.leaf_dmma else 0, "global_rows": args.global_rows})
    ctx.set_stream(stream.cuda_stream)
    rp = torch.from_numpy(A.rowptr).to(dev)
    ci = torch.from_numpy(A.col).to(dev)
    va = torch.from_numpy(A.val).to(dev)
    a_view = (A.m, A.n, rp, ci, va)

    # L2 (126 MB): inputs larger than it are re-read from HBM every step; a
    # smaller input gets a 256 MB buffer written before each step (inside the
    # timed region, about 0.04 ms) so that no step starts with it in L2
    a_bytes = 4 * (A.m + 1) + 12 * A.nnz
    flush = None if a_bytes > 126e6 else torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    l2_note = ("inputs larger than L2 (A CSR %.0f MB > 126 MB), no flush" % (a_bytes / 1e6)
               if flush is None else
               "inputs smaller than L2 (A CSR %.0f MB): 256 MB written before each step, "
               "inside the timed region" % (a_bytes / 1e6))

    def step():
        if flush is not None:
            flush.fill_(1)
        nnz, _ = ctx.symbolic(a_view, None, op)
        crp = torch.empty(A.m + 1, dtype=torch.int32, device=dev)
        cci = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
        cva = torch.empty(max(nnz, 1), dtype=torch.float64, device=dev)
        ctx.numeric(crp, cci, cva)
        return nnz, (crp, cci, cva)

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
        uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    except Exception:
        pass
    # the clock sampler starts before the warm-up steps: its own start-up
    # (a process that queries the driver) stays out of the timed steps
    sampler = ClockSampler(uuid)
    sampler.start()
    nnz_c = 0
    # the warm-up keeps the previous step's C alive exactly as the timed loop
    # does, so that the allocator holds both output buffers before timing
    last = None
    for _ in range(args.warmup):
        nnz_c, last = step()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    stage = {"csr2tile_ms": [], "symbolic_ms": [], "numeric_kernel_ms": []}
    launches = 0
    ev0.record(stream)
    step_ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    for i in range(args.steps):
        step_ev[i].record(stream)
        nnz_c, last = step()
        st = ctx.stats()
        for k in stage:
            stage[k].append(st[k])
        launches += st["kernel_launches"]
    step_ev[args.steps].record(stream)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    step_ms = [step_ev[i].elapsed_time(step_ev[i + 1]) for i in range(args.steps)]
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    # the last timed step's C, kept for the parity check below
    got = tuple(t.cpu().numpy() for t in last)
    got = (got[0], got[1][:nnz_c], got[2][:nnz_c])
    del last
    ms = shards.max_over_ranks(ev0.elapsed_time(ev1) / args.steps)
    value = shards.replica_throughput(world, flops, ms)

    st = ctx.stats()
    peaks = load_peaks()
    abytes = alg_bytes(A.m, A.nnz, A.nnz, nnz_c)
    num_ms = statistics.mean(stage["numeric_kernel_ms"])
    achieved = abytes / (num_ms * 1e-3) / 1e9
    traffic = (None if args.staging or args.unfused or args.leaf_dmma
               else load_traffic(args.workload))

    # repeated product with the same structure and new values (values-only
    # update, rtt_spgemm_numeric_values): no csr2tile counting, no symbolic
    upd = None
    got_upd = None
    if not args.staging and not args.unfused and not args.no_update:
        nnz_u, _ = ctx.symbolic(a_view, None, op)
        urp = torch.empty(A.m + 1, dtype=torch.int32, device=dev)
        uci = torch.empty(max(nnz_u, 1), dtype=torch.int32, device=dev)
        uva = torch.empty(max(nnz_u, 1), dtype=torch.float64, device=dev)
        ctx.numeric(urp, uci, uva)
        new_vals = va * 0.5
        for _ in range(args.warmup):
            ctx.numeric_values(new_vals, None, urp, uci, uva)
        u0 = torch.cuda.Event(enable_timing=True)
        u1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        u0.record(stream)
        for _ in range(args.steps):
            ctx.numeric_values(new_vals, None, urp, uci, uva)
        u1.record(stream)
        torch.cuda.synchronize(dev)
        u_ms = shards.max_over_ranks(u0.elapsed_time(u1) / args.steps)
        upd = {"value": shards.replica_throughput(world, flops, u_ms), "unit": "GFLOP/s",
               "ms_per_step": u_ms,
               "what": "same structure, new values of A: tiles refilled, numeric step only"}
        got_upd = (urp.cpu().numpy(), uci[:nnz_u].cpu().numpy(), uva[:nnz_u].cpu().numpy())
        del urp, uci, uva

    # end to end through the host-buffer C-ABI call (rtt_spgemm_csr_host):
    # H2D of A from pinned memory, the product, D2H of C into malloc'd arrays
    e2e = None
    got_e2e = None
    if not args.no_e2e:
        pin_rp = torch.from_numpy(A.rowptr).pin_memory()
        pin_ci = torch.from_numpy(A.col).pin_memory()
        pin_va = torch.from_numpy(A.val).pin_memory()
        Ah = R.CSR(A.m, A.n, pin_rp.numpy(), pin_ci.numpy(), pin_va.numpy())
        ctx.spgemm_csr_host(Ah, None, op)  # warm
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        n_e2e = max(1, min(3, args.steps))
        e0.record(stream)
        for _ in range(n_e2e):
            Ch = ctx.spgemm_csr_host(Ah, None, op)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        e2e_ms = shards.max_over_ranks(e0.elapsed_time(e1) / n_e2e)
        e2e = {"value": shards.replica_throughput(world, flops, e2e_ms), "unit": "GFLOP/s",
               "h2d_bytes_per_step": 4 * (A.m + 1) + 12 * A.nnz,
               "d2h_bytes_per_step": 4 * (A.m + 1) + 12 * int(Ch.nnz), "ms_per_step": e2e_ms}
        got_e2e = (Ch.rowptr, Ch.col, Ch.val)
        # the same through rtt_spgemm_csr_host_into: C into page-locked host
        # arrays the caller keeps from one product to the next
        nz = int(Ch.nnz)
        outs = (torch.empty(A.m + 1, dtype=torch.int32).pin_memory().numpy(),
                torch.empty(max(nz, 1), dtype=torch.int32).pin_memory().numpy(),
                torch.empty(max(nz, 1), dtype=torch.float64).pin_memory().numpy())
        ctx.spgemm_csr_host_into(Ah, outs, None, op)  # warm
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(n_e2e):
            ctx.spgemm_csr_host_into(Ah, outs, None, op)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        into_ms = shards.max_over_ranks(e0.elapsed_time(e1) / n_e2e)
        e2e["into_caller_buffers"] = {
            "value": shards.replica_throughput(world, flops, into_ms), "unit": "GFLOP/s",
            "ms_per_step": into_ms,
            "what": "rtt_spgemm_csr_host_into: the same H2D and D2H, C into page-locked host "
                    "arrays the caller reuses (no fresh pages to fault in)"}
        del outs

    control = None
    if rank == 0 and not args.no_control:
        b_view = None
        if aat:
            At = A.transpose()
            b_view = (At.m, At.n, torch.from_numpy(At.rowptr).to(dev),
                      torch.from_numpy(At.col).to(dev), torch.from_numpy(At.val).to(dev))
        control = cusparse_control(a_view, b_view, max(1, min(3, args.steps)), 1, flops, got)
        del b_view
    cpu = None
    checks = None
    if rank == 0:
        B = A.transpose() if aat else A
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline_port(A, flops, B if aat else None)
            cpu.pop("seconds", None)
        # every result of this run against the oracle (the checker): the
        # timed product, the values-only update and the host-buffer call
        if not args.no_parity:
            want = oracle_product(A, B)
            what = "full product vs the oracle's FP64 row SPA"
            checks = parity(*got, want, what)
            if e2e is not None:
                e2e["parity"] = parity(*got_e2e, want, what)
            del want
            if upd is not None:
                from rtt_spgemm import generators as G
                A2 = G.CSR(A.m, A.n, A.rowptr, A.col, A.val * 0.5)
                want = oracle_product(A2, A2.transpose() if aat else A2)
                upd["parity"] = parity(*got_upd, want, what + " (A values x 0.5)")
                del want

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    step_frac = abytes / (ms * 1e-3) / 1e9 / peaks["hbm_gbs"]
    line = {
        "metric": "SpGEMM GFLOP/s", "value": value, "unit": "GFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator; no public matrix collection available)",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                   "n": A.m, "nnz_a": A.nnz, "nnz_c": nnz_c, "nnz_cub": cub, "flops": flops,
                   "tiles_a": st["tiles_a"], "tiles_c": st["tiles_c"],
                   "alg_bytes": abytes, "parallelism": f"replicas x{world}",
                   "l2": l2_note,
                   "dmma_pair_cutoff": args.dmma_cutoff, "fused_tile2csr": not args.unfused,
                   "b_staging": bool(args.staging)},
        "roofline": {"bound": "hbm",
                     "kernel": ("k_numeric_rows (TMA-staged numeric + fused tile2csr)" if args.staging
                                else "k_numeric_leaf (FP64 DMMA from hybrid leaves; the leaf "
                                     "build and tile2csr outside the kernel time)" if args.leaf_dmma
                                else "k_numeric_flat (numeric + fused tile2csr)"),
                     "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "peak_source": peaks["source"], "kernel_ms": num_ms,
                     "step_frac": step_frac},
        "stages_ms": {k: statistics.mean(v) for k, v in stage.items()},
        "step_ms": {"min": min(step_ms), "median": statistics.median(step_ms),
                    "max": max(step_ms), "each": [round(x, 3) for x in step_ms]},
        "dmma_pairs": st["dmma_pairs"], "sparse_pairs": st["sparse_pairs"],
        "host_syncs_per_step": st["host_syncs"],
        "gpu_launches": launches,
        "clocks": clocks,
        "parity": checks,
        "cusparse_control": control,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "values_only_update": upd,
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="stencil27_96", choices=list(WORKLOADS))
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--dmma-cutoff", type=int, default=0)
    ap.add_argument("--unfused", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the check of the results against the oracle")
    ap.add_argument("--mtx", default=None,
                    help="Matrix Market file for --workload mtx / mtx_aat")
    ap.add_argument("--mtx-ref-values", action="store_true",
                    help="overwrite the file's values with i %% 10, as the reference's benchmark does")
    ap.add_argument("--no-control", action="store_true",
                    help="skip the cuSPARSE SpGEMM control on the same product")
    ap.add_argument("--no-update", action="store_true",
                    help="skip the values-only update timing")
    ap.add_argument("--tune", action="store_true",
                    help="batched: configurations chosen by the autotuner (tuned in warm-up)")
    ap.add_argument("--batch-count", type=int, default=1024)
    ap.add_argument("--serve-count", type=int, default=200)
    ap.add_argument("--serve-nmax", type=int, default=2000000)
    ap.add_argument("--serve-repeats", type=int, default=3,
                    help="served: timed runs of each arm (median and spread reported)")
    ap.add_argument("--wave-rows", type=int, default=4_000_000)
    ap.add_argument("--sym-window-slots", type=int, default=0,
                    help="symbolic step 2: C tiles per window of the wide-window CTAs "
                         "(0 = default, -1 = off)")
    ap.add_argument("--persistent-rows", action="store_true",
                    help="numeric step: one resident wave of tile-row CTAs over a device queue")
    ap.add_argument("--global-rows", type=int, default=0,
                    help="heavy tile rows accumulated in C's values in device memory "
                         "(1 read-modify-write, 2 atomic adds)")
    ap.add_argument("--leaf-dmma", action="store_true",
                    help="numeric step: FP64 DMMA straight from 8x4 / 4x8 hybrid leaves")
    ap.add_argument("--segment-walk", action="store_true",
                    help="numeric step: walk B's row segments where that applies")
    ap.add_argument("--staging", action="store_true",
                    help="TMA-staged numeric kernel instead of the default flat one")
    ap.add_argument("--ref-tile-rows", type=int, default=256)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload.startswith("mtx"):
        if not args.mtx:
            raise SystemExit("--workload mtx needs --mtx PATH")
        MTX.update(path=args.mtx, value_mode=1 if args.mtx_ref_values else 0)
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "served":
        run_served(args)
    elif args.workload == "rmat20_aat":
        run_wide(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
