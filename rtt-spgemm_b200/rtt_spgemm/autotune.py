"""Autotuner of the numeric step's knobs, per shape class, persisted.

The knobs (rtt_config fields):

* ``dmma_pair_cutoff`` - the DMMA fill cutoff: tile pairs with
  nnz(A tile) * nnz(B tile) at or above it go to the FP64 tensor-core path
  (0: scalar only);
* ``b_staging`` - the accumulator / kernel switch: 0 is the flat kernel
  (warp-private Gustavson, direct B row loads), 1 the kernel with B's rows
  streamed through a TMA stage ring (the one that also runs DMMA pairs);
* ``split_target`` - the tile-row bucket threshold of the early split: tile
  rows whose windows walk more products than this are cut into window tasks
  (0: the library default, negative: never);
* ``sym_window_slots`` - the tile-row bucket threshold of symbolic step 2:
  tile rows with more C tiles than 254 run in wide-window CTAs of this many
  slots (0: 2045, -1: never);
* ``persistent_rows`` - tile-row CTAs as one resident wave over a device
  queue instead of one CTA per tile row;
* ``global_rows`` - tile rows that need several shared-memory windows
  accumulate in C's values in device memory (2: atomic adds, the values to
  the FP64 bound but not bit for bit).

A shape class is the operation (A*A, A*A^T, A*B), and the base-2 buckets of
the row count, the mean entries per row and the row-length skew (longest row
/ mean).  The first product of a class times every candidate configuration
once the operands are resident (after one untimed run each), keeps the
fastest, and stores it with the candidates' times in a JSON file keyed by the
GPU's name; later products of the class use the stored choice.  The file is
``$RTT_TUNE_CACHE`` or ``~/.cache/rtt_spgemm/tune.json``.  All
configurations give results within the same FP64 bound (the DMMA path sums
some products in another order).
"""
from __future__ import annotations

import json
import math
import os
import threading
import time
from pathlib import Path

CANDIDATES = [
    {"dmma_pair_cutoff": 0, "b_staging": 0, "split_target": 0},
    {"dmma_pair_cutoff": 0, "b_staging": 0, "split_target": 1 << 18},
    {"dmma_pair_cutoff": 0, "b_staging": 0, "split_target": 1 << 22},
    {"dmma_pair_cutoff": 0, "b_staging": 0, "split_target": -1},
    {"dmma_pair_cutoff": 3072, "b_staging": 0, "split_target": 0},
    {"dmma_pair_cutoff": 0, "b_staging": 1, "split_target": 0},
    {"dmma_pair_cutoff": 0, "b_staging": 0, "split_target": 0, "sym_window_slots": -1},
    {"dmma_pair_cutoff": 0, "b_staging": 0, "split_target": 0, "sym_window_slots": 4093},
    {"dmma_pair_cutoff": 0, "b_staging": 0, "split_target": 0, "persistent_rows": 1},
    {"dmma_pair_cutoff": 0, "b_staging": 0, "split_target": 0, "global_rows": 2},
]

OPS = {0: "AB", 1: "AAT"}


def _bucket(x: float) -> int:
    return int(math.floor(math.log2(x))) if x >= 1 else 0


def shape_class(op: str, rows: int, nnz: int, max_row: int) -> str:
    """'op|r<log2 rows>|d<log2 mean row>|s<log2 skew>'."""
    mean = nnz / max(rows, 1)
    skew = max_row / mean if mean > 0 else 1.0
    return f"{op}|r{_bucket(rows)}|d{_bucket(mean)}|s{_bucket(skew)}"


def default_path() -> Path:
    env = os.environ.get("RTT_TUNE_CACHE")
    return Path(env) if env else Path.home() / ".cache" / "rtt_spgemm" / "tune.json"


class Tuner:
    """Picks and persists a configuration per shape class.

    runner(ctx, config) -> seconds runs the product once with the context
    configured as given and returns its time; the default runner is supplied
    by configure()/configure_batch() (symbolic + numeric on the device)."""

    def __init__(self, path: str | os.PathLike | None = None, candidates=None,
                 device_name: str | None = None, repeats: int = 2):
        self.path = Path(path) if path is not None else default_path()
        self.candidates = [dict(c) for c in (candidates or CANDIDATES)]
        self.repeats = repeats
        self.device_name = device_name
        self.lock = threading.Lock()
        self.table = self._load()

    # -- persistence -------------------------------------------------------
    def _load(self) -> dict:
        try:
            return json.loads(self.path.read_text())
        except (OSError, ValueError):
            return {"version": 1, "devices": {}}

    def _save(self) -> None:
        self.path.parent.mkdir(parents=True, exist_ok=True)
        tmp = self.path.with_suffix(".tmp")
        tmp.write_text(json.dumps(self.table, indent=1, sort_keys=True))
        os.replace(tmp, self.path)

    def _entries(self) -> dict:
        dev = self.device_name or "unknown-device"
        return self.table.setdefault("devices", {}).setdefault(dev, {})

    def lookup(self, key: str):
        with self.lock:
            e = self._entries().get(key)
            return dict(e["config"]) if e else None

    # -- tuning --------------------------------------------------------------
    def tune(self, key: str, runner) -> dict:
        """Times every candidate with runner(config) -> seconds (one untimed
        run first, then the best of `repeats`), stores and returns the best."""
        times = []
        for cfg in self.candidates:
            try:
                runner(cfg)
                t = min(runner(cfg) for _ in range(self.repeats))
            except Exception as e:  # a configuration the product cannot take
                t = float("inf")
                cfg = dict(cfg, error=str(e)[:120])
            times.append((t, cfg))
        best_t, best = min(times, key=lambda x: x[0])
        best = {k: v for k, v in best.items() if k != "error"}
        with self.lock:
            self._entries()[key] = {
                "config": best, "ms": best_t * 1e3,
                "candidates": [{"config": {k: v for k, v in c.items() if k != "error"},
                                "ms": None if math.isinf(t) else t * 1e3} for t, c in times],
                "tuned_at": time.strftime("%Y-%m-%dT%H:%M:%S")}
            self._save()
        return dict(best)

    def choose(self, key: str, runner) -> dict:
        cfg = self.lookup(key)
        return cfg if cfg is not None else self.tune(key, runner)

    # -- device products ---------------------------------------------------
    def _device(self, ctx):
        if self.device_name is None:
            import torch
            self.device_name = torch.cuda.get_device_name(ctx.device)

    def configure(self, ctx, a, b=None, op: int = 0) -> dict:
        """Configures ctx for C = a*b (op 0) or a*a^T (op 1), tuning the shape
        class on first sight.  a, b: device CSR tuples."""
        import torch

        self._device(ctx)
        rows, _, rp, _, _ = a
        lens = torch.diff(rp)
        key = shape_class(OPS.get(op, "AB"), rows, int(rp[-1]),
                          int(lens.max()) if rows else 0)

        def runner(cfg):
            ctx.configure(cfg)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            nnz, _ = ctx.symbolic(a, b, op)
            crp = torch.empty(rows + 1, dtype=torch.int32, device=rp.device)
            cci = torch.empty(max(nnz, 1), dtype=torch.int32, device=rp.device)
            cva = torch.empty(max(nnz, 1), dtype=torch.float64, device=rp.device)
            ctx.numeric(crp, cci, cva)
            torch.cuda.synchronize()
            return time.perf_counter() - t0

        cfg = self.choose(key, runner)
        ctx.configure(cfg)
        return cfg

    def configure_batch(self, ctx, As, Bs=None) -> dict:
        """Configures ctx for a batched product (the block diagonal's class)."""
        import torch

        from . import spgemm_batched

        self._device(ctx)
        rows = sum(int(a[0]) for a in As)
        nnz = sum(int(a[2][-1]) for a in As)
        max_row = max((int(torch.diff(a[2]).max()) for a in As if a[0] > 0), default=0)
        key = "batch:" + shape_class("AB", rows, nnz, max_row)

        def runner(cfg):
            ctx.configure(cfg)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            spgemm_batched(ctx, As, Bs)
            torch.cuda.synchronize()
            return time.perf_counter() - t0

        cfg = self.choose(key, runner)
        ctx.configure(cfg)
        return cfg
