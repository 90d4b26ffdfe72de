"""Serving loop: SpGEMM requests of different sizes, batched as they arrive.

The served form of the product (the reference has none; it runs one product
per process): requests C = A^2 or C = A*A^T arrive over time; whenever a worker is
free it takes every request that has arrived and fits the device pool, and
runs them as ONE batched product (rtt_spgemm_batched_symbolic / _numeric: one
csr2tile, one symbolic and one numeric pass over the block diagonal of the
batch).  Two workers, each with its own context and CUDA stream, keep two
batches in flight, so requests that arrive while one batch is on the GPU are
admitted into the next one as soon as a worker and pool memory free up, and
the two batches' work overlaps on the device.

Repeated products of one A keep its tile structure resident: the request
that uses a reuse key for the third time runs alone on a context of its own,
whose csr2tile and symbolic state then stays on the device (least recently
used first out, bounded in count and bytes; an evicted structure's context
is kept for the next one); every later request with that key runs the
numeric step only on that context (rtt_spgemm_numeric, or
rtt_spgemm_numeric_values when the request brings other values of the same
structure), without csr2tile or the symbolic phase.  Keys used once or twice
stay in the batches.

Admission is bounded by memory: a request reserves, for the time its batch
runs, its operands plus the exact upper bound of the symbolic phase for C
(nnzCub entries of 12 bytes: C cannot have more entries than products) plus
its row pointer, against a fixed pool.  Operands that a request marks with a
reuse key stay resident on the device (with A^T for A*A^T requests) and are
not copied again.  Each context's own workspace (tile index, symbolic
structure, the window cursors of the numeric step's persistent workers:
4 bytes per A entry up to 32,768 per worker CTA) sits outside this
accounting, so pool_bytes should leave room for it below the device's
memory.

A request whose bound exceeds a quarter of the pool (exclusive_share) runs
alone once nothing else is in flight, and a batch of one request runs
through the plain path (no block-diagonal assembly); a batch that runs out
of device memory beside other work is queued again, its requests to run
alone, and a request alone that still runs out of memory releases what the
server keeps (resident structures and operands, grown buffers) and tries
once more.

A batch's product is one CSR with int32 offsets, so a batch also keeps the
sum of its requests' entry bounds (nnzCub) within 2^31 - 1.  A request whose
own result cannot be represented, or any other failing request, is finished
with its error recorded (Request.error) instead of a result; a failing batch
is retried one request at a time so that only the failing request fails.

Latency of a request = time its result is on the device minus its arrival.
"""
from __future__ import annotations

import threading
import time
from collections import OrderedDict, deque
from dataclasses import dataclass, field

import numpy as np

from . import Context, RttError, spgemm_batched
from .generators import CSR

INT32_MAX = 2**31 - 1


@dataclass
class Request:
    a: CSR                    # host CSR operand
    op: str = "A2"            # "A2" (C = A*A) or "AAT" (C = A*A^T)
    key: object = None        # reuse key of A's structure: operands (and tiles) stay resident
    arrival: float = 0.0      # seconds after the start of the run
    done: float = -1.0
    result: tuple = None      # device (rowptr, col, val) of C
    error: str = None         # set instead of result when the product failed
    bound: int = field(default=0, repr=False)
    entries: int = field(default=0, repr=False)
    exclusive: bool = field(default=False, repr=False)  # runs alone, nothing else in flight
    uses: int = field(default=-1, repr=False)  # requests with its key before it (-1: not yet counted)


def product_cub(a: CSR, op: str) -> int:
    """nnzCub of the request: the products, an upper bound of nnz(C).  Raises
    ValueError for a CSR the library would reject (row pointer not monotone
    or past the entries, a column outside [0, n), A^2 of a non-square A)."""
    rp, col = np.asarray(a.rowptr), np.asarray(a.col)
    if (rp.size != a.m + 1 or rp[0] < 0 or np.any(np.diff(rp) < 0) or rp[-1] > col.size
            or (col.size and (col.min() < 0 or col.max() >= a.n))):
        raise ValueError("invalid CSR operand")
    if op == "A2" and a.m != a.n:
        raise ValueError("A^2 of a non-square matrix")
    if op == "A2":
        return int(np.diff(a.rowptr).astype(np.int64)[a.col].sum())
    # A * A^T: row i's products = sum over k in A(i) of nnz(A^T row k) = colcount(k)
    cc = np.bincount(a.col, minlength=a.n).astype(np.int64)
    return int(cc[a.col].sum())


def product_bound(a: CSR, op: str) -> int:
    """Upper bound of C's bytes from the structure alone: nnz(C) <= nnzCub."""
    return 12 * product_cub(a, op) + 4 * (a.m + 1)


class _OutOfMemory(Exception):
    """A batch ran out of device memory while other work was in flight."""


@dataclass
class _Structure:
    """A reuse key's resident tile structure: a context after its symbolic
    phase on the key's A, with the device operand it borrows."""
    ctx: Context
    cur: CSR                  # the host operand whose values the device tiles hold
    a: tuple                  # device operand (borrowed by ctx)
    op: str
    nnz: int
    bytes: int
    vals: object = None       # device values of the last values-only update (borrowed)
    lock: threading.Lock = field(default_factory=threading.Lock)


class Server:
    def __init__(self, device: int = 0, pool_bytes: float = 120e9, max_batch: int = 512,
                 workers: int = 2, config: dict | None = None, keep_results: bool = True,
                 max_structures: int = 16, structure_bytes: float | None = None,
                 exclusive_share: float = 0.25):
        import torch

        self.torch = torch
        self.device = torch.device("cuda", device)
        self.pool = float(pool_bytes)
        # a request whose bound exceeds this share of the pool runs alone
        self.exclusive_share = exclusive_share
        self.max_batch = max_batch
        self.config = config
        self.nworkers = workers
        self.keep_results = keep_results
        # reuse key -> device operands (LRU, bounded by bytes; counted against the pool)
        self.resident: OrderedDict = OrderedDict()
        self.resident_bytes = pool_bytes / 8
        self.lock = threading.Lock()
        # reuse key -> _Structure (LRU), bounded by count and by the bytes of
        # their products' bounds
        self.structures: OrderedDict = OrderedDict()
        self.max_structures = max_structures
        self.structure_bytes = pool_bytes / 4 if structure_bytes is None else structure_bytes
        self.uses: dict = {}     # reuse key -> requests seen with it
        self._spare: list = []   # contexts of evicted structures, for the next one
        # one (stream, context) per worker, kept across run() calls: their
        # grow-only device buffers stay sized for the traffic seen so far
        self._slots = []
        self.events: dict = {}   # what the last run() did (counts and seconds)

    def _event(self, name: str, seconds: float = 0.0, n: int = 1):
        with self.lock:
            e = self.events.setdefault(name, [0, 0.0])
            e[0] += n
            e[1] += seconds

    def _slot(self, i):
        torch = self.torch
        with self.lock:
            while len(self._slots) <= i:
                stream = torch.cuda.Stream(device=self.device)
                ctx = Context(self.device.index or 0, self.config)
                ctx.set_stream(stream.cuda_stream)
                self._slots.append((stream, ctx))
            return self._slots[i]

    def reset_reuse(self):
        """Forget every reuse key: use counts, resident operands and resident
        structures (their contexts are kept as spares, up to four).  A new
        request stream starts from here."""
        with self.lock:
            structs = list(self.structures.values())
            self.structures.clear()
            self.resident.clear()
            self.uses.clear()
        for st in structs:
            with st.lock:
                with self.lock:
                    if len(self._spare) < 4:
                        self._spare.append(st.ctx)
                        continue
                st.ctx.close()

    def close(self):
        """Release the workers' contexts, the resident structures and operands."""
        for _, ctx in self._slots:
            ctx.close()
        self._slots = []
        for st in self.structures.values():
            with st.lock:
                st.ctx.close()
        self.structures.clear()
        for ctx in self._spare:
            ctx.close()
        self._spare = []
        self.resident.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- operands -------------------------------------------------------
    def _upload(self, a: CSR, ctx: Context):
        t = self.torch
        d = self.device
        va = (a.m, a.n, t.from_numpy(a.rowptr).to(d, non_blocking=True),
              t.from_numpy(a.col).to(d, non_blocking=True),
              t.from_numpy(a.val).to(d, non_blocking=True))
        return va

    def _operands(self, r: Request, ctx: Context, need_at: bool = True):
        """Device operands of a request.  A reuse key names a structure: a
        request whose host operand is another object than the resident one
        brings new values, which replace the resident values (and A^T).
        need_at=False leaves A^T out (the single-request path multiplies
        with RTT_OP_AAT)."""
        with self.lock:
            hit = self.resident.get(r.key) if r.key is not None else None
            if hit is not None:
                self.resident.move_to_end(r.key)
        if hit is not None and hit[2] is not r.a:
            a0 = hit[0]
            a = (a0[0], a0[1], a0[2], a0[3],
                 self.torch.from_numpy(np.ascontiguousarray(r.a.val)).to(self.device,
                                                                         non_blocking=True))
            hit = (a, None, r.a)
        elif hit is None:
            hit = (self._upload(r.a, ctx), None, r.a)
        a, at, src = hit
        if r.op == "AAT" and at is None and need_at:
            at = ctx.transpose(a)
        if r.key is not None:
            with self.lock:
                self.resident[r.key] = (a, at, src)
                self.resident.move_to_end(r.key)
                # least recently used operands leave first (a batch in flight
                # keeps its own references)
                nbytes = lambda e: sum(t.numel() * t.element_size()
                                       for x in (e[0], e[1]) if x is not None for t in x[2:5])
                total = sum(nbytes(e) for e in self.resident.values())
                while len(self.resident) > 1 and total > self.resident_bytes:
                    _, old = self.resident.popitem(last=False)
                    total -= nbytes(old)
        return a, (at if r.op == "AAT" else a)

    # -- resident tile structures -----------------------------------------
    def _count(self, r: Request) -> int:
        """Requests with r's reuse key before r (and count r)."""
        if r.key is None:
            return 0
        if r.uses >= 0:  # a request queued again counts once
            return r.uses
        with self.lock:
            n = self.uses.get(r.key, 0)
            self.uses[r.key] = n + 1
        r.uses = n
        return n

    def _structure(self, r: Request):
        with self.lock:
            st = self.structures.get(r.key) if r.key is not None else None
            if st is not None and st.op == r.op:
                self.structures.move_to_end(r.key)
                return st
        return None

    def _outputs(self, m: int, nnz: int):
        t = self.torch
        return (t.empty(m + 1, dtype=t.int32, device=self.device),
                t.empty(max(nnz, 1), dtype=t.int32, device=self.device),
                t.empty(max(nnz, 1), dtype=t.float64, device=self.device))

    def _finish(self, r: Request, out, nnz: int, t0: float):
        r.done = time.perf_counter() - t0
        r.result = (out[0], out[1][:nnz], out[2][:nnz]) if self.keep_results else None

    @staticmethod
    def _is_oom(e: Exception) -> bool:
        return (isinstance(e, RttError) and e.status == 4) or "out of memory" in str(e)

    def _run_resident(self, st: _Structure, stream, r: Request, t0: float):
        """Numeric step only, on the key's resident structure."""
        with st.lock:
            try:
                st.ctx.set_stream(stream.cuda_stream)
                out = self._outputs(r.a.m, st.nnz)
                if r.a is st.cur:  # the values on the device
                    st.ctx.numeric(*out)
                else:  # other values of the same structure
                    vals = self.torch.from_numpy(np.ascontiguousarray(r.a.val)).to(
                        self.device, non_blocking=True)
                    st.ctx.numeric_values(vals, None, *out)
                    # the tiles (and, for A*A, B's values) now come from vals
                    st.vals, st.cur = vals, r.a
                stream.synchronize()
            except (RttError, RuntimeError) as e:
                if self._is_oom(e):  # the output did not fit beside other work
                    raise _OutOfMemory() from e
                r.error, r.done = str(e), time.perf_counter() - t0
                return
        self._finish(r, out, st.nnz, t0)

    def _build_resident(self, stream, r: Request, t0: float):
        """Run a reused key's product alone on a context of its own and keep
        that context's structure resident."""
        with self.lock:
            hit = self.resident.get(r.key)
        if hit is not None and hit[2] is r.a:
            a = hit[0]
        elif hit is not None:  # the resident structure with the request's values
            a = hit[0][:4] + (self.torch.from_numpy(np.ascontiguousarray(r.a.val)).to(
                self.device, non_blocking=True),)
        else:
            a = self._upload(r.a, None)
        with self.lock:
            ctx = self._spare.pop() if self._spare else None
        if ctx is None:
            ctx = Context(self.device.index or 0, self.config)
        try:
            ctx.set_stream(stream.cuda_stream)
            nnz, _ = ctx.symbolic(a, None, 1 if r.op == "AAT" else 0)
            out = self._outputs(r.a.m, nnz)
            ctx.numeric(*out)
            stream.synchronize()
        except (RttError, RuntimeError) as e:
            ctx.trim()
            with self.lock:
                self._spare.append(ctx)
            if self._is_oom(e):  # queued again, to run alone in the plain batch path
                raise _OutOfMemory() from e
            r.error, r.done = str(e), time.perf_counter() - t0
            return
        self._finish(r, out, nnz, t0)
        st = _Structure(ctx, r.a, a, r.op, nnz, int(r.bound))
        evict = []
        with self.lock:
            old = self.structures.pop(r.key, None)
            if old is not None:
                evict.append(old)
            self.structures[r.key] = st
            total = sum(x.bytes for x in self.structures.values())
            while len(self.structures) > 1 and (len(self.structures) > self.max_structures
                                                or total > self.structure_bytes):
                _, x = self.structures.popitem(last=False)
                total -= x.bytes
                evict.append(x)
        for x in evict:
            with x.lock:  # not in use by another worker
                with self.lock:
                    if len(self._spare) < 4:
                        self._spare.append(x.ctx)
                        continue
                x.ctx.close()

    def _run_batch(self, ctx, stream, batch, t0):
        # keys with a resident structure: the numeric step on it; keys used
        # twice before: a product of their own that makes one resident
        rest = []
        for r in batch:
            uses = self._count(r)
            # a request that ran out of memory beside other work runs alone,
            # in the plain batch path, after every structure was released
            st = None if r.exclusive else self._structure(r)
            t1 = time.perf_counter()
            if st is not None:
                self._run_resident(st, stream, r, t0)
                self._event("resident_numeric", time.perf_counter() - t1)
            elif (uses >= 2 and not r.exclusive and self.max_structures > 0
                  and r.bound <= self.structure_bytes / 4):
                # a structure is kept only when at least four of its size
                # fit the structure budget, so that keys are not evicted by
                # every large newcomer
                self._build_resident(stream, r, t0)
                self._event("resident_build", time.perf_counter() - t1)
            else:
                rest.append(r)
        if rest:
            t1 = time.perf_counter()
            self._run_batch_plain(ctx, stream, rest, t0)
            self._event("batch" if len(rest) > 1 else "batch_of_one", time.perf_counter() - t1)
            self._event("batched_requests", n=len(rest))

    def _run_single(self, ctx, stream, r: Request, t0: float, retried: bool = False):
        """One request through the plain path on the worker's context (no
        block-diagonal assembly, A*A^T as RTT_OP_AAT)."""
        try:
            a, _ = self._operands(r, ctx, need_at=False)
            nnz, _ = ctx.symbolic(a, None, 1 if r.op == "AAT" else 0)
            out = self._outputs(r.a.m, nnz)
            ctx.numeric(*out)
            stream.synchronize()
        except (RttError, RuntimeError) as e:
            if self._is_oom(e):
                if not r.exclusive:  # queued again, to run alone
                    raise _OutOfMemory() from e
                if not retried:  # alone and still short: release what is kept, once
                    out = None
                    self._release_memory()
                    return self._run_single(ctx, stream, r, t0, True)
            r.error, r.done = str(e), time.perf_counter() - t0
            return
        self._finish(r, out, nnz, t0)

    def _run_batch_plain(self, ctx, stream, batch, t0):
        if len(batch) == 1:
            return self._run_single(ctx, stream, batch[0], t0)
        try:
            As, Bs = [], []
            for r in batch:
                a, b = self._operands(r, ctx)
                As.append(a)
                Bs.append(b)
            outs = spgemm_batched(ctx, As, Bs)
            stream.synchronize()
        except (RttError, RuntimeError) as e:
            # device memory short while other work is in flight: the worker
            # queues the requests again, to run alone (see run())
            oom = self._is_oom(e)
            if oom and not all(r.exclusive for r in batch):
                raise _OutOfMemory() from e
            if len(batch) > 1:  # find the failing request(s): one at a time
                for r in batch:
                    self._run_batch_plain(ctx, stream, [r], t0)
                return
            batch[0].error = str(e)
            batch[0].done = time.perf_counter() - t0
            return
        t = time.perf_counter() - t0
        for r, o in zip(batch, outs):
            r.done = t
            r.result = o if self.keep_results else None

    def _release_memory(self):
        """Before a request that ran out of memory runs alone (nothing else
        in flight): drop the resident structures, spare contexts and operands,
        shrink the workers' grown buffers, and hand torch's cache back."""
        with self.lock:
            structs = list(self.structures.values())
            self.structures.clear()
            spare, self._spare = self._spare, []
            self.resident.clear()
        t1 = time.perf_counter()
        for st in structs:
            st.ctx.close()
        for ctx in spare:
            ctx.close()
        for _, ctx in self._slots:
            ctx.trim()
        self.torch.cuda.empty_cache()
        self._event("release_memory", time.perf_counter() - t1)

    # -- the loop ---------------------------------------------------------
    def run(self, requests: list[Request]) -> dict:
        """Serve requests (sorted by arrival) in real time; returns latency
        percentiles and throughput."""
        for r in requests:
            try:
                r.entries = product_cub(r.a, r.op)
            except ValueError as e:  # rejected at admission, finished on arrival
                r.error, r.done = str(e), r.arrival
                continue
            r.bound = 12 * r.entries + 4 * (r.a.m + 1) + 12 * r.a.nnz + 4 * (r.a.m + 1)
            # a product this large would crowd the others out of the pool:
            # it runs alone, when nothing else is in flight
            r.exclusive = r.bound > self.pool * self.exclusive_share
        self.events = {}
        pending = deque()
        nxt = 0
        reserved = [0.0]
        done = [0]
        cv = threading.Condition()
        t0 = time.perf_counter()
        n = len(requests)

        def take_batch():
            # called with cv held: admit arrived requests that fit the pool
            nonlocal nxt
            now = time.perf_counter() - t0
            while nxt < n and requests[nxt].arrival <= now:
                if requests[nxt].error is None:
                    pending.append(requests[nxt])
                nxt += 1
            batch, need, entries = [], 0.0, 0
            if pending and pending[0].exclusive:
                # a request that ran out of memory beside other work runs
                # alone once everything else has finished
                if reserved[0] > 0:
                    return [], 0.0
                batch = [pending.popleft()]
                reserved[0] += self.pool
                return batch, self.pool
            while pending and len(batch) < self.max_batch:
                r = pending[0]
                if r.exclusive:
                    break
                if batch and reserved[0] + need + r.bound > self.pool:
                    break
                if batch and entries + r.entries > INT32_MAX:
                    break  # the batch's C must keep int32 offsets
                entries += r.entries
                if not batch and reserved[0] + r.bound > self.pool and reserved[0] > 0:
                    break  # wait for memory to free up
                batch.append(pending.popleft())
                need += r.bound
            reserved[0] += need
            return batch, need

        def worker(i):
            torch = self.torch
            torch.cuda.set_device(self.device)
            stream, ctx = self._slot(i)
            with torch.cuda.stream(stream):
                while True:
                    with cv:
                        batch, need = take_batch()
                        while not batch:
                            if nxt >= n and not pending:
                                return
                            wait = 0.0005
                            if nxt < n and not pending:
                                wait = max(0.0, requests[nxt].arrival - (time.perf_counter() - t0))
                            cv.wait(timeout=min(wait, 0.01) if wait > 0 else 0.0005)
                            batch, need = take_batch()
                    retry = []
                    try:
                        self._run_batch(ctx, stream, batch, t0)
                    except _OutOfMemory:
                        retry = [r for r in batch if r.done < 0]
                        for r in retry:
                            r.exclusive = True
                        self._event("out_of_memory_requeued", n=len(retry))
                    except Exception as e:  # any other failure finishes the batch's requests
                        now = time.perf_counter() - t0
                        for r in batch:
                            if r.done < 0:
                                r.error, r.done = f"{type(e).__name__}: {e}", now
                    with cv:
                        for r in reversed(retry):
                            pending.appendleft(r)
                        done[0] -= len(retry)
                        reserved[0] -= need
                        done[0] += len(batch)
                        cv.notify_all()

        threads = [threading.Thread(target=worker, args=(i,)) for i in range(self.nworkers)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        span = max(r.done for r in requests) if requests else 0.0
        out = summarize(requests, span)
        out["events"] = {k: {"count": v[0], "seconds": round(v[1], 4)}
                         for k, v in sorted(self.events.items())}
        return out


def serve_plain(requests: list[Request], device: int = 0, config: dict | None = None,
                keep_results: bool = True, ctx: Context | None = None) -> dict:
    """The plain path under the same arrivals: one product per call, FIFO.
    A caller-owned ctx is used and kept (its buffers stay grown)."""
    import torch

    dev = torch.device("cuda", device)
    own = ctx is None
    if own:
        ctx = Context(device, config)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)
    resident = {}
    t0 = time.perf_counter()
    for r in requests:
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        hit = resident.get(r.key) if r.key is not None else None
        if hit is None:
            a = (r.a.m, r.a.n, torch.from_numpy(r.a.rowptr).to(dev),
                 torch.from_numpy(r.a.col).to(dev), torch.from_numpy(r.a.val).to(dev))
        elif hit[1] is not r.a:  # the key's structure with new values
            a = hit[0][:4] + (torch.from_numpy(np.ascontiguousarray(r.a.val)).to(dev),)
        else:
            a = hit[0]
        if r.key is not None:
            resident[r.key] = (a, r.a)
        try:
            nnz, _ = ctx.symbolic(a, None, 1 if r.op == "AAT" else 0)
            rp = torch.empty(r.a.m + 1, dtype=torch.int32, device=dev)
            ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
            va = torch.empty(max(nnz, 1), dtype=torch.float64, device=dev)
            ctx.numeric(rp, ci, va)
            stream.synchronize()
            r.result = (rp, ci[:nnz], va[:nnz]) if keep_results else None
        except RttError as e:
            r.error = str(e)
        r.done = time.perf_counter() - t0
    if own:
        ctx.close()
    return summarize(requests, max(r.done for r in requests) if requests else 0.0)


def summarize(requests, span: float) -> dict:
    """Throughput over all requests; latency percentiles over the requests
    that produced a result."""
    ok = [r for r in requests if r.error is None and r.done >= 0]
    lat = np.array([r.done - r.arrival for r in ok]) * 1e3
    errors = {}
    for r in requests:
        if r.error is not None:
            k = r.error.split(":")[0][:60]
            errors[k] = errors.get(k, 0) + 1
    return {"requests": len(requests), "seconds": span,
            "failed": sum(r.error is not None for r in requests),
            "errors": errors,
            "completed": len(ok),
            "spgemms_per_s": len(ok) / span if span > 0 else 0.0,
            "p50_ms": float(np.percentile(lat, 50)) if lat.size else 0.0,
            "p99_ms": float(np.percentile(lat, 99)) if lat.size else 0.0}


def poisson_requests(count: int, rate: float, n_lo: int, n_hi: int, reuse: float = 0.3,
                     aat_share: float = 0.5, seed: int = 0) -> list[Request]:
    """The served configuration's request stream: Poisson arrivals, mixed A^2 /
    A*A^T, n log-uniform in [n_lo, n_hi], nnz/row 4..64 from the generators
    (2-D / 3-D stencils, R-MAT, banded plus scatter); a share of requests
    reuses an earlier request's A (its reuse key)."""
    from . import generators as G

    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=count))
    reqs = []
    for i in range(count):
        if reqs and rng.random() < reuse:
            j = int(rng.integers(0, len(reqs)))
            src = reqs[j]
            reqs.append(Request(src.a, src.op, src.key, float(t[i])))
            continue
        n = int(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
        kind = int(rng.integers(0, 4))
        if kind == 0:
            side = max(4, int(round(np.sqrt(n))))
            a = G.laplacian_2d(side)
        elif kind == 1:
            side = max(3, int(round(n ** (1 / 3))))
            a = G.stencil_27(side, int(rng.integers(0, 1 << 30)))
        elif kind == 2:
            scale = max(8, int(np.log2(n)))
            a = G.rmat(scale, int(rng.integers(4, 17)), seed=int(rng.integers(0, 1 << 30)))
        else:
            a = G.banded_scatter(n, int(rng.integers(2, 32)), seed=int(rng.integers(0, 1 << 30)))
        op = "AAT" if rng.random() < aat_share else "A2"
        reqs.append(Request(a, op, ("req", i), float(t[i])))
    return reqs
