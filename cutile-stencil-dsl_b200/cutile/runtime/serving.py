"""Continuous-batching stencil solve server (device-resident, HBM-admitted).

A *solve* is one request: a stencil kind, a dtype, an initial state and a
step count.  The server keeps every admitted solve's fields resident on the
device and advances all of them together, one time step per *iteration*:
each (kind, dtype) group of active solves is one persistent batched launch
over a device work list (``csd_launch_batch``), so many small grids share a
launch and large ones stream beside them.  Solves that arrive while others
are running are admitted at the next iteration boundary, first come first
served, as long as their fields fit the HBM budget; a finished solve frees
its memory at the iteration that completes it.  That is iteration-level
(continuous) batching: nothing waits for a whole batch to drain.

The reference has no serving layer (it launches one grid per call,
``launch_<name>`` in target_to_python.py:305-348); every kernel here is the
same stencil kernel a single launch runs, so a solve's result is bit-identical
alone and in the mix.

State rotation: a kind with ``nstate`` state fields (1 for a plain update,
2 for a leapfrog ``u_new = f(u, u_prev)``) keeps ``nstate + 1`` buffers; at
phase p the state is ``bufs[p], bufs[p-1], ...`` (newest first) and the step
writes ``bufs[p+1]`` (indices mod ``nstate + 1``).  Buffers are allocated
zeroed, so a zero Dirichlet halo stays zero (kernels write interiors only).
"""

from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

from cutile.runtime import native
from cutile.runtime.rk_runtime import batch_zchunk


@dataclass
class SolveKind:
    """A stencil kind the server can run: compiled results per dtype
    (``{"float32": CompileResult, "float64": CompileResult}``), each taking
    ``nstate`` input fields and producing one output field."""

    name: str
    results: dict
    nstate: int = 1


@dataclass
class SolveRequest:
    kind: str
    dtype: str                 # "float32" or "float64"
    shape: tuple               # array shape, halo included
    steps: int
    arrival: float = 0.0       # seconds after the server starts
    init: object = None        # tuple of state arrays (newest first) or None
    seed: int = 0              # device Uniform[0,1) interior when init is None
    rid: int = -1


@dataclass
class SolveResult:
    rid: int
    kind: str
    dtype: str
    shape: tuple
    steps: int
    arrival: float
    admitted: float = math.nan
    completed: float = math.nan
    state: tuple = ()          # device tensors, newest first (interior + zero halo)
    error: str | None = None

    @property
    def latency(self) -> float:
        return self.completed - self.arrival


@dataclass
class _Active:
    req: SolveRequest
    res: SolveResult
    flat: object
    bufs: list
    desc: object               # numpy uint8 [phases, grid_size]
    items: int
    phase: int = 0
    done: int = 0
    nbytes: int = 0
    slot: int = -1             # first of its `phases` descriptor slots in the device pool


@dataclass
class ServerStats:
    iterations: int = 0
    launches: int = 0
    peak_bytes: int = 0
    max_active: int = 0
    admitted: int = 0
    rejected: int = 0
    wall: float = 0.0
    host_s: float = 0.0        # building and issuing iterations
    admit_s: float = 0.0       # admitting solves (allocation, initial fields, descriptors)
    wait_s: float = 0.0        # waiting for the GPU to finish iterations
    trace: list = field(default_factory=list)   # (time, active, used_bytes) per iteration


def percentile(values, q: float) -> float:
    """Nearest-rank percentile (q in [0, 100]) of a non-empty sequence."""
    v = sorted(values)
    if not v:
        return math.nan
    k = max(0, min(len(v) - 1, math.ceil(q / 100.0 * len(v)) - 1))
    return v[k]


class StencilServer:
    """Run solve requests with continuous batching under an HBM budget."""

    def __init__(self, kinds, budget_bytes: float = 150e9, device=None):
        import torch

        self.kinds = {k.name: k for k in kinds}
        self.budget = int(budget_bytes)
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = torch.device(device)
        self._progs: dict = {}
        self._idx_bufs: dict = {}
        self._host_bufs: dict = {}  # pinned staging of the index lists, per group and parity
        self._pool = None          # device descriptors of every active solve, all phases
        self._pool_top = 0
        self._pool_free: dict = {}  # phases -> free slot blocks
        self._gen = None
        self._reserved = False
        # host time admissions may take before the next iteration is issued,
        # so that a burst of arrivals does not leave the GPU idle
        self.admit_budget_s = 0.002
        self.stats = ServerStats()

    # -- programs ----------------------------------------------------------
    def program(self, kind: str, dtype: str):
        key = (kind, dtype)
        p = self._progs.get(key)
        if p is None:
            k = self.kinds[kind]
            if dtype not in k.results:
                raise KeyError(f"kind {kind!r} has no {dtype} program")
            prog = k.results[dtype].load_module().program()
            if prog.spec["inputs"] != k.nstate or prog.spec["outputs"] != 1:
                raise ValueError(f"kind {kind!r}: the stencil must read {k.nstate} field(s) and "
                                 f"write one")
            kern = prog.kernel("main")
            p = (prog, kern, batch_zchunk(kern))
            self._progs[key] = p
        return p

    def memory_of(self, req: SolveRequest) -> int:
        """Device bytes a request holds while active (its rotating buffers,
        rows padded to 128 bytes)."""
        esz = 8 if req.dtype == "float64" else 4
        per_row = -(-req.shape[-1] * esz // 128) * 128
        outer = 1
        for x in req.shape[:-1]:
            outer *= x
        span = -(-outer * per_row // 256) * 256
        return (self.kinds[req.kind].nstate + 1) * span

    # -- admission ---------------------------------------------------------
    def _admit(self, req: SolveRequest, res: SolveResult, now: float) -> _Active:
        import numpy as np
        import torch

        from cutile.runtime.rk_runtime import pack_grids

        kind = self.kinds[req.kind]
        prog, kern, zc = self.program(req.kind, req.dtype)
        tdt = torch.float64 if req.dtype == "float64" else torch.float32
        P = kind.nstate + 1
        flat, (bufs,) = pack_grids([req.shape], P, tdt, self.device)
        bufs = list(bufs)
        halo = prog.spec["halo"]
        inner = tuple(slice(h, s - h) for h, s in zip(halo, req.shape))
        if req.init is not None:
            init = tuple(req.init)
            if len(init) != kind.nstate:
                raise ValueError(f"request {req.rid}: {kind.nstate} initial field(s) expected")
            for k, a in enumerate(init):
                t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a))
                bufs[(-k) % P].copy_(t.to(device=self.device, dtype=tdt), non_blocking=True)
        else:
            if self._gen is None:
                self._gen = torch.Generator(device=self.device)
            self._gen.manual_seed(int(req.seed))
            interior = tuple(s - 2 * h for h, s in zip(halo, req.shape))
            u = torch.rand(interior, generator=self._gen, device=self.device, dtype=tdt)
            for k in range(kind.nstate):
                bufs[(-k) % P][inner].copy_(u)
        gsz = native.grid_size()
        desc = np.zeros((P, gsz), dtype=np.uint8)
        items = 0
        for p in range(P):
            ins = [bufs[(p - k) % P] for k in range(kind.nstate)]
            out = [bufs[(p + 1) % P]]
            items, loader = native.grid_build(kern, ins, out, halo, desc[p].ctypes.data,
                                              zchunk=zc, loader=native.CSD_LOADER_TMA)
        res.admitted = now
        slot = self._pool_alloc(P)
        gsz = native.grid_size()
        self._pool[slot * gsz:(slot + P) * gsz].copy_(
            torch.from_numpy(desc.reshape(-1)).pin_memory(), non_blocking=True)
        return _Active(req=req, res=res, flat=flat, bufs=bufs, desc=desc, items=items,
                       nbytes=flat.numel() * flat.element_size(), slot=slot)

    # -- the device descriptor pool ---------------------------------------
    def _pool_alloc(self, n: int) -> int:
        """First slot of `n` consecutive descriptor slots.  Growing copies the
        pool on the stream, after the launches that read the old one."""
        import torch

        free = self._pool_free.get(n)
        if free:
            return free.pop()
        gsz = native.grid_size()
        cap = 0 if self._pool is None else self._pool.numel() // gsz
        if self._pool_top + n > cap:
            new_cap = max(256, 2 * cap, self._pool_top + n)
            pool = torch.empty(new_cap * gsz, dtype=torch.uint8, device=self.device)
            if self._pool is not None:
                pool[:self._pool_top * gsz].copy_(self._pool[:self._pool_top * gsz])
            self._pool = pool
        slot = self._pool_top
        self._pool_top += n
        return slot

    def _pool_release(self, slot: int, n: int) -> None:
        self._pool_free.setdefault(n, []).append(slot)

    # -- one iteration -----------------------------------------------------
    def _iterate(self, active: list, stream) -> None:
        """Issue one step of every active solve: per (kind, dtype) group, the
        batch's descriptor indices (pool slot + phase) and item prefix sums go
        up in one pinned copy and one batched launch reads the resident
        descriptors.  Index buffers alternate between iterations; the loop
        keeps at most two iterations in flight, so a buffer is rewritten only
        after the launch that read it has finished."""
        import numpy as np
        import torch

        groups: dict = {}
        for a in active:
            groups.setdefault((a.req.kind, a.req.dtype), []).append(a)
        parity = self.stats.iterations & 1
        for key, members in groups.items():
            prog, kern, zc = self.program(*key)
            n = len(members)
            size = 2 * n + 1
            # pinned staging buffers alternate like the device ones: the copy
            # that read a buffer two iterations ago has finished
            hbufs = self._host_bufs.setdefault(key, [None, None])
            hb = hbufs[parity]
            if hb is None or hb.numel() < size:
                hb = torch.empty(max(2 * size, 1024), dtype=torch.int32, pin_memory=True)
                hbufs[parity] = hb
            host = hb.numpy()[:size]
            host[:n] = [a.slot + a.phase for a in members]
            host[n] = 0
            np.cumsum([a.items for a in members], out=host[n + 1:])
            bufs = self._idx_bufs.setdefault(key, [None, None])
            buf = bufs[parity]
            if buf is None or buf.numel() < size:
                buf = torch.empty(max(2 * size, 1024), dtype=torch.int32, device=self.device)
                bufs[parity] = buf
            buf[:size].copy_(hb[:size], non_blocking=True)
            native.launch_batch(kern, self._pool.data_ptr(), buf.data_ptr() + 4 * n, n,
                                int(host[-1]), stream, loader=native.CSD_LOADER_TMA,
                                grid_index_ptr=buf.data_ptr())
            self.stats.launches += 1

    def _stream(self):
        import torch

        return torch.cuda.current_stream(self.device)

    def _reserve(self) -> None:
        """Have the caching allocator hold the budget's memory as one free
        segment before serving: admissions then split it instead of calling
        cudaMalloc (which synchronises the device) in the request loop."""
        import torch

        if self._reserved:
            return
        self._reserved = True
        free, _total = torch.cuda.mem_get_info(self.device)
        nbytes = int(min(self.budget, 0.9 * free))
        if nbytes > 0:
            block = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            del block

    def _record(self, stream):
        """A marker after the work issued so far on ``stream``."""
        import torch

        ev = torch.cuda.Event(enable_timing=True)
        ev.record(stream)
        return ev

    def _wait(self, mark) -> None:
        mark.synchronize()

    def _done(self, mark) -> bool:
        """Whether the GPU has passed ``mark`` (no waiting)."""
        return mark.query()

    def _mark_time(self, mark, start, t_start: float) -> float:
        """Seconds after the loop start at which the GPU passed ``mark``."""
        return t_start + start.elapsed_time(mark) / 1e3

    # -- the request loop --------------------------------------------------
    def run(self, requests, *, realtime: bool = True, keep_state=True):
        """Serve ``requests`` (any order; admitted by arrival, FIFO) and
        return their results in request order.  ``realtime``: a request is
        admissible only once the wall clock passes its arrival time.
        ``keep_state``: True, False or a set of request ids whose final
        fields the results keep (kept fields stay allocated after the budget
        has released them).  The host builds and issues iteration k + 1 while
        the GPU runs iteration k; a solve's completion time is when the GPU
        passed the end of its last iteration."""
        reqs = list(requests)
        for i, r in enumerate(reqs):
            if r.rid < 0:
                r.rid = i
        results = {r.rid: SolveResult(rid=r.rid, kind=r.kind, dtype=r.dtype, shape=tuple(r.shape),
                                      steps=r.steps, arrival=r.arrival) for r in reqs}
        queue = deque(sorted(reqs, key=lambda r: (r.arrival, r.rid)))
        active: list[_Active] = []
        in_flight: deque = deque()          # (marker, solves finished by it)
        used = 0
        stream = self._stream()
        self._reserve()
        start = self._record(stream)
        self._wait(start)           # the GPU clock's zero is the loop start
        t0 = time.perf_counter()
        st = self.stats
        def admit_one() -> bool:
            """Admit (or reject) the head of the queue if it has arrived and
            fits; False when nothing could be done."""
            nonlocal used
            now = time.perf_counter() - t0
            if not queue or (realtime and queue[0].arrival > now):
                return False
            r = queue[0]
            need = self.memory_of(r)
            if need > self.budget:
                queue.popleft()
                results[r.rid].error = (f"needs {need} bytes, more than the "
                                        f"{self.budget}-byte budget")
                st.rejected += 1
                return True
            if used + need > self.budget:
                return False                    # first come, first served
            queue.popleft()
            ta = time.perf_counter()
            a = self._admit(r, results[r.rid], now)
            st.admit_s += time.perf_counter() - ta
            active.append(a)
            used += a.nbytes
            st.admitted += 1
            return True

        while queue or active or in_flight:
            # admit arrived requests in order while they fit (a bounded amount
            # of host time per pass while solves are running)
            admit_until = time.perf_counter() + self.admit_budget_s
            while queue:
                if (active or in_flight) and time.perf_counter() > admit_until:
                    break
                if not admit_one():
                    break
            st.peak_bytes = max(st.peak_bytes, used)
            st.max_active = max(st.max_active, len(active))
            if active:
                th = time.perf_counter()
                self._iterate(active, stream)
                mark = self._record(stream)
                st.host_s += time.perf_counter() - th
                st.iterations += 1
                st.trace.append((time.perf_counter() - t0, len(active), used))
                finished, keep = [], []
                for a in active:
                    a.done += 1
                    a.phase = (a.phase + 1) % len(a.bufs)
                    if a.done >= a.req.steps:
                        P = len(a.bufs)
                        nstate = self.kinds[a.req.kind].nstate
                        if keep_state is True or (keep_state and a.req.rid in keep_state):
                            a.res.state = tuple(a.bufs[(a.phase - k) % P] for k in range(nstate))
                        # later work on the stream is ordered after this
                        # iteration, so the memory and slots can be reused now
                        used -= a.nbytes
                        if a.slot >= 0:
                            self._pool_release(a.slot, P)
                        finished.append(a.res)
                    else:
                        keep.append(a)
                active = keep
                in_flight.append((mark, finished))
            # keep one iteration in flight while the next is prepared; the
            # host time until the oldest one finishes admits arrived requests
            # (their set-up work queues behind the running iteration), so
            # admission costs no GPU time unless the host is the slower side
            while in_flight and (len(in_flight) > 1 or not active):
                mark, finished = in_flight.popleft()
                while not self._done(mark):
                    if not admit_one():
                        break
                tw = time.perf_counter()
                self._wait(mark)
                st.wait_s += time.perf_counter() - tw
                if finished:
                    tdone = self._mark_time(mark, start, 0.0)
                    for res in finished:
                        res.completed = tdone
            if not active and not in_flight and queue and realtime:
                now = time.perf_counter() - t0
                time.sleep(max(0.0, min(queue[0].arrival - now, 0.01)))
        st.wall = time.perf_counter() - t0
        return [results[r.rid] for r in reqs]

    # -- the plain path --------------------------------------------------------
    def run_alone(self, req: SolveRequest):
        """One request by itself through the drop-in launch (one
        ``launch_<name>`` per step on C-contiguous fields): returns
        ``(state, device_ms)``."""
        import numpy as np
        import torch

        kind = self.kinds[req.kind]
        prog, _kern, _zc = self.program(req.kind, req.dtype)
        tdt = torch.float64 if req.dtype == "float64" else torch.float32
        P = kind.nstate + 1
        bufs = [torch.zeros(req.shape, dtype=tdt, device=self.device) for _ in range(P)]
        halo = prog.spec["halo"]
        inner = tuple(slice(h, s - h) for h, s in zip(halo, req.shape))
        if req.init is not None:
            for k, a in enumerate(req.init):
                t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a))
                bufs[(-k) % P].copy_(t.to(device=self.device, dtype=tdt))
        else:
            g = torch.Generator(device=self.device)
            g.manual_seed(int(req.seed))
            interior = tuple(s - 2 * h for h, s in zip(halo, req.shape))
            u = torch.rand(interior, generator=g, device=self.device, dtype=tdt)
            for k in range(kind.nstate):
                bufs[(-k) % P][inner].copy_(u)
        stream = torch.cuda.current_stream(self.device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for s in range(req.steps):
            p = s % P
            prog.launch([bufs[(p - k) % P] for k in range(kind.nstate)], [bufs[(p + 1) % P]],
                        stream)
        e1.record(stream)
        e1.synchronize()
        p = req.steps % P
        return tuple(bufs[(p - k) % P] for k in range(kind.nstate)), e0.elapsed_time(e1)


__all__ = ["SolveKind", "SolveRequest", "SolveResult", "StencilServer", "ServerStats",
           "percentile", "batch_zchunk"]
