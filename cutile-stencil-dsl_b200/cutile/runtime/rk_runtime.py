"""Runtime of generated Runge-Kutta modules: single grids and batches.

``RKProgram`` runs the stage kernels of ``RKIntegrator.compile`` on one grid
(``step``) with lazily allocated workspace.  ``RKBatch`` advances many
independent grids of uneven sizes together: every stage is ONE persistent
launch over a device-resident work list (``csd_launch_batch``), ``dt`` is a
per-grid device scalar (optionally recomputed each step from a CFL
max-reduction, also one batched launch), and a whole multi-step loop can be
captured into a CUDA graph and replayed.
"""

from __future__ import annotations

import ctypes
import threading

from cutile.runtime import native
from cutile.runtime.rk_integrator import stage_table


def _as_tuple(u):
    return tuple(u) if isinstance(u, (tuple, list)) else (u,)


class RKProgram:
    def __init__(self, cuda_source: str, spec: dict):
        self.source = cuda_source
        self.spec = spec
        self.table = stage_table(spec["method"])
        self._modules: dict = {}
        self._lock = threading.Lock()
        self._work: dict = {}
        self._dt: dict = {}
        self.bc_odd: tuple = ()
        self.bc_value = 0.0

    # -- kernels ---------------------------------------------------------------
    def kernel(self, stage: int) -> native.NativeKernel:
        import torch

        dev = torch.cuda.current_device()
        with self._lock:
            m = self._modules.get(dev)
            if m is None:
                m = native.NativeModule(self.source)
                self._modules[dev] = m
        return m.kernel(self.spec["stages"][stage])

    # -- buffers -------------------------------------------------------------
    def copy_state(self, u0):
        t = tuple(x.clone() for x in _as_tuple(u0))
        return t if isinstance(u0, (tuple, list)) else t[0]

    def workspace(self, state: tuple) -> dict:
        import torch

        key = tuple((x.data_ptr(), tuple(x.shape), x.dtype) for x in state)
        ws = self._work.get(key)
        if ws is None:
            names = {n for row in self.table for n in (row[4], row[5], row[6], row[7])
                     if n not in (None, "u")}
            # same strides as the state (row-pitched batches included)
            ws = {n: tuple(torch.empty_strided(x.size(), x.stride(), dtype=x.dtype,
                                               device=x.device).zero_() for x in state)
                  for n in sorted(names)}
            self._work[key] = ws
        return ws

    def stage_io(self, k: int, bufs: dict, aux: tuple):
        a, b, c, w, base, stage, acc_in, out = self.table[k]
        inputs = list(bufs[stage]) + list(aux)
        if a != 0.0 and base != stage:
            inputs += list(bufs[base])
        if w is not None:
            inputs += list(bufs[acc_in])
        outputs = list(bufs[out])
        if w is not None:
            outputs += list(bufs["acc"])
        return inputs, outputs

    def _scalars(self, scalars: dict | None) -> list:
        names = self.spec.get("scalars", [])
        scalars = scalars or {}
        missing = [n for n in names if n not in scalars]
        if missing:
            raise TypeError(f"missing scalar parameter(s) {missing}")
        return [float(scalars[n]) for n in names]

    # -- one grid --------------------------------------------------------------
    def step(self, u, dt, stream=None, scalars: dict | None = None, aux=()) -> None:
        """One RK step of the state ``u`` in place; ``dt`` is a float or a
        device float64 tensor of one element."""
        import torch

        fields = _as_tuple(u)
        m = self.spec["state_fields"]
        if len(fields) + len(aux) != self.spec["fields"]:
            raise TypeError(f"the operator reads {self.spec['fields']} fields")
        state = fields[:m]
        if isinstance(dt, torch.Tensor):
            dyn = dt
        else:
            dyn = self._dt.get(state[0].device)
            if dyn is None:
                dyn = torch.empty(1, dtype=torch.float64, device=state[0].device)
                self._dt[state[0].device] = dyn
            dyn.fill_(float(dt))
        bufs = dict(self.workspace(state))
        bufs["u"] = state
        sv = self._scalars(scalars)
        halo = self.spec["halo"]
        for k in range(len(self.table)):
            inputs, outputs = self.stage_io(k, bufs, tuple(fields[m:]) + tuple(aux))
            native.launch(self.kernel(k), inputs, outputs, halo, stream, scalars=sv, dyn=dyn,
                          bc_odd=self.bc_odd, bc_value=self.bc_value)
        last_out = self.table[-1][7]
        if last_out != "u":
            inner = tuple(slice(h, s - h) for h, s in zip(halo, state[0].shape))
            for dst, src in zip(state, bufs[last_out]):
                dst[inner].copy_(src[inner])


def pack_grids(shapes, nfields: int, dtype, device, row_align_bytes: int = 128):
    """Fields of many grids in one flat device buffer, rows padded to
    ``row_align_bytes`` so that every grid qualifies for the TMA loader and
    16-byte vector stores.  Returns ``(flat, grids)``: ``grids[g]`` is a tuple
    of ``nfields`` row-pitched views of shape ``shapes[g]`` (halo included);
    the pad columns are never read or written by the engine."""
    import torch

    esz = torch.empty((), dtype=dtype).element_size()
    align = max(1, row_align_bytes // esz)
    layout, total = [], 0
    for shp in shapes:
        shp = tuple(int(x) for x in shp)
        pitch = -(-shp[-1] // align) * align
        outer = 1
        for x in shp[:-1]:
            outer *= x
        span = outer * pitch
        offs = []
        for _ in range(nfields):
            offs.append(total)
            total += -(-span * esz // 256) * 256 // esz
        layout.append((shp, pitch, offs))
    flat = torch.zeros(max(total, 1), dtype=dtype, device=device)
    grids = []
    for shp, pitch, offs in layout:
        strides, acc = [1], pitch
        for x in reversed(shp[1:-1]):
            strides.insert(0, acc)
            acc *= x
        if len(shp) > 1:
            strides.insert(0, acc)
        strides = tuple(strides[-len(shp):])
        grids.append(tuple(flat.as_strided(shp, strides, off) for off in offs))
    return flat, grids


class BatchLaunch:
    """Device descriptors of one kernel over many grids (one persistent launch)."""

    def __init__(self, kernel: native.NativeKernel, per_grid: list, halo, *, zchunk: int = 0,
                 bc_value: float = 0.0):
        import torch

        self.kernel = kernel
        gsz = native.grid_size()
        n = len(per_grid)
        host = (ctypes.c_ubyte * (gsz * n))()

        def build(loader):
            starts, used = [0], set()
            for i, g in enumerate(per_grid):
                dest = ctypes.addressof(host) + i * gsz
                items, ld = native.grid_build(kernel, g["inputs"], g["outputs"], halo, dest,
                                              zchunk=zchunk, scalars=g.get("scalars", ()),
                                              dyn=g.get("dyn"), red=g.get("red"),
                                              bc_odd=g.get("bc_odd", ()), bc_value=bc_value,
                                              loader=loader)
                starts.append(starts[-1] + items)
                used.add(ld)
            return starts, used

        # one copy path per batch: TMA when every grid qualifies, else cp.async
        starts, used = build(-1)
        self.loader = native.CSD_LOADER_TMA
        if len(used) > 1 or native.CSD_LOADER_LDG in used:
            starts, _ = build(native.CSD_LOADER_LDG)
            self.loader = native.CSD_LOADER_LDG
        dev = per_grid[0]["inputs"][0].device
        # 64-byte aligned device copy (torch allocations are 256-byte aligned)
        self.grids = torch.frombuffer(bytearray(host), dtype=torch.uint8).to(dev)
        self.item_start = torch.tensor(starts, dtype=torch.int32, device=dev)
        self.ngrids = n
        self.total_items = starts[-1]

    def launch(self, stream=None, grid: int = 0) -> None:
        native.launch_batch(self.kernel, self.grids.data_ptr(), self.item_start.data_ptr(),
                            self.ngrids, self.total_items, stream, grid=grid, loader=self.loader)


def batch_zchunk(kernel: native.NativeKernel) -> int:
    """Rows per work item in a batched launch: short items for issue-bound
    bodies (kernels whose default asks for several items per resident
    block), long ones for memory-bound bodies.  Measured on the 256-grid
    shallow-water batch (8-row steps): 32-row items 130 solves/s, 16-row 124,
    64-row 128, 8-row 107."""
    d = kernel.desc
    return 4 * d["rows"] if d["zchunk"] < 0 else 64


class RKBatch:
    """Many independent grids advanced together, one launch per stage.

    ``states``: per grid, the tuple of state fields (any sizes, same ndim and
    dtype).  ``scalars``: per grid, the operator's scalar parameters (dict).
    ``dt``: a float (same for all grids), or ``cfl=(speed_program, scale,
    cfl)`` to recompute ``dt = cfl * scale[g] / max speed`` per grid and step
    on the device, where ``speed_program`` is a ``compile(..., reduce="max")``
    program of a pointwise signal-speed stencil over the state fields.
    """

    def __init__(self, rk_result, states: list, scalars: list | None = None, *, dt=None,
                 cfl=None, bc_odd=(), bc_value: float = 0.0, zchunk: int | None = None,
                 dt_max: float = 1e30):
        import torch

        self.prog = rk_result.load_module().program()
        self.states = [tuple(s) for s in states]
        n = len(self.states)
        dev = self.states[0][0].device
        self.dt = torch.zeros(n, dtype=torch.float64, device=dev)
        if dt is not None:
            self.dt.fill_(float(dt))
        self.cfl = cfl
        self.dt_max = dt_max
        self.smax = torch.zeros(n, dtype=torch.float64, device=dev)
        self.zchunk = zchunk
        scalars = scalars or [{}] * n
        m = self.prog.spec["state_fields"]
        self.ws = [self.prog.workspace(s) for s in self.states]
        self.stage_launches = []
        for k in range(len(self.prog.table)):
            per = []
            for g, (st, ws) in enumerate(zip(self.states, self.ws)):
                bufs = dict(ws)
                bufs["u"] = st[:m]
                inputs, outputs = self.prog.stage_io(k, bufs, st[m:])
                per.append({"inputs": inputs, "outputs": outputs,
                            "scalars": self.prog._scalars(scalars[g]),
                            "dyn": self.dt.data_ptr() + 8 * g, "bc_odd": bc_odd})
            kern = self.prog.kernel(k)
            self.stage_launches.append(BatchLaunch(kern, per, self.prog.spec["halo"],
                                                   zchunk=zchunk or batch_zchunk(kern),
                                                   bc_value=bc_value))
        self.speed_launch = None
        if cfl is not None:
            speed_program, scale, self.cfl_number = cfl
            self.scale = torch.as_tensor(scale, dtype=torch.float64, device=dev)
            per = [{"inputs": list(st[:m]), "outputs": [], "red": self.smax.data_ptr() + 8 * g}
                   for g, st in enumerate(self.states)]
            kern = speed_program.kernel("main")
            self.speed_launch = BatchLaunch(kern, per, speed_program.spec["halo"],
                                            zchunk=zchunk or batch_zchunk(kern))
        last_out = self.prog.table[-1][7]
        if last_out != "u":
            raise NotImplementedError("batched stepping needs a method whose last stage writes "
                                      "the state (rk2, rk4, ssprk3)")

    def update_dt(self, stream=None) -> None:
        if self.speed_launch is not None:
            self.speed_launch.launch(stream)
            native.cfl_update(self.smax, self.scale, self.cfl_number, self.dt, self.dt_max, stream)

    def step(self, stream=None) -> None:
        self.update_dt(stream)
        for bl in self.stage_launches:
            bl.launch(stream)

    def launches_per_step(self) -> int:
        return len(self.stage_launches) + (2 if self.speed_launch is not None else 0)

    def capture(self, steps: int):
        """A CUDA graph of ``steps`` steps (replay with ``graph.replay()``)."""
        import torch

        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            for _ in range(steps):
                self.step(s)
        return g


__all__ = ["RKProgram", "RKBatch", "BatchLaunch", "pack_grids", "batch_zchunk"]
