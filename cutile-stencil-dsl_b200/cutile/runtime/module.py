"""Runtime behind a generated stencil module.

The reference's generated module is cuTile Python with ``launch_<name>``
(stencil_to_target.py:650-843), ``apply_boundary_<name>``
(target_to_python.py:199-297) and, for bricked layouts,
``launch_<name>_bricked`` (multigpu_emitter.py:426-473).  Here the generated
module is a small Python file whose functions call a ``StencilProgram``: it
holds the CUDA source, JIT-loads it per device through libcsd, checks the
arrays against the kernel's contract and launches on the caller's stream.
"""

from __future__ import annotations

import threading

from cutile.runtime import native

_DTYPES = {"float64": "torch.float64", "float32": "torch.float32"}


class StencilProgram:
    """Launchable stencil kernels of one generated module.

    ``spec`` keys: ``name``, ``ndim``, ``dtype``, ``halo`` (array halo),
    ``stencil_halo``, ``inputs`` (count), ``outputs``, ``temporal_steps``,
    ``boundary`` (dict or None), ``kernels`` (entry names in the source:
    ``main`` and optionally ``fused_bc``), ``zchunk``.
    """

    def __init__(self, cuda_source: str, spec: dict, cubin: str | None = None,
                 cubin_sha256: str | None = None):
        self.source = cuda_source
        self.spec = dict(spec)
        # a prebuilt cubin of ``cuda_source`` (ahead-of-time build) replaces the
        # NVRTC compile; it is checked against its recorded hash at load
        self.cubin = cubin
        self.cubin_sha256 = cubin_sha256
        self._modules: dict[int, native.NativeModule] = {}
        self._lock = threading.Lock()

    # -- loading -------------------------------------------------------------
    def _module(self) -> native.NativeModule:
        import torch

        if not torch.cuda.is_available():
            raise native.CsdError("no CUDA device: the B200 stencil backend has no CPU fallback")
        dev = torch.cuda.current_device()
        with self._lock:
            m = self._modules.get(dev)
            if m is None:
                torch.cuda.init()
                if self.cubin is not None:
                    m = native.NativeModule(self.source, image=native.read_image(
                        self.cubin, self.cubin_sha256))
                else:
                    m = native.NativeModule(self.source)
                self._modules[dev] = m
        return m

    def kernel(self, which: str = "main") -> native.NativeKernel:
        return self._module().kernel(self.spec["kernels"][which])

    # -- checks --------------------------------------------------------------
    def _check(self, arrays, role: str) -> None:
        import torch

        want = torch.float64 if self.spec["dtype"] in ("float64", "fp64") else torch.float32
        ndim = self.spec["ndim"]
        shape = None
        for a in arrays:
            if not isinstance(a, torch.Tensor):
                raise TypeError(f"{role} arrays must be torch CUDA tensors, got {type(a).__name__}")
            if a.dtype != want:
                raise TypeError(f"{self.spec['name']}: {role} dtype {a.dtype} does not match the "
                                f"compiled dtype {want}")
            if a.dim() != ndim:
                raise ValueError(f"{self.spec['name']}: expected {ndim}-D arrays, got {a.dim()}-D")
            if shape is None:
                shape = tuple(a.shape)
            elif tuple(a.shape) != shape:
                raise ValueError(f"{self.spec['name']}: all arrays must share one shape")
        for n, h in zip(shape, self.spec["halo"]):
            if n - 2 * h < 1:
                raise ValueError(f"{self.spec['name']}: extent {n} leaves no interior with halo {h}")

    # -- entry points --------------------------------------------------------
    def scalar_values(self, scalars: dict | None) -> list:
        names = self.spec.get("scalars", [])
        scalars = scalars or {}
        missing = [n for n in names if n not in scalars]
        if missing:
            raise TypeError(f"{self.spec['name']}: missing scalar parameter(s) {missing}")
        extra = set(scalars) - set(names)
        if extra:
            raise TypeError(f"{self.spec['name']}: unknown scalar parameter(s) {sorted(extra)}")
        return [float(scalars[n]) for n in names]

    def launch(self, inputs, outputs, stream=None, *, zchunk: int = 0, grid: int = 0,
               loader: int = -1, scalars: dict | None = None, which: str = "main",
               dyn=None, red=None, bc_odd=(), timeout_ns: int = 0,
               withhold_chunk: int = 0) -> None:
        """``launch_<name>``: ``temporal_steps`` steps from ``inputs`` into the
        interiors of ``outputs`` (halos untouched).

        ``timeout_ns`` bounds every device wait for input (0: 2 s); a wait
        that runs out stops its CTA and sets the device error word
        (``native.error_word``).  ``withhold_chunk`` is the failure-test hook
        of ``csd_launch_opts`` (one input chunk of CTA 0 is never requested)."""
        self._check(list(inputs) + list(outputs), "stencil")
        if len(inputs) != self.spec["inputs"] or len(outputs) != self.spec["outputs"]:
            raise TypeError(f"launch_{self.spec['name']} takes {self.spec['inputs']} input(s) and "
                            f"{self.spec['outputs']} output(s)")
        for o in outputs:
            for i in inputs:
                if o.data_ptr() == i.data_ptr():
                    raise ValueError("outputs must not alias inputs (the kernel reads neighbours)")
        native.launch(self.kernel(which), inputs, outputs, self.spec["halo"], stream,
                      zchunk=zchunk, grid=grid, loader=loader,
                      scalars=self.scalar_values(scalars), dyn=dyn, red=red, bc_odd=bc_odd,
                      timeout_ns=timeout_ns, withhold_chunk=withhold_chunk)

    def step(self, inputs, outputs, stream=None, *, scalars: dict | None = None, **kw) -> None:
        """One step with the declared boundary condition fused into staging:
        ``out = stencil(apply_boundary(in))`` without writing the inputs' halos."""
        if "fused_bc" not in self.spec["kernels"]:
            raise ValueError(f"{self.spec['name']} declares no boundary condition")
        self._check(list(inputs) + list(outputs), "stencil")
        bc = self.spec["boundary"] or {}
        native.launch(self.kernel("fused_bc"), inputs, outputs, self.spec["halo"], stream,
                      bc_value=float(bc.get("value", 0.0)),
                      scalars=self.scalar_values(scalars), **kw)

    def reduce(self, inputs, out=None, stream=None, scalars: dict | None = None):
        """Max-reduce the body over the interior into the device scalar ``out``."""
        import torch

        self._check(list(inputs), "reduction")
        if out is None:
            out = torch.zeros((), dtype=torch.float64, device=inputs[0].device)
        native.launch(self.kernel("main"), inputs, [], self.spec["halo"], stream,
                      scalars=self.scalar_values(scalars), red=out)
        return out

    # -- graph-captured time loops --------------------------------------------
    def capture_steps(self, set_a, set_b, steps: int, *, boundary: bool = False,
                      scalars: dict | None = None):
        """A CUDA graph of ``steps`` launches that ping-pong between two field
        sets: step k reads set ``a`` (k even) or ``b`` and writes the other, so
        after an even count the state is back in ``set_a``.  ``boundary``
        launches the fused-boundary kernel (``step_<name>``).  Replay with
        ``graph.replay()``; the launches are the eager ones, so results are
        bit-identical to calling them in a loop."""
        import torch

        set_a, set_b = list(set_a), list(set_b)
        nin, nout = self.spec["inputs"], self.spec["outputs"]
        if len(set_a) != nin or len(set_b) != nin or nin != nout:
            raise ValueError(f"{self.spec['name']}: a ping-pong loop needs as many outputs as "
                             f"inputs and two sets of {nin} field(s)")
        run = self.step if boundary else self.launch
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):       # load the module outside the capture
            run(set_a, set_b, side, scalars=scalars)
        side.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=side):
            cur, nxt = set_a, set_b
            for _ in range(steps):
                run(cur, nxt, side, scalars=scalars)
                cur, nxt = nxt, cur
        # the graph holds raw addresses: keep the fields alive with it
        graph.csd_fields = (tuple(set_a), tuple(set_b))
        return graph

    # -- bricked layout ------------------------------------------------------
    def _brick(self, brick_size) -> int:
        bs = int(brick_size)
        if self.spec.get("layout") != "bricked" or "bricked" not in self.spec["kernels"]:
            raise ValueError(f"{self.spec['name']} was not compiled with layout='bricked'")
        if bs != self.spec["brick_size"]:
            raise ValueError(f"{self.spec['name']}: compiled for brick size "
                             f"{self.spec['brick_size']}, got {bs}")
        return bs

    def to_bricks(self, flat, brick_size, stream=None):
        return native.to_bricks(flat, int(brick_size), stream)

    def from_bricks(self, bricked, shape, brick_size, stream=None):
        return native.from_bricks(bricked, shape, int(brick_size), stream=stream)

    def launch_on_bricks(self, inputs, outputs, shape, stream=None, *,
                         scalars: dict | None = None, loader: int = -1, zchunk: int = 0,
                         halo=None) -> None:
        """The bricked kernel on bricked fields of a ``shape`` array: writes
        the interior cells of the outputs' bricks (halo and padding cells
        untouched).  ``loader``: -1 picks TMA brick staging where the kernel
        has it, else per-group cp.async copies.  ``halo``: the arrays' halo
        widths when they differ from the compiled ``halo_widths`` (each at
        least the stencil's reach); a halo of whole bricks starts the
        interior on a brick, so that every column tile of the TMA staging
        holds interior points."""
        bs = self._brick(self.spec["brick_size"])
        shape = tuple(int(n) for n in shape)
        if len(shape) != self.spec["ndim"]:
            raise ValueError(f"{self.spec['name']}: expected a {self.spec['ndim']}-D shape")
        if len(inputs) != self.spec["inputs"] or len(outputs) != self.spec["outputs"]:
            raise TypeError(f"{self.spec['name']} takes {self.spec['inputs']} input(s) and "
                            f"{self.spec['outputs']} output(s)")
        for o in outputs:
            for i in inputs:
                if o.data_ptr() == i.data_ptr():
                    raise ValueError("outputs must not alias inputs (the kernel reads neighbours)")
        want = "float64" if self.spec["dtype"] in ("float64", "fp64") else "float32"
        for t in list(inputs) + list(outputs):
            if str(t.dtype).replace("torch.", "") != want:
                raise TypeError(f"{self.spec['name']}: bricked field dtype {t.dtype} does not "
                                f"match the compiled dtype {want}")
        fin = [native.bricked_field(t, shape, bs) for t in inputs]
        fout = [native.bricked_field(t, shape, bs) for t in outputs]
        halo = list(self.spec["halo"]) if halo is None else [int(h) for h in halo]
        if len(halo) != len(shape):
            raise ValueError(f"{self.spec['name']}: halo {halo} does not match the {len(shape)}-D "
                             "shape")
        native.launch_fields(self.kernel("bricked"), fin, fout, halo, stream,
                             loader=loader, zchunk=zchunk, scalars=self.scalar_values(scalars))

    def launch_bricked(self, inputs, outputs, brick_size, stream=None, *,
                       scalars: dict | None = None) -> None:
        """``launch_<name>_bricked`` (multigpu_emitter.py:426-473): flat in,
        flat out; every output is overwritten whole, interior with the
        result and halo with zeros, as the reference's write-back of the
        bricked result does."""
        bs = self._brick(brick_size)
        self._check(list(inputs) + list(outputs), "stencil")
        shape = tuple(inputs[0].shape)
        ins = [native.to_bricks(t.contiguous(), bs, stream) for t in inputs]
        outs = [_zeros(native.bricked_shape(shape, bs), o) for o in outputs]
        self.launch_on_bricks(ins, outs, shape, stream, scalars=scalars)
        for o, ob in zip(outputs, outs):
            native.from_bricks(ob, shape, bs, out=o, stream=stream)

    def apply_boundary(self, u, stream=None) -> None:
        """``apply_boundary_<name>(u)``: fill the halo of ``u`` in place."""
        bc = self.spec["boundary"]
        if bc is None:
            raise ValueError(f"{self.spec['name']} declares no boundary condition")
        self._check([u], "boundary")
        native.apply_boundary(u, self.spec["halo"], bc["type"], float(bc.get("value", 0.0)),
                              stream)


def _zeros(shape, like):
    import torch

    return torch.zeros(tuple(shape), dtype=like.dtype, device=like.device)


__all__ = ["StencilProgram"]
