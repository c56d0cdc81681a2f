"""A small SSA IR: attributes, types, values, operations, blocks and regions.

The reference builds its three dialects on xDSL (cutile/dialects/*/dialect.py,
cutile/frontend/parser.py:15-36).  This module provides the subset of that
object model the stencil compiler needs, with the same spelling where callers
touch it (``.data`` on attributes, ``op.attributes`` / ``op.properties``,
``module.walk()``, ``module.clone()``, ``str(module)``, ``Block.args``,
``Region.blocks``), so passes and tests read like the reference's.

Ops are generic: an ``Operation`` has a name, operands, results, properties,
attributes and regions.  Dialect modules subclass it to add typed accessors.
"""

from __future__ import annotations

import itertools
from dataclasses import dataclass
from typing import Any, Iterable, Iterator, Sequence


# --------------------------------------------------------------------------- #
# Attributes
# --------------------------------------------------------------------------- #


class Attribute:
    """Base class of IR attributes; immutable value objects."""

    name = "attr"

    def __eq__(self, other):
        return type(self) is type(other) and self._key() == other._key()

    def __hash__(self):
        return hash((type(self).__name__, self._key()))

    def _key(self):  # pragma: no cover - overridden
        return ()

    def __repr__(self):
        return self.print()

    def print(self) -> str:  # pragma: no cover - overridden
        return self.name


class IntAttr(Attribute):
    name = "builtin.int"

    def __init__(self, data: int):
        self.data = int(data)

    def _key(self):
        return (self.data,)

    def print(self) -> str:
        return str(self.data)


class StringAttr(Attribute):
    name = "builtin.string"

    def __init__(self, data: str):
        self.data = str(data)

    def _key(self):
        return (self.data,)

    def print(self) -> str:
        return '"' + self.data.replace("\\", "\\\\").replace('"', '\\"') + '"'


class _FloatData:
    __slots__ = ("data",)

    def __init__(self, data: float):
        self.data = data


class FloatType(Attribute):
    """``f32`` / ``f64`` element types."""

    def __init__(self, width: int):
        self.width = width
        self.name = f"f{width}"

    def _key(self):
        return (self.width,)

    def print(self) -> str:
        return self.name

    @property
    def bytes(self) -> int:
        return self.width // 8


f32 = FloatType(32)
f64 = FloatType(64)


class IndexType(Attribute):
    name = "index"

    def _key(self):
        return ()

    def print(self) -> str:
        return "index"


class IntegerType(Attribute):
    """``i1`` for comparison results."""

    def __init__(self, width: int):
        self.width = width
        self.name = f"i{width}"

    def _key(self):
        return (self.width,)

    def print(self) -> str:
        return self.name


i1 = IntegerType(1)


class FloatAttr(Attribute):
    """A float constant with its element type.  ``.value.data`` is the Python
    float (the reference reads constants that way, stencil_to_target.py:200-202)."""

    name = "builtin.float"

    def __init__(self, value: float, type: FloatType = f64):
        self.value = _FloatData(float(value))
        self.type = type

    @property
    def data(self) -> float:
        return self.value.data

    def _key(self):
        return (self.value.data, self.type)

    def print(self) -> str:
        return f"{self.value.data!r} : {self.type.print()}"


class ArrayAttr(Attribute):
    name = "builtin.array"

    def __init__(self, data: Iterable[Attribute]):
        self.data = tuple(data)

    def __iter__(self):
        return iter(self.data)

    def __len__(self):
        return len(self.data)

    def __getitem__(self, k):
        return self.data[k]

    def _key(self):
        return self.data

    def print(self) -> str:
        return "[" + ", ".join(a.print() for a in self.data) + "]"


class DictionaryAttr(Attribute):
    name = "builtin.dict"

    def __init__(self, data: dict):
        self.data = dict(data)

    def _key(self):
        return tuple(sorted(self.data.items(), key=lambda kv: kv[0]))

    def print(self) -> str:
        return "{" + ", ".join(f"{k} = {v.print()}" for k, v in self.data.items()) + "}"


class IndexAttr(Attribute):
    """Stencil offset ``<[-1, 0]>`` (xdsl.dialects.stencil.IndexAttr)."""

    name = "stencil.index"

    def __init__(self, offsets: Sequence[int]):
        self.offsets = tuple(int(o) for o in offsets)
        # xDSL layout: ``parameters[0].data`` is the tuple of IntAttr offsets
        self.parameters = (ArrayAttr([IntAttr(o) for o in self.offsets]),)

    @classmethod
    def from_indices(cls, *offsets: int) -> "IndexAttr":
        return cls(offsets)

    def __iter__(self):
        return iter(self.offsets)

    def __len__(self):
        return len(self.offsets)

    def _key(self):
        return self.offsets

    def print(self) -> str:
        return "<[" + ", ".join(str(o) for o in self.offsets) + "]>"


class TempType(Attribute):
    """``!stencil.temp<?x?xf64>``: an N-D field temporary."""

    name = "stencil.temp"

    def __init__(self, ndim: int, element_type: FloatType):
        self.ndim = int(ndim)
        self.element_type = element_type

    def _key(self):
        return (self.ndim, self.element_type)

    def print(self) -> str:
        return "!stencil.temp<" + "x".join(["?"] * self.ndim) + "x" + self.element_type.print() + ">"


class FunctionType(Attribute):
    name = "builtin.function_type"

    def __init__(self, inputs: Sequence[Attribute], outputs: Sequence[Attribute]):
        self.inputs = tuple(inputs)
        self.outputs = tuple(outputs)

    @classmethod
    def from_lists(cls, inputs, outputs) -> "FunctionType":
        return cls(inputs, outputs)

    def _key(self):
        return (self.inputs, self.outputs)

    def print(self) -> str:
        return ("(" + ", ".join(t.print() for t in self.inputs) + ") -> ("
                + ", ".join(t.print() for t in self.outputs) + ")")


class FileLineColLoc(Attribute):
    """Source location of an op (file, line, column)."""

    name = "loc"

    def __init__(self, filename: str, line: int, col: int):
        self.filename = StringAttr(filename)
        self.line = IntAttr(line)
        self.col = IntAttr(col)

    def _key(self):
        return (self.filename.data, self.line.data, self.col.data)

    def print(self) -> str:
        return f'loc("{self.filename.data}":{self.line.data}:{self.col.data})'


def to_attr(value: Any) -> Attribute:
    """Wrap a Python value as an attribute (ints, floats, strings, sequences)."""
    if isinstance(value, Attribute):
        return value
    if isinstance(value, bool):
        return IntAttr(int(value))
    if isinstance(value, int):
        return IntAttr(value)
    if isinstance(value, float):
        return FloatAttr(value, f64)
    if isinstance(value, str):
        return StringAttr(value)
    if isinstance(value, dict):
        return DictionaryAttr({k: to_attr(v) for k, v in value.items()})
    if isinstance(value, (list, tuple)):
        return ArrayAttr(to_attr(v) for v in value)
    raise TypeError(f"cannot convert {value!r} to an attribute")


# --------------------------------------------------------------------------- #
# Values, blocks, regions, operations
# --------------------------------------------------------------------------- #


class SSAValue:
    """A value defined by an op result or a block argument."""

    __slots__ = ("type", "owner", "index", "uses")

    def __init__(self, type: Attribute, owner, index: int):
        self.type = type
        self.owner = owner
        self.index = index
        self.uses: list = []

    def __repr__(self):
        return f"<SSAValue {self.type.print()} #{self.index} of {getattr(self.owner, 'name', 'block')}>"


class BlockArgument(SSAValue):
    __slots__ = ()


class OpResult(SSAValue):
    __slots__ = ()


class Block:
    def __init__(self, ops: Iterable["Operation"] = (), arg_types: Sequence[Attribute] = ()):
        self._args: list[BlockArgument] = []
        self._ops: list[Operation] = []
        self.parent: Region | None = None
        for t in arg_types:
            self.insert_arg(t, len(self._args))
        for op in ops:
            self.add_op(op)

    @property
    def args(self) -> tuple[BlockArgument, ...]:
        return tuple(self._args)

    @property
    def ops(self) -> tuple["Operation", ...]:
        return tuple(self._ops)

    @property
    def first_op(self):
        return self._ops[0] if self._ops else None

    def insert_arg(self, type: Attribute, index: int) -> BlockArgument:
        arg = BlockArgument(type, self, index)
        self._args.insert(index, arg)
        for k, a in enumerate(self._args):
            a.index = k
        return arg

    def add_op(self, op: "Operation") -> None:
        if op.parent is not None:
            raise ValueError(f"op {op.name} already has a parent block")
        op.parent = self
        self._ops.append(op)

    def add_ops(self, ops: Iterable["Operation"]) -> None:
        for op in ops:
            self.add_op(op)

    def detach_op(self, op: "Operation") -> "Operation":
        self._ops.remove(op)
        op.parent = None
        return op

    def walk(self) -> Iterator["Operation"]:
        for op in list(self._ops):
            yield from op.walk()

    def parent_op(self):
        return self.parent.parent if self.parent is not None else None


class Region:
    def __init__(self, blocks: Block | Iterable[Block] = ()):
        if isinstance(blocks, Block):
            blocks = [blocks]
        self._blocks: list[Block] = []
        self.parent: Operation | None = None
        for b in blocks:
            self.add_block(b)

    @property
    def blocks(self) -> tuple[Block, ...]:
        return tuple(self._blocks)

    @property
    def block(self) -> Block:
        return self._blocks[0]

    def add_block(self, b: Block) -> None:
        b.parent = self
        self._blocks.append(b)

    def walk(self) -> Iterator["Operation"]:
        for b in self._blocks:
            yield from b.walk()


_ids = itertools.count()


class Operation:
    """Generic op.  Subclasses set ``name`` and may add typed accessors."""

    name = "builtin.unregistered"

    def __init__(
        self,
        operands: Sequence[SSAValue] = (),
        result_types: Sequence[Attribute] = (),
        properties: dict | None = None,
        attributes: dict | None = None,
        regions: Sequence[Region] = (),
    ):
        self.operands: tuple[SSAValue, ...] = tuple(_as_value(o) for o in operands)
        for o in self.operands:
            o.uses.append(self)
        self.results: tuple[OpResult, ...] = tuple(
            OpResult(t, self, k) for k, t in enumerate(result_types))
        self.properties: dict[str, Attribute] = {
            k: to_attr(v) for k, v in (properties or {}).items() if v is not None}
        self.attributes: dict[str, Attribute] = {
            k: to_attr(v) for k, v in (attributes or {}).items() if v is not None}
        self.regions: tuple[Region, ...] = tuple(regions)
        for r in self.regions:
            r.parent = self
        self.parent: Block | None = None
        self.location: FileLineColLoc | None = None
        self._uid = next(_ids)

    # -- convenience ------------------------------------------------------
    @property
    def result(self) -> OpResult:
        return self.results[0]

    @property
    def res(self) -> OpResult:
        return self.results[0]

    @property
    def body(self) -> Region:
        return self.regions[0]

    def prop(self, key: str, default=None):
        a = self.properties.get(key)
        return default if a is None else a

    def walk(self) -> Iterator["Operation"]:
        yield self
        for r in self.regions:
            yield from r.walk()

    def parent_block(self) -> Block | None:
        return self.parent

    def parent_op(self) -> "Operation | None":
        if self.parent is None or self.parent.parent is None:
            return None
        return self.parent.parent.parent

    def detach(self) -> "Operation":
        if self.parent is not None:
            self.parent.detach_op(self)
        return self

    def erase(self) -> None:
        self.detach()
        for o in self.operands:
            if self in o.uses:
                o.uses.remove(self)

    def clone(self, value_map: dict | None = None) -> "Operation":
        """Deep copy, remapping operands through *value_map* (filled in with
        the clone's results and block arguments)."""
        if value_map is None:
            value_map = {}
        new = object.__new__(type(self))
        new.operands = tuple(value_map.get(o, o) for o in self.operands)
        for o in new.operands:
            o.uses.append(new)
        new.results = tuple(OpResult(r.type, new, r.index) for r in self.results)
        for old, nr in zip(self.results, new.results):
            value_map[old] = nr
        new.properties = dict(self.properties)
        new.attributes = dict(self.attributes)
        new.parent = None
        new.location = self.location
        new._uid = next(_ids)
        regions = []
        for r in self.regions:
            nr = Region()
            for b in r.blocks:
                nb = Block()
                for a in b.args:
                    value_map[a] = nb.insert_arg(a.type, a.index)
                nr.add_block(nb)
            for b, nb in zip(r.blocks, nr.blocks):
                for op in b.ops:
                    nb.add_op(op.clone(value_map))
            regions.append(nr)
        new.regions = tuple(regions)
        for r in new.regions:
            r.parent = new
        for k, v in vars(self).items():
            if k not in new.__dict__:
                new.__dict__[k] = v
        return new

    def __str__(self) -> str:
        from cutile.ir.printer import Printer

        return Printer().print_op_to_string(self)

    def __repr__(self) -> str:
        return f"<{self.name} op>"

    # Subclasses may override to print a custom form (``name`` + rest).
    def print_custom(self, printer) -> str | None:
        return None


def _as_value(v) -> SSAValue:
    if isinstance(v, SSAValue):
        return v
    if isinstance(v, Operation):
        return v.results[0]
    raise TypeError(f"expected an SSA value, got {v!r}")


class ModuleOp(Operation):
    """``builtin.module``: a single-block region of top-level ops."""

    name = "builtin.module"

    def __init__(self, ops: Region | Iterable[Operation] = ()):
        if isinstance(ops, Region):
            region = ops
        else:
            region = Region(Block(list(ops)))
        super().__init__(regions=[region])

    @property
    def ops(self) -> tuple[Operation, ...]:
        return self.body.block.ops


class Context:
    """Pass context (kept for the ``apply(ctx, module)`` signature)."""


class ModulePass:
    """Base class of passes: ``apply(ctx, module)`` mutates the module."""

    name = "pass"

    def apply(self, ctx: Context, op: ModuleOp) -> None:  # pragma: no cover
        raise NotImplementedError
