"""Helpers shared by the dialect definitions."""

from __future__ import annotations

from cutile.ir.core import Attribute, Operation, to_attr


class prop:
    """Descriptor: ``op.<name>`` reads (and assigns) ``op.properties[name]``
    (``None`` when absent), like an xDSL ``prop_def``/``opt_prop_def``."""

    def __init__(self, key: str | None = None):
        self.key = key

    def __set_name__(self, owner, name):
        if self.key is None:
            self.key = name

    def __get__(self, obj, objtype=None):
        if obj is None:
            return self
        return obj.properties.get(self.key)

    def __set__(self, obj, value):
        if value is None:
            obj.properties.pop(self.key, None)
        else:
            obj.properties[self.key] = to_attr(value)


class attr:
    """Descriptor over ``op.attributes[name]`` (an xDSL ``attr_def``)."""

    def __init__(self, key: str | None = None):
        self.key = key

    def __set_name__(self, owner, name):
        if self.key is None:
            self.key = name

    def __get__(self, obj, objtype=None):
        if obj is None:
            return self
        return obj.attributes.get(self.key)

    def __set__(self, obj, value):
        if value is None:
            obj.attributes.pop(self.key, None)
        else:
            obj.attributes[self.key] = to_attr(value)


class Dialect:
    """A named collection of op and attribute classes."""

    def __init__(self, name: str, ops, attributes=()):
        self.name = name
        self.operations = tuple(ops)
        self.attributes = tuple(attributes)

    def __repr__(self):
        return f"Dialect({self.name!r}, {len(self.operations)} ops)"


def build(cls, *, operands=(), result_types=(), properties=None, attributes=None, regions=()):
    """Generic constructor used by ``Op.build(...)`` (xDSL's ``IRDLOperation.build``)."""
    op = object.__new__(cls)
    Operation.__init__(op, operands=operands, result_types=result_types, properties=properties,
                       attributes=attributes, regions=regions)
    return op


class BuildMixin:
    @classmethod
    def build(cls, *, operands=(), result_types=(), properties=None, attributes=None, regions=()):
        flat = []
        for o in operands:
            if isinstance(o, (list, tuple)):
                flat.extend(o)
            else:
                flat.append(o)
        return build(cls, operands=flat, result_types=result_types, properties=properties,
                     attributes=attributes, regions=regions)


__all__ = ["prop", "attr", "Dialect", "build", "BuildMixin", "Attribute"]
