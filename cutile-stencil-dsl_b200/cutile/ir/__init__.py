"""Minimal SSA IR used by the stencil dialects (stands in for xDSL)."""

from cutile.ir.core import (
    ArrayAttr,
    Attribute,
    Block,
    BlockArgument,
    Context,
    DictionaryAttr,
    FileLineColLoc,
    FloatAttr,
    FloatType,
    FunctionType,
    IndexAttr,
    IndexType,
    IntAttr,
    IntegerType,
    ModuleOp,
    ModulePass,
    OpResult,
    Operation,
    Region,
    SSAValue,
    StringAttr,
    TempType,
    f32,
    f64,
    i1,
    to_attr,
)
from cutile.ir.printer import Printer, print_module

__all__ = [
    "ArrayAttr", "Attribute", "Block", "BlockArgument", "Context", "DictionaryAttr",
    "FileLineColLoc", "FloatAttr", "FloatType", "FunctionType", "IndexAttr", "IndexType",
    "IntAttr", "IntegerType", "ModuleOp", "ModulePass", "OpResult", "Operation", "Region",
    "SSAValue", "StringAttr", "TempType", "f32", "f64", "i1", "to_attr", "Printer",
    "print_module",
]
