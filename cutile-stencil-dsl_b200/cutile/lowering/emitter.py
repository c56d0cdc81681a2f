"""Indentation-aware source builder (reference: cutile/lowering/emitter.py:13-63)."""

from __future__ import annotations

from contextlib import contextmanager
from typing import Iterator


class CodeEmitter:
    def __init__(self, indent_str: str = "    ") -> None:
        self._lines: list[str] = []
        self._indent_str = indent_str
        self._level = 0

    def line(self, text: str = "") -> None:
        self._lines.append(self._indent_str * self._level + text if text else "")

    def blank(self) -> None:
        self._lines.append("")

    @contextmanager
    def indent(self) -> Iterator[None]:
        self._level += 1
        try:
            yield
        finally:
            self._level -= 1

    def render(self) -> str:
        return "\n".join(self._lines) + "\n"
