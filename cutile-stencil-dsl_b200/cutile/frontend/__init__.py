"""Frontend: Python ``@stencil`` functions to Dialect 1 IR."""

from cutile.frontend.decorator import stencil
from cutile.frontend.parser import parse_stencil

__all__ = ["stencil", "parse_stencil"]
