"""B200-native stencil DSL: ``@stencil`` functions compiled to sm_100a CUDA.

Drop-in for the reference package's public API (cutile/__init__.py:9-17):
``stencil, compile, compile_fused, Pipeline, RKIntegrator, BoundarySpec,
maximum, minimum, where`` (plus ``sqrt``).
"""

from cutile.frontend.decorator import stencil
from cutile.frontend.elementwise import maximum, minimum, sqrt, where
from cutile.frontend.types import BoundarySpec
from cutile.runtime.launcher import compile, compile_fused, load_aot
from cutile.runtime.pipeline import Pipeline


def __getattr__(name):
    if name == "RKIntegrator":
        from cutile.runtime.rk_integrator import RKIntegrator

        return RKIntegrator
    raise AttributeError(name)


__all__ = ["stencil", "compile", "compile_fused", "load_aot", "Pipeline", "RKIntegrator", "BoundarySpec",
           "maximum", "minimum", "where", "sqrt"]
