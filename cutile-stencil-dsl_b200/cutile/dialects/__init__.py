"""Stencil dialects: D1 ``cutile_stencil``, D2 ``stencil``, D3 ``cutile`` target,
``layout``, and the ``arith``/``math`` ops used in stencil bodies."""
