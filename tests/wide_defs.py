"""Wide and very wide stencils for the engine's next tier: dense boxes of
radius r (27 and 125 points) generated as Python source with coefficients by
distance class, and a compressible-flow style update reading eight fields and
writing five through compile_fused.  The box bodies are written grouped by
coefficient, the way a person writes them, so the DSL's term order is the
grouped order."""

from __future__ import annotations

import importlib.util
import os
import tempfile
from itertools import product


def _idx(name: str, off: int) -> str:
    return name if off == 0 else (f"{name} + {off}" if off > 0 else f"{name} - {-off}")


def box_source(name: str, radius: int, ndim: int = 3, decorated: bool = True,
               dtype: str = "float64") -> str:
    """Source of a dense (2r+1)^ndim box stencil; the coefficient of an
    offset depends on its squared distance d2: 0.3 / (2 + 3 * d2), rounded to
    4 decimals, and the terms of one class are summed together."""
    idx = ["i", "j", "k"][:ndim]
    classes: dict = {}
    for off in product(range(-radius, radius + 1), repeat=ndim):
        d2 = sum(o * o for o in off)
        classes.setdefault(d2, []).append(off)
    groups = []
    for d2 in sorted(classes):
        c = round(0.3 / (2 + 3 * d2), 4)
        acc = " + ".join("u[" + ", ".join(_idx(v, o) for v, o in zip(idx, off)) + "]"
                         for off in classes[d2])
        groups.append(f"{c!r} * ({acc})")
    body = "\n        + ".join(groups)
    head = "from cutile import stencil\n\n\n"
    dec = f"@stencil(ndim={ndim}, order={2 * radius}, dtype={dtype!r})\n" if decorated else ""
    return (f"{head}{dec}def {name}(u, {', '.join(idx)}):\n"
            f"    return ({body})\n")


def load_box(name: str, radius: int, ndim: int = 3, decorated: bool = True,
             dtype: str = "float64", directory: str | None = None):
    """The box stencil as a function (decorated: a ``@stencil`` object)."""
    directory = directory or tempfile.mkdtemp(prefix="wide_defs_")
    path = os.path.join(directory, f"{name}.py")
    with open(path, "w") as f:
        f.write(box_source(name, radius, ndim, decorated, dtype))
    spec = importlib.util.spec_from_file_location(f"wide_{name}_{os.getpid()}", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return getattr(mod, name)


# Compressible-flow style explicit update: density, three momenta and total
# energy advanced by central flux differences, with pressure p, temperature t
# and viscosity mu as auxiliary fields (eight fields in, five out).
C_DT = 0.05     # dt / (2 dx)
C_VIS = 0.01    # dt / dx^2


def cns_rho(rho, mx, my, mz, i, j, k):
    return rho[i, j, k] - C_DT * ((mx[i + 1, j, k] - mx[i - 1, j, k])
                                  + (my[i, j + 1, k] - my[i, j - 1, k])
                                  + (mz[i, j, k + 1] - mz[i, j, k - 1]))


def cns_mx(rho, mx, my, mz, p, mu, i, j, k):
    fe = mx[i + 1, j, k] * mx[i + 1, j, k] / rho[i + 1, j, k] + p[i + 1, j, k]
    fw = mx[i - 1, j, k] * mx[i - 1, j, k] / rho[i - 1, j, k] + p[i - 1, j, k]
    gn = mx[i, j + 1, k] * my[i, j + 1, k] / rho[i, j + 1, k]
    gs = mx[i, j - 1, k] * my[i, j - 1, k] / rho[i, j - 1, k]
    hu = mx[i, j, k + 1] * mz[i, j, k + 1] / rho[i, j, k + 1]
    hd = mx[i, j, k - 1] * mz[i, j, k - 1] / rho[i, j, k - 1]
    lap = (mx[i + 1, j, k] + mx[i - 1, j, k] + mx[i, j + 1, k] + mx[i, j - 1, k]
           + mx[i, j, k + 1] + mx[i, j, k - 1] - 6.0 * mx[i, j, k])
    return mx[i, j, k] - C_DT * ((fe - fw) + (gn - gs) + (hu - hd)) + C_VIS * mu[i, j, k] * lap


def cns_my(rho, mx, my, mz, p, mu, i, j, k):
    fe = my[i + 1, j, k] * mx[i + 1, j, k] / rho[i + 1, j, k]
    fw = my[i - 1, j, k] * mx[i - 1, j, k] / rho[i - 1, j, k]
    gn = my[i, j + 1, k] * my[i, j + 1, k] / rho[i, j + 1, k] + p[i, j + 1, k]
    gs = my[i, j - 1, k] * my[i, j - 1, k] / rho[i, j - 1, k] + p[i, j - 1, k]
    hu = my[i, j, k + 1] * mz[i, j, k + 1] / rho[i, j, k + 1]
    hd = my[i, j, k - 1] * mz[i, j, k - 1] / rho[i, j, k - 1]
    lap = (my[i + 1, j, k] + my[i - 1, j, k] + my[i, j + 1, k] + my[i, j - 1, k]
           + my[i, j, k + 1] + my[i, j, k - 1] - 6.0 * my[i, j, k])
    return my[i, j, k] - C_DT * ((fe - fw) + (gn - gs) + (hu - hd)) + C_VIS * mu[i, j, k] * lap


def cns_mz(rho, mx, my, mz, p, mu, i, j, k):
    fe = mz[i + 1, j, k] * mx[i + 1, j, k] / rho[i + 1, j, k]
    fw = mz[i - 1, j, k] * mx[i - 1, j, k] / rho[i - 1, j, k]
    gn = mz[i, j + 1, k] * my[i, j + 1, k] / rho[i, j + 1, k]
    gs = mz[i, j - 1, k] * my[i, j - 1, k] / rho[i, j - 1, k]
    hu = mz[i, j, k + 1] * mz[i, j, k + 1] / rho[i, j, k + 1] + p[i, j, k + 1]
    hd = mz[i, j, k - 1] * mz[i, j, k - 1] / rho[i, j, k - 1] + p[i, j, k - 1]
    lap = (mz[i + 1, j, k] + mz[i - 1, j, k] + mz[i, j + 1, k] + mz[i, j - 1, k]
           + mz[i, j, k + 1] + mz[i, j, k - 1] - 6.0 * mz[i, j, k])
    return mz[i, j, k] - C_DT * ((fe - fw) + (gn - gs) + (hu - hd)) + C_VIS * mu[i, j, k] * lap


def cns_e(rho, mx, my, mz, e, p, t, mu, i, j, k):
    fe = (e[i + 1, j, k] + p[i + 1, j, k]) * mx[i + 1, j, k] / rho[i + 1, j, k]
    fw = (e[i - 1, j, k] + p[i - 1, j, k]) * mx[i - 1, j, k] / rho[i - 1, j, k]
    gn = (e[i, j + 1, k] + p[i, j + 1, k]) * my[i, j + 1, k] / rho[i, j + 1, k]
    gs = (e[i, j - 1, k] + p[i, j - 1, k]) * my[i, j - 1, k] / rho[i, j - 1, k]
    hu = (e[i, j, k + 1] + p[i, j, k + 1]) * mz[i, j, k + 1] / rho[i, j, k + 1]
    hd = (e[i, j, k - 1] + p[i, j, k - 1]) * mz[i, j, k - 1] / rho[i, j, k - 1]
    lap_t = (t[i + 1, j, k] + t[i - 1, j, k] + t[i, j + 1, k] + t[i, j - 1, k]
             + t[i, j, k + 1] + t[i, j, k - 1] - 6.0 * t[i, j, k])
    return e[i, j, k] - C_DT * ((fe - fw) + (gn - gs) + (hu - hd)) + C_VIS * mu[i, j, k] * lap_t


CNS_FIELDS = ["rho", "mx", "my", "mz", "e", "p", "t", "mu"]
CNS_MEMBERS = [cns_rho, cns_mx, cns_my, cns_mz, cns_e]


def cns_init(n: int, seed: int = 7, halo=(1, 1, 1), dtype="float64"):
    """Positive density, pressure, temperature and viscosity near 1, small
    momenta, energy near 2.5 (seeded)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    shape = tuple(n + 2 * h for h in halo)
    base = {"rho": 1.0, "mx": 0.0, "my": 0.0, "mz": 0.0, "e": 2.5, "p": 1.0, "t": 1.0,
            "mu": 1.0}
    amp = {"rho": 0.1, "mx": 0.05, "my": 0.05, "mz": 0.05, "e": 0.1, "p": 0.1, "t": 0.1,
           "mu": 0.1}
    out = {}
    for name in CNS_FIELDS:
        a = np.full(shape, base[name])
        a = a + amp[name] * (rng.random(shape) - 0.5)
        out[name] = a.astype(dtype)
    return out
