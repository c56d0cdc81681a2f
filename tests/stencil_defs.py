"""Stencil bodies used by the tests, as plain Python functions.

They are shared by the golden-fixture generator (which hands them to the
reference's NumPy executor) and by the tests (which wrap them with
``@stencil``).  The formulas are the configurations' own (heat, 7-point
Laplacian, Gray-Scott, shallow water, upwind advection, leapfrog wave) and
small cases covering every element-wise operation the DSL lowers.
"""

# Constants referenced as module globals (the parser picks up numeric globals).
CFL = 0.5
DU, DV, F_GS, K_GS, DT_GS = 0.16, 0.08, 0.037, 0.06, 1.0
SW_COEFF = 0.01 * 1.0 / (2 * 0.1)
G_COEFF = 0.01 * 9.81 / (2 * 0.1)
WAVE_C = 0.1


def heat1d(u, i):
    return 0.25 * u[i - 1] + 0.5 * u[i] + 0.25 * u[i + 1]


def heat2d(u, i, j):
    return 0.25 * (u[i - 1, j] + u[i + 1, j] + u[i, j - 1] + u[i, j + 1])


def lap7(u, i, j, k):
    return u[i, j, k] + 0.1 * (u[i - 1, j, k] + u[i + 1, j, k] + u[i, j - 1, k] + u[i, j + 1, k]
                               + u[i, j, k - 1] + u[i, j, k + 1] - 6 * u[i, j, k])


def lap3d(u, i, j, k):
    return (u[i - 1, j, k] + u[i + 1, j, k] + u[i, j - 1, k] + u[i, j + 1, k]
            + u[i, j, k - 1] + u[i, j, k + 1]) / 6.0


def lap4_1d(u, i):
    return (-u[i - 2] + 16 * u[i - 1] - 30 * u[i] + 16 * u[i + 1] - u[i + 2]) / 12.0


def advect(u, i):
    return u[i] - CFL * (u[i] - u[i - 1])


def advect2d(u, i, j):
    return u[i, j] - 0.25 * (u[i, j] - u[i - 1, j]) - 0.125 * (u[i, j] - u[i, j - 1])


def wave4(u, i, j):
    return (WAVE_C * (-1 / 12) * u[i - 2, j] + WAVE_C * (4 / 3) * u[i - 1, j]
            + WAVE_C * (-5 / 2) * u[i, j] + WAVE_C * (4 / 3) * u[i + 1, j]
            + WAVE_C * (-1 / 12) * u[i + 2, j] + WAVE_C * (-1 / 12) * u[i, j - 2]
            + WAVE_C * (4 / 3) * u[i, j - 1] + WAVE_C * (-5 / 2) * u[i, j]
            + WAVE_C * (4 / 3) * u[i, j + 1] + WAVE_C * (-1 / 12) * u[i, j + 2])


# Heat diffusion with a small step (alpha * dt / dx^2 = 0.02): each update is
# a tiny fraction of u, which is where a compensated FP32 update pays.
KD_HEAT = 0.02


def heat_small_dt(u, i, j):
    return u[i, j] + KD_HEAT * (u[i - 1, j] + u[i + 1, j] + u[i, j - 1] + u[i, j + 1] - 4.0 * u[i, j])


def heat_bump_init(n: int, halo=(1, 1), dtype="float64"):
    """u = 1 + 0.1 * Gaussian bump (width 0.08) on an n x n interior, zero halo."""
    import numpy as np

    y = (np.arange(n) + 0.5) / n
    r2 = (y[:, None] - 0.5) ** 2 + (y[None, :] - 0.45) ** 2
    u = np.zeros((n + 2 * halo[0], n + 2 * halo[1]))
    u[halo[0]:halo[0] + n, halo[1]:halo[1] + n] = 1.0 + 0.1 * np.exp(-r2 / (2 * 0.08 ** 2))
    return u.astype(dtype)


def leapfrog(u, up, i, j):
    return 2.0 * u[i, j] - up[i, j] + 0.25 * (u[i - 1, j] + u[i + 1, j] + u[i, j - 1]
                                              + u[i, j + 1] - 4.0 * u[i, j])


def gs_u(u, v, i, j):
    return u[i, j] + DT_GS * (DU * (u[i - 1, j] + u[i + 1, j] + u[i, j - 1] + u[i, j + 1]
                                    - 4 * u[i, j]) - u[i, j] * v[i, j] * v[i, j]
                              + F_GS * (1.0 - u[i, j]))


def gs_v(u, v, i, j):
    return v[i, j] + DT_GS * (DV * (v[i - 1, j] + v[i + 1, j] + v[i, j - 1] + v[i, j + 1]
                                    - 4 * v[i, j]) + u[i, j] * v[i, j] * v[i, j]
                              - (F_GS + K_GS) * v[i, j])


def sw_h(h, hu, hv, i, j):
    return h[i, j] - SW_COEFF * (hu[i + 1, j] - hu[i - 1, j]) - SW_COEFF * (hv[i, j + 1] - hv[i, j - 1])


def sw_hu(h, hu, i, j):
    return hu[i, j] - G_COEFF * (h[i + 1, j] - h[i - 1, j])


def update_e(E, H, i):
    return E[i] + (0.005 / (1.0 * 0.01)) * (H[i] - H[i - 1])


def cond3d(u, i, j, k):
    return abs(0.5 * max(u[i, j, k], 0.0) + 0.25 * max(u[i + 1, j, k], 0.0)
               + 0.25 * max(u[i - 1, j, k], 0.0) - 0.125 * min(u[i, j + 1, k], 0.0))


def clip1d(u, i):
    return where(u[i] > 0.5, u[i - 1], u[i + 1]) + where(u[i] <= 0.0, 1.0, 0.0)  # noqa: F821


def box27(u, i, j, k):
    return (0.3 * u[i, j, k]
            + 0.05 * (u[i - 1, j, k] + u[i + 1, j, k] + u[i, j - 1, k] + u[i, j + 1, k]
                      + u[i, j, k - 1] + u[i, j, k + 1])
            + 0.02 * (u[i - 1, j - 1, k] + u[i - 1, j + 1, k] + u[i + 1, j - 1, k]
                      + u[i + 1, j + 1, k] + u[i - 1, j, k - 1] + u[i - 1, j, k + 1]
                      + u[i + 1, j, k - 1] + u[i + 1, j, k + 1] + u[i, j - 1, k - 1]
                      + u[i, j - 1, k + 1] + u[i, j + 1, k - 1] + u[i, j + 1, k + 1])
            + 0.01 * (u[i - 1, j - 1, k - 1] + u[i - 1, j - 1, k + 1] + u[i - 1, j + 1, k - 1]
                      + u[i - 1, j + 1, k + 1] + u[i + 1, j - 1, k - 1] + u[i + 1, j - 1, k + 1]
                      + u[i + 1, j + 1, k - 1] + u[i + 1, j + 1, k + 1]))


# name -> (function, ndim, number of input arrays)
CASES = {
    "heat1d": (heat1d, 1, 1), "heat2d": (heat2d, 2, 1), "lap7": (lap7, 3, 1),
    "lap3d": (lap3d, 3, 1), "lap4_1d": (lap4_1d, 1, 1), "advect": (advect, 1, 1),
    "advect2d": (advect2d, 2, 1), "wave4": (wave4, 2, 1), "leapfrog": (leapfrog, 2, 2),
    "gs_u": (gs_u, 2, 2), "gs_v": (gs_v, 2, 2), "sw_h": (sw_h, 2, 3), "sw_hu": (sw_hu, 2, 2),
    "update_e": (update_e, 1, 2), "cond3d": (cond3d, 3, 1), "clip1d": (clip1d, 1, 1),
    "box27": (box27, 3, 1),
}


# Increments of the Gray-Scott updates (gs_u = u + gs_u_incr, gs_v = v + gs_v_incr);
# the Kahan-compensated FP32 mode adds the increment with compensation.
def gs_u_incr(u, v, i, j):
    return DT_GS * (DU * (u[i - 1, j] + u[i + 1, j] + u[i, j - 1] + u[i, j + 1] - 4 * u[i, j])
                    - u[i, j] * v[i, j] * v[i, j] + F_GS * (1.0 - u[i, j]))


def gs_v_incr(u, v, i, j):
    return DT_GS * (DV * (v[i - 1, j] + v[i + 1, j] + v[i, j - 1] + v[i, j + 1] - 4 * v[i, j])
                    + u[i, j] * v[i, j] * v[i, j] - (F_GS + K_GS) * v[i, j])


def gray_scott_init(n: int, seed: int = 2, halo=(1, 1), dtype="float64"):
    """4096^2-style Gray-Scott start: u=1, v=0, then 20 random 32x32 squares set
    to u=0.5, v=0.25 with +-1% uniform noise (seeded)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    shape = (n + 2 * halo[0], n + 2 * halo[1])
    u = np.ones(shape)
    v = np.zeros(shape)
    for _ in range(20):
        y, x = rng.integers(0, n - 32, size=2)
        sl = (slice(halo[0] + y, halo[0] + y + 32), slice(halo[1] + x, halo[1] + x + 32))
        u[sl] = 0.5 * (1 + rng.uniform(-0.01, 0.01, (32, 32)))
        v[sl] = 0.25 * (1 + rng.uniform(-0.01, 0.01, (32, 32)))
    return u.astype(dtype), v.astype(dtype)


# Nonlinear shallow water (h, hu, hv) on a square grid, x = j (columns),
# y = i (rows): the right-hand side with local Lax-Friedrichs (Rusanov) fluxes
# and the signal speed for the CFL step.  `sqrt` comes from the executor.
G_SW = 9.81


def sw_rhs(h, hu, hv, dx, i, j):
    hC = h[i, j]; huC = hu[i, j]; hvC = hv[i, j]
    hE = h[i, j + 1]; huE = hu[i, j + 1]; hvE = hv[i, j + 1]
    hW = h[i, j - 1]; huW = hu[i, j - 1]; hvW = hv[i, j - 1]
    hN = h[i + 1, j]; huN = hu[i + 1, j]; hvN = hv[i + 1, j]
    hS = h[i - 1, j]; huS = hu[i - 1, j]; hvS = hv[i - 1, j]
    uC = huC / hC; vC = hvC / hC; cC = sqrt(G_SW * hC)  # noqa: F821
    uE = huE / hE; cE = sqrt(G_SW * hE)  # noqa: F821
    uW = huW / hW; cW = sqrt(G_SW * hW)  # noqa: F821
    vN = hvN / hN; cN = sqrt(G_SW * hN)  # noqa: F821
    vS = hvS / hS; cS = sqrt(G_SW * hS)  # noqa: F821
    pC = 0.5 * G_SW * hC * hC
    fuC = huC * uC + pC; fvC = huC * vC
    fuE = huE * uE + 0.5 * G_SW * hE * hE; fvE = hvE * uE
    fuW = huW * uW + 0.5 * G_SW * hW * hW; fvW = hvW * uW
    guC = hvC * uC; gvC = hvC * vC + pC
    guN = huN * vN; gvN = hvN * vN + 0.5 * G_SW * hN * hN
    guS = huS * vS; gvS = hvS * vS + 0.5 * G_SW * hS * hS
    aE = max(abs(uC) + cC, abs(uE) + cE)
    aW = max(abs(uW) + cW, abs(uC) + cC)
    bN = max(abs(vC) + cC, abs(vN) + cN)
    bS = max(abs(vS) + cS, abs(vC) + cC)
    FhE = 0.5 * (huC + huE) - 0.5 * aE * (hE - hC)
    FhW = 0.5 * (huW + huC) - 0.5 * aW * (hC - hW)
    FuE = 0.5 * (fuC + fuE) - 0.5 * aE * (huE - huC)
    FuW = 0.5 * (fuW + fuC) - 0.5 * aW * (huC - huW)
    FvE = 0.5 * (fvC + fvE) - 0.5 * aE * (hvE - hvC)
    FvW = 0.5 * (fvW + fvC) - 0.5 * aW * (hvC - hvW)
    GhN = 0.5 * (hvC + hvN) - 0.5 * bN * (hN - hC)
    GhS = 0.5 * (hvS + hvC) - 0.5 * bS * (hC - hS)
    GuN = 0.5 * (guC + guN) - 0.5 * bN * (huN - huC)
    GuS = 0.5 * (guS + guC) - 0.5 * bS * (huC - huS)
    GvN = 0.5 * (gvC + gvN) - 0.5 * bN * (hvN - hvC)
    GvS = 0.5 * (gvS + gvC) - 0.5 * bS * (hvC - hvS)
    return (-(FhE - FhW) / dx - (GhN - GhS) / dx,
            -(FuE - FuW) / dx - (GuN - GuS) / dx,
            -(FvE - FvW) / dx - (GvN - GvS) / dx)


def sw_speed(h, hu, hv, i, j):
    return max(abs(hu[i, j] / h[i, j]), abs(hv[i, j] / h[i, j])) + sqrt(G_SW * h[i, j])  # noqa: F821


def sw_init(n: int, rng, halo=(1, 1), dtype="float32"):
    """h = 1 + 0.1 * Gaussian bump at a random centre, hu = hv = 0."""
    import numpy as np

    y = (np.arange(n) + 0.5) / n
    cy, cx = rng.uniform(0.2, 0.8, size=2)
    r2 = (y[:, None] - cy) ** 2 + (y[None, :] - cx) ** 2
    shape = (n + 2 * halo[0], n + 2 * halo[1])
    h = np.ones(shape)
    h[halo[0]:halo[0] + n, halo[1]:halo[1] + n] = 1.0 + 0.1 * np.exp(-r2 / (2 * 0.05 ** 2))
    z = np.zeros(shape)
    return h.astype(dtype), z.astype(dtype), z.astype(dtype)


# Serving mix: 2-D heat 5-pt, 2-D first-order upwind advection with velocity
# (1, 0.5) at Courant number 0.4 in x, 2-D leapfrog wave (c = 1, Courant^2
# 0.25, state u, u_prev) and the 3-D 7-point Laplacian.
def upwind2d(u, i, j):
    return u[i, j] - 0.4 * (u[i, j] - u[i, j - 1]) - 0.2 * (u[i, j] - u[i - 1, j])


SERVE_KINDS = {"heat2d": (heat2d, 2, 1), "upwind2d": (upwind2d, 2, 1),
               "wave2d": (leapfrog, 2, 2), "lap7": (lap7, 3, 1)}


def serving_kinds(align_halo: bool = False):
    """SolveKind objects (FP32 and FP64 programs) for the serving mix."""
    from cutile import compile as stencil_compile
    from cutile import stencil
    from cutile.runtime.serving import SolveKind

    kinds = []
    for name, (fn, ndim, nstate) in SERVE_KINDS.items():
        res = {dt: stencil_compile(stencil(ndim=ndim, dtype=dt)(fn), temporal_blocking=False,
                                   align_halo=align_halo)
               for dt in ("float32", "float64")}
        kinds.append(SolveKind(name, res, nstate))
    return kinds
