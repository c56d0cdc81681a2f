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
