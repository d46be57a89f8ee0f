"""Problem setup: initial primitive states for the two reference problems.

The reference defines problems with device hooks compiled into the solver
(``set_initial_condition`` etc., e.g.
src/application/kepler_disk_demo/mhd_solver.curb:10-33).  Hooks cannot cross a
C ABI, so here a problem is a :class:`~nmhd_b200.config.SolverConfig` plus an
initial state generated on the host in float64 and rounded to float32, in the
reference's ``.bin`` array layout (8, Sz, Sy, Sx).

Axes follow the reference's shearing-box convention: X azimuthal (the shear
direction), Y radial (shearing-periodic, with margins), Z vertical.
"""
from __future__ import annotations

import math

import numpy as np

from .config import SolverConfig


def orszag_tang_3d(n=64, ny=None, nz=None, extent=1.0, gamma=5.0 / 3.0, cfl=0.4, b0=None):
    """3-D Orszag-Tang-type vortex on a periodic box of side ``extent``.

    rho = 25/(36 pi), p = 5/(12 pi),
    v = (-sin 2pi y, sin 2pi x, 0.1 sin 2pi z),
    B = B0 (-sin 2pi y, sin 4pi x, 0) with B0 = 1/sqrt(4 pi).
    Face B comes from A_z = B0 (cos(2pi y)/(2pi) + cos(4pi x)/(4pi)) by exact
    edge differences, so the discrete divergence is zero before rounding.
    Coordinates are scaled so one period spans the box.
    """
    nx = n
    ny = n if ny is None else ny
    nz = n if nz is None else nz
    b0 = 1.0 / math.sqrt(4.0 * math.pi) if b0 is None else b0
    cfg = SolverConfig(size_x=nx, size_y=ny, size_z=nz, extent_x=extent, extent_y=extent,
                       extent_z=extent, gamma=gamma, cfl=cfl)
    dx, dy, dz = extent / nx, extent / ny, extent / nz
    k = 2.0 * math.pi / extent
    xc = (np.arange(nx) + 0.5) * dx
    yc = (np.arange(ny) + 0.5) * dy
    zc = (np.arange(nz) + 0.5) * dz
    xf = np.arange(nx + 1) * dx
    yf = np.arange(ny + 1) * dy
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    state = np.empty((8, nz, ny, nx), dtype=np.float64)
    state[0] = 25.0 / (36.0 * math.pi)
    state[1] = -np.sin(k * Y)
    state[2] = np.sin(k * X)
    state[3] = 0.1 * np.sin(k * Z)
    state[4] = 5.0 / (12.0 * math.pi)

    def az(x, y):
        return b0 * (np.cos(k * y) / k + np.cos(2.0 * k * x) / (2.0 * k))

    # Bx on the lower x-face of cell (i, j): (Az(x_i, y_{j+1}) - Az(x_i, y_j)) / dy
    xi = xf[:nx][None, :]
    bx = (az(xi, yf[1:ny + 1][:, None]) - az(xi, yf[:ny][:, None])) / dy
    # By on the lower y-face of cell (i, j): -(Az(x_{i+1}, y_j) - Az(x_i, y_j)) / dx
    yj = yf[:ny][:, None]
    by = -(az(xf[1:nx + 1][None, :], yj) - az(xf[:nx][None, :], yj)) / dx
    state[5] = bx[None, :, :]
    state[6] = by[None, :, :]
    state[7] = 0.0
    return cfg, state.astype(np.float32)


def shearing_box(n_radial=128, n_azimuthal=256, n_vertical=64, l_radial=1.0, l_azimuthal=4.0,
                 l_vertical=1.0, q=1.5, omega=1.0, beta=400.0, density=1.0, pressure=1.0,
                 gamma=5.0 / 3.0, cfl=0.4, noise=0.01, seed=1, margin=4):
    """MRI shearing box with a net vertical field and seeded velocity noise.

    Background: rho, p uniform; azimuthal velocity v_X = -q Omega y, with y the
    radial coordinate of the cell centre measured from the centre of the
    margin-inclusive box (the coordinate the reference's tidal term uses,
    src/application/kepler_disk_demo/mhd_solver.curb:18-21, 76-79), so the
    background is an exact equilibrium.  B = (0, 0, sqrt(2 p / beta)).
    Noise: U(-noise, noise) * c_s added to each velocity component of every
    interior cell, c_s = sqrt(gamma p / rho), numpy PCG64(seed).
    Margin rows are overwritten by the shearing-periodic fill before the first
    step; they are set to the background here.
    """
    sx, sy, sz = n_azimuthal, n_radial + 2 * margin, n_vertical
    cfg = SolverConfig(size_x=sx, size_y=sy, size_z=sz, margin_y=margin,
                       extent_x=l_azimuthal, extent_y=l_radial, extent_z=l_vertical,
                       gamma=gamma, cfl=cfl, problem="shearing_box", q=q, omega=omega)
    d = cfg.derived()
    # radial cell-centre coordinate, in float32 exactly as the solver computes it
    y_idx = np.arange(sy, dtype=np.float32)
    y_loc = np.float32(d["corner_y"]) + np.float32(d["dy"]) * (y_idx + np.float32(0.5))
    v_shear = (np.float32(-q) * np.float32(omega)) * y_loc
    state = np.zeros((8, sz, sy, sx), dtype=np.float64)
    state[0] = density
    state[4] = pressure
    state[1] = v_shear.astype(np.float64)[None, :, None]
    state[7] = math.sqrt(2.0 * pressure / beta)
    cs = math.sqrt(gamma * pressure / density)
    rng = np.random.Generator(np.random.PCG64(seed))
    pert = rng.uniform(-noise, noise, size=(3, sz, n_radial, sx)) * cs
    state[1:4, :, margin:margin + n_radial, :] += pert
    return cfg, state.astype(np.float32)


def shearing_box_slabs(n_slabs, n_radial=128, n_azimuthal=256, n_vertical=64, l_radial=1.0,
                       l_azimuthal=4.0, l_vertical=1.0, q=1.5, omega=1.0, beta=400.0, density=1.0,
                       pressure=1.0, gamma=5.0 / 3.0, cfl=0.4, noise=0.01, seed=1, margin=4, only=None):
    """The box of :func:`shearing_box` split into ``n_slabs`` radial slabs, as
    the reference's ranks along Y hold it: each slab in its own frame (v_X =
    -q Omega y with y measured from the slab's own margin-inclusive centre),
    the noise of the whole box (same seed and draw) cut into the slabs' rows.
    Returns (one slab's config, [state of rank 0, ..., rank n_slabs - 1]);
    with ``only`` = r the list holds rank r's state alone."""
    from .slab import slab_config
    whole, _ = shearing_box(n_radial=n_radial, n_azimuthal=n_azimuthal, n_vertical=n_vertical,
                            l_radial=l_radial, l_azimuthal=l_azimuthal, l_vertical=l_vertical, q=q,
                            omega=omega, beta=beta, density=density, pressure=pressure, gamma=gamma,
                            cfl=cfl, noise=0.0, seed=seed, margin=margin)
    cfg = slab_config(whole, n_slabs)
    d = cfg.derived()
    rows = n_radial // n_slabs
    sx, sy, sz = cfg.size_x, cfg.size_y, cfg.size_z
    y_idx = np.arange(sy, dtype=np.float32)
    y_loc = np.float32(d["corner_y"]) + np.float32(d["dy"]) * (y_idx + np.float32(0.5))
    v_shear = (np.float32(-q) * np.float32(omega)) * y_loc
    cs = math.sqrt(gamma * pressure / density)
    rng = np.random.Generator(np.random.PCG64(seed))
    pert = rng.uniform(-noise, noise, size=(3, sz, n_radial, sx)) * cs
    states = []
    for r in range(n_slabs) if only is None else [only]:
        state = np.zeros((8, sz, sy, sx), dtype=np.float64)
        state[0] = density
        state[4] = pressure
        state[1] = v_shear.astype(np.float64)[None, :, None]
        state[7] = math.sqrt(2.0 * pressure / beta)
        state[1:4, :, margin:margin + rows, :] += pert[:, :, r * rows:(r + 1) * rows, :]
        states.append(state.astype(np.float32))
    return cfg, states


def mri_ensemble(n_boxes=64, seed=0, sides=(32, 48, 64, 96), ratios=(2, 3, 4), beta_range=(1e2, 1e4),
                 q_range=(1.2, 1.8), noise=0.01, margin=4):
    """Ensemble of independent MRI shearing boxes of uneven sizes.

    Per box: radial and vertical cell counts drawn from ``sides``, azimuthal =
    k * radial with k from ``ratios``; extents radial 1, azimuthal k, vertical 1
    (cubic cells); beta log-uniform in ``beta_range``; q uniform in ``q_range``;
    noise seed 1000 + box.  The draws use numpy PCG64(seed).
    Returns (list of (config, state), list of per-box parameter dicts).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    boxes, params = [], []
    for b in range(n_boxes):
        nr = int(rng.choice(sides))
        nz = int(rng.choice(sides))
        k = int(rng.choice(ratios))
        beta = float(10.0 ** rng.uniform(math.log10(beta_range[0]), math.log10(beta_range[1])))
        q = float(rng.uniform(*q_range))
        cfg, state = shearing_box(n_radial=nr, n_azimuthal=k * nr, n_vertical=nz, l_radial=1.0,
                                  l_azimuthal=float(k), l_vertical=1.0, q=q, beta=beta, noise=noise,
                                  seed=1000 + b, margin=margin)
        boxes.append((cfg, state))
        params.append({"n_radial": nr, "n_azimuthal": k * nr, "n_vertical": nz, "beta": beta, "q": q,
                       "seed": 1000 + b})
    return boxes, params
