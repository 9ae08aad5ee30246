"""Seeded synthetic inputs for the implicit-step workloads.

No dataset is involved: every input is generated from a seed with the shapes
and value distributions of the benchmark configurations.

* ``gaussian_diffusion``: transient diffusion on the unit cube, Gaussian bump
  (centre 0.5, sigma 0.1) plus N(0, 1e-3) noise, Dirichlet 1 / 0 on x = 0 / 1,
  zero-gradient elsewhere, constant D (64^3, D = 1e-3, dt = 1e-2, 10 steps).
* ``tvd_convection_diffusion``: periodic cube, divergence-free face velocities
  from the discrete curl of a seeded vector potential made of 8 Fourier modes,
  scaled to a cell Peclet number (|u|max dx / D) and a CFL number; a smooth
  seeded scalar in [0, 1]; van Leer TVD (256^3, D = 1e-4, Pe 5, CFL 0.5).
* ``heterogeneous``: as above with a log-normal diffusivity (mu = ln 1e-4,
  sigma = 1) smoothed by a periodic 5-cell box filter, face D = mean of the
  two adjacent cells.

Arrays are float64 in the layouts of ``include/dare_gpu.h``: ghosted fields
(n+4 per active dimension), faces (n+1 along the face normal).  ``xp`` may be
``numpy`` or ``torch`` (for on-device generation of the large cases).
"""
from __future__ import annotations

import math

import numpy as np


def _backend(device):
    if device is None:
        return np, None
    import torch
    return torch, torch.device(device)


def _arange(xp, dev, n):
    if xp is np:
        return np.arange(n, dtype=np.float64)
    return xp.arange(n, dtype=xp.float64, device=dev)


def _roll(xp, a, shift, axis):
    if xp is np:
        return np.roll(a, shift, axis=axis)
    return xp.roll(a, shifts=shift, dims=axis)


def _abs_max(xp, a):
    return float(np.abs(a).max()) if xp is np else float(a.abs().max().item())


def ghosted(xp, dev, interior, ng=2):
    """Embed an interior 3D array into a zero ghosted array (ghosts untouched)."""
    nx, ny, nz = interior.shape
    if xp is np:
        out = np.zeros((nx + 2 * ng, ny + 2 * ng, nz + 2 * ng), dtype=np.float64)
    else:
        out = xp.zeros((nx + 2 * ng, ny + 2 * ng, nz + 2 * ng), dtype=xp.float64, device=dev)
    out[ng:ng + nx, ng:ng + ny, ng:ng + nz] = interior
    return out


def periodic_ghosts(xp, a, ng=2):
    """Fill the face ghosts of a ghosted 3D array periodically (halo exchange)."""
    n = [a.shape[d] - 2 * ng for d in range(3)]
    a[:ng, ng:ng + n[1], ng:ng + n[2]] = a[n[0]:n[0] + ng, ng:ng + n[1], ng:ng + n[2]]
    a[n[0] + ng:, ng:ng + n[1], ng:ng + n[2]] = a[ng:2 * ng, ng:ng + n[1], ng:ng + n[2]]
    a[ng:ng + n[0], :ng, ng:ng + n[2]] = a[ng:ng + n[0], n[1]:n[1] + ng, ng:ng + n[2]]
    a[ng:ng + n[0], n[1] + ng:, ng:ng + n[2]] = a[ng:ng + n[0], ng:2 * ng, ng:ng + n[2]]
    a[ng:ng + n[0], ng:ng + n[1], :ng] = a[ng:ng + n[0], ng:ng + n[1], n[2]:n[2] + ng]
    a[ng:ng + n[0], ng:ng + n[1], n[2] + ng:] = a[ng:ng + n[0], ng:ng + n[1], ng:2 * ng]
    return a


def _mode_field(xp, dev, rng, n, offsets, num_modes=8, kmax=8, decay=2.0):
    """Sum of separable periodic modes A prod_d sin(2 pi k_d x_d + phase_d),
    sampled at x_d = (i + offsets[d]) / n_d."""
    coords = [(_arange(xp, dev, n[d]) + offsets[d]) / n[d] for d in range(3)]
    out = None
    for _ in range(num_modes):
        k = rng.integers(1, kmax + 1, size=3)
        ph = rng.uniform(0.0, 2.0 * math.pi, size=3)
        amp = rng.normal() / float(np.dot(k, k)) ** (decay / 2.0)
        fx = xp.sin(2.0 * math.pi * float(k[0]) * coords[0] + float(ph[0]))
        fy = xp.sin(2.0 * math.pi * float(k[1]) * coords[1] + float(ph[1]))
        fz = xp.sin(2.0 * math.pi * float(k[2]) * coords[2] + float(ph[2]))
        term = amp * fx[:, None, None] * fy[None, :, None] * fz[None, None, :]
        out = term if out is None else out + term
    return out


def divergence_free_velocity(n, seed, u_max, device=None):
    """Face velocities (x-, y-, z-faces, each with n+1 entries along its normal,
    face n == face 0) as the discrete curl of an edge-sampled vector potential."""
    xp, dev = _backend(device)
    rng = np.random.default_rng(seed)
    dx = [1.0 / n[d] for d in range(3)]
    # psi_x on x-edges ((i+1/2), j, k); psi_y on y-edges (i, j+1/2, k); psi_z on z-edges (i, j, k+1/2)
    psi_x = _mode_field(xp, dev, rng, n, (0.5, 0.0, 0.0))
    psi_y = _mode_field(xp, dev, rng, n, (0.0, 0.5, 0.0))
    psi_z = _mode_field(xp, dev, rng, n, (0.0, 0.0, 0.5))
    ux = (_roll(xp, psi_z, -1, 1) - psi_z) / dx[1] - (_roll(xp, psi_y, -1, 2) - psi_y) / dx[2]
    uy = (_roll(xp, psi_x, -1, 2) - psi_x) / dx[2] - (_roll(xp, psi_z, -1, 0) - psi_z) / dx[0]
    uz = (_roll(xp, psi_y, -1, 0) - psi_y) / dx[0] - (_roll(xp, psi_x, -1, 1) - psi_x) / dx[1]
    scale = u_max / max(_abs_max(xp, ux), _abs_max(xp, uy), _abs_max(xp, uz))
    faces = []
    for d, u in enumerate((ux, uy, uz)):
        u = u * scale
        first = [slice(None)] * 3
        first[d] = slice(0, 1)
        if xp is np:
            faces.append(np.concatenate([u, u[tuple(first)]], axis=d))
        else:
            faces.append(xp.cat([u, u[tuple(first)]], dim=d))
    return faces


def smooth_scalar(n, seed, device=None):
    """Seeded smooth periodic scalar rescaled to [0, 1] (cell centres)."""
    xp, dev = _backend(device)
    rng = np.random.default_rng(seed + 7919)
    f = _mode_field(xp, dev, rng, n, (0.5, 0.5, 0.5), decay=1.0)
    lo, hi = (float(f.min()), float(f.max())) if xp is np else (float(f.min().item()), float(f.max().item()))
    return (f - lo) / (hi - lo)


def gaussian_diffusion(n=64, seed=0, D=1e-3, dt=1e-2, steps=10, noise=1e-3):
    """Config: 3D transient diffusion, Dirichlet x (1 at x=0, 0 at x=1), Neumann elsewhere."""
    rng = np.random.default_rng(seed)
    c = (np.arange(n, dtype=np.float64) + 0.5) / n
    r2 = (c[:, None, None] - 0.5) ** 2 + (c[None, :, None] - 0.5) ** 2 + (c[None, None, :] - 0.5) ** 2
    phi = np.exp(-r2 / (2.0 * 0.1 ** 2)) + rng.normal(0.0, noise, size=(n, n, n))
    return {
        "n": (n, n, n), "size": (1.0, 1.0, 1.0), "periodic": (0, 0, 0), "D": D, "dt": dt, "steps": steps,
        "phi0": ghosted(np, None, phi),
        "bc": {1: (1, 1.0), 2: (1, 0.0), 3: (2, 0.0), 4: (2, 0.0), 5: (2, 0.0), 6: (2, 0.0)},
        "rel_tol": 1e-10,
    }


def tvd_convection_diffusion(n=256, seed=0, D=1e-4, peclet=5.0, cfl=0.5, steps=20, device=None):
    """Config: periodic convection-diffusion with van Leer TVD (deferred correction)."""
    xp, dev = _backend(device)
    nn = (n, n, n)
    dx = 1.0 / n
    u_max = peclet * D / dx
    dt = cfl * dx / u_max
    faces = divergence_free_velocity(nn, seed, u_max, device=device)
    phi = periodic_ghosts(xp, ghosted(xp, dev, smooth_scalar(nn, seed, device=device)))
    return {
        "n": nn, "size": (1.0, 1.0, 1.0), "periodic": (1, 1, 1), "D": D, "dt": dt, "steps": steps,
        "u_max": u_max, "face_vel": faces, "phi0": phi, "limiter": "VANLEER", "rel_tol": 1e-10,
    }


def lognormal_diffusivity(n, seed, mu=math.log(1e-4), sigma=1.0, box=5, device=None):
    """Cell diffusivity exp(N(mu, sigma)) smoothed by a periodic box filter of `box` cells."""
    xp, dev = _backend(device)
    rng = np.random.default_rng(seed + 104729)
    g = np.exp(rng.normal(mu, sigma, size=n))
    a = g if xp is np else xp.from_numpy(g).to(dev)
    h = box // 2
    for axis in range(3):
        acc = a * 0.0
        for s in range(-h, h + 1):
            acc = acc + _roll(xp, a, s, axis)
        a = acc / box
    return a


def heterogeneous(n=512, seed=0, peclet=5.0, cfl=0.5, steps=1, device=None):
    """Config: heterogeneous log-normal D (periodic), velocity for Pe at the median D."""
    xp, dev = _backend(device)
    nn = (n, n, n)
    dx = 1.0 / n
    Dc = lognormal_diffusivity(nn, seed, device=device)
    med = float(np.median(Dc)) if xp is np else float(Dc.median().item())
    u_max = peclet * med / dx
    dt = cfl * dx / u_max
    faces = divergence_free_velocity(nn, seed, u_max, device=device)
    phi = periodic_ghosts(xp, ghosted(xp, dev, smooth_scalar(nn, seed, device=device)))
    return {
        "n": nn, "size": (1.0, 1.0, 1.0), "periodic": (1, 1, 1), "cell_D": Dc, "median_D": med, "dt": dt,
        "steps": steps, "u_max": u_max, "face_vel": faces, "phi0": phi, "limiter": "VANLEER", "rel_tol": 1e-10,
    }


def batched_diffusion(count=4096, seed=0, sides=(16, 24, 32, 48, 64), dt=1e-2, d_range=(1e-5, 1e-2)):
    """Batch of independent cubes: side uniform from `sides`, unit size, D
    log-uniform in `d_range`, one random face Dirichlet with a U[0,1] value,
    Neumann on the other five, phi_0 = 0, one implicit step of `dt`."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        side = int(rng.choice(sides))
        D = float(np.exp(rng.uniform(np.log(d_range[0]), np.log(d_range[1]))))
        face = int(rng.integers(1, 7))
        val = float(rng.uniform(0.0, 1.0))
        bc = {f: (2, 0.0) for f in range(1, 7)}
        bc[face] = (1, val)
        out.append({"n": (side, side, side), "size": (1.0, 1.0, 1.0), "D": D, "dt": dt, "bc": bc})
    return out
