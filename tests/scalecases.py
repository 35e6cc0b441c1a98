"""Parity cases at the sizes of the benchmark configurations (shared by the digest
generator tests/golden/make_config_digests.py and tests/test_gpu_config_parity.py).

* ``kolmogorov64``: 3-D Kolmogorov flow, D3Q19 BGK fluid only, 64^3 periodic, FP64,
  tau = 0.6 (nu = 1/30), body force F_x = 1e-5 sin(2 pi (y + 1/2) / 64), rho = 1 and
  u = 0 plus seeded uniform +-1e-4 velocity noise (populations f = feq(1, u0)), 2000
  steps -- the plain-method configuration, run through the compiled reference.
* ``*_multiblock``: lattices wider than one 128-thread block row (NX > 128, NX not a
  multiple of 128), so that several x-blocks and a partial last block are compared
  with the reference cell for cell.

The reference's own output is kept as SHA-256 digests of the FP64 arrays in the
layout the Python API returns (AoS populations [z][y][x][q], vectors [z][y][x][3],
scalars [z][y][x]), little-endian bytes; an FP64 run that is bit-identical to the
reference reproduces every digest.
"""
import hashlib

import numpy as np

import oracle as O
from lbcases import make_case

W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
C = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
              [1, 1, 0], [1, -1, 0], [-1, 1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1], [-1, 0, -1],
              [0, 1, 1], [0, 1, -1], [0, -1, 1], [0, -1, -1]], dtype=float)
TWO_PI = 2 * 3.14159265359  # the reference's two_pi literal (src/typedef.h:367)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def kinetic_energy(u):
    """Total kinetic energy 1/2 sum |u|^2 over the cells (fixed numpy order)."""
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 3)
    return float(0.5 * np.sum(u[:, 0] * u[:, 0] + u[:, 1] * u[:, 1] + u[:, 2] * u[:, 2]))


def feq(rho, u):
    """D3Q19 equilibrium w rho (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u^2), elementwise."""
    cu = u @ C.T
    u2 = (u * u).sum(axis=-1)[..., None]
    return W * rho[..., None] * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * u2)


def kolmogorov64(seed=2000, n=64):
    """(flagset, config, state, steps) of the plain-method configuration."""
    tau = 0.6
    nu = (tau - 0.5) / 3.0
    amp = 1e-5 / (nu * (TWO_PI / n) ** 2)  # F_x = Amp_x nu (2 pi / LY)^2 sin(...), src/forcing.c:390-400
    cfg = O.make_config(n, n, n, O.FLAGSETS["kolmogorov"], tau_u=tau, Amp_x=amp, Amp_y=0.0, Amp_z=0.0)
    rng = np.random.default_rng(seed)
    u0 = rng.uniform(-1e-4, 1e-4, size=(n, n, n, 3))
    p = np.ascontiguousarray(feq(np.ones((n, n, n)), u0))
    return "kolmogorov", cfg, {"p": p}, 2000


# name -> (lbcases case, lattice, steps, seed)
MULTIBLOCK = {
    "rb_multiblock": ("rb", (200, 10, 6), 100, 21),
    "hit_multiblock": ("hit", (300, 6, 5), 60, 22),
    "les_multiblock": ("les", (160, 9, 5), 60, 23),
    "particles_multiblock": ("particles", (140, 8, 6), 30, 24),
    # walls on x and z (the x walls on both ends of a multi-block row); shear-improved LES,
    # whose running mean is read across block boundaries in the reference's loop order
    "duct_multiblock": ("duct", (150, 8, 6), 60, 25),
    "sism_multiblock": ("les_kalman", (170, 9, 5), 60, 26),
}


def multiblock(name):
    case, dims, steps, seed = MULTIBLOCK[name]
    flagset, cfg, state = make_case(case, seed=seed, dims=dims)
    if "part" in state:  # twice the particles of the small case, over the wider box
        from lbcases import make_particles
        state["part"] = make_particles(np.random.default_rng(seed + 100), 600, *dims)
        cfg.particle_number = 600
    return flagset, cfg, state, steps


def case(name):
    return kolmogorov64() if name == "kolmogorov64" else multiblock(name)


NAMES = ["kolmogorov64"] + sorted(MULTIBLOCK)
# outputs compared per case (when the run has them)
OUTPUTS = ("p", "g", "h", "u", "dens", "t", "phi")
PARTICLE_OUTPUTS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "ux", "uy", "uz")
