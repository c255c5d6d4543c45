"""Synthetic initial conditions for the hydro hot path (host side, numpy).

Every workload is a seeded cubic lattice with uniform jitter, built the way the reference lays out its regular grid
(main/src/init/grid.hpp:101-131: lattice point k along an axis sits at -r + (k + 0.5) * step, index order z-major,
then y, then x) and filled with the field values of its test case. Random numbers come from a counter-based
splitmix64 hash, so the same (seed, particle, axis) always gives the same jitter on every machine.

Fields are returned as a dict of numpy arrays, in lattice order, with the names of the reference's particle fields
(sph/include/sph/particles_data.hpp:262-266), plus scalar settings under "params".
"""
from __future__ import annotations

import math

import numpy as np

#: gas constant used for the ideal-gas heat capacity (sph/include/sph/eos.hpp:19)
GAS_R = 8.317e7

_MASK64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser applied elementwise to a uint64 array (Steele, Lea & Flood 2014)."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & _MASK64
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _MASK64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _MASK64
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, index: np.ndarray, stream: int) -> np.ndarray:
    """Uniform doubles in [0, 1) from the counter (seed, particle index, stream), 53 random bits each."""
    with np.errstate(over="ignore"):
        ctr = (np.uint64(seed) * np.uint64(0xD1B54A32D192ED03)) ^ (index.astype(np.uint64) * np.uint64(4)
                                                                    + np.uint64(stream))
    bits = splitmix64(ctr) >> np.uint64(11)
    return bits.astype(np.float64) * (1.0 / 9007199254740992.0)


def ideal_gas_cv(mui: float, gamma: float) -> float:
    """Heat capacity cv = R / mui / (gamma - 1) (sph/include/sph/eos.hpp:16-21)."""
    return GAS_R / mui / (gamma - 1.0)


def jittered_lattice(side: int, r: float, seed: int, jitter: float = 0.05):
    """side^3 lattice over [-r, r]^3 plus uniform jitter of +-jitter * spacing per coordinate."""
    step = 2.0 * r / side
    idx = np.arange(side ** 3, dtype=np.int64)
    k = idx % side
    j = (idx // side) % side
    i = idx // (side * side)
    r_ini = -r + 0.5 * step
    x = r_ini + k * step
    y = r_ini + j * step
    z = r_ini + i * step
    amp = jitter * step
    x = x + (2.0 * uniform01(seed, idx, 0) - 1.0) * amp
    y = y + (2.0 * uniform01(seed, idx, 1) - 1.0) * amp
    z = z + (2.0 * uniform01(seed, idx, 2) - 1.0) * amp
    return x, y, z, step


def _common(n: int, h0: float, m: float, alphamin: float):
    zeros = np.zeros(n, dtype=np.float64)
    return {
        "h": np.full(n, h0), "m": np.full(n, m),
        "vx": zeros.copy(), "vy": zeros.copy(), "vz": zeros.copy(),
        "x_m1": zeros.copy(), "y_m1": zeros.copy(), "z_m1": zeros.copy(),
        "du_m1": zeros.copy(), "alpha": np.full(n, alphamin),
        "id": np.arange(n, dtype=np.uint64),
    }


def default_params(**over) -> dict:
    """Physics settings with the reference's defaults (particles_data.hpp:85-143)."""
    p = dict(ng0=100, ngmax=150, gamma=5.0 / 3.0, mui=10.0, minDt=1e-6, minDt_m1=1e-6, Kcour=0.2, Krho=0.06,
             alphamin=0.05, alphamax=1.0, decay_constant=0.2, sincIndex=6.0)
    p.update(over)
    return p


def sedov(side: int, seed: int = 0, energy: float = 1.0, gamma: float = 5.0 / 3.0, ng0: int = 100,
          ngmax: int = 150) -> dict:
    """Sedov blast in the periodic box [-0.5, 0.5]^3.

    Uniform density 1 (m = 1/N), zero velocity, alpha = alphamin, h0 = 0.5 * cbrt(3/(4 pi) * ng0 * V / N)
    (main/src/init/sedov_init.hpp:57). Internal energy u = 1e-8 everywhere plus the blast energy deposited with a
    normalised Gaussian weight g = exp(-r^2 / (2 s)^2), s = lattice spacing: u_i += E g_i / (m sum_j g_j).
    Stored as temp = u / cv since the VE propagator conserves temp (main/src/propagator/ve_hydro.hpp:73).
    """
    r = 0.5
    n = side ** 3
    x, y, z, step = jittered_lattice(side, r, seed)
    p = default_params(gamma=gamma, ng0=ng0, ngmax=ngmax)
    m = 1.0 / n
    h0 = 0.5 * math.pow(3.0 / (4.0 * math.pi) * ng0 * (2 * r) ** 3 / n, 1.0 / 3.0)
    f = _common(n, h0, m, p["alphamin"])
    width = 2.0 * step
    g = np.exp(-(x * x + y * y + z * z) / (width * width))
    u = 1e-8 + energy * g / (m * g.sum())
    f.update(x=x, y=y, z=z, temp=u / ideal_gas_cv(p["mui"], gamma))
    f["box"] = (-r, r, -r, r, -r, r)
    f["periodic"] = True
    f["params"] = p
    f["name"] = f"sedov{side}"
    return f


def noh(side: int, seed: int = 0, ng0: int = 100, ngmax: int = 150) -> dict:
    """Noh implosion: the side^3 lattice over [-0.5, 0.5]^3 cut to r <= 0.5, open box.

    Density 1 (m = 1/N_kept), u = 1e-6, velocity -r_hat with |r| floored at 1e-10, x_m1 = v * dt0 with dt0 = 1e-4,
    h0 = 0.5 * cbrt(3/(4 pi) * ng0 * (4 pi / 3 * 0.5^3) / N) (main/src/init/noh_init.hpp:59-114).
    """
    r = 0.5
    x, y, z, step = jittered_lattice(side, r, seed)
    keep = (x * x + y * y + z * z) <= r * r
    x, y, z = x[keep], y[keep], z[keep]
    n = x.size
    dt0 = 1e-4
    p = default_params(ng0=ng0, ngmax=ngmax, minDt=dt0, minDt_m1=dt0)
    m = 1.0 / n
    vol = 4.0 * math.pi / 3.0 * r ** 3
    h0 = 0.5 * math.pow(3.0 / (4.0 * math.pi) * ng0 * vol / n, 1.0 / 3.0)
    f = _common(n, h0, m, p["alphamin"])
    rad = np.maximum(np.sqrt(x * x + y * y + z * z), 1e-10)
    vx, vy, vz = -x / rad, -y / rad, -z / rad
    f.update(x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, x_m1=vx * dt0, y_m1=vy * dt0, z_m1=vz * dt0,
             temp=np.full(n, 1e-6 / ideal_gas_cv(p["mui"], p["gamma"])))
    f["box"] = (float(x.min()), float(x.max()), float(y.min()), float(y.max()), float(z.min()), float(z.max()))
    f["periodic"] = False
    f["params"] = p
    f["name"] = f"noh{side}"
    return f


#: order of the conserved per-particle fields exchanged with the C ABIs
CONSERVED_FIELDS = ("x", "y", "z", "h", "m", "temp", "vx", "vy", "vz", "x_m1", "y_m1", "z_m1", "du_m1", "alpha")
