"""Seeded synthetic SPME systems (the five benchmark/parity configurations).

No public dataset is involved: every system is generated here from a fixed
numpy seed, with the shapes, sizes and value distributions of the
configurations the reference path is measured on.

Each generator returns a ``System`` (positions in nm, charges, the 6-vector
box ``L = [ax, by, cz, bx, cx, cy]`` of the reference's Cell, sfac.hpp:37-52,
the grid ``K``, the B-spline ``order``, the Ewald ``beta`` and the
influence-function cutoff ``max_m``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# max_m = beta * sqrt(ln 1e16) / pi: reciprocal vectors beyond it have
# f(m^2) < 1e-16 f(0+) relative weight.
MAX_M_FACTOR = math.sqrt(math.log(1e16)) / math.pi


@dataclass
class System:
    name: str
    x: np.ndarray  # (N, 3) float64 positions
    q: np.ndarray  # (N,) float64 charges
    L: np.ndarray  # (6,) float64 box
    K: tuple
    order: int
    beta: float
    max_m: float
    extra: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.q.shape[0])


def LofS(L):
    return np.array([[L[0], 0.0, 0.0], [L[3], L[1], 0.0], [L[4], L[5], L[2]]])


def smooth_235(n: int) -> int:
    """Smallest integer >= n whose prime factors are all 2, 3 or 5."""
    m = max(1, int(n))
    while True:
        r = m
        for p in (2, 3, 5):
            while r % p == 0:
                r //= p
        if r == 1:
            return m
        m += 1


def cfg1_plain() -> System:
    """1000 alternating +-1 charges, cubic 3.0 nm box, 32^3, order 4, beta 3.47."""
    rng = np.random.default_rng(1)
    n = 1000
    x = rng.uniform(0.0, 3.0, size=(n, 3))
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    beta = 3.47
    return System("plain_1000_32cube_p4", x, q, np.array([3.0, 3.0, 3.0, 0.0, 0.0, 0.0]),
                  (32, 32, 32), 4, beta, MAX_M_FACTOR * beta)


def _random_rotations(rng, n):
    """Uniform random rotation matrices from uniform unit quaternions."""
    u1, u2, u3 = rng.uniform(size=(3, n))
    a = np.sqrt(1 - u1) * np.sin(2 * np.pi * u2)
    b = np.sqrt(1 - u1) * np.cos(2 * np.pi * u2)
    c = np.sqrt(u1) * np.sin(2 * np.pi * u3)
    d = np.sqrt(u1) * np.cos(2 * np.pi * u3)
    w, x, y, z = d, a, b, c
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def cfg2_water(n_mol: int = 32768) -> System:
    """Rigid 3-site water box: 32768 molecules in a 10 nm cube, 96^3, order 4,
    beta 3.12 (O -0.834, H +0.417, O-H 0.09572 nm, H-O-H 104.52 deg)."""
    rng = np.random.default_rng(2)
    side = 10.0
    centers = rng.uniform(0.0, side, size=(n_mol, 3))
    R = _random_rotations(rng, n_mol)
    d, theta = 0.09572, math.radians(104.52)
    h1 = np.array([d * math.sin(theta / 2), d * math.cos(theta / 2), 0.0])
    h2 = np.array([-d * math.sin(theta / 2), d * math.cos(theta / 2), 0.0])
    x = np.empty((n_mol, 3, 3))
    x[:, 0] = centers
    x[:, 1] = centers + R @ h1
    x[:, 2] = centers + R @ h2
    q = np.tile(np.array([-0.834, 0.417, 0.417]), n_mol)
    beta = 3.12
    return System(f"water_{3 * n_mol}_96cube_p4", x.reshape(-1, 3), q,
                  np.array([side, side, side, 0.0, 0.0, 0.0]), (96, 96, 96), 4, beta,
                  MAX_M_FACTOR * beta)


def cfg3_triclinic(n: int = 1048576, K: int = 256) -> System:
    """1,048,576 charges N(0, 0.5^2) (neutralised) in a triclinic cell
    a=b=c=20 nm, gamma=60 deg; 256^3, order 6, beta 3.5."""
    rng = np.random.default_rng(3)
    q = rng.normal(0.0, 0.5, size=n)
    q -= q.mean()
    s = rng.uniform(0.0, 1.0, size=(n, 3))
    L = np.array([20.0, 17.320508075688775, 20.0, 10.0, 0.0, 0.0])
    x = s @ LofS(L)
    beta = 3.5
    return System(f"triclinic_{n}_{K}cube_p6", x, q, L, (K, K, K), 6, beta, MAX_M_FACTOR * beta)


def cfg4_batch(count: int = 64) -> list:
    """64 small periodic systems: N log-uniform in [64, 2048], cubic sides
    U[1.5, 4.0] nm, charges U[-1, 1] neutralised, K = 2/3/5-smooth >= L/0.1
    clamped to [24, 48], order 4, beta 3.47."""
    rng = np.random.default_rng(4)
    out = []
    beta = 3.47
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(64), math.log(2048)))))
        side = float(rng.uniform(1.5, 4.0))
        q = rng.uniform(-1.0, 1.0, size=n)
        q -= q.mean()
        x = rng.uniform(0.0, side, size=(n, 3))
        k = min(48, max(24, smooth_235(math.ceil(side / 0.1))))
        out.append(System(f"batch{i}", x, q, np.array([side, side, side, 0.0, 0.0, 0.0]),
                          (k, k, k), 4, beta, MAX_M_FACTOR * beta))
    return out


def cfg5_specs(count: int = 10000, seed: int = 5) -> list:
    """Serving-stream request shapes: N log-uniform in [500, 200000] (even),
    density 100 atoms/nm^3 (cubic side (N/100)^(1/3) nm), K = 2/3/5-smooth >=
    round(side/0.1) clamped to [24, 128], order 4 or 6 uniformly, beta 3.12."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(500), math.log(200000)))))
        n += n % 2
        side = (n / 100.0) ** (1.0 / 3.0)
        k = min(128, max(24, smooth_235(int(round(side / 0.1)))))
        order = int(rng.choice([4, 6]))
        beta = 3.12
        out.append(dict(id=i, n=n, side=side, K=(k, k, k), order=order, beta=beta, max_m=MAX_M_FACTOR * beta))
    return out


CFG5_POOL_ATOMS = 200000


def cfg5_pool(seed: int = 5) -> np.ndarray:
    """Unit-cube fractional positions shared by all serving requests: request
    i uses the first N_i of them scaled by its box side."""
    return np.random.default_rng(10_000 + seed).uniform(0.0, 1.0, size=(CFG5_POOL_ATOMS, 3))


def cfg5_charges(n: int) -> np.ndarray:
    return np.where(np.arange(n) % 2 == 0, 1.0, -1.0)


def cfg5_request(spec: dict, pool: np.ndarray) -> System:
    n, side = spec["n"], spec["side"]
    return System(f"req_{spec['id']}_{n}_{spec['K'][0]}_p{spec['order']}", pool[:n] * side, cfg5_charges(n),
                  np.array([side, side, side, 0.0, 0.0, 0.0]), spec["K"], spec["order"], spec["beta"],
                  spec["max_m"])


BY_NAME = {
    "plain": cfg1_plain,
    "water": cfg2_water,
    "triclinic": cfg3_triclinic,
}
