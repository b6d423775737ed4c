"""Seeded synthetic particle sets with the shapes of the benchmark workloads.

There is no public dataset for this path; these generators stand in for the
reference's initial conditions (polytropes on an hcp lattice,
parallel_bleeding_edge/src/initialize_polyes.f:66-170, Lane-Emden profile
:545-595).  Particles are drawn at random instead of on a lattice; smoothing
lengths follow the reference's neighbour-count rule: ``2 hp`` is the distance
to the 64th nearest neighbour, so each particle has ~64 neighbours within
2 hp, and ``range2 = 4 hp^2`` (grav.f:15-18; negated for point masses).

Workloads (G = 1):
  config1  N=16,384 equal-mass n=1.5 polytrope (M=1, R=1)
  config2  N=262,144 two-star collision snapshot: n=3 (M=1, R=1) at x=-1.5 and
           n=1.5 (M=0.5, R=0.6) at x=+1.5, 131,072 particles each
  config3  N=1,048,576 red-giant envelope + point-mass core (m=0.3, hp=0.05)
  config4  64 stellar models, N log-uniform in [4,096, 131,072], n in [1, 3]
  config5  16 collision snapshots, N log-uniform in [65,536, 524,288]
"""
from __future__ import annotations

import hashlib
import os
import tempfile
from dataclasses import dataclass, field
from functools import lru_cache
from typing import List

import numpy as np

KNN = 64


@lru_cache(maxsize=32)
def lane_emden(n_index: float, dxi: float = 2e-4):
    """Solve theta'' + (2/xi) theta' + theta^n = 0 (RK4) up to the first zero.

    Returns (xi, theta, dtheta, xi1) on a uniform grid ending at the surface.
    """
    xi0 = 1e-6
    th = 1.0 - xi0 * xi0 / 6.0
    dth = -xi0 / 3.0

    def f(x, t, d):
        return d, -(np.maximum(t, 0.0) ** n_index) - 2.0 * d / x

    xs, ts, ds = [xi0], [th], [dth]
    x = xi0
    while th > 0.0:
        k1 = f(x, th, dth)
        k2 = f(x + dxi / 2, th + dxi / 2 * k1[0], dth + dxi / 2 * k1[1])
        k3 = f(x + dxi / 2, th + dxi / 2 * k2[0], dth + dxi / 2 * k2[1])
        k4 = f(x + dxi, th + dxi * k3[0], dth + dxi * k3[1])
        th_new = th + dxi / 6 * (k1[0] + 2 * k2[0] + 2 * k3[0] + k4[0])
        dth = dth + dxi / 6 * (k1[1] + 2 * k2[1] + 2 * k3[1] + k4[1])
        x += dxi
        if th_new <= 0.0:
            # linear interpolation to the zero
            frac = th / (th - th_new)
            x1 = x - dxi + frac * dxi
            xs.append(x1)
            ts.append(0.0)
            ds.append(dth)
            break
        th = th_new
        xs.append(x)
        ts.append(th)
        ds.append(dth)
        if x > 50.0:
            raise RuntimeError("Lane-Emden integration did not reach the surface")
    xs, ts, ds = np.array(xs), np.array(ts), np.array(ds)
    return xs, ts, ds, xs[-1]


def _isotropic(rng: np.random.Generator, r: np.ndarray) -> np.ndarray:
    v = rng.normal(size=(r.shape[0], 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v * r[:, None]


def polytrope_equal_mass(rng: np.random.Generator, n: int, n_index: float, mass: float = 1.0,
                         radius: float = 1.0):
    """Equal-mass particles with the Lane-Emden density profile: radii by
    inverse CDF of the enclosed mass m(xi) ~ -xi^2 theta'(xi)."""
    xi, th, dth, xi1 = lane_emden(float(n_index))
    menc = -xi * xi * dth
    menc = np.maximum.accumulate(menc / menc[-1])
    u = rng.random(n)
    r = np.interp(u, menc, xi) / xi1 * radius
    pos = _isotropic(rng, r)
    m = np.full(n, mass / n)
    return pos, m


def knn_range2(pos: np.ndarray, k: int = KNN) -> np.ndarray:
    """range2 = (2 hp)^2 with 2 hp = distance to the k-th nearest other particle."""
    from scipy.spatial import cKDTree
    tree = cKDTree(pos)
    d, _ = tree.query(pos, k=k + 1, workers=-1)
    return d[:, k] ** 2


@dataclass
class ParticleSets:
    """Concatenated particle sets: set s is [offsets[s], offsets[s+1])."""
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    m: np.ndarray
    range2: np.ndarray
    offsets: np.ndarray
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.offsets[-1])

    @property
    def nsets(self) -> int:
        return len(self.offsets) - 1

    @property
    def pairs(self) -> int:
        d = np.diff(self.offsets).astype(np.int64)
        return int(np.sum(d * d))

    def subset(self, s: int) -> "ParticleSets":
        a, b = int(self.offsets[s]), int(self.offsets[s + 1])
        return ParticleSets(self.x[a:b].copy(), self.y[a:b].copy(), self.z[a:b].copy(),
                            self.m[a:b].copy(), self.range2[a:b].copy(),
                            np.array([0, b - a], dtype=np.int32), f"{self.name}[{s}]")


def _pack(parts: List[tuple], name: str, meta: dict) -> ParticleSets:
    xs, ms, rs, offs = [], [], [], [0]
    for pos, m, r2 in parts:
        xs.append(pos)
        ms.append(m)
        rs.append(r2)
        offs.append(offs[-1] + pos.shape[0])
    pos = np.concatenate(xs)
    return ParticleSets(np.ascontiguousarray(pos[:, 0]), np.ascontiguousarray(pos[:, 1]),
                        np.ascontiguousarray(pos[:, 2]), np.concatenate(ms), np.concatenate(rs),
                        np.array(offs, dtype=np.int32), name, meta)


def from_snapshots(paths: List[str]) -> ParticleSets:
    """Real models as a batch: one set per dump file (sph.start*u, out*.sph),
    with range2 built as the gravity call builds it (grav.f:15-18)."""
    from .snapshot import read_snapshot
    parts = []
    for path in paths:
        s = read_snapshot(path)
        pos = np.stack([s.data["x"], s.data["y"], s.data["z"]], axis=1)
        parts.append((pos, s.data["am"].copy(), s.range2()))
    return _pack(parts, "snapshots", {"paths": list(paths)})


def single_polytrope(n: int, n_index: float = 1.5, seed: int = 1, mass: float = 1.0,
                     radius: float = 1.0) -> ParticleSets:
    rng = np.random.default_rng(seed)
    pos, m = polytrope_equal_mass(rng, n, n_index, mass, radius)
    return _pack([(pos, m, knn_range2(pos))], f"polytrope_n{n_index}_N{n}",
                 {"n_index": n_index})


def config1(seed: int = 1) -> ParticleSets:
    """N=16,384 equal-mass n=1.5 polytrope, M=1, R=1."""
    s = single_polytrope(16384, 1.5, seed)
    s.name = "config1_polytrope_n1.5_N16384"
    return s


def collision_pair(rng: np.random.Generator, n1: int, n2: int, idx1: float, m1: float, r1: float,
                   idx2: float, m2: float, r2_: float, x1: float, x2: float):
    p1, ma = polytrope_equal_mass(rng, n1, idx1, m1, r1)
    p2, mb = polytrope_equal_mass(rng, n2, idx2, m2, r2_)
    p1[:, 0] += x1
    p2[:, 0] += x2
    pos = np.concatenate([p1, p2])
    return pos, np.concatenate([ma, mb])


def config2(seed: int = 2, n_each: int = 131072) -> ParticleSets:
    """Two-star collision snapshot: n=3 (M=1,R=1) at x=-1.5 and n=1.5
    (M=0.5, R=0.6) at x=+1.5; kNN smoothing on the combined set."""
    rng = np.random.default_rng(seed)
    pos, m = collision_pair(rng, n_each, n_each, 3.0, 1.0, 1.0, 1.5, 0.5, 0.6, -1.5, 1.5)
    return _pack([(pos, m, knn_range2(pos))], f"config2_collision_N{2 * n_each}", {})


def red_giant(n: int = 1048576, seed: int = 3, core_mass: float = 0.3, core_hp: float = 0.05,
              span_h: float = 1e-3, span_m: float = 1e-4) -> ParticleSets:
    """Red-giant envelope (n=3 polytrope, R=1) with a point-mass core.

    n-1 gas particles with radii log-uniform in [span_h * r_t, r_t], where r_t
    is the radius at which rho/rho_c = span_m (equal particle counts per
    logarithmic radius shell, so kNN smoothing lengths grow ~ r and span
    ~1/span_h); particle masses m ~ rho(r) r^3 (= rho / number density),
    floored at span_m * max(m) so they span 1/span_m, and normalised to
    1 - core_mass.  The core sits at the origin with m = core_mass,
    hp = core_hp (range2 = -(2 hp)^2: a point mass, u = 0)."""
    rng = np.random.default_rng(seed)
    xi, th, _, xi1 = lane_emden(3.0)
    thr = span_m ** (1.0 / 3.0)
    r_t = float(np.interp(-thr, -th, xi)) / xi1
    ng = n - 1
    r = np.exp(rng.uniform(np.log(span_h * r_t), np.log(r_t), size=ng))
    rho = np.interp(r * xi1, xi, th) ** 3
    m = rho * r ** 3
    m = np.maximum(m, span_m * m.max())
    m *= (1.0 - core_mass) / m.sum()
    pos = _isotropic(rng, r)
    r2 = knn_range2(pos)
    pos = np.concatenate([np.zeros((1, 3)), pos])
    m = np.concatenate([[core_mass], m])
    r2 = np.concatenate([[-(2.0 * core_hp) ** 2], r2])
    return _pack([(pos, m, r2)], f"config3_redgiant_N{n}",
                 {"r_t": r_t, "core_mass": core_mass, "core_hp": core_hp})


def config3(seed: int = 3) -> ParticleSets:
    return red_giant(1048576, seed)


def batch_models(nsets: int = 64, nmin: int = 4096, nmax: int = 131072, seed: int = 4,
                 scale: float = 1.0) -> ParticleSets:
    """Independent stellar models: N log-uniform in [nmin, nmax] (times
    ``scale`` for reduced test versions), polytropic index U[1, 3], M=1, R=1."""
    rng = np.random.default_rng(seed)
    parts = []
    ns, idx = [], []
    for _ in range(nsets):
        n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax))) * scale))
        n = max(n, 2)
        ni = float(rng.uniform(1.0, 3.0))
        pos, m = polytrope_equal_mass(rng, n, ni)
        parts.append((pos, m, knn_range2(pos)))
        ns.append(n)
        idx.append(ni)
    return _pack(parts, f"config4_batch_{nsets}sets", {"n": ns, "n_index": idx})


def config4(seed: int = 4) -> ParticleSets:
    return batch_models(64, 4096, 131072, seed)


def collision_snapshots(nsnap: int = 16, nmin: int = 65536, nmax: int = 524288, seed: int = 5,
                        scale: float = 1.0) -> ParticleSets:
    """Collision snapshots: total N log-uniform in [nmin, nmax] (times
    ``scale``), mass ratio q ~ U[0.2, 1], separation ~ U[2, 4]; primary n=3
    (M=1, R=1), secondary n=1.5 (M=q, R=q); equal-mass particles; centre of
    mass at the origin."""
    rng = np.random.default_rng(seed)
    parts, meta = [], []
    for _ in range(nsnap):
        n = max(4, int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax))) * scale)))
        q = float(rng.uniform(0.2, 1.0))
        sep = float(rng.uniform(2.0, 4.0))
        n1 = int(round(n / (1.0 + q)))
        n2 = n - n1
        x1, x2 = -sep * q / (1.0 + q), sep / (1.0 + q)
        pos, m = collision_pair(rng, n1, n2, 3.0, 1.0, 1.0, 1.5, q, q, x1, x2)
        parts.append((pos, m, knn_range2(pos)))
        meta.append({"n": n, "q": q, "sep": sep})
    return _pack(parts, f"config5_sweep_{nsnap}snapshots", {"snapshots": meta})


def config5(seed: int = 5) -> ParticleSets:
    return collision_snapshots(16, 65536, 524288, seed)


CONFIGS = {"config1": config1, "config2": config2, "config3": config3, "config4": config4,
           "config5": config5}


def cached(name: str, seed: int | None = None, **kw) -> ParticleSets:
    """Generate (or reload from a temp-dir cache) a named workload."""
    fn = CONFIGS[name]
    args = {} if seed is None else {"seed": seed}
    args.update(kw)
    key = hashlib.sha1(repr((name, sorted(args.items()), 2)).encode()).hexdigest()[:16]
    path = os.path.join(tempfile.gettempdir(), f"sphgrav_b200_{name}_{key}.npz")
    if os.path.exists(path):
        try:
            d = np.load(path, allow_pickle=False)
            return ParticleSets(d["x"], d["y"], d["z"], d["m"], d["range2"], d["offsets"],
                                str(d["name"]))
        except Exception:
            pass
    s = fn(**args)
    tmp = path + f".{os.getpid()}.tmp.npz"
    np.savez(tmp, x=s.x, y=s.y, z=s.z, m=s.m, range2=s.range2, offsets=s.offsets,
             name=np.array(s.name))
    os.replace(tmp, path)
    return s
