"""Seeded synthetic point clouds with the shapes, sizes and value distributions
of the benchmark configurations (FP64 coordinates in [0, 1)^3, duplicates
removed keeping the first occurrence).

  uniform(n, seed)          i.i.d. U[0,1)^3                       (100k config)
  mixed(n, seed)            half uniform, half N(0.5, 0.1^2) per axis clipped
                            to [0,1)                               (1M config)
  degenerate(n, seed)       50% on the sphere r=0.4 about the cube centre, 30%
                            snapped to the 1/1024 lattice, 20% uniform (500k)
  clustered(n, k, sigma)    60% uniform, 40% k-cluster Gaussian mixture (8M)
  batch_sizes(count, seed)  cloud sizes log-uniform in [64, 50000] (4096 clouds)
  batch_cloud(n, kind, seed) uniform / Gaussian sigma=0.1 / 8-cluster sigma=0.02
"""
import numpy as np

_ONE_MINUS = np.nextafter(1.0, 0.0)


def _dedup(p):
    _, first = np.unique(p, axis=0, return_index=True)
    return np.ascontiguousarray(p[np.sort(first)])


def _clip01(p):
    return np.clip(p, 0.0, _ONE_MINUS)


def uniform(n, seed=1):
    rng = np.random.default_rng(seed)
    return _dedup(rng.random((n, 3)))


def mixed(n, seed=1):
    rng = np.random.default_rng(seed)
    h = n // 2
    a = rng.random((h, 3))
    b = _clip01(rng.normal(0.5, 0.1, size=(n - h, 3)))
    return _dedup(np.concatenate([a, b]))


def degenerate(n, seed=1):
    rng = np.random.default_rng(seed)
    ns, nl = n // 2, (3 * n) // 10
    nu = n - ns - nl
    d = rng.normal(size=(ns, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    sph = 0.5 + 0.4 * d
    lat = np.floor(rng.random((nl, 3)) * 1024.0) / 1024.0
    uni = rng.random((nu, 3))
    p = np.concatenate([sph, lat, uni])
    rng.shuffle(p)
    return _dedup(p)


def clustered(n, k=64, sigma=0.01, seed=1, uniform_frac=0.6):
    rng = np.random.default_rng(seed)
    nu = int(round(n * uniform_frac))
    centers = 0.1 + 0.8 * rng.random((k, 3))
    lab = rng.integers(0, k, size=n - nu)
    g = _clip01(centers[lab] + rng.normal(0.0, sigma, size=(n - nu, 3)))
    return _dedup(np.concatenate([rng.random((nu, 3)), g]))


def batch_sizes(count=4096, seed=1, lo=64, hi=50000):
    rng = np.random.default_rng(seed)
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))).astype(np.int64)


def batch_clouds(count=4096, seed=1, hi=50000):
    """The 4,096-cloud batch: sizes log-uniform in [64, hi], each cloud uniform,
    Gaussian (sigma 0.1) or an 8-cluster mixture (sigma 0.02) by a seeded draw.
    Returns (list of clouds, concatenated points, int64 offsets)."""
    sizes = batch_sizes(count, seed=seed, hi=hi)
    kinds = np.random.default_rng(seed + 7).integers(0, 3, size=count)
    clouds = [batch_cloud(int(n), int(k), seed * 100003 + i) for i, (n, k) in enumerate(zip(sizes, kinds))]
    offs = np.zeros(count + 1, np.int64)
    offs[1:] = np.cumsum([len(c) for c in clouds])
    return clouds, np.concatenate(clouds), offs


def batch_cloud(n, kind, seed):
    rng = np.random.default_rng(seed)
    if kind == 0:
        p = rng.random((n, 3))
    elif kind == 1:
        p = _clip01(rng.normal(0.5, 0.1, size=(n, 3)))
    else:
        centers = 0.1 + 0.8 * rng.random((8, 3))
        p = _clip01(centers[rng.integers(0, 8, size=n)] + rng.normal(0.0, 0.02, size=(n, 3)))
    return _dedup(p)


def config_cloud(name, scale=1.0, seed=1):
    """Cloud of a named benchmark configuration; `scale` shrinks the point count
    (used for CPU-sized parity cases)."""
    if name == "uniform100k":
        return uniform(int(100_000 * scale), seed), 256
    if name == "mixed1m":
        return mixed(int(1_000_000 * scale), seed), 512
    if name == "degenerate500k":
        return degenerate(int(500_000 * scale), seed), 512
    if name == "clustered8m":
        return clustered(int(8_000_000 * scale), seed=seed), 1024
    raise KeyError(name)
