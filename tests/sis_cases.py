"""Sequential indicator simulation cases shared by the oracle and GPU tests:
seeded codes and informed masks, per-category variograms (different
types, ranges and neighbour counts so every category has its own template
and table), and optional per-category mean cubes."""

import numpy as np

BASE = dict(cov_type=0, ranges=(8.0, 8.0, 4.0), angles=(0.0, 0.0, 0.0), sill=1.0, nugget=0.0, radii=(10, 10, 5),
            max_neighbours=12)


def params(K, big=False):
    ps = [dict(BASE, marginal_prob=0.3),
          dict(BASE, marginal_prob=0.45, cov_type=1, max_neighbours=8, angles=(30.0, 0.0, 0.0)),
          dict(BASE, marginal_prob=0.15, ranges=(5.0, 5.0, 3.0), cov_type=2, max_neighbours=16),
          dict(BASE, marginal_prob=0.1, ranges=(6.0, 4.0, 3.0), max_neighbours=10)]
    ps = [dict(p) for p in ps[:K]]
    if big:
        ps[0]["max_neighbours"] = 40
        ps[0]["radii"] = (12, 12, 6)
    return ps


def case(shape=(18, 16, 6), K=3, seed=5, informed=0.1):
    rng = np.random.default_rng(seed)
    n = int(np.prod(shape))
    codes = rng.integers(0, K, n).astype(np.uint8)
    mask = (rng.random(n) < informed).astype(np.uint8)
    return dict(shape=shape, codes=codes, mask=mask, values=None, kind="ik")


def means(shape, K, seed=7):
    rng = np.random.default_rng(seed)
    n = int(np.prod(shape))
    cubes = [np.clip(1.0 / K + 0.1 * rng.normal(size=n), 0, 1).astype(np.float32) for _ in range(K)]
    cubes[0][:7] = 0.0
    cubes[1][7:11] = 1.0
    return cubes
