"""Seeded inputs for the experimental-variogram tests: grids of values with
an informed mask (Fortran and C order, a strided view), point sets, search
templates, and layer thickness maps the reference stacks without writing out
of bounds."""

import numpy as np

# (lag width, separation, tolerance, lags, first lag, radii (R1, R2, R3), angles (az, dip, rot))
TEMPLATES = {
    "x_narrow": (2.0, 2.0, 0.8, 8, 0.0, (20.0, 3.0, 2.0), (30.0, 0.0, 0.0)),
    "overlapping_lags": (3.0, 1.5, 0.5, 10, 1.0, (15.0, 4.0, 2.0), (0.0, 0.0, 0.0)),
    "dipping": (4.0, 4.0, 0.3, 6, 2.0, (30.0, 6.0, 4.0), (45.0, 30.0, 10.0)),
    "vertical": (1.0, 1.0, 0.9, 5, 0.0, (6.0, 2.0, 2.0), (0.0, 90.0, 0.0)),
}


def grid(shape, informed, seed, order="F"):
    rng = np.random.default_rng(seed)
    x = np.arange(shape[0])[:, None, None]
    v = (rng.normal(size=shape) + 0.05 * x).astype(np.float32)
    m = (rng.random(shape) < informed).astype(np.uint8)
    return np.require(v, requirements=order), np.require(m, requirements=order)


def points(n, seed, extent=(60.0, 40.0, 10.0)):
    rng = np.random.default_rng(seed)
    xs = (rng.random(n) * extent[0]).astype(np.float32)
    ys = (rng.random(n) * extent[1]).astype(np.float32)
    zs = (rng.random(n) * extent[2]).astype(np.float32)
    vals = (rng.normal(size=n) + 0.02 * xs).astype(np.float32)
    return xs, ys, zs, vals


def layers(nx, ny, n, seed):
    """Thickness maps: positive layers, and erosions (negative) no deeper
    than what lies below them."""
    rng = np.random.default_rng(seed)
    out = []
    for l in range(n):
        a = rng.uniform(0.2, 4.0, (nx, ny)).astype(np.float32)
        if l % 3 == 2:
            a = -rng.uniform(0.0, 1.5, (nx, ny)).astype(np.float32)
        out.append(np.asfortranarray(a))
    return out
