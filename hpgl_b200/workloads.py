"""Seeded synthetic kriging workloads.

No public dataset exists for the reference's kriging path; these generators
stand in for it with the grid shapes, informed fractions, value
distributions and variogram/search parameters of the five benchmark cases:

* ``ok_50x50x20``      ordinary kriging, 50x50x20, 2 % uniform informed
                       cells, values N(0,1) + 0.01*x, spherical (10,10,5),
                       radii (20,20,10), 12 neighbours.
* ``sk_ok_256x256x64`` simple / ordinary kriging, 256x256x64, 1 % informed,
                       values from an FFT Gaussian random field (exponential
                       covariance, range 30), exponential (40,20,8) azimuth
                       30, sill 1, nugget 0.05, radii (80,40,16), 32
                       neighbours, SK mean 0.
* ``ik_200x200x100``   4-category indicator kriging, 200x200x100, codes from
                       thresholding a Gaussian field at its 0.25/0.5/0.75
                       quantiles, 1.5 % informed, spherical (25,25,6) sill
                       0.1875 for every category, radii (25,25,6), 24
                       neighbours, marginal probabilities 0.25.
* ``lvm_512x512x32``   LVM kriging, 512x512x32, mean cube = 8 low-frequency
                       sinusoids (total amplitude 0.5), 0.5 % informed cells
                       in 200 Gaussian blobs (sigma 3 cells), values = mean +
                       N(0, 0.3), Gaussian (30,30,4), nugget 0.01, radii
                       (40,40,5), 64 neighbours.
* ``serve_stream``     a Poisson stream of mixed jobs (see ``serve_stream``).

Arrays are Fortran-ordered (index = x + nx*(y + ny*z)), float32 values or
uint8 codes, uint8 masks, exactly as the reference's Python layer hands them
to the library.  Every generator takes a ``shape`` override so tests can run
the same statistics on grids small enough for the CPU oracle.
"""

import math

import numpy as np

SPHERICAL, EXPONENTIAL, GAUSSIAN = 0, 1, 2


def _choose_cells(rng, size, fraction):
    n = max(1, int(round(size * fraction)))
    return rng.choice(size, size=n, replace=False)


def gaussian_field(rng, shape, corr_range, cov="exponential"):
    """Stationary Gaussian random field with unit variance on ``shape``
    (periodic FFT method): white noise filtered by the square root of the
    covariance's spectrum, exponential ``exp(-3h/range)`` or Gaussian."""
    axes = [np.fft.fftfreq(n) * n for n in shape]
    gx, gy, gz = np.meshgrid(*axes, indexing="ij")
    h = np.sqrt(gx * gx + gy * gy + gz * gz)
    if cov == "gaussian":
        c = np.exp(-3.0 * (h / corr_range) ** 2)
    else:
        c = np.exp(-3.0 * h / corr_range)
    spec = np.fft.rfftn(c).real
    spec[spec < 0] = 0
    noise = rng.standard_normal(shape)
    f = np.fft.irfftn(np.sqrt(spec) * np.fft.rfftn(noise), s=shape, axes=(0, 1, 2))
    f = (f - f.mean()) / (f.std() + 1e-30)
    return f


def cov_params(cov_type, ranges, angles=(0.0, 0.0, 0.0), sill=1.0, nugget=0.0, radii=(1, 1, 1),
               max_neighbours=12, marginal_prob=0.0):
    return dict(cov_type=int(cov_type), ranges=tuple(float(r) for r in ranges),
                angles=tuple(float(a) for a in angles), sill=float(sill), nugget=float(nugget),
                radii=tuple(int(r) for r in radii), max_neighbours=int(max_neighbours),
                marginal_prob=float(marginal_prob))


def ok_50x50x20(shape=(50, 50, 20), seed=1):
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    size = nx * ny * nz
    values = np.full(size, -99.0, dtype=np.float32)
    mask = np.zeros(size, dtype=np.uint8)
    cells = _choose_cells(rng, size, 0.02)
    x = cells % nx
    values[cells] = (rng.standard_normal(len(cells)) + 0.01 * x).astype(np.float32)
    mask[cells] = 1
    return dict(name="ok_50x50x20", kind="ok", shape=shape, values=values, mask=mask,
                params=[cov_params(SPHERICAL, (10, 10, 5), radii=(20, 20, 10), max_neighbours=12)])


def sk_ok_256x256x64(shape=(256, 256, 64), seed=2, kind="sk"):
    rng = np.random.default_rng(seed)
    size = int(np.prod(shape))
    field = gaussian_field(rng, shape, 30.0).reshape(-1, order="F").astype(np.float32)
    values = np.full(size, -99.0, dtype=np.float32)
    mask = np.zeros(size, dtype=np.uint8)
    cells = _choose_cells(rng, size, 0.01)
    values[cells] = field[cells]
    mask[cells] = 1
    p = cov_params(EXPONENTIAL, (40, 20, 8), angles=(30, 0, 0), sill=1.0, nugget=0.05, radii=(80, 40, 16),
                   max_neighbours=32)
    return dict(name="sk_ok_256x256x64", kind=kind, shape=shape, values=values, mask=mask, params=[p],
                sk_mean=0.0)


def ik_200x200x100(shape=(200, 200, 100), seed=3, categories=4):
    rng = np.random.default_rng(seed)
    size = int(np.prod(shape))
    field = gaussian_field(rng, shape, 25.0).reshape(-1, order="F")
    qs = np.quantile(field, [(k + 1) / categories for k in range(categories - 1)])
    codes_all = np.searchsorted(qs, field).astype(np.uint8)
    codes = np.zeros(size, dtype=np.uint8)
    mask = np.zeros(size, dtype=np.uint8)
    cells = _choose_cells(rng, size, 0.015)
    codes[cells] = codes_all[cells]
    mask[cells] = 1
    p = [cov_params(SPHERICAL, (25, 25, 6), sill=0.1875, nugget=0.0, radii=(25, 25, 6), max_neighbours=24,
                    marginal_prob=1.0 / categories) for _ in range(categories)]
    return dict(name="ik_200x200x100", kind="ik", shape=shape, codes=codes, mask=mask, params=p)


def lvm_512x512x32(shape=(512, 512, 32), seed=4, blobs=200, sigma=3.0):
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    size = nx * ny * nz
    x = np.arange(nx, dtype=np.float64)[:, None, None]
    y = np.arange(ny, dtype=np.float64)[None, :, None]
    z = np.arange(nz, dtype=np.float64)[None, None, :]
    mean = np.zeros(shape)
    for _ in range(8):
        fx, fy, fz = rng.uniform(0.2, 2.0, 3) * np.array([1.0 / nx, 1.0 / ny, 0.5 / nz])
        ph = rng.uniform(0, 2 * math.pi)
        mean += np.sin(2 * math.pi * (fx * x + fy * y + fz * z) + ph)
    mean = (0.5 / 8.0 * mean).astype(np.float32).reshape(-1, order="F")
    target = max(1, int(round(size * 0.005)))
    centers = np.stack([rng.uniform(0, n, blobs) for n in shape], axis=1)
    chosen = np.zeros(size, dtype=bool)
    count = 0
    while count < target:
        b = rng.integers(0, blobs, 4096)
        p = centers[b] + rng.normal(0, sigma, (4096, 3))
        p = np.floor(p).astype(np.int64)
        ok = (p[:, 0] >= 0) & (p[:, 0] < nx) & (p[:, 1] >= 0) & (p[:, 1] < ny) & (p[:, 2] >= 0) & (p[:, 2] < nz)
        p = p[ok]
        idx = p[:, 0] + nx * (p[:, 1] + ny * p[:, 2])
        for i in idx:
            if count >= target:
                break
            if not chosen[i]:
                chosen[i] = True
                count += 1
    cells = np.nonzero(chosen)[0]
    values = np.full(size, -99.0, dtype=np.float32)
    values[cells] = (mean[cells] + rng.normal(0, 0.3, len(cells))).astype(np.float32)
    mask = chosen.astype(np.uint8)
    p = cov_params(GAUSSIAN, (30, 30, 4), sill=1.0, nugget=0.01, radii=(40, 40, 5), max_neighbours=64)
    return dict(name="lvm_512x512x32", kind="lvm", shape=shape, values=values, mask=mask, mean=mean, params=[p])


# Search radius = the extent along each axis where the model's covariance
# falls to 1 % of C(0), rounded up: f * range with f = 1.0 (spherical, zero at
# the range), 1.54 (exponential, exp(-3h/a) = 0.01) and 1.24 (Gaussian,
# exp(-3(h/a)^2) = 0.01) -- the extent of the reference's search template.
_RADIUS_FACTOR = {SPHERICAL: 1.0, EXPONENTIAL: 1.54, GAUSSIAN: 1.24}


def serve_job(rng, job_id=0, max_cells=256 * 256 * 64):
    """One job of the serving stream: grid log-uniform between 32^3 and
    256x256x64 cells, informed fraction 0.5-3 %, variogram type uniform over
    spherical/exponential/Gaussian, ranges 5-60, nugget 0-0.1, 8-64
    neighbours, search radii = the 1 % covariance extents (rounded up); kind 50 % OK, 25 % SK,
    25 % 4-category IK."""
    lo, hi = math.log(min(32 ** 3, max_cells)), math.log(max_cells)
    cells = math.exp(rng.uniform(lo, hi))
    aspect = np.array([4.0, 4.0, 1.0]) * rng.uniform(0.8, 1.25, 3)
    s = (cells / np.prod(aspect)) ** (1.0 / 3.0)
    shape = tuple(int(max(8, min(m, round(a * s)))) for a, m in zip(aspect, (256, 256, 64)))
    frac = rng.uniform(0.005, 0.03)
    cov_type = int(rng.integers(0, 3))
    ranges = rng.uniform(5, 60, 3)
    ranges[2] = min(ranges[2], ranges[0])
    nugget = rng.uniform(0, 0.1)
    nmax = int(rng.integers(8, 65))
    radii = tuple(int(math.ceil(_RADIUS_FACTOR[cov_type] * r)) for r in ranges)
    u = rng.uniform()
    kind = "ok" if u < 0.5 else ("sk" if u < 0.75 else "ik")
    size = int(np.prod(shape))
    cells_i = _choose_cells(rng, size, frac)
    mask = np.zeros(size, dtype=np.uint8)
    mask[cells_i] = 1
    if kind == "ik":
        codes = np.zeros(size, dtype=np.uint8)
        codes[cells_i] = rng.integers(0, 4, len(cells_i)).astype(np.uint8)
        sill = 0.1875
        p = [cov_params(cov_type, ranges, sill=sill, nugget=min(nugget, 0.5 * sill), radii=radii,
                        max_neighbours=nmax, marginal_prob=0.25) for _ in range(4)]
        return dict(name="serve_%d" % job_id, kind="ik", shape=shape, codes=codes, mask=mask, params=p)
    values = np.full(size, -99.0, dtype=np.float32)
    values[cells_i] = rng.standard_normal(len(cells_i)).astype(np.float32)
    p = cov_params(cov_type, ranges, sill=1.0, nugget=nugget, radii=radii, max_neighbours=nmax)
    return dict(name="serve_%d" % job_id, kind=kind, shape=shape, values=values, mask=mask, params=[p],
                sk_mean=0.0)


def serve_stream(n_jobs, rate_per_s, seed=5, max_cells=256 * 256 * 64):
    """Poisson arrivals at ``rate_per_s``: list of (arrival_time_s, job)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for j in range(n_jobs):
        t += rng.exponential(1.0 / rate_per_s)
        out.append((t, serve_job(rng, j, max_cells=max_cells)))
    return out


CONFIGS = {
    "ok_50x50x20": ok_50x50x20,
    "sk_ok_256x256x64": sk_ok_256x256x64,
    "ik_200x200x100": ik_200x200x100,
    "lvm_512x512x32": lvm_512x512x32,
}


def cokriging_job(shape=(48, 48, 12), mark=1, seed=6, informed=0.02, secondary_informed=0.9,
                  max_neighbours=16, correlation=0.7):
    """Colocated simple cokriging (Markov model I or II): a sparse primary
    property and a dense, correlated secondary one on the same grid.  The
    primary is a seeded Gaussian field (spherical covariance), the secondary
    0.7 x the same field + 0.7 x an independent one, informed at
    `secondary_informed` of the cells; means and the secondary variance are
    those of the informed values."""
    rng = np.random.default_rng(seed)
    size = int(np.prod(shape))
    f1 = gaussian_field(rng, shape, 12.0).reshape(-1, order="F")
    f2 = gaussian_field(rng, shape, 12.0).reshape(-1, order="F")
    prim = (2.0 + f1).astype(np.float32)
    sec = (5.0 + 0.7 * f1 + 0.7 * f2).astype(np.float32)
    values = np.full(size, -99.0, dtype=np.float32)
    mask = np.zeros(size, dtype=np.uint8)
    cells = _choose_cells(rng, size, informed)
    values[cells] = prim[cells]
    mask[cells] = 1
    smask = (rng.uniform(size=size) < secondary_informed).astype(np.uint8)
    svalues = np.where(smask > 0, sec, np.float32(-99.0)).astype(np.float32)
    p = cov_params(SPHERICAL, (14, 14, 5), sill=1.0, nugget=0.0, radii=(14, 14, 5), max_neighbours=max_neighbours)
    job = dict(name="cok%d_%dx%dx%d" % ((mark,) + tuple(shape)), kind="cok%d" % mark, shape=tuple(shape),
               values=values, mask=mask, secondary_values=svalues, secondary_mask=smask, params=[p],
               primary_mean=float(values[cells].astype(np.float64).mean()),
               secondary_mean=float(svalues[smask > 0].astype(np.float64).mean()),
               correlation=float(correlation))
    if mark == 1:
        job["secondary_variance"] = float(svalues[smask > 0].astype(np.float64).var())
    else:
        job["secondary_cov"] = cov_params(EXPONENTIAL, (20, 20, 6), sill=1.0, nugget=0.05)
    return job
