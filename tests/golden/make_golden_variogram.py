"""Generates golden fixtures of the experimental variograms and layer
stacking from the reference's own _cvariogram sources compiled by
oracle/build_ref.sh: seeded grids (Fortran and C order), point sets and
thickness maps, and the reference's results for them.

    python tests/golden/make_golden_variogram.py      # needs the reference build

Writes tests/golden/variogram/<case>.npz."""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import oracle as O  # noqa: E402
import variogram_cases as VC  # noqa: E402

OUT = os.path.join(HERE, "variogram")


def spec_vec(spec):
    return np.array([spec[0], spec[1], spec[2], spec[3], spec[4], *spec[5], *spec[6]], np.float64)


def main():
    os.makedirs(OUT, exist_ok=True)
    for i, (name, spec) in enumerate(VC.TEMPLATES.items()):
        t = O.cv_template(*spec)
        v, m = VC.grid((30, 24, 8), 0.25, seed=40 + i, order="F" if i % 2 == 0 else "C")
        r = O.ref_variograms(t, v, m)
        np.savez_compressed(os.path.join(OUT, "grid_%s.npz" % name), kind=np.array("grid"), template=spec_vec(spec),
                            values=v, mask=m, result=r)
        xs, ys, zs, vals = VC.points(500, seed=50 + i)
        r = O.ref_variograms_points(t, xs, ys, zs, vals)
        np.savez_compressed(os.path.join(OUT, "points_%s.npz" % name), kind=np.array("points"),
                            template=spec_vec(spec), xs=xs, ys=ys, zs=zs, vals=vals, result=r)
        print("variograms", name)
    ls = VC.layers(21, 16, 8, seed=60)
    res = np.asfortranarray(np.full((21, 16, 14), -5, np.float32))
    O.stack_layers(ls, list(range(1, 9)), 14, 1.5, -1, res, reference=True)
    np.savez_compressed(os.path.join(OUT, "stack_layers.npz"), kind=np.array("stack"),
                        template=spec_vec(list(VC.TEMPLATES.values())[0]), layers=np.array(ls),
                        markers=np.arange(1, 9), nz=14, scalez=1.5, blank=-1, result=res)
    print("stack layers")


if __name__ == "__main__":
    main()
