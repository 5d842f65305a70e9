"""The host side of sequential simulation (hpgl_b200/csrc/sgs_host.cpp: the
reference's random path walked from jump-ahead starts on several threads,
boost's mt11213b draws and their quantiles computed behind the generator,
the normal-score transforms with their bucketed lower bounds), built for the
host by tests/cpp/sim_host_check.cpp and compared with the restatement."""

import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(ROOT, "hpgl_b200", "csrc")


@pytest.fixture(scope="module")
def shc(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("shc") / "sim_host_check.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-pthread", "-o", out,
                    "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "cpp", "sim_host_check.cpp"),
                    os.path.join(SRC, "sgs_host.cpp"), os.path.join(SRC, "plan.cpp"),
                    os.path.join(SRC, "task_pool.cpp")], check=True,
                   capture_output=True)
    lib = C.CDLL(out)
    lib.shc_path.restype = C.c_longlong
    return lib


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def _path(shc, shape, mask, seed, quantiles, sim_mask=None):
    n = int(np.prod(shape))
    nodes = np.zeros(n, np.int32)
    u = np.zeros(n)
    sm = None if sim_mask is None else np.ascontiguousarray(sim_mask, np.uint8)
    cnt = shc.shc_path(*shape, _ptr(mask, C.c_ubyte), _ptr(sm, C.c_ubyte), C.c_longlong(seed), int(quantiles),
                       _ptr(nodes, C.c_int), _ptr(u, C.c_double))
    return (nodes[:cnt], u[:cnt]) if cnt >= 0 else cnt


@pytest.mark.parametrize("shape,seed", [((166, 141, 30), 3439275), ((17, 11, 5), 99), ((64, 64, 64), 2 ** 32 + 5),
                                        ((7, 3, 2), 0), ((250, 1, 1), 12345), ((5, 1, 1), 8), ((4, 1, 1), 3),
                                        ((1, 1, 1), 1), ((2, 1, 1), 1), ((3, 2, 1), 4), ((2, 2, 2), 5),
                                        ((3, 2, 2), 6), ((9, 1, 1), 2)])
def test_path_and_quantiles_match_restatement(shc, shape, seed):
    rng = np.random.default_rng(1)
    n = int(np.prod(shape))
    mask = (rng.random(n) < 0.02).astype(np.uint8)
    sm = (rng.random(n) < 0.8).astype(np.uint8) if n > 1000 else None
    nodes, xp = _path(shc, shape, mask, seed, True, sm)
    job = dict(shape=shape, values=np.zeros(n, np.float32), mask=mask,
               params=[dict(cov_type=0, ranges=(2.0, 2.0, 2.0), angles=(0.0, 0.0, 0.0), sill=1.0, nugget=0.0,
                            radii=(1, 1, 1), max_neighbours=1)])
    _, _, order = O.sgs(job, seed=seed, sim_mask=sm)
    assert np.array_equal(nodes, order)
    assert np.array_equal(xp.view(np.uint64), O.sgs_draws(seed, nodes.size).view(np.uint64))
    nodes2, u = _path(shc, shape, mask, seed, False, sm)
    assert np.array_equal(nodes2, nodes) and ((u >= 0) & (u <= 1)).all()


def test_repeating_walks_skip_simulated_nodes(shc):
    # sizes 2, 4, 6, 8, 12 fall back to C = 2, which divides the size: the walk
    # repeats nodes and the reference simulates each once
    for n in (2, 4, 6, 8, 12):
        mask = np.zeros(n, np.uint8)
        for seed in range(n):
            nodes, _ = _path(shc, (n, 1, 1), mask, seed, True)
            assert len(set(nodes.tolist())) == nodes.size


def test_path_refusals(shc):
    mask = np.zeros(8, np.uint8)
    assert _path(shc, (2, 2, 2), mask, -3, True) == -2
    assert _path(shc, (2, 2, 2), mask, 2 ** 31, True) == -2


@pytest.mark.parametrize("dup", [False, True])
def test_cdf_transforms_match_restatement(shc, dup):
    rng = np.random.default_rng(2)
    vals = np.sort(rng.normal(size=5000).astype(np.float32))
    if dup:
        vals[100:140] = vals[100]
    u, c = np.unique(vals, return_counts=True)
    cv = u[:-1].copy()
    cp = np.cumsum(c[:-1] / float(vals.size)).astype(np.float32)
    if dup:
        cp[200:230] = cp[200]  # repeated probabilities
    x = np.concatenate([rng.normal(size=200000).astype(np.float32) * 1.5, cv[::7], cv[::11] + 1e-7,
                        np.array([-0.0, 0.0, cv[0], cv[-1], cv[0] - 1, cv[-1] + 1, np.inf, -np.inf],
                                 np.float32)]).astype(np.float32)
    mask = (rng.random(x.size) < 0.9).astype(np.uint8)
    for direction, m in ((0, mask), (0, None), (1, mask)):
        got = x.copy()
        shc.shc_cdf(_ptr(cv, C.c_float), _ptr(cp, C.c_float), C.c_longlong(cv.size), _ptr(got, C.c_float),
                    _ptr(m, C.c_ubyte), C.c_longlong(got.size), direction, 4)
        want = O.cdf_transform(x, (cv, cp), direction, m)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), direction
