"""Argument checks of the simulation wrappers (hpgl_b200.geo_bsd.sgs / sis /
cdf) that run before the library is called, and the CDF the wrappers build
(the reference's calc_cdf) -- no GPU needed."""

import numpy as np
import pytest

from hpgl_b200.geo_bsd import cdf, geo, sgs, sis


def _prop(shape=(4, 3, 2)):
    rng = np.random.default_rng(0)
    data = np.asfortranarray(rng.normal(size=shape).astype(np.float32))
    mask = np.asfortranarray((rng.random(shape) < 0.5).astype(np.uint8))
    return geo.ContProperty(data, mask)


def test_calc_cdf_drops_the_largest_value_and_accumulates_in_order():
    data = np.asfortranarray(np.array([3, 1, 2, 2, 5, 1], np.float32).reshape(6, 1, 1))
    mask = np.asfortranarray(np.array([1, 1, 1, 1, 0, 1], np.uint8).reshape(6, 1, 1))
    c = cdf.calc_cdf(geo.ContProperty(data, mask))
    # informed values 3, 1, 2, 2, 1: distinct 1, 2, 3; the largest dropped
    assert c.values.tolist() == [1.0, 2.0]
    assert np.allclose(c.probs, [2 / 5, 4 / 5]) and c.probs.dtype == np.float32


def test_calc_cdf_single_value_is_kept():
    data = np.asfortranarray(np.full((3, 1, 1), 7, np.float32))
    mask = np.asfortranarray(np.ones((3, 1, 1), np.uint8))
    c = cdf.calc_cdf(geo.ContProperty(data, mask))
    assert c.values.tolist() == [7.0] and np.allclose(c.probs, [1.0])


def test_normed_cov_model_scales_to_unit_sill_minus_nugget():
    m = sgs.normed_cov_model(geo.CovarianceModel(type=1, ranges=(5, 5, 2), sill=0.5, nugget=0.1))
    assert abs((m.sill - m.nugget) - 1.0) < 1e-12 and abs(m.nugget - 0.25) < 1e-12


def test_sgs_rejects_mismatched_sizes():
    prop = _prop()
    cov = geo.CovarianceModel(type=0, ranges=(3, 3, 2))
    with pytest.raises(RuntimeError):
        sgs.sgs_simulation(prop, geo.SugarboxGrid(5, 3, 2), None, (2, 2, 1), 4, cov, 1)
    with pytest.raises(RuntimeError):
        sgs.sgs_simulation(prop, geo.SugarboxGrid(4, 3, 2), None, (2, 2, 1), 4, cov, 1, mask=np.ones(5, np.uint8))
    with pytest.raises(RuntimeError):
        sgs.sgs_simulation(prop, geo.SugarboxGrid(4, 3, 2), None, (2, 2, 1), 4, cov, 1, mean=np.zeros(7, np.float32))
    with pytest.raises(ValueError):
        sgs.sgs_simulation(prop, geo.SugarboxGrid(4, 3, 2), cdf.CdfData([1, 2], [0.5]), (2, 2, 1), 4, cov, 1)


def test_sis_rejects_mismatched_categories():
    data = np.asfortranarray(np.zeros((4, 3, 2), np.uint8))
    prop = geo.IndProperty(data, data.copy(), 2)
    cats = [{"cov_model": geo.CovarianceModel(type=0, ranges=(3, 3, 2)), "radiuses": (2, 2, 1),
             "max_neighbours": 4}] * 2
    with pytest.raises(ValueError):
        sis.sis_simulation(prop, geo.SugarboxGrid(4, 3, 2), cats, 1, [0.5])
    with pytest.raises(RuntimeError):
        sis.sis_simulation(prop, geo.SugarboxGrid(4, 3, 2), cats, 1, [0.5, 0.5], mask=np.ones(3, np.uint8))
