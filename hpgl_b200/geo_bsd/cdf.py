"""Cumulative distributions of a property with the names of the reference's
geo_bsd/cdf.py: ``CdfData`` (cdf.py:3-6) and ``calc_cdf`` (:8-33) -- the
sorted distinct informed values without the largest one, each with the
cumulative frequency of the values up to it (float32 arrays).  The frequencies
accumulate in double in increasing value order, as the reference's loop did
(its values are the keys of a dict, so -0.0 and 0.0 count as one value).
"""

import numpy

__all__ = ["CdfData", "calc_cdf"]


class CdfData:
    def __init__(self, values, probs):
        self.values = numpy.require(values, "float32")
        self.probs = numpy.require(probs, "float32")


def calc_cdf(prop):
    data = numpy.asarray(prop.data)
    mask = numpy.asarray(prop.mask)
    informed = data[mask != 0].astype(numpy.float32, copy=False)
    values, counts = numpy.unique(informed, return_counts=True)
    size = values.size - 1 if values.size > 1 else values.size
    full_count = float(informed.size)
    # add.accumulate sums left to right, like the reference's running total
    probs = numpy.cumsum(counts[:size] / full_count)
    return CdfData(values=values[:size], probs=probs)
