"""Python-3 drop-in for the kriging entry points of the reference's
``geo_bsd`` package (geo_bsd/geo.py), running on the B200 library."""

from .geo import *  # noqa: F401,F403
