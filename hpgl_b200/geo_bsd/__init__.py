"""Python-3 drop-in for the entry points of the reference's ``geo_bsd``
package (geo_bsd/geo.py, sgs.py, sis.py, cdf.py), running on the B200 library."""

from .cdf import *  # noqa: F401,F403
from .geo import *  # noqa: F401,F403
from .sgs import *  # noqa: F401,F403
from .sis import *  # noqa: F401,F403
