from cmmdft_b200.units import *  # noqa: F401,F403
from cmmdft_b200.units import parse_unit  # noqa: F401
