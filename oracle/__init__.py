"""FP64 CPU oracle of the TurboGAP SOAP-GAP path (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` leg may
load this package; the product path in ``turbogap_b200`` never does.
"""
from .oracle import *  # noqa: F401,F403
