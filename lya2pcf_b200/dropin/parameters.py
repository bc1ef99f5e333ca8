"""Top-level ``parameters`` module for the reference's drivers: re-exports
:mod:`lya2pcf_b200.parameters` (the constants of lya2pcf ``parameters.py``)."""
import os
import sys

_root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if _root not in sys.path:
    sys.path.insert(0, _root)

from lya2pcf_b200.parameters import *   # noqa: E402,F401,F403
