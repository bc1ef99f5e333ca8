"""Access to the drop-in module directory (``lya2pcf_b200/dropin``).

The drop-in directory holds top-level modules named as the reference's
(``forest_class``, ``parameters``, ``correlation_procedures_pycuda``, ...), so
that pickled catalogues and the reference's drivers resolve to this package.
"""
import os
import sys

DROPIN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'dropin')


def ensure_on_path():
    if DROPIN_DIR not in sys.path:
        sys.path.insert(0, DROPIN_DIR)


def quasar_class():
    ensure_on_path()
    import forest_class
    return forest_class.quasar
