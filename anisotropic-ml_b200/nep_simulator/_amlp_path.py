"""Makes the ``amlp`` package importable for the flat, script-style modules of
this directory (the reference runs ``python sim_input.py`` from inside
``nep_simulator/`` and imports its modules by bare name)."""
import os
import sys

_PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if _PKG_ROOT not in sys.path:
    sys.path.insert(0, _PKG_ROOT)
