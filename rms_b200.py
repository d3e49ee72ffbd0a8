"""Import name for the package directory ``monte-carlo-simulation-3d-rms_b200/``.

That directory name is not a Python identifier, so this module loads the
package from it under the name ``rms_b200`` and replaces itself in
``sys.modules``; ``import rms_b200`` and ``from rms_b200 import runio`` then
work from the repository root.
"""
import importlib.util as _ilu
import os as _os
import sys as _sys

_DIR = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)),
                     "monte-carlo-simulation-3d-rms_b200")
_spec = _ilu.spec_from_file_location(__name__, _os.path.join(_DIR, "__init__.py"),
                                     submodule_search_locations=[_DIR])
_mod = _ilu.module_from_spec(_spec)
_sys.modules[__name__] = _mod
_spec.loader.exec_module(_mod)
