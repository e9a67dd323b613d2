"""
Import name for the package kept in ``q-pop-diffraction_b200/``.

A directory name with hyphens cannot be imported directly, so this module loads
``q-pop-diffraction_b200/__init__.py`` as the package ``qpop_diffraction_b200``
(its submodules resolve from that directory) and puts it in ``sys.modules``.
"""

import importlib.util
import os
import sys

_dir = os.path.join(os.path.dirname(os.path.abspath(__file__)), "q-pop-diffraction_b200")
_spec = importlib.util.spec_from_file_location(__name__, os.path.join(_dir, "__init__.py"),
                                               submodule_search_locations=[_dir])
_pkg = importlib.util.module_from_spec(_spec)
sys.modules[__name__] = _pkg
_spec.loader.exec_module(_pkg)
