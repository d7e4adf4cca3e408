"""Import name for the package directory ``iblbm-mechanism-resolved_b200/``.

The directory name is not a Python identifier, so this module loads the
package from it under the importable name ``iblbm_b200`` (submodules such as
``iblbm_b200.engine`` resolve inside that directory).
"""
import importlib.util
import os
import sys

_ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "iblbm-mechanism-resolved_b200")
_spec = importlib.util.spec_from_file_location(
    __name__, os.path.join(_ROOT, "__init__.py"), submodule_search_locations=[_ROOT])
_module = importlib.util.module_from_spec(_spec)
sys.modules[__name__] = _module
_spec.loader.exec_module(_module)
