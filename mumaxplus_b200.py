"""Import shim: `import mumaxplus_b200` loads the package in ./mumax-plus_b200/.

The package directory carries a hyphen, which `import` cannot name, so this
module loads it under the importable name and replaces itself with it.
"""
import importlib.util as _util
import os as _os
import sys as _sys

_here = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "mumax-plus_b200")
_spec = _util.spec_from_file_location(__name__, _os.path.join(_here, "__init__.py"),
                                      submodule_search_locations=[_here])
_mod = _util.module_from_spec(_spec)
_sys.modules[__name__] = _mod
_spec.loader.exec_module(_mod)
