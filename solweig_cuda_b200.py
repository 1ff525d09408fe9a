"""Import name of the package that lives in the directory ``solweig-cuda_b200/``.

The directory name is not a Python identifier, so this module stands in for
the package: it points the package search path at that directory and runs
its ``__init__.py``.  ``import solweig_cuda_b200.svf`` and friends then
resolve inside ``solweig-cuda_b200/``.
"""
import os as _os

__path__ = [_os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "solweig-cuda_b200")]
_init = _os.path.join(__path__[0], "__init__.py")
with open(_init, encoding="utf-8") as _f:
    exec(compile(_f.read(), _init, "exec"))
del _f, _init
