"""B200-native explicit MPM ductile-fracture substep (Python host binding).

The product is the C-ABI library ``libgmpm.so`` (include/gmpm.h) built from
``csrc/`` for sm_100a; this package loads it through ctypes for tests and
benchmarks.  The directory name contains hyphens, so callers import it by
path with ``importlib.util.spec_from_file_location``.
"""
from . import gmpm, scenes  # noqa: F401
from .gmpm import Context, Scene, lib  # noqa: F401
