"""Loader for the unmodified reference (bempp_cl) installed under ``baseline/_ref``.

TEST AND BASELINE INFRASTRUCTURE ONLY: the tests use the real reference to
check the drop-in boundary (its grids, spaces and operator API driving the
cuda device interface) and its Numba path as a live oracle; bench.py's CPU
legs time its Numba path.  The product package never imports this.

The install is ``pip install --no-index --no-build-isolation --no-deps
--target baseline/_ref <copy of the reference>`` (``install()`` below, run by
``__graft_entry__.build()`` when the reference sources are present); numba,
numpy and scipy come from the environment.  ``meshio`` is absent here and
only used by the reference's grid file I/O (bempp_cl/api/grid/io.py:3), so an
empty module stands in for it.  Bytecode and Numba caches are kept out of the
install.
"""

import contextlib as _contextlib
import io as _io
import os as _os
import shutil as _shutil
import subprocess as _sp
import sys as _sys
import tempfile as _tempfile
import types as _types

ROOT = _os.path.dirname(_os.path.dirname(_os.path.abspath(__file__)))
INSTALL = _os.path.join(ROOT, "baseline", "_ref")

_module = None
_reason = None


def install(source):
    """pip-install the reference sources at ``source`` (read-only) into baseline/_ref, offline."""
    if _os.path.isdir(_os.path.join(INSTALL, "bempp_cl")):
        return
    with _tempfile.TemporaryDirectory() as tmp:
        copy = _os.path.join(tmp, "src")
        _shutil.copytree(source, copy, ignore=_shutil.ignore_patterns("__pycache__", ".git"))
        _sp.run([_sys.executable, "-m", "pip", "install", "-q", "--no-index", "--no-build-isolation", "--no-deps",
                 "--target", INSTALL, copy], check=True)


def load():
    """The ``bempp_cl`` package of the install, or None (``reason()`` says why)."""
    global _module, _reason
    if _module is not None or _reason is not None:
        return _module
    if not _os.path.isdir(_os.path.join(INSTALL, "bempp_cl")):
        _reason = "bempp_cl is not installed under baseline/_ref"
        return None
    _sys.dont_write_bytecode = True
    _os.environ.setdefault("NUMBA_CACHE_DIR", _os.path.join(_tempfile.gettempdir(), "bempp_cl_numba_cache"))
    if INSTALL not in _sys.path:
        _sys.path.append(INSTALL)
    try:
        import meshio  # noqa: F401
    except ImportError:
        _sys.modules["meshio"] = _types.ModuleType("meshio")
    try:
        import numba  # noqa: F401

        # the reference prints a notice about optional packages (gmsh, plotting) when imported;
        # keep stdout for the callers' own output
        with _contextlib.redirect_stdout(_io.StringIO()):
            import bempp_cl.api  # noqa: F401
    except Exception as exc:  # pragma: no cover - depends on the environment
        _reason = "bempp_cl does not import: %s: %s" % (type(exc).__name__, exc)
        return None
    import bempp_cl

    _module = bempp_cl
    return _module


def reason():
    return _reason


def grid_from(grid):
    """A reference ``bempp_cl.api.Grid`` with the vertices and elements of ``grid``."""
    import numpy as np

    bempp_cl = load()
    return bempp_cl.api.Grid(np.asarray(grid.vertices, dtype=np.float64), np.asarray(grid.elements, dtype=np.uint32))
