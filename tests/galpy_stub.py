"""Import galpy without matplotlib (TEST ONLY).

galpy imports matplotlib at module level (galpy/util/plot.py) only for
plotting; none of the orbit or potential code used by the tests needs it.
This installs inert stand-ins for matplotlib / mpl_toolkits before importing
galpy from, in this order: the reference checkout (GALPY_REFERENCE_TREE,
where it exists), or the pure-Python galpy installed into baseline/_ref
(``pip install --no-deps --target baseline/_ref <galpy tree>``: git-ignored,
but copied with the working tree to GPU machines, so galpy's own
Orbit.integrate can drive the engine there).  Without either the galpy-based
tests are skipped."""
import os
import subprocess
import sys
import types


def _reference_tree():
    """The reference checkout the oracle's recipe reads (oracle/Makefile's
    REF: GALPY_REFERENCE_TREE, else its default); it need not exist."""
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    try:
        r = subprocess.run(["make", "-s", "-C", os.path.join(here, "oracle"), "print-ref"],
                           stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        return r.stdout.strip()
    except OSError:  # no make: only the installed copy can serve
        return ""


REFERENCE = _reference_tree()
INSTALLED = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                         "baseline", "_ref")


class _InertMeta(type):
    def __getattr__(cls, name):
        if name.startswith("__"):
            raise AttributeError(name)
        if name[:1].isupper():
            return _InertMeta(name, (_Inert,), {})
        return _Inert()


class _Inert(metaclass=_InertMeta):
    def __init__(self, *a, **k):
        pass

    def __call__(self, *a, **k):
        return _Inert()

    def __getattr__(self, name):
        return _Inert()


class _StubModule(types.ModuleType):
    def __getattr__(self, name):
        if name == "__version__":
            return "3.8.0"
        if name.startswith("__"):
            raise AttributeError(name)
        if name[:1].isupper():
            return _InertMeta(name, (_Inert,), {})
        return _Inert()


_STUBS = ["matplotlib", "matplotlib.pyplot", "matplotlib.ticker", "matplotlib.cm",
          "matplotlib.colors", "matplotlib.patches", "matplotlib.animation", "mpl_toolkits",
          "mpl_toolkits.mplot3d", "matplotlib.projections", "matplotlib.transforms",
          "matplotlib.lines", "matplotlib.collections", "matplotlib.projections.polar",
          "mpl_toolkits.axes_grid1", "matplotlib.gridspec"]


def galpy_root():
    """Directory to put on sys.path for galpy, or None."""
    for root in (REFERENCE, INSTALLED):
        if os.path.isfile(os.path.join(root, "galpy", "__init__.py")):
            return root
    return None


def import_galpy():
    """Return the galpy module, or None if no copy is available."""
    if "galpy" in sys.modules:
        return sys.modules["galpy"]
    root = galpy_root()
    if root is None:
        return None
    try:
        import matplotlib  # noqa: F401
    except ImportError:
        for name in _STUBS:
            sys.modules.setdefault(name, _StubModule(name))
    os.environ.setdefault("HOME", "/tmp")
    if root not in sys.path:
        sys.path.insert(0, root)
    import galpy

    return galpy
