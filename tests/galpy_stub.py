"""Import galpy from the reference tree without matplotlib (TEST ONLY).

galpy imports matplotlib at module level (galpy/util/plot.py) only for
plotting; none of the orbit or potential code used by the tests needs it.
This installs inert stand-ins for matplotlib / mpl_toolkits before importing
galpy from the reference checkout, when that checkout exists (it does in the
build container; it does not on GPU machines, where the galpy-based tests
are skipped)."""
import os
import sys
import types

REFERENCE = os.environ.get("GALPY_REFERENCE_TREE", "/root/reference")


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


def import_galpy():
    """Return the galpy module from the reference tree, or None if absent."""
    if "galpy" in sys.modules:
        return sys.modules["galpy"]
    if not os.path.isdir(os.path.join(REFERENCE, "galpy")):
        return None
    try:
        import matplotlib  # noqa: F401
    except ImportError:
        for name in _STUBS:
            sys.modules.setdefault(name, _StubModule(name))
    os.environ.setdefault("HOME", "/tmp")
    if REFERENCE not in sys.path:
        sys.path.insert(0, REFERENCE)
    import galpy

    return galpy
