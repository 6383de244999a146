"""CPU checks of the drop-in boundary: the C-ABI library loads without a GPU and exports
every entry point include/*.h declares; the ctypes binding covers them all."""
import ctypes
import glob
import os
import re

import pytest

from cabanadem_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(dem_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("library not built")
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(_declared()) if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert _declared() <= set(_lib.exported_symbols()), sorted(_declared() - set(_lib.exported_symbols()))


def test_no_gpu_means_loud_failure():
    """Without a device the product path raises instead of falling back to the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from cabanadem_b200 import api
    with pytest.raises(_lib.DemError):
        api.Context(0)


def test_closing_a_context_closes_its_objects_first():
    """Objects created on a context are closed (newest first) when it closes, and closing one
    afterwards does nothing: no destroy call can reach a freed context."""
    from cabanadem_b200 import api

    class Ctx(api.Context):
        def __init__(self):   # no device needed: a context with a fake handle
            self.h = object()
            self._children = []

    order = []

    class Obj:
        def __init__(self, ctx, name):
            self.ctx, self.name, self.h = ctx, name, True
            ctx.adopt(self)

        def close(self):
            if self.h and self.ctx.alive:
                order.append(self.name)
            self.h = None

    import cabanadem_b200.api as A
    ctx = Ctx()
    a, b = Obj(ctx, "particles"), Obj(ctx, "solver")
    real = A.lib
    A.lib = lambda: type("L", (), {"dem_ctx_destroy": staticmethod(lambda h: None)})()
    try:
        ctx.close()
    finally:
        A.lib = real
    assert order == ["solver", "particles"]
    a.close()
    b.close()
    assert order == ["solver", "particles"] and not ctx.alive
