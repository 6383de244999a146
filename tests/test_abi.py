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
