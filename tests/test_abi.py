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


_STRUCTS = (("ForceParams", "dem_force_params"), ("SolverParams", "dem_solver_params"),
            ("SceneParams", "dem_scene_params"), ("BondParams", "dem_bond_params"), ("RunStats", "dem_run_stats"),
            ("NnRows", "dem_nn_rows"), ("NnMlp", "dem_nn_mlp"), ("SurrogateParams", "dem_surrogate_params"),
            ("RolloutStats", "dem_rollout_stats"))


def test_constants_and_struct_layouts_match_the_header(tmp_path):
    """Every ctypes structure of the binding has the size and field offsets of its C struct in
    include/b200dem.h, and the field, wall-field, precision, status and quirk constants of the
    Python side have the header's values (a C program built from the header prints them)."""
    import re
    import subprocess
    from cabanadem_b200 import scenarios as S
    hdr_path = os.path.join(ROOT, "include", "b200dem.h")
    consts = {"DEM_F_" + k.upper(): v for k, v in _lib.F.items()}
    consts.update({"DEM_W_" + k.upper(): v for k, v in _lib.W.items()})
    consts.update({"DEM_FP64": _lib.DEM_FP64, "DEM_MIXED": _lib.DEM_MIXED, "DEM_REF_COMPAT": S.REF_COMPAT,
                   "DEM_NOALLOC_MAX_PARTICLES": _lib.NOALLOC_MAX_PARTICLES,
                   "DEM_NOALLOC_MAX_NEIGHBORS": _lib.NOALLOC_MAX_NEIGHBORS})
    consts.update({"DEM_" + k: getattr(S, k) for k in dir(S) if re.fullmatch(r"Q\d_[A-Z_]+", k)})
    errs = re.findall(r"#define\s+(DEM_ERR_[A-Z_]+)\s", open(hdr_path).read())
    consts.update({name: code for code, name in _lib.ERR.items()})
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "b200dem.h"', 'int main(void) {']
    for name in sorted(set(consts) | set(errs)):
        lines.append('    printf("C %s %%ld\\n", (long)(%s));' % (name, name))
    for py, c in _STRUCTS:
        lines.append('    printf("S %s %%zu\\n", sizeof(%s));' % (c, c))
        for f, _ in getattr(_lib, py)._fields_:
            lines.append('    printf("O %s.%s %%zu\\n", offsetof(%s, %s));' % (c, f, c, f))
    lines += ['    return 0;', '}']
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I" + os.path.dirname(hdr_path), str(src), "-o", str(tmp_path / "abi")],
                   check=True)
    out = dict(l.split(" ", 1)[1].rsplit(" ", 1) for l in
               subprocess.run([str(tmp_path / "abi")], check=True, capture_output=True, text=True).stdout.splitlines())
    assert set(errs) <= set(_lib.ERR.values()), sorted(set(errs) - set(_lib.ERR.values()))
    for name, v in consts.items():
        assert int(out[name]) == v, name
    for py, c in _STRUCTS:
        cls = getattr(_lib, py)
        assert int(out[c]) == ctypes.sizeof(cls), c
        for f, _ in cls._fields_:
            assert int(out[c + "." + f]) == getattr(cls, f).offset, (c, f)
