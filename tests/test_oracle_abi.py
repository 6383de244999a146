"""The oracle's ctypes wrapper (oracle/oracle.py) against its C header (oracle/dem_oracle.h):
every structure has the size and field offsets of its C struct, and the wrapper's constants
have the header's values (a C program built from the header prints them)."""
import ctypes
import os
import subprocess

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = (("_Particles", "orc_particles"), ("_Walls", "orc_walls"), ("_ForceParams", "orc_force_params"),
           ("_Mesh", "orc_mesh"), ("_Hooks", "orc_hooks"), ("_Bonds", "orc_bonds"),
           ("_BondParams", "orc_bond_params"))
CONSTS = {"ORC_REF_COMPAT": O.REF_COMPAT, "ORC_POW_LIBM": O.POW_LIBM, "ORC_POW_SQRT": O.POW_SQRT,
          "ORC_BOND_REF_COMPAT": O.BOND_REF_COMPAT}


def test_oracle_wrapper_matches_its_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "dem_oracle.h"', 'int main(void) {']
    for name in CONSTS:
        lines.append('    printf("%s %%ld\\n", (long)(%s));' % (name, name))
    for py, c in STRUCTS:
        lines.append('    printf("%s %%zu\\n", sizeof(%s));' % (c, c))
        for f, _ in getattr(O, py)._fields_:
            lines.append('    printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (c, f, c, f))
    lines += ['    return 0;', '}']
    src = tmp_path / "orc.c"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I" + os.path.join(ROOT, "oracle"), str(src), "-o", str(tmp_path / "orc")],
                   check=True)
    out = dict(l.rsplit(" ", 1) for l in
               subprocess.run([str(tmp_path / "orc")], check=True, capture_output=True, text=True).stdout.splitlines())
    for name, v in CONSTS.items():
        assert int(out[name]) == v, name
    for py, c in STRUCTS:
        cls = getattr(O, py)
        assert int(out[c]) == ctypes.sizeof(cls), c
        for f, _ in cls._fields_:
            assert int(out[c + "." + f]) == getattr(cls, f).offset, (c, f)
