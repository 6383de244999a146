"""The C++ interface (include/CabanaDEM_B200.hpp): the example driver builds against the
header and library on the CPU; on the GPU it reproduces the head-on impact of the reference's
first validation case bit for bit against the oracle."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "examples", "01_two_sphere_head_on")


def _build():
    if not os.path.exists(os.path.join(ROOT, "cabanadem_b200", "libb200dem.so")):
        pytest.skip("library not built")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "examples")], check=True)


def test_example_driver_builds():
    _build()
    assert os.access(EXE, os.X_OK)


@pytest.mark.gpu
def test_example_driver_matches_oracle(tmp_path, example_inputs):
    _build()
    from cabanadem_b200 import scenarios as S
    from oracle import oracle as O
    raw = json.load(open(os.path.join(ROOT, "tests", "golden", "example_inputs.json")))
    key = "01_elastic_normal_impact_of_two_identical_particles"
    inp = tmp_path / "in.json"
    inp.write_text(json.dumps(raw[key]))
    out = tmp_path / "out.csv"
    subprocess.run([EXE, str(inp), str(out)], check=True, capture_output=True)
    got = np.loadtxt(out, delimiter=",", skiprows=1)
    sc = S.example01(example_inputs[key])
    st = sc.state
    ref = []
    for _ in range(sc.nsteps):
        O.run(st, sc.walls, sc.params, sc.dt, 1, delta=sc.delta, pow_mode=O.POW_SQRT)
        ref.append(st.force[1, 0])
    assert got.shape[0] == sc.nsteps
    assert np.array_equal(got[:, 2], np.array(ref))
    assert got[:, 2].max() > 1e4
