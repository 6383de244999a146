"""The C++ interface (include/CabanaDEM_B200.hpp) and the example drivers on it.

On the CPU every driver builds against the header and library, the snapshot reader parses
the drivers' output format, and the header's XDMF writer round-trips through the reader.  On the GPU each driver runs with the reference's command
line and input file; every snapshot it writes (particles_<k>.csv after each step divisible by
output_frequency) is compared bit for bit with the oracle stepped the same way, and the
observables the reference's automate.py reads from those files are checked: restitution
out = in for example 03 (automate.py:315), the rebound spin peak for example 04 (:447), the
contact slots of tst_03 (:531)."""
import json
import math
import os
import subprocess

import numpy as np
import pytest

from cabanadem_b200 import snapshots

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXDIR = os.path.join(ROOT, "examples")
EXE = os.path.join(EXDIR, "01_two_sphere_head_on")
DRIVERS = ("01_two_sphere_head_on", "01ElasticNormalImpactOfTwoIdenticalParticles",
           "02ElasticNormalImpactOfParticleWall", "03NormalParticleWallDifferentCOR",
           "04ObliqueParticleWallDifferentAngles", "Tst01ParticleInsertion", "Tst03MultipleParticlesContacts",
           "Tst04GranularDamBreak2d", "Tst01BDEMTwoParticlesTensile3D")
K01 = "01_elastic_normal_impact_of_two_identical_particles"
K02 = "02_elastic_normal_impact_of_particle_wall"
K03 = "03_normal_particle_wall_different_cor"
K04 = "04_oblique_particle_wall_different_angles"
KT3 = "tst_03_multiple_particles_contacts"
KT4 = "tst_04_granular_dam_break_2d"


def _build():
    if not os.path.exists(os.path.join(ROOT, "cabanadem_b200", "libb200dem.so")):
        pytest.skip("library not built")
    subprocess.run(["make", "-s", "-C", EXDIR], check=True)


def _raw_inputs():
    with open(os.path.join(ROOT, "tests", "golden", "example_inputs.json")) as f:
        return json.load(f)


def _run(tmp_path, exe, key, extra=()):
    tmp_path.mkdir(parents=True, exist_ok=True)
    inp = tmp_path / "in.json"
    inp.write_text(json.dumps(_raw_inputs()[key]))
    out = tmp_path / "out"
    subprocess.run([os.path.join(EXDIR, exe), str(inp), str(out), *extra], check=True, capture_output=True)
    return [snapshots.read(f) for f in snapshots.files(str(out))]


def test_example_drivers_build():
    _build()
    for d in DRIVERS:
        assert os.access(os.path.join(EXDIR, d), os.X_OK), d


def test_snapshot_reader(tmp_path):
    (tmp_path / "particles_12.csv").write_text(
        "# time 0.25\n"
        "id,positions_0,positions_1,positions_2,velocities_0,velocities_1,velocities_2,omega_0,omega_1,omega_2,"
        "forces_0,forces_1,forces_2,mass,density,radius,total_no_tangential_contacts\n"
        "0,1,2,3,4,5,6,7,8,9,10,11,12,13,14,15,2\n"
        "1,0.1,0.2,0.30000000000000004,0,0,0,0,0,0,0,0,0,1,1,1,0\n")
    (tmp_path / "particles_3.csv").write_text((tmp_path / "particles_12.csv").read_text())
    (tmp_path / "other.csv").write_text("x")
    fs = snapshots.files(str(tmp_path))
    assert [os.path.basename(f) for f in fs] == ["particles_3.csv", "particles_12.csv"]
    s = snapshots.read(fs[1])
    assert s["time"] == 0.25
    assert s["positions"].shape == (2, 3) and s["positions"][1, 2] == 0.30000000000000004
    assert s["forces"][0].tolist() == [10., 11., 12.]
    assert s["total_no_tangential_contacts"].tolist() == [2, 0]
    assert s["radius"].tolist() == [15., 1.]


_XDMF_PROG = r"""
#include "CabanaDEM_B200.hpp"
#include <cstdlib>
int main(int argc, char **argv) {
    const int n = 5;
    std::vector<double> x(3 * n), u(3 * n), w(3 * n), f(3 * n), m(n), rho(n), r(n);
    std::vector<int> tc(n);
    for (int i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d) {
            x[3 * i + d] = 0.1 * i + d + 1.0 / 3.0;
            u[3 * i + d] = -2.5 * i + d;
            w[3 * i + d] = 1e-300 * (i + 1) * (d + 1);
            f[3 * i + d] = 1e9 / (i + d + 1);
        }
        m[i] = 0.5 + i; rho[i] = 2500.0; r[i] = 1e-3 * (i + 1); tc[i] = i % 3;
    }
    CabanaDEM::writeXdmfSnapshot(argv[1], std::atoi(argv[2]), 0.1 + 0.2, n,
        {{"positions", x.data(), 3, false}, {"velocities", u.data(), 3, false}, {"omega", w.data(), 3, false},
         {"forces", f.data(), 3, false}, {"mass", m.data(), 1, false}, {"density", rho.data(), 1, false},
         {"radius", r.data(), 1, false}, {"total_no_tangential_contacts", tc.data(), 1, true}});
    CabanaDEM::writeCsvSnapshot(argv[1], std::atoi(argv[2]), 0.1 + 0.2, n, x.data(), u.data(), w.data(), f.data(),
                                m.data(), rho.data(), r.data(), tc.data());
    return 0;
}
"""


def test_xdmf_snapshot_round_trip(tmp_path):
    """writeXdmfSnapshot (the C++ interface's XDMF output) read back by snapshots.read_xdmf:
    every dataset bit for bit, the time, the Polyvertex topology and the grid's layout."""
    import xml.etree.ElementTree as ET
    src = tmp_path / "xdmf.cpp"
    src.write_text(_XDMF_PROG)
    exe = tmp_path / "xdmf"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    for step in (7, 12):
        subprocess.run([str(exe), str(tmp_path), str(step)], check=True)
    fs = snapshots.files(str(tmp_path), ".xmf")
    assert [os.path.basename(f) for f in fs] == ["particles_7.xmf", "particles_12.xmf"]
    s = snapshots.read_xdmf(fs[1])
    n, i = 5, np.arange(5)[:, None]
    d = np.arange(3)[None, :]
    assert s["time"] == 0.1 + 0.2
    assert np.array_equal(s["positions"], 0.1 * i + d + 1.0 / 3.0)
    assert np.array_equal(s["velocities"], -2.5 * i + d)
    assert np.array_equal(s["omega"], 1e-300 * (i + 1) * (d + 1))
    assert np.array_equal(s["forces"], 1e9 / (i + d + 1))
    assert np.array_equal(s["mass"], 0.5 + np.arange(n)) and np.array_equal(s["density"], np.full(n, 2500.0))
    assert np.array_equal(s["radius"], 1e-3 * (np.arange(n) + 1))
    assert s["total_no_tangential_contacts"].dtype == np.int32
    assert s["total_no_tangential_contacts"].tolist() == [0, 1, 2, 0, 1]
    grid = ET.parse(fs[1]).getroot().find("Domain/Grid")
    topo = grid.find("Topology")
    assert topo.get("TopologyType") == "Polyvertex" and topo.get("NumberOfElements") == "5"
    assert grid.find("Geometry").get("GeometryType") == "XYZ"
    kinds = {a.get("Name"): a.get("AttributeType") for a in grid.findall("Attribute")}
    assert kinds["velocities"] == "Vector" and kinds["mass"] == "Scalar"
    assert os.path.getsize(tmp_path / "particles_12.bin") == n * (4 * 3 * 8 + 3 * 8 + 4)


def test_python_writers_match_the_cpp_interface(tmp_path):
    """snapshots.write_xdmf and write_csv write the same bytes as the C++ interface's
    writeXdmfSnapshot and writeCsvSnapshot (what Particles::output calls) for the same data, and
    the CSV reads back bit for bit."""
    from cabanadem_b200.state import ParticleState
    src = tmp_path / "xdmf.cpp"
    src.write_text(_XDMF_PROG)
    exe = tmp_path / "xdmf"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    (tmp_path / "cpp").mkdir()
    (tmp_path / "py").mkdir()
    subprocess.run([str(exe), str(tmp_path / "cpp"), "5"], check=True)
    n = 5
    st = ParticleState.create(n, max_cnts=1, max_walls=1)
    for i in range(n):
        for d in range(3):
            st.x[i, d] = 0.1 * i + d + 1.0 / 3.0
            st.u[i, d] = -2.5 * i + d
            st.omega[i, d] = 1e-300 * (i + 1) * (d + 1)
            st.force[i, d] = 1e9 / (i + d + 1)
        st.m[i], st.rho[i], st.rad[i], st.tng_count[i] = 0.5 + i, 2500.0, 1e-3 * (i + 1), i % 3
    snapshots.write_xdmf(str(tmp_path / "py"), 5, 0.1 + 0.2, st)
    for ext in (".xmf", ".bin"):
        assert (tmp_path / "py" / ("particles_5" + ext)).read_bytes() == \
            (tmp_path / "cpp" / ("particles_5" + ext)).read_bytes(), ext
    csv = snapshots.write_csv(str(tmp_path / "py"), 5, 0.1 + 0.2, st)
    assert open(csv, "rb").read() == (tmp_path / "cpp" / "particles_5.csv").read_bytes()
    got = snapshots.read(csv)
    assert got["time"] == 0.1 + 0.2
    for name, f in (("positions", "x"), ("velocities", "u"), ("omega", "omega"), ("forces", "force"),
                    ("mass", "m"), ("density", "rho"), ("radius", "rad"), ("total_no_tangential_contacts", "tng_count")):
        assert np.array_equal(got[name], getattr(st, f)), name


_JSON_PROG = r"""
#include "CabanaDEM_B200.hpp"
#include <cstdio>
static void dump(const CabanaDEM::JsonValue &v, const std::string &path) {
    using K = CabanaDEM::JsonValue;
    switch (v.kind) {
        case K::Object: for (const auto &kv : v.obj) dump(kv.second, path + "/" + kv.first); break;
        case K::Array: for (size_t k = 0; k < v.arr.size(); ++k) dump(v.arr[k], path + "/" + std::to_string(k)); break;
        case K::Number: std::printf("%s N %.17g\n", path.c_str(), v.num); break;
        case K::String: std::printf("%s S ", path.c_str()); for (unsigned char c : v.str) std::printf("%02x", c);
                        std::printf("\n"); break;
        case K::Bool: std::printf("%s B %d\n", path.c_str(), int(v.num)); break;
        case K::Null: std::printf("%s Z\n", path.c_str()); break;
    }
}
int main(int argc, char **argv) {
    std::ifstream f(argv[1]);
    std::stringstream ss;
    ss << f.rdbuf();
    dump(CabanaDEM::JsonValue::parse(ss.str()), "");
    CabanaDEM::Inputs in(argv[1]);
    std::printf("num_steps %d\n", int(in["num_steps"]));
    return 0;
}
"""


def _flatten(v, path=""):
    if isinstance(v, dict):
        return [x for k in sorted(v) for x in _flatten(v[k], path + "/" + k)]
    if isinstance(v, list):
        return [x for k, e in enumerate(v) for x in _flatten(e, path + "/" + str(k))]
    if isinstance(v, bool):
        return ["%s B %d" % (path, v)]
    if v is None:
        return ["%s Z" % path]
    if isinstance(v, str):
        return ["%s S %s" % (path, v.encode("utf-8").hex())]
    return ["%s N %s" % (path, "%.17g" % float(v))]


def test_json_reader_matches_python(tmp_path):
    """The C++ interface's JSON reader (Inputs; the reference uses nlohmann::json,
    Input.hpp:58-62) gives every value of the seven example inputs and of a file with escapes,
    exponents, nesting and literals as Python's json does; num_steps = int(final_time /
    timestep) truncates as Input.hpp:50-54 (0.3 / 0.1 -> 2)."""
    src = tmp_path / "json.cpp"
    src.write_text(_JSON_PROG)
    exe = tmp_path / "json"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    tricky = ('{ "final_time": {"value": 0.3}, "timestep" :{"value":1e-1},\n'
              ' "a": {"value": -1.5E-3, "units": "m\\/s\\u00b2 \\"x\\" \\ud83d\\ude00\\n\\t\\\\"},\n'
              ' "arr": [1, 2.5, [true, false, null], {}, "\\u0041"], "big": 12345678901234567890}')
    cases = dict(_raw_inputs())
    cases["tricky"] = None
    for name, raw in cases.items():
        f = tmp_path / ("%s.json" % name)
        f.write_text(tricky if raw is None else json.dumps(raw, indent=2))
        data = json.loads(f.read_text())
        out = subprocess.run([str(exe), str(f)], check=True, capture_output=True, text=True).stdout.splitlines()
        assert out[:-1] == _flatten(data), name
        assert out[-1] == "num_steps %d" % int(float(data["final_time"]["value"]) / float(data["timestep"]["value"]))
    assert out[-1] == "num_steps 2"


_PHASE_PROG = r"""
#include "CabanaDEM_B200.hpp"
struct mem {};
struct exe {};
// the reference loop (Solver.hpp:81-94) written with the phase-level calls
template <class S, class P>
void loop(std::shared_ptr<S> solver, P &particles, int nsteps) {
    CabanaDEM::Integrator<S> integrator(solver);
    for (int step = 0; step < nsteps; ++step) {
        integrator.stage1(particles);
        integrator.stage2(particles);
        solver->buildNeighbors();
        CabanaDEM::computeForceParticleParticleInfiniteWall(*solver);
        integrator.stage3(particles);
    }
}
int main(int argc, char **argv) {
    CabanaDEM::Inputs inputs(argv[1]);
    auto force = std::make_shared<CabanaDEM::Force<exe>>(0.8, 0.8, 0.3, 0.3);
    auto particles = std::make_shared<CabanaDEM::Particles<mem, 3, 6, 1>>(exe(), 2, argv[2]);
    particles->setOutputFormat("both");
    std::shared_ptr<CabanaDEM::Wall<mem, 3>> wall;
    auto solver = CabanaDEM::createSolverDEM<mem>(inputs, particles, wall, force, 3e-3);
    loop(solver, *particles, 3);
    particles->output(0, 0.0);
    return 0;
}
"""


def test_phase_level_interface_builds(tmp_path):
    """The reference loop written with Integrator<Solver>, buildNeighbors and
    computeForceParticleParticleInfiniteWall builds and links against the library (it runs
    only with a GPU)."""
    _build()
    src = tmp_path / "phases.cpp"
    src.write_text(_PHASE_PROG)
    lib = os.path.join(ROOT, "cabanadem_b200")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I" + os.path.join(ROOT, "include"), str(src), "-o",
                    str(tmp_path / "phases"), "-L" + lib, "-lb200dem", "-Wl,-rpath," + lib], check=True)
    assert os.access(tmp_path / "phases", os.X_OK)


def _oracle_snapshots(sc):
    """The oracle stepped as SolverDEM::run: steps 0..num_steps, a snapshot after every step
    divisible by output_frequency (Solver.hpp:79-108)."""
    from oracle import oracle as O
    st, freq = sc.state.copy(), sc.output_frequency
    last = sc.nsteps - 1
    out, step = [], 0
    while step <= last:
        stop = min(last, -(-step // freq) * freq)
        O.run(st, sc.walls, sc.params, sc.dt, stop - step + 1, delta=sc.delta, pow_mode=O.POW_SQRT)
        if stop % freq == 0:
            out.append((stop * sc.dt, st.copy()))
        step = stop + 1
    return out


def _assert_snapshots(got, ref):
    assert len(got) == len(ref)
    for k, (g, (t, r)) in enumerate(zip(got, ref)):
        assert g["time"] == t, k
        for name, f in (("positions", "x"), ("velocities", "u"), ("omega", "omega"), ("forces", "force")):
            assert np.array_equal(g[name], getattr(r, f)), (k, name, np.abs(g[name] - getattr(r, f)).max())
        assert np.array_equal(g["total_no_tangential_contacts"], r.tng_count), k
        assert np.array_equal(g["mass"], r.m) and np.array_equal(g["radius"], r.rad)


def _cases():
    from cabanadem_b200 import scenarios as S
    return [
        ("01", "01ElasticNormalImpactOfTwoIdenticalParticles", K01, (), lambda I: S.example01(I[K01])),
        ("02", "02ElasticNormalImpactOfParticleWall", K02, (), lambda I: S.example02(I[K02])),
        ("03_cor0.4", "03NormalParticleWallDifferentCOR", K03, ("--cor_pw=0.4",), lambda I: S.example03(I[K03], 0.4)),
        ("04_30deg", "04ObliqueParticleWallDifferentAngles", K04, ("--angle=30",),
         lambda I: S.example04(I[K04], 30.0)),
        ("tst03", "Tst03MultipleParticlesContacts", KT3, (), lambda I: S.tst03(I[KT3])),
        ("tst04", "Tst04GranularDamBreak2d", KT4, (), lambda I: S.tst04(I[KT4])),
        ("tst04_box", "Tst04GranularDamBreak2d", KT4, ("--walls=box",), lambda I: S.tst04(I[KT4], box_walls=True)),
    ]


CASE_IDS = ["01", "02", "03_cor0.4", "04_30deg", "tst03", "tst04", "tst04_box"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASE_IDS)
def test_driver_snapshots_match_oracle(tmp_path, example_inputs, case):
    _build()
    _, exe, key, extra, make = next(c for c in _cases() if c[0] == case)
    got = _run(tmp_path, exe, key, extra)
    sc = make(example_inputs)
    _assert_snapshots(got, _oracle_snapshots(sc))
    if case == "tst03":
        counts = np.array([g["total_no_tangential_contacts"] for g in got])
        assert counts[:, 0].max() == 2 and counts[-1].sum() == 0


@pytest.mark.gpu
def test_driver_03_restitution_out_equals_in(tmp_path, example_inputs):
    """automate.py:303-343: the last snapshot's velocities[0][1] / velocity_p against cor_pw."""
    _build()
    v = float(example_inputs[K03]["velocity_p"])
    for cor in (0.01, 0.2, 0.4, 0.6, 0.8, 1.0):
        got = _run(tmp_path / ("c%g" % cor), "03NormalParticleWallDifferentCOR", K03, ("--cor_pw=%g" % cor,))
        assert abs(got[-1]["velocities"][0, 1] / v - cor) < 0.02, cor


@pytest.mark.gpu
def test_driver_04_rebound_spin_peaks_near_30_degrees(tmp_path, example_inputs):
    """automate.py:427-478 plots omega[0][2] of the last snapshot against the incident angle;
    the oracle run of the same cases is pinned to the Lethe and experimental curves on the CPU."""
    _build()
    angles = [10., 20., 25., 30., 35., 40., 50.]
    om = []
    for a in angles:
        got = _run(tmp_path / ("a%g" % a), "04ObliqueParticleWallDifferentAngles", K04, ("--angle=%g" % a,))
        om.append(got[-1]["omega"][0, 2])
    assert 25.0 <= angles[int(np.argmax(om))] <= 35.0


@pytest.mark.gpu
def test_particle_insertion_driver(tmp_path):
    """tst_01_particle_insertion: snapshots of 1, 20, 20 (moved by 2 u) and 15 particles."""
    _build()
    raw = _raw_inputs()[K04]
    got = _run(tmp_path, "Tst01ParticleInsertion", K04, ("--angle=30",))
    r = raw["particle_radius"]["value"]
    assert [g["positions"].shape[0] for g in got] == [1, 20, 20, 15]
    assert [g["time"] for g in got] == [0.0, 0.1, 0.2, 0.3]
    assert got[0]["positions"][0, 1] == r + r / 1000000.
    a = 30. / 180. * math.pi
    assert got[0]["velocities"][0, :2].tolist() == [3.9 * math.sin(a), -3.9 * math.cos(a)]
    i = np.arange(20)
    assert np.array_equal(got[1]["positions"][:, 1], 3 * i * r + r / 1000000.)
    assert np.array_equal(got[2]["positions"][:, 1], 3 * i * r + r / 1000000. + 2.)
    assert np.array_equal(got[3]["positions"][:, 1], 5 * np.arange(15) * r + r / 1000000.)
    assert got[1]["mass"][0] > 0 and got[1]["mass"][1] == 0.0     # added particles start zeroed


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [[], ["--hooks=device"], ["--fused"]], ids=["reference_loop", "device_hooks", "fused"])
def test_bdem_driver_matches_oracle(tmp_path, mode):
    """tst_01_BDEM written as the reference's loop (BondedDEMIntegrator stages,
    resetForcesAndTorques, the example's hooks through the force slice, computeBondedForce):
    the driver's snapshots every 100 steps against the bonded oracle, bit for bit; the same
    with the hooks on the device, and with the loop fused."""
    _build()
    from cabanadem_b200 import scenarios as S
    from oracle import oracle as O
    out = tmp_path / "bdem"
    subprocess.run([os.path.join(EXDIR, "Tst01BDEMTwoParticlesTensile3D"), str(out)] + mode, check=True,
                   capture_output=True)
    got = [snapshots.read(f) for f in snapshots.files(str(out))]
    case = S.bdem_two_particles()
    st, b = case["state"].copy(), case["bonds"].copy()
    O.setup_bonds(b, st, case["bond_factor"], case["search_cutoff"])
    last = case["nsteps"] - 1
    assert len(got) == last // 100 + 1
    done = 0
    for k, g in enumerate(got):
        O.bonded_run(st, b, case["bparams"], case["dt"], k * 100 + 1 - done, ext_force=case["ext_force"],
                     fix_flags=case["fix_flags"], pow_mode=O.POW_SQRT)
        done = k * 100 + 1
        for name, f in (("positions", "x"), ("velocities", "u"), ("omega", "omega"), ("forces", "force")):
            assert np.array_equal(g[name], getattr(st, f)), (k, name)


@pytest.mark.gpu
def test_example_driver_matches_oracle(tmp_path, example_inputs):
    """01_two_sphere_head_on records sphere 1's force at every step."""
    _build()
    from cabanadem_b200 import scenarios as S
    from oracle import oracle as O
    inp = tmp_path / "in.json"
    inp.write_text(json.dumps(_raw_inputs()[K01]))
    out = tmp_path / "out.csv"
    subprocess.run([EXE, str(inp), str(out)], check=True, capture_output=True)
    got = np.loadtxt(out, delimiter=",", skiprows=1)
    sc = S.example01(example_inputs[K01])
    st = sc.state
    ref = []
    for _ in range(sc.nsteps):
        O.run(st, sc.walls, sc.params, sc.dt, 1, delta=sc.delta, pow_mode=O.POW_SQRT)
        ref.append(st.force[1, 0])
    assert got.shape[0] == sc.nsteps
    assert np.array_equal(got[:, 2], np.array(ref))
    assert got[:, 2].max() > 1e4
