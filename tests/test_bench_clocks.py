"""bench.py's clock sampler on CPU, with a stand-in for nvidia-smi that prints one sample line
and keeps running: samples taken before the timed region are skipped, stop() ends the sampler
and removes its file, and a timed region that raises still ends the sampler at exit."""
import os
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LINE = "0, 1965, 1965, 512.3, 0x0, Not Active, Not Active, Not Active, Active"
FAKE = ["sh", "-c", "echo '%s'; sleep 2; echo '%s'; exec sleep 60" % (LINE, LINE.replace("1965, 1965", "1800, 1965"))]


def test_sampler_skips_early_samples_and_cleans_up():
    sys.path.insert(0, ROOT)
    import bench
    c = bench.ClockSampler(0, cmd=FAKE)
    c.start()
    pid, path = c.proc.pid, c.path
    import time
    time.sleep(3)
    ck = c.stop()
    assert ck["samples"] == 1 and ck["sm_mhz"] == 1800.0 and ck["sm_max_mhz"] == 1965.0
    assert ck["reasons"] == ["sw_power_cap"]
    assert not os.path.exists(path) and c.proc.poll() is not None
    c._end()                                   # the exit hook after a normal stop does nothing
    assert pid > 0


def test_sampler_ends_when_the_timed_region_raises(tmp_path):
    prog = tmp_path / "raise.py"
    prog.write_text(textwrap.dedent("""
        import sys
        sys.path.insert(0, %r)
        import bench
        c = bench.ClockSampler(0, cmd=%r)
        c.start()
        print(c.proc.pid, c.path, flush=True)
        raise RuntimeError("timed region failed")
    """ % (ROOT, FAKE)))
    r = subprocess.run([sys.executable, str(prog)], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "timed region failed" in r.stderr
    pid, path = r.stdout.split()
    assert not os.path.exists(path)
    assert not os.path.exists("/proc/%s" % pid) or open("/proc/%s/stat" % pid).read().split()[2] == "Z"
