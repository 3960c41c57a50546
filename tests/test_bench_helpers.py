"""Host-side pieces of bench.py: the bounded CPU sample and the reference arm's
isolation from this package's native library."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_cpu_sample_is_the_whole_device_when_a_sweep_is_short():
    # N = 221, N_z = 800: one oracle sweep ~7 s, sampled whole
    assert bench.cpu_sample_nz(221, 800) == 800
    assert bench.sweep_scale(800, 800) == 1.0


def test_cpu_sample_cuts_long_sweeps_to_fewer_slices():
    # N = 797, N_z = 400: ~160 s per sweep on one core, cut to about CPU_SAMPLE_S
    nz = bench.cpu_sample_nz(797, 400)
    assert 8 <= nz < 400
    est = 16.0 * 797 ** 3 * nz / 20e9
    assert est <= 1.5 * bench.CPU_SAMPLE_S
    # nz inverses and nz - 1 block products against 400 and 399
    assert bench.sweep_scale(nz, 400) == pytest.approx((2 * nz - 1) / 799.0)


def test_reference_arm_loads_no_library_of_this_package():
    """--impl reference times the oracle on inputs built by the oracle's own
    set-up: no libnegfgpu.so is mapped into its process."""
    code = (
        "import runpy, sys\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0',\n"
        "            '--workload', 'small:1.2:16', '--cpu-threads', '2']\n"
        f"runpy.run_path({os.path.join(ROOT, 'bench.py')!r}, run_name='__main__')\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('NATIVE', 'libnegfgpu' in maps, 'liboracle' in maps)\n"
    )
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, env=env,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = [l for l in out.stdout.splitlines() if l.startswith("NATIVE")][-1]
    assert line == "NATIVE False True", line
    assert '"impl": "reference"' in out.stdout
