"""The C ABI on a machine without a GPU: the library builds and loads,
exports every entry point include/sparc_gpu.h declares, its structs match
the ctypes mirror, and it refuses to run without an sm_100 device."""
import ctypes as C
import os
import re
import subprocess

import pytest

from sparc2_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sparc_gpu.h")
HEADERS = [HEADER, os.path.join(ROOT, "include", "sparc_trol.h")]


@pytest.fixture(scope="module")
def lib():
    from sparc2_b200 import build
    build.build()
    return abi.load()


def declared():
    text = "".join(open(h).read() for h in HEADERS)
    return sorted(set(re.findall(r"\b(sparc_[a-z_0-9]+)\s*\(", text)))


def test_every_declared_entry_point_is_exported(lib):
    names = declared()
    assert len(names) >= 19
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(abi.EXPORTS) == names


def _c_layout(tmp_path):
    fields = {
        "sparc_params": [f for f, _ in abi.SparcParams._fields_],
        "sparc_pulse": [f for f, _ in abi.SparcPulse._fields_],
        "sparc_source": [f for f, _ in abi.SparcSource._fields_],
        "sparc_diag": [f for f, _ in abi.SparcDiag._fields_],
        "sparc_trol": [f for f, _ in abi.SparcTrol._fields_],
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>',
             f'#include "{HEADERS[1]}"', 'int main(void) {']
    for s, fs in fields.items():
        lines.append(f'printf("{s} size %zu\\n", sizeof({s}));')
        for f in fs:
            lines.append(f'printf("{s} {f} %zu\\n", offsetof({s}, {f}));')
    lines += ['return 0;', '}']
    src = tmp_path / "layout.c"
    exe = tmp_path / "layout"
    src.write_text("\n".join(lines))
    subprocess.check_call(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"),
                           "-o", str(exe), str(src)])
    out = subprocess.check_output([str(exe)]).decode().split("\n")
    res = {}
    for line in out:
        if line:
            parts = line.split()
            res[tuple(parts[:-1])] = int(parts[-1])
    return res


def test_struct_layout_matches_header(tmp_path):
    lay = _c_layout(tmp_path)
    for cname, cls in (("sparc_params", abi.SparcParams),
                       ("sparc_pulse", abi.SparcPulse),
                       ("sparc_source", abi.SparcSource),
                       ("sparc_diag", abi.SparcDiag),
                       ("sparc_trol", abi.SparcTrol)):
        assert lay[(cname, "size")] == C.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert lay[(cname, f)] == getattr(cls, f).offset, (cname, f)


def test_create_without_device_fails_loudly(lib):
    from sparc2_b200 import workloads as W
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p, _, _ = W.cfg0(nx=32, ny=32, nz=48, blocks=(2, 2, 2))
    h = C.c_void_p()
    r = lib.sparc_create(C.byref(p), 0, C.byref(h))
    assert r == abi.SPARC_ERR_NODEVICE
    assert lib.sparc_last_error(None)
    from sparc2_b200 import Simulation
    with pytest.raises(abi.SparcError):
        Simulation(p, W.quiet_background(32, 32, 48))


def test_invalid_parameters_are_rejected_before_any_device_call(lib):
    from sparc2_b200 import workloads as W
    p, _, _ = W.cfg0(nx=32, ny=32, nz=48, blocks=(2, 2, 2))
    p.filter_mode_z = 3
    h = C.c_void_p()
    assert lib.sparc_create(C.byref(p), 0, C.byref(h)) == abi.SPARC_ERR_INVALID
    p.filter_mode_z = 1
    p.block_z = 1
    assert lib.sparc_create(C.byref(p), 0, C.byref(h)) == abi.SPARC_ERR_INVALID
    assert b"block" in lib.sparc_last_error(None)
    p.block_z = 2
    p.precision = 7
    assert lib.sparc_create(C.byref(p), 0, C.byref(h)) == abi.SPARC_ERR_INVALID
    assert b"precision" in lib.sparc_last_error(None)
    p.precision = abi.SPARC_FP32
    p.nx = p.ny = 4096
    p.nz = 4096
    assert lib.sparc_create(C.byref(p), 0, C.byref(h)) == abi.SPARC_ERR_INVALID
    assert b"precision form" in lib.sparc_last_error(None)


def test_c_driver_builds_and_reports_the_missing_device(tmp_path):
    """The C caller of the ABI (the driver.f90 loop) compiles against the
    header and the library; without a device it stops at sparc_create with
    its documented exit status 3."""
    import torch
    from sparc2_b200 import workloads as W
    from tests import c_driver, cases
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    exe = c_driver.build(tmp_path)
    p, bg, src = cases.quiet_periodic()
    c_driver.write_inputs(tmp_path, p, bg, src)
    r = c_driver.run(exe, tmp_path, 0, 3)
    assert r.returncode == 3, (r.returncode, r.stderr)
    assert "sparc_create" in r.stderr
    (tmp_path / "params.bin").write_bytes(b"short")
    assert c_driver.run(exe, tmp_path, 0, 3).returncode == 1


@pytest.mark.parametrize("name", ["quiet_periodic", "mhd_hpml", "quiet_random"])
def test_c_driver_reads_every_source_kind(tmp_path, name):
    """The C caller's input files for the pulse, PULSE = 2 and PULSE = 0
    sources read back as written (its --dry-run needs no device)."""
    import numpy as np
    from tests import c_driver, cases
    exe = c_driver.build(tmp_path)
    p, bg, src = cases.CASES[name]()
    c_driver.write_inputs(tmp_path, p, bg, src)
    r = c_driver.run(exe, tmp_path, 0, 1, "--dry-run")
    assert r.returncode == 0, r.stderr
    words = r.stdout.replace(",", "").replace("(", "").replace(")", "").split()
    assert words[:2] == ["inputs", "ok:"]
    assert int(words[words.index("source") + 1]) == src.kind
    npl = int(words[words.index("pulses") + 1])
    nser = int(words[words.index("series") + 1])
    if src.kind == abi.SPARC_SRC_PSR:
        assert npl == len(src._keep) == src.npulses
    elif src.kind == abi.SPARC_SRC_RANDOM:
        assert nser == src.nseries
        assert float(words[words.index("sum") + 1]) == pytest.approx(float(np.sum(src._keep)),
                                                                    rel=1e-12, abs=1e-9)
    if src.kind == abi.SPARC_SRC_RANDOM:
        (tmp_path / "series.bin").write_bytes(b"\0" * 16)
        assert c_driver.run(exe, tmp_path, 0, 1, "--dry-run").returncode == 1


@pytest.mark.parametrize("name", ["quiet_periodic", "mhd_hpml"])
def test_c_driver_reads_a_trol_file(tmp_path, name):
    """The C caller started from a .trol control file: the grid, physics,
    source kind and the run's iteration range (init .. maxtime) come from
    the file (its --dry-run needs no device)."""
    from tests import c_driver, cases
    exe = c_driver.build(tmp_path)
    p, bg, src = cases.CASES[name]()
    c_driver.write_inputs(tmp_path, p, bg, src)
    (tmp_path / "params.bin").write_bytes(b"not read with --trol")
    (tmp_path / "run.trol").write_text(c_driver.trol_text(p, src, solartime_h=0.01))
    r = c_driver.run(exe, tmp_path, "-", "-", "--dry-run", "--trol", str(tmp_path / "run.trol"))
    assert r.returncode == 0, r.stderr
    words = r.stdout.replace(",", "").replace("(", "").replace(")", "").split()
    assert words[2:5] == [str(p.nx), "x", str(p.ny)] and words[6] == str(p.nz)
    assert int(words[words.index("magnetic") + 1]) == p.magnetic
    assert int(words[words.index("source") + 1]) == src.kind
    maxtime = 2 * (int(36.0 / p.timestep) // 2)
    assert words[-1] == f"0..{maxtime}"
