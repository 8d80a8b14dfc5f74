"""The .trol reader (sparc_read_trol / sparc_parse_trol, include/sparc_trol.h)
against hand-checked values: READ_SPARC_PARAMETERS (initialize.f90:1385-1924)
and the run quantities of driver.f90:38-39, 64-69.  CPU only (the reader
touches no device)."""
import ctypes as C
import os

import pytest

from sparc2_b200 import abi

SAMPLE = "/root/reference/sparc_parameters"


@pytest.fixture(scope="module")
def lib():
    from sparc2_b200 import build
    build.build()
    return abi.load()


def parse(lib, text):
    t = abi.SparcTrol()
    err = C.create_string_buffer(256)
    r = lib.sparc_parse_trol(text.encode(), C.byref(t), err, 256)
    return r, t, err.value.decode()


BASE = """nx = 64
ny = 48
nz = 100
timestep = 0.5
"""


@pytest.mark.skipif(not os.path.exists(SAMPLE), reason="reference sample not present")
def test_reference_sample_file(lib):
    t = abi.SparcTrol()
    err = C.create_string_buffer(256)
    assert lib.sparc_read_trol(SAMPLE.encode(), C.byref(t), err, 256) == abi.SPARC_OK, err.value
    p, s = t.params, t.source
    assert (p.nx, p.ny, p.nz) == (128, 128, 220)
    assert p.xlength == 200.0e8 and p.ylength == 200.0e8
    assert p.timestep == 0.75
    assert t.restart == 0 and t.time0 == 0 and t.init == 0
    assert t.wall_time == 1.0e8 * 3600 and t.solartime == 4.0
    assert p.stabilise == 1 and t.damping == 0 and p.magnetic == 2
    assert p.maxva == 5000.0e5
    assert t.twod == 0 and t.twop5d == 0 and t.displ == 0 and t.flows == 0
    assert (p.block_x, p.block_y, p.block_z) == (2, 2, 4)
    # USE_HPML = 0 keeps USE_PML on; PERIODIC = 1 stands without HPMLs;
    # the x/y PML widths are zeroed without HPMLs, the z ones kept
    assert p.use_pml == 1 and p.use_hpml == 0 and p.periodic == 1
    assert (p.npml_xb, p.npml_xt, p.npml_yb, p.npml_yt) == (0, 0, 0, 0)
    assert (p.npml_zb, p.npml_zt) == (10, 10)
    assert list(p.pml_xb) == [15.0, 3.0, 8.0, 0.1]
    assert list(p.pml_zt) == [5.0, 2.0, 8.0, 0.1]
    assert s.kind == abi.SPARC_SRC_PULSE and t.pulse == 1 and s.dir == 3
    assert (s.t0, s.t1, s.st) == (600.0, 300.0, 75.0)
    assert (s.px, s.py, s.pz) == (35.0e8, 35.0e8, -0.4e8)
    assert (s.sr, s.sz, s.amp) == (2.0e8, 0.15e8, 1.0e4)
    assert (p.sp_str, p.sp_length, p.sp_decay) == (0.0, 10.0e8, 0.008)
    assert (p.filter_mode_xy, p.filter_mode_z) == (1, 1)
    assert (p.s_xy, p.s_z, p.t_xy, p.t_z) == (1.0, 1.0, 15.0, 7.5)
    assert t.dir_bkg == b"./TEST_CASE/test_for_matthias_30_Bmod_10.h5"
    assert t.dir_out == b"./TEST_CASE/"
    assert t.simname == b"pml_test_N10_RC5_kappa8_3D_vm_"
    assert t.forcingfunc == b"/short/y94/dfp565/forcing256_200_18hrs.fits"
    assert t.fulloutputcad == 600.0 and t.chunkoutputcad == 30.0
    assert t.minsavtime == 0.0 and t.timestamp_size == 4
    assert (t.xcb, t.xct, t.ycb, t.yct, t.zcb, t.zct) == (1, 256, 1, 256, 269, 269)
    # derived: 4 h / 0.75 s = 19200 iterations; cadences floor(t/dt + 1e-5)
    assert t.maxtime == 19200
    assert (t.xyfreq, t.zfreq) == (20, 10)
    assert (t.fulloutputsteps, t.chunkoutputsteps) == (800, 40)
    assert t.fullout == 1 and t.chunkout == 1
    # driver.f90:38-39: floor(19200*0.75/60) + 2 = 242 -> 2*121 + 2
    assert t.num_steps == 244
    assert t.stopped_line == 0 and t.psr_npulses == 500


def test_missing_grid_is_an_error(lib):
    r, _, err = parse(lib, "timestep = 1.0\nnx = 8\n")
    assert r == abi.SPARC_ERR_INVALID and "nx, ny, nz" in err


def test_key_matching_rules(lib):
    text = BASE + "\n".join([
        "  nz = 7",                       # indented: the name keeps its blanks
        "NX = 9",                         # case-sensitive
        "unknown_key = 5",
        "!! a comment = with an equals sign",
        "xlength   =   2.5d9  trailing words",
        "ylength=1.5D+09",
        "simname = \"my run\"",
        "dir_out = ./out/  ignored",      # undelimited: a '/' ends the item
        "block_x = 3",
        "a_very_long_name_that_is_cut_at_thirty_chars = 1",
    ]) + "\n"
    r, t, _ = parse(lib, text)
    assert r == abi.SPARC_OK
    p = t.params
    assert (p.nx, p.ny, p.nz) == (64, 48, 100)
    assert p.xlength == 2.5e9 and p.ylength == 1.5e9
    assert t.simname == b"my run_3D_vt_"       # MAGNETIC unset: thermal
    assert t.dir_out == b"."
    assert p.block_x == 3


def test_failed_value_ends_the_file(lib):
    text = BASE + "block_y = 2\nblock_x = two\nblock_z = 5\n"
    r, t, _ = parse(lib, text)
    assert r == abi.SPARC_OK
    assert t.stopped_line == 6
    assert t.params.block_y == 2 and t.params.block_x == 0 and t.params.block_z == 0
    # an integer key given a real fails too, as a list-directed integer read
    r, t, _ = parse(lib, BASE + "time0 = 1.5\nblock_z = 5\n")
    assert t.stopped_line == 5 and t.params.block_z == 0
    # an empty value is an end of record: the read fails
    r, t, _ = parse(lib, BASE + "maxva =\nblock_z = 5\n")
    assert t.stopped_line == 5 and t.params.block_z == 0


def test_order_sensitive_keys(lib):
    # HPML on before PERIODIC: periodic is dropped; x/y PMLs read after it
    r, t, _ = parse(lib, BASE + "USE_HPML = 1\nPERIODIC = 1\nxpmlb = 8, 15.0, 3.0, 8.0, 0.1\n")
    assert t.params.use_hpml == 1 and t.params.periodic == 0 and t.params.npml_xb == 8
    # PERIODIC before HPML stands; a PML line before USE_HPML is zeroed
    r, t, _ = parse(lib, BASE + "PERIODIC = 1\nypmlt = 8,15.0,3.0,8.0,0.1\nUSE_HPML = 1\n")
    assert t.params.periodic == 1 and t.params.npml_yt == 0 and t.params.use_hpml == 1
    # USE_HPML = 0 turns USE_PML on; z PML widths need USE_PML first
    r, t, _ = parse(lib, BASE + "zpmlb = 10,5.0,2.0,8.0,0.1\nUSE_HPML = 0\nzpmlt = 12,5.0,2.0,8.0,0.1\n")
    assert t.params.use_pml == 1 and t.params.npml_zb == 0 and t.params.npml_zt == 12
    # pulse_* are read only once PULSE is set, else take 1.0 (amp 0, dir 1)
    r, t, _ = parse(lib, BASE + "pulse_t0 = 600.0\npulse_amp = 5.0\npulse_dir = 2\n"
                    "PULSE = 1\npulse_t1 = 300.0\n")
    s = t.source
    assert s.kind == abi.SPARC_SRC_PULSE
    assert s.t0 == 1.0 and s.amp == 0.0 and s.dir == 1 and s.t1 == 300.0
    # t_xy / t_z below the timestep read so far become that timestep
    r, t, _ = parse(lib, "t_z = 0.1\n" + BASE + "t_xy = 0.25\n")
    assert t.params.t_z == 0.1 and t.params.t_xy == 0.5
    assert t.zfreq == 0 and t.xyfreq == 1


def test_sources_and_run_length(lib):
    # PULSE = 0: the random source, its series length from driver.f90:38-39
    text = BASE + ("PULSE = 0\nsolartime = 1.0\ncadforcing = 45.0\n"
                   "randomexciteampl = 1.0d4\nrandomexcitedepth = -0.15d8\n"
                   "randomexcitesigma = 0.075d8\n")
    r, t, _ = parse(lib, text)
    s = t.source
    assert s.kind == abi.SPARC_SRC_RANDOM and t.pulse == 0 and s.dir == 3
    assert (s.rnd_ampl, s.rnd_depth, s.rnd_sigma) == (1.0e4, -0.15e8, 0.075e8)
    assert t.maxtime == 7200
    assert s.nseries == t.num_steps == 2 * ((80 + 2) // 2) + 2
    # PULSE = 2: the PSR field (its table is drawn by the caller)
    r, t, _ = parse(lib, BASE + "PULSE = 2\npulse_dir = 3\nTWOD = 1\n")
    assert t.source.kind == abi.SPARC_SRC_PSR and t.source.psr_st == 120.0
    assert t.psr_npulses == 100 and t.params.ny == 1 and t.params.ylength == 0.0
    # odd run lengths are made even; a restart starts after snapshot time0
    r, t, _ = parse(lib, BASE + "solartime = 0.00375\nrestart = 1\ntime0 = 3\n"
                    "fulloutputcad = 5.0\n")
    assert t.maxtime == 26 and t.fulloutputsteps == 10 and t.init == 31
    assert t.source.init == 31
    # a zero output cadence switches that output off (steps 1)
    assert t.chunkout == 0 and t.chunkoutputsteps == 1


def test_crlf_and_filter_modes(lib):
    text = BASE.replace("\n", "\r\n") + "filter_mode_xy = 2\r\nfilter_mode_z = 7\r\nMAGNETIC = 0\r\n"
    r, t, _ = parse(lib, text)
    assert r == abi.SPARC_OK
    assert t.params.filter_mode_xy == 2 and t.params.filter_mode_z == 0
    assert t.params.magnetic == 0 and t.simname == b"_3D_vq_"


def test_damping_key_reaches_the_parameters(lib):
    """DAMPING (initialize.f90:1512-1517, an integer switch: 0 off, any other
    value on): the FFT damping the library runs in the FP64 plain form."""
    r, t, _ = parse(lib, BASE + "DAMPING = 2\n")
    assert r == abi.SPARC_OK and t.damping == 1 and t.params.damping == 1
    r, t, _ = parse(lib, BASE + "DAMPING = 0\n")
    assert r == abi.SPARC_OK and t.damping == 0 and t.params.damping == 0
