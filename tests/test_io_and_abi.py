"""Host-side pieces: .LBMBin format, block-tiled order, case files, C ABI."""
import ctypes
import os
import re

import numpy as np
import pytest

from cudalbm_b200 import _lib, casefiles, lbmbin

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_block_tiled_index_is_a_permutation():
    idx = lbmbin.block_tiled_index(16, 24, 8)
    assert sorted(idx.ravel().tolist()) == list(range(16 * 24 * 8))
    # first 8 entries of a block are one x-row of the first block
    assert idx[0, 0, :8].tolist() == list(range(8))
    assert idx[0, 1, 0] == 8 and idx[1, 0, 0] == 64 and idx[0, 0, 8] == 512


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_lbmbin_roundtrip(tmp_path, dtype):
    rng = np.random.default_rng(0)
    data = rng.standard_normal((3, 8, 16, 24)).astype(dtype)
    p = tmp_path / "f_7.LBMBin"
    lbmbin.write(str(p), ["a", "b", "c"], data, 7, "timeAverage")
    f = lbmbin.read(str(p))
    assert f.names == ["a", "b", "c"] and f.time_step == 7 and f.time_type == "timeAverage"
    assert (f.nx, f.ny, f.nz) == (24, 16, 8)
    assert np.array_equal(f.data, data)
    raw = p.read_bytes()
    assert raw.startswith(b"systemInformation\n{\n\tbinaryType\tlittleEndian;")
    assert b"\tfield[9216][3][8][16][24]\n\t{\n" in raw


def test_lbmbin_truncated_file_is_rejected(tmp_path):
    data = np.zeros((1, 8, 8, 8), np.float32)
    p = tmp_path / "t_0.LBMBin"
    lbmbin.write(str(p), ["x"], data, 0)
    p.write_bytes(p.read_bytes()[:-200])
    with pytest.raises(ValueError):
        lbmbin.read(str(p))


def test_case_files_grammar(tmp_path):
    spec = casefiles.CaseSpec(nx=16, ny=24, nz=32, Re=100.0, u_inf=0.05, n_steps=11, save_interval=5,
                              info_interval=5, function_objects=("S", "kMean"))
    casefiles.write_case(str(tmp_path), spec)
    pc = (tmp_path / "programControl").read_text()
    assert re.search(r"^nTimeSteps\s+11;$", pc, re.M)
    fo = (tmp_path / "functionObjects").read_text()
    assert "    S;\n" in fo and "    // SMean;\n" in fo and "    kMean;\n" in fo
    ic = (tmp_path / "initialConditions").read_text()
    assert "field m_xx\n{" in ic and "value   equilibrium;" in ic


def test_scaled_region_values():
    rv = casefiles.scaled_region_values(casefiles.lid_cavity_values(0.05))
    assert rv.shape == (10, 7) and rv.dtype == np.float32
    north = casefiles.REGIONS.index("North")
    assert rv[1, north] == np.float32(0.05) * np.float32(3)
    assert rv[4, north] == np.float32(4.5) * (np.float32(0.05) * np.float32(0.05))
    assert np.count_nonzero(rv) == 2


def _declared_functions():
    text = open(os.path.join(ROOT, "include", "lbm_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbm_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    declared = _declared_functions()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(L, name), name
    assert set(declared) == set(_lib.EXPORTS)


def test_abi_calls_that_need_no_gpu():
    L = _lib.lib()
    cfg = _lib.Config()
    L.lbm_config_default(ctypes.byref(cfg))
    assert cfg.lattice == 19 and cfg.nx == 64 and abs(cfg.u_inf - 0.05) < 1e-7
    assert L.lbm_status_string(4) == b"device wait timed out"
    assert [L.lbm_field_set_vars(i) for i in range(6)] == [10, 6, 6, 1, 1, 10]
    # invalid sizes are rejected before any device work
    cfg.nx = 12
    h = ctypes.c_void_p()
    assert L.lbm_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    assert b"multiples of 8" in L.lbm_last_error()
    cfg.nx, cfg.lattice = 16, 15
    assert L.lbm_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    assert L.lbm_create(None, ctypes.byref(h)) == 1
    # node offsets within a field are 32-bit: 2^32 nodes or more are refused
    cfg.lattice, cfg.nx, cfg.ny, cfg.nz = 19, 2048, 2048, 1024
    assert L.lbm_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    assert b"at most 2^32 - 1 nodes" in L.lbm_last_error()


def test_batch_calls_that_need_no_gpu():
    L = _lib.lib()
    cfgs = (_lib.Config * 2)()
    for c in cfgs:
        L.lbm_config_default(ctypes.byref(c))
    b = ctypes.c_void_p()
    assert L.lbm_batch_create(None, 2, ctypes.byref(b)) == 1
    assert L.lbm_batch_create(cfgs, 0, ctypes.byref(b)) == 1
    cfgs[1].lattice = 27
    assert L.lbm_batch_create(cfgs, 2, ctypes.byref(b)) == 1
    assert b"share the lattice" in L.lbm_last_error()
    cfgs[1].lattice = 19
    cfgs[0].function_objects = _lib.FO_K
    assert L.lbm_batch_create(cfgs, 2, ctypes.byref(b)) == 1
    assert b"plain method" in L.lbm_last_error()
    cfgs[0].function_objects = 0
    cfgs[0].storage = 1
    assert L.lbm_batch_create(cfgs, 2, ctypes.byref(b)) == 1
    assert L.lbm_batch_destroy(None) == 0


def test_seeded_batch_workload():
    # MT19937-64: the C++ standard's check value (10000th draw, default seed)
    g = casefiles.MT19937_64(5489)
    for _ in range(9999):
        g.next()
    assert g.next() == 9981545732273789042
    cav = casefiles.random_cavities(64, seed=0)
    assert len(cav) == 64
    assert {c["nx"] for c in cav} == set(casefiles.BATCH_EDGES)
    assert all(c["nx"] == c["ny"] == c["nz"] for c in cav)
    assert all(100.0 <= c["Re"] < 2000.0 for c in cav)
    assert 35e6 < sum(c["nx"] ** 3 for c in cav) < 50e6
    assert cav == casefiles.random_cavities(64, seed=0)
