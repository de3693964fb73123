"""The library's case-file reader and .LBMBin writer (host C++ behind the C
ABI), checked on CPU: same values as the reference grammar gives, same bytes
as the reference writer's layout, and the reference's error behaviour."""
import ctypes
import os

import numpy as np
import pytest

from cudalbm_b200 import _lib, casefiles, lbmbin

# case directories shipped with the reference, read from a checkout named by
# LBM_REFERENCE_DIR (the tests that need them skip when it is unset)
REF_CASES = ["lidDrivenCavity/D3Q19", "lidDrivenCavity/D3Q27", "unitTests/ComputeSanitizerTest"]


def reference_case(rel):
    ref = os.environ.get("LBM_REFERENCE_DIR")
    if not ref:
        pytest.skip("LBM_REFERENCE_DIR is not set (no reference checkout to read the shipped cases from)")
    path = os.path.join(ref, rel)
    if not os.path.isdir(path):
        pytest.skip(f"{path} is not a directory")
    return path


def write(tmp_path, **kw):
    spec = casefiles.CaseSpec(**{**dict(nx=16, ny=24, nz=32, Re=250.0, u_inf=0.05, n_steps=101, save_interval=50,
                                        info_interval=10), **kw})
    casefiles.write_case(str(tmp_path), spec)
    return spec


def test_reads_generated_case(tmp_path):
    spec = write(tmp_path, function_objects=("S", "kMean", "momentsMean"), lid_ic=0.0064)
    c = _lib.read_case(str(tmp_path))
    assert c["case_name"] == "lidDrivenCavity"
    assert (c["nx"], c["ny"], c["nz"]) == (16, 24, 32)
    assert c["Re"] == np.float32(250.0) and c["u_inf"] == np.float32(0.05)
    assert (c["n_time_steps"], c["save_interval"], c["info_interval"]) == (101, 50, 10)
    assert c["function_objects"] == _lib.FO_S | _lib.FO_KMEAN | _lib.FO_MOMENTSMEAN
    assert np.array_equal(c["region"], casefiles.scaled_region_values(spec.initial_values()))
    assert c["has_restart"] == 0


@pytest.mark.parametrize("rel", REF_CASES)
def test_reads_the_reference_shipped_cases(rel):
    path = reference_case(rel)
    c = _lib.read_case(path)
    assert c["nx"] in (64, 256) and c["function_objects"] == 0
    north = casefiles.REGIONS.index("North")
    lid = 0.0256 if "lidDriven" in path else 0.0064
    assert c["region"][1, north] == np.float32(lid) * np.float32(3)
    assert c["region"][4, north] == np.float32(4.5) * np.float32(lid) * np.float32(lid)


def test_latest_time_and_restart_detection(tmp_path):
    write(tmp_path)
    for t in (0, 50, 100, 7):
        (tmp_path / f"lidDrivenCavity_{t}.LBMBin").write_bytes(b"")
    (tmp_path / "lidDrivenCavity_x1.LBMBin").write_bytes(b"")
    (tmp_path / "other_200.LBMBin").write_bytes(b"")
    c = _lib.read_case(str(tmp_path))
    assert c["has_restart"] == 1 and c["latest_time"] == 100


def test_substring_key_lookup_like_the_reference(tmp_path):
    """Keys are found by substring: the first line containing 'Re' wins."""
    write(tmp_path)
    pc = tmp_path / "programControl"
    pc.write_text("// Refine later\n" + pc.read_text())
    with pytest.raises(_lib.LBMError):
        _lib.read_case(str(tmp_path))  # '// Refine' has no ';'-terminated value token


def test_function_object_lines_must_match_exactly(tmp_path):
    write(tmp_path)
    (tmp_path / "functionObjects").write_text("functionObjectList\n{\n    S;\n    // k;\n    SMean ;\n    kMeanX;\n};\n")
    c = _lib.read_case(str(tmp_path))
    assert c["function_objects"] == _lib.FO_S | _lib.FO_SMEAN


def test_missing_and_malformed_files(tmp_path):
    with pytest.raises(_lib.LBMError) as e:
        _lib.read_case(str(tmp_path))
    assert e.value.status == 5  # I/O
    write(tmp_path)
    ic = tmp_path / "initialConditions"
    ic.write_text(ic.read_text().replace("value   equilibrium;", "value   banana;"))
    with pytest.raises(_lib.LBMError) as e:
        _lib.read_case(str(tmp_path))
    assert e.value.status == 6 and b"not a valid numerical value" in _lib.lib().lbm_last_error()
    write(tmp_path)
    ic.write_text(ic.read_text().replace("field m_yz\n{", "field m_yz\n"))
    with pytest.raises(_lib.LBMError):
        _lib.read_case(str(tmp_path))


@pytest.mark.parametrize("time_average", [0, 1])
def test_lbmbin_writer_bytes_match(tmp_path, time_average):
    rng = np.random.default_rng(1)
    data = rng.standard_normal((3, 8, 16, 24)).astype(np.float32)
    names = ["S_xx", "S_xy", "S_xz"]
    a = tmp_path / "a_12.LBMBin"
    b = tmp_path / "b_12.LBMBin"
    lbmbin.write(str(a), names, data, 12, "timeAverage" if time_average else "instantaneous")
    flat = np.ascontiguousarray(lbmbin.global_to_tiled(data))
    arr = (ctypes.c_char_p * 3)(*[n.encode() for n in names])
    _lib.check(_lib.lib().lbm_lbmbin_write(str(b).encode(), 24, 16, 8, 3, arr, flat.ctypes.data, 12, time_average))
    assert a.read_bytes() == b.read_bytes()
