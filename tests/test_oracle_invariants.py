"""Invariants of the FP64 oracle (independent of the reference's rounding)."""
import numpy as np
import pytest

from cudalbm_b200 import casefiles
from pyoracle import Oracle


def lid_oracle(q, n=(16, 16, 16), Re=100.0, u=0.05):
    o = Oracle(q, *n, Re, u)
    m = o.initial(casefiles.scaled_region_values(casefiles.lid_cavity_values(u)))
    return o, m


def test_rest_state_stays_at_rest_d3q19():
    o = Oracle(19, 16, 16, 16, 100.0, 0.0)
    m = o.initial(casefiles.scaled_region_values(casefiles.lid_cavity_values(0.0)))
    assert not m.any()
    o.run(m, 10)
    assert np.max(np.abs(m)) < 1e-14


def test_rest_state_d3q27_lid_corner_quirk():
    """D3Q27 at rest stays at rest except at the four North (lid) corners:
    the reference's lid-corner formula rho = -24 rho_I / (-14 - 8U + 9U^2)
    (boundaryConditions.cuh:403-455) carries the D3Q19 constant 12/7 for both
    lattices, while the South corners use 216/125 for D3Q27.  At rest the
    known populations of a D3Q27 corner sum to 125/216, so those nodes get
    rho = 12/7 * 125/216."""
    o = Oracle(27, 16, 16, 16, 100.0, 0.0)
    m = o.initial(casefiles.scaled_region_values(casefiles.lid_cavity_values(0.0)))
    o.run(m, 1)
    corners = [(z, 15, x) for z in (0, 15) for x in (0, 15)]
    for c in corners:
        assert abs(m[0][c] - (12 / 7 * 125 / 216 - 1)) < 1e-14
        m[0][c] = 0.0
    assert np.max(np.abs(m)) < 1e-14


@pytest.mark.parametrize("q", [19, 27])
def test_boundary_classes_give_finite_positive_density(q):
    o, m = lid_oracle(q, (16, 24, 32))
    o.run(m, 20)
    rho = m[0] + 1.0
    assert np.all(np.isfinite(m))
    assert rho.min() > 0.5 and rho.max() < 1.5  # the impulsive lid start swings the lid corners by ~15%
    # every one of the 26 boundary classes + interior is present
    nz, ny, nx = rho.shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    t = (x == 0) * 1 | (x == nx - 1) * 2 | (y == 0) * 4 | (y == ny - 1) * 8 | (z == 0) * 16 | (z == nz - 1) * 32
    assert len(np.unique(t)) == 27


@pytest.mark.parametrize("q", [19, 27])
def test_mirror_symmetry_about_mid_z(q):
    """The lid moves in x on the North (y = max) face: the cavity is symmetric
    under z -> nz-1-z with w, m_xz, m_yz changing sign."""
    o, m = lid_oracle(q)
    o.run(m, 50)
    r = m[:, ::-1]
    sign = np.array([1, 1, 1, -1, 1, 1, -1, 1, -1, 1])[:, None, None, None]
    assert np.max(np.abs(m - sign * r)) < 1e-12


@pytest.mark.parametrize("q", [19, 27])
def test_mass_drift_is_small(q):
    o, m = lid_oracle(q)
    m0 = (m[0] + 1).sum()
    o.run(m, 200)
    assert abs((m[0] + 1).sum() - m0) / m0 < 5e-3


@pytest.mark.parametrize("q", [19, 27])
def test_lid_drives_positive_u_below_the_lid(q):
    o, m = lid_oracle(q)
    o.run(m, 100)
    nz, ny, nx = m.shape[1:]
    u_below_lid = m[1, nz // 2, ny - 2, nx // 2] / 3.0
    assert 0.0 < u_below_lid < 0.05


def test_function_objects_formulas():
    """S, k and the running means follow the reference's definitions."""
    o, m = lid_oracle(19, (8, 8, 8))
    fo = o.new_function_objects(["S", "SMean", "k", "kMean", "momentsMean"])
    snaps = []
    for t in range(3):
        o.run(m, 1, t, fo)
        snaps.append(m.copy())
    u, v, w = m[1], m[2], m[3]
    tau = float(o.p.tau)
    np.testing.assert_allclose(fo["k"][0], 0.5 * np.sqrt(u * u + v * v + w * w), rtol=1e-12)
    np.testing.assert_allclose(fo["S"][1], 3 * (u * v - m[5]) / (18 * tau), rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(fo["momentsMean"], np.mean(snaps, axis=0), rtol=1e-10, atol=1e-14)
