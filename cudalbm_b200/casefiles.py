"""Writer for cudaLBM case directories.

A case directory holds the four text files the solvers read from their working
directory (``programControl``, ``latticeMesh``, ``initialConditions`` and the
optional ``functionObjects``).  The layout written here is the one the
reference ships in ``lidDrivenCavity/D3Q19/*`` and parses with
``src/strings.cuh:311-414`` (blocks) and ``src/strings.cuh:561-585``
(``key value;`` lines), so the same directory runs unchanged under the
reference executables and under this project's ``momentBasedD3Q19`` /
``momentBasedD3Q27``.

The product's own parser is C++ (``cudalbm_b200/csrc/casefile.cpp``); this
module exists for tests, the benchmark and fixture generation.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Dict, Iterable, Optional

_BANNER = (
    "/*---------------------------------------------------------------------------*\\\n"
    "|                                                                             |\n"
    "| lid-driven cavity case (moment-representation LBM)                          |\n"
    "|                                                                             |\n"
    "\\*---------------------------------------------------------------------------*/\n"
    "\n"
)

MOMENT_NAMES = ("rho", "u", "v", "w", "m_xx", "m_xy", "m_xz", "m_yy", "m_yz", "m_zz")
REGIONS = ("internalField", "North", "South", "East", "West", "Front", "Back")
FUNCTION_OBJECTS = ("S", "SMean", "k", "kMean", "momentsMean")


def lid_cavity_values(u_lid: float) -> Dict[str, Dict[str, object]]:
    """Initial/boundary values of the shipped lid-driven cavity case.

    Every field is 0 everywhere except ``u`` on North (the lid velocity) and
    ``m_xx`` on North, which is ``equilibrium`` (reference
    ``lidDrivenCavity/D3Q19/initialConditions:12-390``).
    """
    vals: Dict[str, Dict[str, object]] = {
        name: {region: 0 for region in REGIONS} for name in MOMENT_NAMES
    }
    vals["u"]["North"] = u_lid
    vals["m_xx"]["North"] = "equilibrium"
    return vals


@dataclass
class CaseSpec:
    """Everything needed to write one cavity case directory."""

    nx: int
    ny: int
    nz: int
    Re: float
    u_inf: float
    n_steps: int
    save_interval: int
    info_interval: int
    case_name: str = "lidDrivenCavity"
    function_objects: Iterable[str] = ()
    lid_ic: Optional[float] = None  # North 'u' in initialConditions (defaults to u_inf)
    values: Optional[Dict[str, Dict[str, object]]] = None
    L: tuple = (1.0, 1.0, 1.0)
    extra_files: Dict[str, str] = field(default_factory=dict)

    def initial_values(self) -> Dict[str, Dict[str, object]]:
        if self.values is not None:
            return self.values
        return lid_cavity_values(self.u_inf if self.lid_ic is None else self.lid_ic)


def _fmt(v: object) -> str:
    if isinstance(v, str):
        return v
    if isinstance(v, int):
        return str(v)
    s = repr(float(v))
    if "e" in s or "E" in s:
        # the reference's isNumber() accepts only [+-]digits[.digits]
        s = f"{float(v):.12f}".rstrip("0")
        if s.endswith("."):
            s += "0"
    return s


def program_control_text(spec: CaseSpec) -> str:
    return _BANNER + (
        "/*---------------------------------------------------------------------------*\\\n\n"
        f"caseName        {spec.case_name};\n\n"
        f"Re              {_fmt(spec.Re)};\n\n"
        f"u_inf           {_fmt(spec.u_inf)};\n\n"
        "startFrom       latestTime;\n\n"
        "startTime       0;\n\n"
        f"nTimeSteps      {int(spec.n_steps)};\n\n"
        f"saveInterval    {int(spec.save_interval)};\n\n"
        f"infoInterval    {int(spec.info_interval)};\n\n"
        "\\*---------------------------------------------------------------------------*/\n"
    )


def lattice_mesh_text(spec: CaseSpec) -> str:
    lx, ly, lz = spec.L
    return _BANNER + (
        "/*---------------------------------------------------------------------------*\\\n\n"
        f"nx              {int(spec.nx)};\n\n"
        f"ny              {int(spec.ny)};\n\n"
        f"nz              {int(spec.nz)};\n\n"
        f"Lx              {_fmt(lx)};\n\n"
        f"Ly              {_fmt(ly)};\n\n"
        f"Lz              {_fmt(lz)};\n\n"
        "\\*---------------------------------------------------------------------------*/\n"
    )


def initial_conditions_text(values: Dict[str, Dict[str, object]]) -> str:
    out = [_BANNER, "/*---------------------------------------------------------------------------*\\\n\n"]
    for name in MOMENT_NAMES:
        out.append(f"field {name}\n{{\n")
        regions = values[name]
        for i, region in enumerate(REGIONS):
            out.append(f"    {region}\n    {{\n        value   {_fmt(regions[region])};\n    }};\n")
            if i != len(REGIONS) - 1:
                out.append("\n")
        out.append("};\n\n")
    out.append("\\*---------------------------------------------------------------------------*/\n")
    return "".join(out)


def function_objects_text(enabled: Iterable[str]) -> str:
    enabled = list(enabled)
    for name in enabled:
        if name not in FUNCTION_OBJECTS:
            raise ValueError(f"unknown function object {name!r}")
    lines = []
    for name in FUNCTION_OBJECTS:
        prefix = "" if name in enabled else "// "
        lines.append(f"    {prefix}{name};\n")
    return _BANNER + (
        "/*---------------------------------------------------------------------------*\\\n\n"
        "functionObjectList\n{\n" + "".join(lines) + "};\n\n"
        "\\*---------------------------------------------------------------------------*/\n"
    )


def write_case(directory: str, spec: CaseSpec) -> str:
    """Write the case files of ``spec`` into ``directory`` (created if needed)."""
    os.makedirs(directory, exist_ok=True)
    files = {
        "programControl": program_control_text(spec),
        "latticeMesh": lattice_mesh_text(spec),
        "initialConditions": initial_conditions_text(spec.initial_values()),
        "functionObjects": function_objects_text(spec.function_objects),
    }
    files.update(spec.extra_files)
    for fname, text in files.items():
        with open(os.path.join(directory, fname), "w") as fh:
            fh.write(text)
    return directory


def scaled_region_values(values: Dict[str, Dict[str, object]]):
    """Per-region initial values scaled the way the reference stores them.

    Returns a float32 array ``[10, 7]`` (fields in moment order, regions in the
    order internalField, North, South, East, West, Front, Back).  Numbers are
    scaled by 1 (rho), 3 (u, v, w), 4.5 (m_aa) or 9 (m_ab); ``equilibrium``
    gives 4.5*u_a*u_b/rho0 from the same region's raw velocities -- 4.5 also
    for the off-diagonal moments, as the reference does
    (src/boundaryConditions/boundaryValue.cuh:147-254).
    """
    import numpy as np

    f32 = np.float32
    scale = {"rho": 1.0, "u": 3.0, "v": 3.0, "w": 3.0, "m_xx": 4.5, "m_xy": 9.0, "m_xz": 9.0,
             "m_yy": 4.5, "m_yz": 9.0, "m_zz": 4.5}
    eq_pair = {"m_xx": ("u", "u"), "m_xy": ("u", "v"), "m_xz": ("u", "w"),
               "m_yy": ("v", "v"), "m_yz": ("v", "w"), "m_zz": ("w", "w")}
    out = np.zeros((10, 7), dtype=np.float32)
    for fi, name in enumerate(MOMENT_NAMES):
        for ri, region in enumerate(REGIONS):
            v = values[name][region]
            if isinstance(v, str):
                if v != "equilibrium" or name not in eq_pair:
                    raise ValueError(f"invalid value {v!r} for {name} in {region}")
                a, b = eq_pair[name]
                ua, ub = f32(float(values[a][region])), f32(float(values[b][region]))
                out[fi, ri] = f32(4.5) * (ua * ub) / f32(1.0)
            else:
                out[fi, ri] = f32(float(v)) * f32(scale[name])
    return out


def relaxation(u_inf: float, Re: float, nx: int):
    """(tau, omega, 1-omega, omega/2) in float32 exactly as the reference
    computes them: nu = u_inf*(nx-1)/Re (src/latticeMesh/latticeMesh.cuh:177-201)."""
    import numpy as np

    f32 = np.float32
    nu = f32(u_inf) * f32(nx - 1) / f32(Re)
    tau = f32(0.5) + f32(3.0) * nu
    omega = f32(1.0) / tau
    return tau, omega, f32(1.0) - omega, omega * f32(0.5)


# ------------------------------------------------------ batched workloads
class MT19937_64:
    """The 64-bit Mersenne Twister (Matsumoto & Nishimura 2004; the engine of
    C++'s std::mt19937_64), so that seeded workloads are reproducible in any
    host language without a library."""

    _N, _M = 312, 156
    _A = 0xB5026F5AA96619E9
    _UPPER, _LOWER = 0xFFFFFFFF80000000, 0x7FFFFFFF
    _MASK = (1 << 64) - 1

    def __init__(self, seed: int):
        mt = [seed & self._MASK]
        for i in range(1, self._N):
            prev = mt[-1]
            mt.append((6364136223846793005 * (prev ^ (prev >> 62)) + i) & self._MASK)
        self._mt, self._i = mt, self._N

    def _twist(self) -> None:
        mt, n, m = self._mt, self._N, self._M
        for i in range(n):
            x = (mt[i] & self._UPPER) | (mt[(i + 1) % n] & self._LOWER)
            xa = (x >> 1) ^ (self._A if x & 1 else 0)
            mt[i] = mt[(i + m) % n] ^ xa
        self._i = 0

    def next(self) -> int:
        if self._i >= self._N:
            self._twist()
        y = self._mt[self._i]
        self._i += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & self._MASK


BATCH_EDGES = (32, 48, 64, 96, 128)


def random_cavities(n: int = 64, seed: int = 0, edges=BATCH_EDGES, re_range=(100.0, 2000.0), u_lid: float = 0.05,
                    lattice: int = 19):
    """Cubic lid-driven cavities of uneven size and Reynolds number.

    MT19937-64 seeded with `seed`; for each cavity in turn, one draw x picks
    the edge edges[x % len(edges)] and the next draw y gives
    Re = lo + (hi - lo) * (y >> 11) / 2^53.  Returns a list of dicts with the
    keys of solver.Cavity."""
    g = MT19937_64(seed)
    lo, hi = re_range
    out = []
    for _ in range(n):
        e = int(edges[g.next() % len(edges)])
        re = lo + (hi - lo) * ((g.next() >> 11) * 2.0 ** -53)
        out.append(dict(lattice=lattice, nx=e, ny=e, nz=e, Re=float(re), u_inf=u_lid))
    return out
