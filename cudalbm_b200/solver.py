"""Python front end of the solver: one lid-driven cavity on one GPU.

Mirrors what the reference executables do in ``main``
(applications/momentBasedD3Q19/momentBasedD3Q19.cu:56-140): read a case,
set up the state, step, write .LBMBin snapshots.  All compute goes through the
C ABI (include/lbm_b200.h); this module only marshals host buffers.
"""
from __future__ import annotations

import ctypes
from typing import Dict, Iterable, Optional

import numpy as np

from . import _lib
from .casefiles import MOMENT_NAMES, lid_cavity_values, scaled_region_values

FIELD_NAMES = {
    "moments": list(MOMENT_NAMES),
    "S": ["S_xx", "S_xy", "S_xz", "S_yy", "S_yz", "S_zz"],
    "SMean": ["S_xxMean", "S_xyMean", "S_xzMean", "S_yyMean", "S_yzMean", "S_zzMean"],
    "k": ["k"],
    "kMean": ["kMean"],
    "momentsMean": [n + "Mean" for n in MOMENT_NAMES],
}
NVARS = {k: len(v) for k, v in FIELD_NAMES.items()}


class Cavity:
    """Device state of one cavity behind an ``lbm_handle``."""

    def __init__(self, lattice: int, nx: int, ny: int, nz: int, Re: float, u_inf: float,
                 function_objects: Iterable[str] = (), mean_bits: int = 32, device: int = 0,
                 start_step: int = 0, tile: Optional[tuple] = None, z_chunk: int = 0, pop_buffers: int = 0,
                 storage: str = "f32"):
        L = _lib.lib()
        cfg = _lib.Config()
        L.lbm_config_default(ctypes.byref(cfg))
        cfg.lattice, cfg.device = int(lattice), int(device)
        cfg.nx, cfg.ny, cfg.nz = int(nx), int(ny), int(nz)
        cfg.Re, cfg.u_inf = float(Re), float(u_inf)
        self.function_objects = list(function_objects)
        mask = 0
        for name in self.function_objects:
            mask |= _lib.FO_BITS[name]
        cfg.function_objects = mask
        cfg.mean_bits = int(mean_bits)
        cfg.start_step = int(start_step)
        if tile:
            cfg.tile_x, cfg.tile_y = int(tile[0]), int(tile[1])
            if len(tile) > 2:
                cfg.stages = int(tile[2])
        cfg.z_chunk = int(z_chunk)
        cfg.pop_buffers = int(pop_buffers)
        cfg.storage = _lib.STORAGE[storage]
        self.storage = storage
        self.cfg = cfg
        self.shape = (nz, ny, nx)
        self.mean_bits = mean_bits
        h = ctypes.c_void_p()
        _lib.check(L.lbm_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h

    @classmethod
    def _borrowed(cls, handle: ctypes.c_void_p, cfg, owner) -> "Cavity":
        """View of a cavity owned by a Batch (closing it releases nothing)."""
        self = cls.__new__(cls)
        self.function_objects = []
        self.storage = "f32"
        self.cfg = cfg
        self.shape = (int(cfg.nz), int(cfg.ny), int(cfg.nx))
        self.mean_bits = int(cfg.mean_bits)
        self._h = handle
        self._owner = owner
        return self

    # ------------------------------------------------------------ lifecycle
    def close(self) -> None:
        if getattr(self, "_owner", None) is not None:
            self._h = None
            return
        if getattr(self, "_h", None):
            _lib.lib().lbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -------------------------------------------------------------- state
    def init_regions(self, region_values=None) -> None:
        """Initial state from per-region values (default: the lid cavity)."""
        if region_values is None:
            region_values = scaled_region_values(lid_cavity_values(self.cfg.u_inf))
        rv = np.ascontiguousarray(region_values, dtype=np.float32).reshape(70)
        _lib.check(_lib.lib().lbm_init_regions(self._h, rv.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def write(self, data: np.ndarray, field_set: str = "moments", tiled: bool = False) -> None:
        data = np.ascontiguousarray(data)
        dtype = _lib.F64 if data.dtype == np.float64 else _lib.F32
        if data.dtype not in (np.float32, np.float64):
            data = data.astype(np.float32)
        _lib.check(_lib.lib().lbm_write_fields(self._h, _lib.FIELD_SET[field_set], data.ctypes.data, data.size,
                                               dtype, _lib.ORDER_TILED if tiled else _lib.ORDER_GLOBAL))

    def read(self, field_set: str = "moments", dtype=np.float32, tiled: bool = False, out=None) -> np.ndarray:
        nv = NVARS[field_set]
        nz, ny, nx = self.shape
        shape = (nv, nx * ny * nz) if tiled else (nv, nz, ny, nx)
        if out is None:
            out = np.empty(shape, dtype=dtype)
        _lib.check(_lib.lib().lbm_read_fields(self._h, _lib.FIELD_SET[field_set], out.ctypes.data, out.size,
                                              _lib.F64 if out.dtype == np.float64 else _lib.F32,
                                              _lib.ORDER_TILED if tiled else _lib.ORDER_GLOBAL))
        return out

    def step(self, n: int = 1) -> None:
        _lib.check(_lib.lib().lbm_step(self._h, int(n)))

    def perturb_velocity(self, amplitude: float, seed: int) -> None:
        """Add U(-amplitude, amplitude) to u, v, w of every interior node."""
        _lib.check(_lib.lib().lbm_perturb_velocity(self._h, float(amplitude), int(seed)))

    def filter_from(self, fine: "Cavity") -> None:
        """This (coarse) state := 2:1 box filter of `fine`'s current state."""
        _lib.check(_lib.lib().lbm_filter_2to1(fine._h, self._h))

    def set_closure(self, net) -> None:
        """Relax every interior node with tau0 + dtau from the network `net`
        (an _lib.MLP) in every following step; None restores the plain method."""
        _lib.check(_lib.lib().lbm_closure_set(self._h, ctypes.byref(net) if net is not None else None))

    def closure_refresh(self, every: int) -> None:
        """Recompute the closure's dtau every `every` steps (1: every step)."""
        _lib.check(_lib.lib().lbm_closure_refresh(self._h, int(every)))

    def closure_fused(self, on: bool = True) -> None:
        """Evaluate the closure network inside the step kernel (True, the
        default) or in a separate inference kernel (False); same results."""
        _lib.check(_lib.lib().lbm_closure_fused(self._h, int(bool(on))))

    def closure_dtau(self) -> np.ndarray:
        nz, ny, nx = self.shape
        out = np.empty((nz, ny, nx), np.float32)
        _lib.check(_lib.lib().lbm_closure_dtau(self._h, out.ctypes.data, out.size))
        return out

    def cut_plane(self, axis: int, position: float, field_set: str = "moments") -> np.ndarray:
        """Plane normal to `axis` (0 x, 1 y, 2 z) at `position` in [0, 1]
        between the first and last node plane, linearly interpolated on the
        device; shape [nvars, b, a] with (a, b) = (y, z), (x, z) or (x, y)."""
        nz, ny, nx = self.shape
        na = ny if axis == 0 else nx
        nb = ny if axis == 2 else nz
        out = np.empty((NVARS[field_set], nb, na), dtype=np.float32)
        _lib.check(_lib.lib().lbm_cut_plane(self._h, _lib.FIELD_SET[field_set], int(axis), float(position),
                                            out.ctypes.data, out.size))
        return out

    def step_monitored(self, n: int, out=None):
        """n steps, each returning (mass, rho*|u_stored|^2, nonfinite) sums
        computed by the step kernel; ``out`` is a structured array of length
        >= n (page-locked for a fully asynchronous call).  Valid after
        synchronize()."""
        if out is None:
            out = np.zeros(n, dtype=_lib.MONITOR_DTYPE)
        _lib.check(_lib.lib().lbm_step_monitored(self._h, int(n), out.ctypes.data))
        return out

    def run_streamed(self, moments: np.ndarray, n: int, outs: Dict[str, np.ndarray], monitor=None,
                     slab: int = 0, z_chunk: int = 0, lead: int = 0) -> None:
        """One job between host arrays with the copies overlapping the steps:
        upload ``moments`` ([10, nz, ny, nx] float32), advance ``n`` steps and
        download each field set named in ``outs`` into its array ([nvars, nz,
        ny, nx]; float64 for the means of an FP64-mean handle); ``monitor``
        (structured array of length n, or None) receives the per-step sums.
        Page-locked arrays (_lib.PinnedArray) let the copies run at full speed."""
        nz, ny, nx = self.shape
        if moments.dtype != np.float32 or not moments.flags.c_contiguous or moments.size != 10 * nx * ny * nz:
            raise ValueError("moments must be a contiguous float32 array of 10 fields")
        ptrs = (ctypes.c_void_p * 6)()
        for name, arr in outs.items():
            want = np.float64 if (self.cfg.mean_bits == 64 and "Mean" in name) else np.float32
            if arr.dtype != want or not arr.flags.c_contiguous or arr.size != NVARS[name] * nx * ny * nz:
                raise ValueError(f"output '{name}' must be a contiguous {np.dtype(want).name} array of "
                                 f"{NVARS[name]} fields")
            ptrs[_lib.FIELD_SET[name]] = arr.ctypes.data
        if monitor is not None and (monitor.dtype != np.dtype(_lib.MONITOR_DTYPE) or monitor.size < n):
            raise ValueError("monitor must be a MONITOR_DTYPE array of at least n entries")
        opts = _lib.StreamOpts(int(slab), int(z_chunk), int(lead))
        _lib.check(_lib.lib().lbm_run_streamed(self._h, moments.ctypes.data, int(n), ptrs,
                                               monitor.ctypes.data if monitor is not None else None,
                                               ctypes.byref(opts)))

    def autotune(self, trial_steps: int = 10) -> Dict[str, object]:
        """Pick the fastest kernel variant for this size class (state unchanged)."""
        t = _lib.Tuning()
        _lib.check(_lib.lib().lbm_autotune(self._h, int(trial_steps), ctypes.byref(t)))
        return {f: getattr(t, f) for f, _ in t._fields_}

    def synchronize(self) -> None:
        _lib.check(_lib.lib().lbm_synchronize(self._h))

    def reduce(self) -> Dict[str, float]:
        out = (ctypes.c_double * 3)()
        _lib.check(_lib.lib().lbm_reduce(self._h, out))
        return {"mass": out[0], "kinetic_energy": out[1], "nonfinite": int(out[2])}

    def info(self) -> Dict[str, object]:
        inf = _lib.Info()
        _lib.check(_lib.lib().lbm_get_info(self._h, ctypes.byref(inf)))
        return {f: getattr(inf, f) for f, _ in inf._fields_}


def write_vts(path: str, fields: np.ndarray, names: Iterable[str], lengths=(1.0, 1.0, 1.0)) -> None:
    """VTK XML structured grid of fields [nvars, nz, ny, nx] (the file format
    of fieldConvert -fileType vts)."""
    fields = np.ascontiguousarray(fields, dtype=np.float32)
    if fields.ndim == 3:  # one plane: [nvars, ny, nx]
        fields = fields.reshape((fields.shape[0], 1) + fields.shape[1:])
    nv, nz, ny, nx = fields.shape
    names = [n.encode() for n in names]
    arr = (ctypes.c_char_p * nv)(*names)
    L = (ctypes.c_float * 3)(*lengths)
    _lib.check(_lib.lib().lbm_vts_write(path.encode(), nx, ny, nz, L, nv, arr, fields.ctypes.data))


def field_statistics(fields: np.ndarray, shape=None, tiled: bool = False, device: int = 0):
    """fieldCalculate's checks of fields [nfields][nz][ny][nx] (or
    [nfields][nodes] in the .LBMBin tiled order with tiled=True and
    shape=(nz, ny, nx)), on the GPU: (NaN count, the reference's spatial mean
    -- left-to-right float sum in global order / float(nodes) --, FP64 mean)
    per field."""
    fields = np.ascontiguousarray(fields, dtype=np.float32)
    nf = fields.shape[0]
    nz, ny, nx = shape if shape is not None else fields.shape[1:]
    nan = np.zeros(nf, np.int32)
    mean_ref = np.zeros(nf, np.float32)
    mean = np.zeros(nf, np.float64)
    _lib.check(_lib.lib().lbm_field_statistics(int(device), fields.ctypes.data, int(nx), int(ny), int(nz), int(nf),
                                               _lib.ORDER_TILED if tiled else _lib.ORDER_GLOBAL, nan.ctypes.data,
                                               mean_ref.ctypes.data, mean.ctypes.data))
    return nan, mean_ref, mean


class Batch:
    """Many independent cavities advanced by one persistent launch per step.

    ``specs`` is a sequence of dicts with the keys of ``Cavity`` (lattice, nx,
    ny, nz, Re, u_inf, ...); all share the lattice, FP32 storage, no function
    objects.  ``batch[i]`` is a ``Cavity`` view of cavity i for state set-up
    and read-back.
    """

    def __init__(self, specs, device: int = 0):
        L = _lib.lib()
        specs = list(specs)
        cfgs = (_lib.Config * len(specs))()
        for c, sp in zip(cfgs, specs):
            L.lbm_config_default(ctypes.byref(c))
            c.lattice = int(sp.get("lattice", 19))
            c.device = int(device)
            c.nx, c.ny, c.nz = int(sp["nx"]), int(sp["ny"]), int(sp["nz"])
            c.Re, c.u_inf = float(sp["Re"]), float(sp.get("u_inf", 0.05))
            c.start_step = int(sp.get("start_step", 0))
            c.z_chunk = int(sp.get("z_chunk", 0))
        self.cfgs = cfgs
        b = ctypes.c_void_p()
        _lib.check(L.lbm_batch_create(cfgs, len(specs), ctypes.byref(b)))
        self._b = b
        self.cavities = []
        for i in range(len(specs)):
            h = ctypes.c_void_p()
            _lib.check(L.lbm_batch_cavity(b, i, ctypes.byref(h)))
            self.cavities.append(Cavity._borrowed(h, cfgs[i], self))

    def __len__(self):
        return len(self.cavities)

    def __getitem__(self, i) -> Cavity:
        return self.cavities[i]

    def close(self) -> None:
        if getattr(self, "_b", None):
            for c in self.cavities:
                c.close()
            _lib.lib().lbm_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def init_regions(self) -> None:
        """Lid-cavity initial state in every cavity."""
        for c in self.cavities:
            c.init_regions()

    def step(self, n: int = 1) -> None:
        _lib.check(_lib.lib().lbm_batch_step(self._b, int(n)))

    def synchronize(self) -> None:
        _lib.check(_lib.lib().lbm_batch_synchronize(self._b))

    def autotune(self, trial_steps: int = 10) -> Dict[str, object]:
        t = _lib.BatchTuning()
        _lib.check(_lib.lib().lbm_batch_autotune(self._b, int(trial_steps), ctypes.byref(t)))
        return {f: getattr(t, f) for f, _ in t._fields_}

    def configure(self, tile_x: int, tile_y: int = 8, stages: int = 2, pop_buffers: int = 1,
                  persistent: bool = True) -> None:
        """Set the batched kernel's shape by hand (instead of autotune)."""
        t = _lib.BatchTuning(tile_x=tile_x, tile_y=tile_y, stages=stages, pop_buffers=pop_buffers,
                             persistent=int(bool(persistent)))
        _lib.check(_lib.lib().lbm_batch_configure(self._b, ctypes.byref(t)))

    def info(self) -> Dict[str, object]:
        inf = _lib.BatchInfo()
        _lib.check(_lib.lib().lbm_batch_get_info(self._b, ctypes.byref(inf)))
        return {f: getattr(inf, f) for f, _ in inf._fields_}
