"""Python binding of the C ABI in ``include/parahpop.h`` (ctypes over the
in-tree ``libparahpop_engine.so``).

The operator surface mirrors the reference's: a run configuration (the JSON
schema of ``example/config/*.json``) plus targets in the reference's target
schema, propagated by the B200 backend to final epochs and states.  There is
no CPU path: the library needs a CUDA device and fails loudly without one.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libparahpop_engine.so"
CLI_PATH = PKG / "bin" / "parahpop_gpu"

_lib = None


class PhopStats(C.Structure):
    _fields_ = [("kernel_ms", C.c_double), ("records_ms", C.c_double), ("total_ms", C.c_double),
                ("object_steps", C.c_int64), ("launches", C.c_int64), ("lanes", C.c_int), ("ctas", C.c_int),
                ("threads", C.c_int), ("split", C.c_int), ("shared_grid", C.c_int), ("tile_in_smem", C.c_int),
                ("tune_ms", C.c_double), ("tile_fallbacks", C.c_int64), ("pair_sh", C.c_int),
                ("deep_registers", C.c_int), ("registers", C.c_int)]


def library() -> C.CDLL:
    """Load the engine library (built by ``parahpop_b200.build``)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m parahpop_b200.build` first")
        lib = C.CDLL(str(LIB_PATH))
        D = C.POINTER(C.c_double)
        lib.phop_create.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]
        lib.phop_create.restype = C.c_int
        lib.phop_destroy.argtypes = [C.c_void_p]
        lib.phop_last_error.argtypes = [C.c_void_p]
        lib.phop_last_error.restype = C.c_char_p
        lib.phop_run_parameters.argtypes = [C.c_void_p, D, D, C.POINTER(C.c_int64)]
        lib.phop_propagate.argtypes = [C.c_void_p, C.c_int64] + [D] * 11
        lib.phop_propagate.restype = C.c_int
        lib.phop_propagate_device.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_double] + [D] * 5 + \
            [C.c_double, C.c_double, D]
        lib.phop_propagate_device.restype = C.c_int
        lib.phop_propagate_trajectory.argtypes = [C.c_void_p, C.c_int64, C.c_double] + [D] * 6 + \
            [C.c_double, C.c_double, C.c_int64, C.c_int64, D, D, C.POINTER(C.c_int64)]
        lib.phop_object_times.argtypes = [C.c_void_p, C.c_int64, D, D, D, D]
        lib.phop_propagate_device_objects.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                                      C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]
        lib.phop_set_option.argtypes = [C.c_void_p, C.c_char_p, C.c_double]
        lib.phop_last_stats.argtypes = [C.c_void_p, C.POINTER(PhopStats)]
        lib.paraHPOP_run.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.c_char_p]
        lib.paraHPOP_setLogLevel.argtypes = [C.c_int]
        lib.phop_fma_peak.argtypes = [C.c_int, D, D]
        lib.phop_nrlmsise00_density.argtypes = [C.c_int, C.c_int64, D, C.c_int, D]
        lib.phop_load_environment.argtypes = [C.c_char_p, C.POINTER(C.c_uint64), D]
        lib.phop_server_create.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.POINTER(C.c_void_p)]
        lib.phop_server_destroy.argtypes = [C.c_void_p]
        lib.phop_server_last_error.argtypes = [C.c_void_p]
        lib.phop_server_last_error.restype = C.c_char_p
        lib.phop_server_submit.argtypes = [C.c_void_p, C.c_int64] + [D] * 9 + [C.POINTER(C.c_int64)]
        lib.phop_server_step.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
        lib.phop_server_status.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_int)]
        lib.phop_server_take.argtypes = [C.c_void_p, C.c_int64, D, D, D, D]
        lib.phop_server_get_stats.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
        _lib = lib
    return _lib


class ServerStats(C.Structure):
    _fields_ = [("queued", C.c_int64), ("running", C.c_int64), ("done", C.c_int64), ("failed", C.c_int64),
                ("active_objects", C.c_int64), ("launches", C.c_int64), ("rounds", C.c_int64),
                ("object_steps", C.c_int64), ("busy_ms", C.c_double), ("lanes", C.c_int)]


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class PhopError(RuntimeError):
    pass


class Propagator:
    """One loaded configuration, resident on one GPU (``phop_create``)."""

    def __init__(self, config_path, device: int = 0, lanes: int | None = None, split: bool = False,
                 threads: int | None = None):
        lib = library()
        h = C.c_void_p()
        if lib.phop_create(str(config_path).encode(), device, C.byref(h)) != 0:
            raise PhopError(lib.phop_last_error(None).decode())
        self._h = h
        d, s, m = C.c_double(), C.c_double(), C.c_int64()
        lib.phop_run_parameters(h, C.byref(d), C.byref(s), C.byref(m))
        self.duration, self.step, self.max_steps = d.value, s.value, m.value
        if lanes is not None:
            self.set_option("lanes", lanes)
        if split:
            self.set_option("split", 1)
        if threads is not None:
            self.set_option("threads", threads)

    def set_option(self, key: str, value: float):
        if library().phop_set_option(self._h, key.encode(), float(value)) != 0:
            raise PhopError(library().phop_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            library().phop_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def propagate(self, epochs, states, mass, drag_area, srp_area, cd, cr, duration=None, step=None):
        """Propagate arrays of targets; returns (final_epochs, final_states)."""
        n = len(epochs)
        f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64))
        ep, st, ma, ad, asr, cdd, crr = map(f, (epochs, states, mass, drag_area, srp_area, cd, cr))
        st = st.reshape(n, 6)
        dur = None if duration is None else f(np.broadcast_to(duration, (n,)))
        stp = None if step is None else f(np.broadcast_to(step, (n,)))
        out_e = np.zeros(n)
        out_s = np.zeros((n, 6))
        rc = library().phop_propagate(self._h, n, _dp(ep), _dp(st), _dp(ma), _dp(ad), _dp(asr), _dp(cdd), _dp(crr),
                                      _dp(dur) if dur is not None else None, _dp(stp) if stp is not None else None,
                                      _dp(out_e), _dp(out_s))
        if rc != 0:
            raise PhopError(library().phop_last_error(self._h).decode())
        return out_e, out_s

    def propagate_targets(self, targets: dict, use_target_times=True):
        """Propagate a reference-schema targets document (dict)."""
        t = targets["targets"]
        g = lambda k: np.array([x[k] for x in t], dtype=np.float64)
        dur = step = None
        if use_target_times and any("duration_seconds" in x for x in t):
            dur = np.array([x.get("duration_seconds", self.duration) for x in t])
        if use_target_times and any("step_seconds" in x for x in t):
            step = np.array([x.get("step_seconds", self.step) for x in t])
        return self.propagate(g("epoch_mjd2000_tdb"), np.array([x["state_km_km_s"] for x in t]), g("mass_kg"),
                              g("drag_area_m2"), g("srp_area_m2"), g("cd"), g("cr"), dur, step)

    def propagate_device(self, d_state_ptr: int, n: int, epoch: float, mass, drag_area, srp_area, cd, cr,
                         duration: float, step: float) -> float:
        """Propagate an SoA state already in device memory (6*n doubles) in place."""
        f = lambda a: np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=np.float64), (n,)))
        ma, ad, asr, cdd, crr = map(f, (mass, drag_area, srp_area, cd, cr))
        out = C.c_double()
        rc = library().phop_propagate_device(self._h, n, C.c_void_p(d_state_ptr), epoch, _dp(ma), _dp(ad), _dp(asr),
                                             _dp(cdd), _dp(crr), duration, step, C.byref(out))
        if rc != 0:
            raise PhopError(library().phop_last_error(self._h).decode())
        return out.value

    def object_times(self, epochs, durations, steps) -> np.ndarray:
        """Per-object time arrays (4*n: current epoch, end epoch, current step
        size, nominal step; TDB seconds past J2000) for
        ``propagate_device_objects``."""
        f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64))
        ep, du, st = map(f, (epochs, durations, steps))
        n = len(ep)
        out = np.empty(4 * n)
        if library().phop_object_times(self._h, n, _dp(ep), _dp(du), _dp(st), _dp(out)) != 0:
            raise PhopError(library().phop_last_error(self._h).decode())
        return out

    def propagate_device_objects(self, n: int, d_state_ptr: int, d_time_ptr: int, d_bc_ptr: int, d_ams_ptr: int,
                                 max_steps: int) -> int:
        """Advance a resident uneven batch by at most ``max_steps`` steps per
        object (device pointers); returns the objects still short of their end."""
        left = C.c_int64()
        rc = library().phop_propagate_device_objects(self._h, n, C.c_void_p(d_state_ptr), C.c_void_p(d_time_ptr),
                                                     C.c_void_p(d_bc_ptr), C.c_void_p(d_ams_ptr), int(max_steps),
                                                     C.byref(left))
        if rc != 0:
            raise PhopError(library().phop_last_error(self._h).decode())
        return left.value

    @staticmethod
    def factors(mass, drag_area, srp_area, cd, cr):
        """Per-object drag and SRP factors (bc, ams) as the library forms them
        (driver.cpp:118-120, PrivateAccelerations.h:41-42): area in km^2,
        cr scaled by srp_area / drag_area."""
        area = np.asarray(drag_area, dtype=np.float64) * 1e-6
        crf = np.asarray(cr, dtype=np.float64) * np.asarray(srp_area, dtype=np.float64) / np.asarray(drag_area)
        return np.asarray(cd) * area / np.asarray(mass), crf * area / np.asarray(mass)

    def trajectory(self, epoch: float, states, mass, drag_area, srp_area, cd, cr, duration: float, step: float,
                   every: int = 1):
        """States of a batch with one epoch, duration and step after every
        ``every``-th fixed step: (epochs (records,), states (records, n, 6))."""
        st = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 6)
        n = len(st)
        f = lambda a: np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=np.float64), (n,)))
        ma, ad, asr, cdd, crr = map(f, (mass, drag_area, srp_area, cd, cr))
        steps = int(np.ceil(duration / step))
        cap = max(1, steps // every) if every > 0 else 1  # the library refuses every <= 0
        ep = np.empty(cap)
        out = np.empty((cap, n, 6))
        got = C.c_int64()
        rc = library().phop_propagate_trajectory(self._h, n, epoch, _dp(st), _dp(ma), _dp(ad), _dp(asr), _dp(cdd),
                                                 _dp(crr), duration, step, every, cap, _dp(ep), _dp(out),
                                                 C.byref(got))
        if rc != 0:
            raise PhopError(library().phop_last_error(self._h).decode())
        return ep[:got.value], out[:got.value]

    def stats(self) -> dict:
        s = PhopStats()
        library().phop_last_stats(self._h, C.byref(s))
        return {k: getattr(s, k) for k, _ in PhopStats._fields_}


class Server:
    """Serving loop over one Propagator (``phop_server_*``): queued requests
    are admitted into a device-resident pool of ``capacity`` objects and
    advanced together in slices of about ``slice_ms``."""

    QUEUED, RUNNING, DONE, FAILED = 0, 1, 2, 3

    def __init__(self, propagator: Propagator, capacity: int, slice_ms: float = 20.0):
        h = C.c_void_p()
        if library().phop_server_create(propagator._h, int(capacity), float(slice_ms), C.byref(h)) != 0:
            raise PhopError(library().phop_last_error(propagator._h).decode())
        self._h = h
        self._prop = propagator
        self._sizes = {}

    def _err(self):
        return PhopError(library().phop_server_last_error(self._h).decode())

    def submit(self, epochs, states, mass, drag_area, srp_area, cd, cr, duration=None, step=None) -> int:
        n = len(epochs)
        f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64))
        ep, st, ma, ad, asr, cdd, crr = map(f, (epochs, states, mass, drag_area, srp_area, cd, cr))
        st = st.reshape(n, 6)
        dur = None if duration is None else f(np.broadcast_to(duration, (n,)))
        stp = None if step is None else f(np.broadcast_to(step, (n,)))
        rid = C.c_int64()
        rc = library().phop_server_submit(self._h, n, _dp(ep), _dp(st), _dp(ma), _dp(ad), _dp(asr), _dp(cdd),
                                          _dp(crr), _dp(dur) if dur is not None else None,
                                          _dp(stp) if stp is not None else None, C.byref(rid))
        if rc != 0:
            raise self._err()
        self._sizes[rid.value] = n
        return rid.value

    def submit_targets(self, targets: dict) -> int:
        t = targets["targets"]
        g = lambda k: np.array([x[k] for x in t], dtype=np.float64)
        dur = np.array([x.get("duration_seconds", self._prop.duration) for x in t])
        step = np.array([x.get("step_seconds", self._prop.step) for x in t])
        return self.submit(g("epoch_mjd2000_tdb"), np.array([x["state_km_km_s"] for x in t]), g("mass_kg"),
                           g("drag_area_m2"), g("srp_area_m2"), g("cd"), g("cr"), dur, step)

    def step(self) -> int:
        f = C.c_int64()
        if library().phop_server_step(self._h, C.byref(f)) != 0:
            raise self._err()
        return f.value

    def status(self, rid: int) -> int:
        s = C.c_int()
        if library().phop_server_status(self._h, rid, C.byref(s)) != 0:
            raise self._err()
        return s.value

    def take(self, rid: int):
        """(final_epochs, final_states, latency_ms, queue_ms) of a finished request."""
        n = self._sizes.pop(rid)
        ep = np.zeros(n)
        st = np.zeros((n, 6))
        lat, q = C.c_double(), C.c_double()
        if library().phop_server_take(self._h, rid, _dp(ep), _dp(st), C.byref(lat), C.byref(q)) != 0:
            raise self._err()
        return ep, st, lat.value, q.value

    def run_until_idle(self, max_rounds: int = 10 ** 7):
        for _ in range(max_rounds):
            self.step()
            s = self.stats()
            if s["queued"] == 0 and s["running"] == 0:
                return
        raise PhopError("server did not become idle")

    def stats(self) -> dict:
        s = ServerStats()
        library().phop_server_get_stats(self._h, C.byref(s))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            library().phop_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fma_peak(device: int = 0) -> tuple[float, float]:
    """Measured (FP64, FP32) FMA throughput in TFLOP/s on `device`."""
    a, b = C.c_double(), C.c_double()
    if library().phop_fma_peak(device, C.byref(a), C.byref(b)) != 0:
        raise PhopError("FMA peak measurement failed")
    return a.value, b.value


def nrlmsise00_density(inputs, lanes: int = 4, device: int = 0) -> np.ndarray:
    """NRLMSISE-00 total mass density (kg/m^3) of input rows {doy, sec, alt,
    g_lat, g_long, lst, f107A, f107, ap, ap_a[0..6]} on the device, through
    the step kernel's per-object model split over `lanes` lanes."""
    a = np.ascontiguousarray(inputs, dtype=np.float64).reshape(-1, 16)
    out = np.empty(len(a))
    lib = library()
    if lib.phop_nrlmsise00_density(device, len(a), _dp(a), lanes, _dp(out)) != 0:
        raise PhopError(lib.phop_last_error(None).decode())
    return out


def load_environment(config) -> tuple:
    """Reads a configuration and its environment files on the host (no device
    needed), with the checks ``Propagator`` applies; returns (digest of
    everything loaded, load wall time in ms).  Raises PhopError with the
    loader's message."""
    digest = C.c_uint64(0)
    ms = C.c_double(0.0)
    lib = library()
    if lib.phop_load_environment(str(config).encode(), C.byref(digest), C.byref(ms)) != 0:
        raise PhopError(lib.phop_last_error(None).decode())
    return digest.value, ms.value


def run(config, targets, output, backend="device") -> int:
    """In-process equivalent of ``parahpop_gpu CONFIG TARGETS OUTPUT``."""
    argv = [b"parahpop_gpu", str(config).encode(), str(targets).encode(), str(output).encode()]
    arr = (C.c_char_p * len(argv))(*argv)
    return library().paraHPOP_run(len(argv), arr, backend.encode())


def run_cli(config, targets, output, env=None) -> subprocess.CompletedProcess:
    """Run the ``parahpop_gpu`` executable."""
    return subprocess.run([str(CLI_PATH), str(config), str(targets), str(output)], stdout=subprocess.PIPE,
                          stderr=subprocess.PIPE, text=True, env=env)
