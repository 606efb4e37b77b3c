"""lcurve-b200 — B200 light-curve engine with the Python interface of lcurve_rs.

Mirrors the reference's Python module (python/src/lib.rs, python/lcurve_rs/
__init__.py): ``Model(path)``, ``Model.light_curve(...)``,
``Model.chisq_batch(data, names, values, scale)``, ``LcResult``,
``set_device`` / ``get_device`` / ``has_cuda``.  Every computation runs
through liblcurve_b200.so on a CUDA device (sm_100a); there is no CPU path,
so ``set_device("cpu")`` raises instead of silently running elsewhere.

Example
-------
>>> import importlib; lc = importlib.import_module("lcurve-rs_b200")
>>> m = lc.Model("model.dat")
>>> r = m.light_curve(time1=-0.2, time2=1.2, ntime=1000)
>>> r.flux
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

from . import _capi
from ._capi import DATUM_DTYPE, LcbError, Result, check, dptr, i64ptr

__all__ = ["Model", "LcResult", "Batch", "set_device", "get_device", "has_cuda", "read_data", "make_data",
           "chisq_batch_ragged", "LcbError", "DATUM_DTYPE"]
__version__ = "0.1.0"

_state = threading.local()
_ctx_lock = threading.Lock()
_contexts: dict[int, C.c_void_p] = {}
_device = 0


def _parse_device(device: str) -> int:  # python/src/lib.rs:30-50
    s = device.strip().lower()
    if s in ("cuda", "gpu"):
        return 0
    if s.startswith("cuda:"):
        try:
            i = int(s[5:])
        except ValueError:
            raise ValueError(f"invalid device id: '{s[5:]}'") from None
        if i < 0:
            raise ValueError(f"device id must be >= 0, got {i}")
        return i
    if s == "cpu":
        raise ValueError("this engine has no CPU path: use 'cuda' or 'cuda:N'")
    raise ValueError(f"unknown device '{s}': expected 'cuda' or 'cuda:N'")


def set_device(device: str = "cuda") -> None:
    """Select the CUDA device ('cuda' or 'cuda:N')."""
    global _device
    _device = _parse_device(device)


def get_device() -> str:
    return f"cuda:{_device}"


def has_cuda() -> bool:
    """True if the library loads and sees at least one CUDA device."""
    try:
        n = C.c_int(0)
        return _capi.load().lcb_device_count(C.byref(n)) == 0 and n.value > 0
    except (ImportError, OSError):
        return False


def _ctx() -> C.c_void_p:
    L = _capi.load()
    with _ctx_lock:
        h = _contexts.get(_device)
        if h is None:
            h = C.c_void_p()
            check(L.lcb_ctx_create(_device, C.byref(h)))
            _contexts[_device] = h
        return h


def transfer_bytes() -> tuple[int, int]:
    """(host->device, device->host) bytes of the last call on the current device's context."""
    h, d = C.c_int64(), C.c_int64()
    check(_capi.load().lcb_ctx_transfer_bytes(_ctx(), C.byref(h), C.byref(d)))
    return h.value, d.value


def fma_peak_tflops(fp64: bool) -> float:
    """Measured FMA throughput of the current device (TFLOP/s)."""
    v = C.c_double()
    check(_capi.load().lcb_measure_fma_peak(_ctx(), int(bool(fp64)), C.byref(v)))
    return v.value


def set_stream(cuda_stream: int) -> None:
    """Issue this device's work on an existing cudaStream_t (e.g. a torch stream's cuda_stream)."""
    check(_capi.load().lcb_ctx_set_stream(_ctx(), C.c_void_p(cuda_stream)))


def make_data(times, expose=0.001, ndiv=1, flux=0.0, ferr=1.0, weight=1.0) -> np.ndarray:
    """Structured array of lcb_datum records."""
    times = np.atleast_1d(np.asarray(times, dtype=np.float64))
    d = np.zeros(times.shape[0], dtype=DATUM_DTYPE)
    d["time"] = times
    d["expose"] = expose
    d["flux"] = flux
    d["ferr"] = ferr
    d["weight"] = weight
    d["ndiv"] = ndiv
    return d


def read_data(path: str | os.PathLike) -> np.ndarray:
    """Read an lcurve data file (crates/lcurve/src/types.rs:229-254)."""
    L = _capi.load()
    p = C.c_void_p()
    n = C.c_int64()
    check(L.lcb_read_data(str(path).encode(), C.byref(p), C.byref(n)))
    try:
        buf = (C.c_char * (n.value * DATUM_DTYPE.itemsize)).from_address(p.value) if n.value else b""
        return np.frombuffer(bytes(buf), dtype=DATUM_DTYPE).copy()
    finally:
        L.lcb_free_data(p)


class LcResult:
    """Result of a light curve computation (python/src/lib.rs:63-117)."""

    def __init__(self, times, calc, res: Result):
        self._times = np.asarray(times, dtype=np.float64)
        self._calc = np.asarray(calc, dtype=np.float64)
        self.wdwarf = res.wdwarf
        self.chisq = res.chisq
        self.wnok = res.wnok
        self.logg1 = res.logg1
        self.logg2 = res.logg2
        self.rv1 = res.rv1
        self.rv2 = res.rv2
        self._sfac = np.array(list(res.sfac))

    @property
    def calc(self) -> np.ndarray:
        return self._calc.copy()

    @property
    def flux(self) -> np.ndarray:
        return self._calc.copy()

    @property
    def times(self) -> np.ndarray:
        return self._times.copy()

    @property
    def sfac(self) -> np.ndarray:
        return self._sfac.copy()

    def __repr__(self):
        return (f"LcResult(npoints={self._calc.size}, wdwarf={self.wdwarf:.6e}, chisq={self.chisq:.4f}, "
                f"logg1={self.logg1:.4f}, logg2={self.logg2:.4f})")


class Model:
    """An lcurve model (crates/lcurve/src/model.rs) evaluated on the GPU."""

    def __init__(self, path: str | os.PathLike | None = None, *, text: str | None = None, _handle=None):
        L = _capi.load()
        self._h = C.c_void_p()
        if _handle is not None:
            self._h = _handle
        elif text is not None:
            check(L.lcb_model_parse(text.encode(), C.byref(self._h)))
        else:
            try:
                check(L.lcb_model_load(str(path).encode(), C.byref(self._h)))
            except LcbError as e:
                raise ValueError(str(e)) from None

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(_capi, "_lib", None) if _capi is not None else None  # None at interpreter exit
        if h and lib is not None:
            lib.lcb_model_destroy(h)
            self._h = None

    # ---- parameters (python/src/lib.rs:263-421)
    def get_param(self, name: str) -> float:
        v = C.c_double()
        rc = _capi.load().lcb_model_get_param(self._h, name.encode(), C.byref(v))
        if rc != 0:
            raise ValueError(f"unknown parameter: '{name}'")
        return v.value

    def set_param(self, name: str, value: float) -> None:
        rc = _capi.load().lcb_model_set_param(self._h, name.encode(), float(value))
        if rc != 0:
            raise ValueError(f"unknown parameter: '{name}'")

    def get_pparam(self, name: str) -> dict:
        v, r, s = C.c_double(), C.c_double(), C.c_double()
        vary, defined = C.c_int(), C.c_int()
        rc = _capi.load().lcb_model_get_pparam(self._h, name.encode(), C.byref(v), C.byref(r), C.byref(s),
                                               C.byref(vary), C.byref(defined))
        if rc != 0:
            raise ValueError(f"unknown parameter: '{name}'")
        return {"value": v.value, "range": r.value, "dstep": s.value, "vary": bool(vary.value),
                "defined": bool(defined.value)}

    def set_pparam(self, name: str, *, value=None, range=None, dstep=None, vary=None) -> None:
        def opt(x, ct):
            return C.byref(ct(x)) if x is not None else None
        rc = _capi.load().lcb_model_set_pparam(self._h, name.encode(), opt(value, C.c_double), opt(range, C.c_double),
                                               opt(dstep, C.c_double),
                                               opt(None if vary is None else int(bool(vary)), C.c_int))
        if rc != 0:
            raise ValueError(f"unknown parameter: '{name}'")

    def get_free_params(self) -> list:
        out = []
        L = _capi.load()
        i = 0
        while True:
            n = L.lcb_param_name(i)
            if n is None:
                break
            p = self.get_pparam(n.decode())
            if p["vary"] and p["defined"]:
                out.append({"name": n.decode(), "value": p["value"], "range": p["range"], "dstep": p["dstep"]})
            i += 1
        return out

    def set_params(self, names, values) -> None:
        if len(names) != len(values):
            raise ValueError(f"names and values must have same length ({len(names)} vs {len(values)})")
        for n, v in zip(names, values):
            self.set_param(n, v)

    def set_comp(self, name: str, value) -> None:
        """Set a computational parameter (nlat1f, delta_phase, limb1, ...) from its .dat text."""
        check(_capi.load().lcb_model_set_comp(self._h, name.encode(), str(value).encode()))

    def get_comp(self, name: str) -> str:
        buf = C.create_string_buffer(64)
        check(_capi.load().lcb_model_get_comp(self._h, name.encode(), buf, 64))
        return buf.value.decode()

    def copy(self) -> "Model":
        h = C.c_void_p()
        check(_capi.load().lcb_model_clone(self._h, C.byref(h)))
        return Model(_handle=h)

    for _n in ("q", "iangle", "r1", "r2", "t1", "t2", "period", "t0", "velocity_scale"):
        locals()[_n] = property(lambda self, n=_n: self.get_param(n),
                                lambda self, v, n=_n: self.set_param(n, v))
    del _n

    # ---- evaluation
    def light_curve(self, *, time1=-0.2, time2=1.2, ntime=500, times=None, expose=0.001, ndiv=1, data=None,
                    scale=False) -> LcResult:
        """Light curve (python/src/lib.rs:617-682; orchestration.rs:36-318)."""
        if data is not None:
            d = data if isinstance(data, np.ndarray) else read_data(data)
            rdata = True
        elif times is not None:
            d = make_data(np.ascontiguousarray(times, dtype=np.float64), expose=expose, ndiv=ndiv, ferr=1.0,
                          weight=0.0)
            rdata = False
        else:
            if ntime == 0:
                raise ValueError("ntime must be > 0")
            if ntime == 1:
                t = np.array([(time1 + time2) / 2.0])
            else:
                t = time1 + (time2 - time1) * np.arange(ntime, dtype=np.float64) / (ntime - 1)
            d = make_data(t, expose=expose, ndiv=ndiv, ferr=1.0, weight=0.0)
            rdata = False
        d = np.ascontiguousarray(d, dtype=DATUM_DTYPE)
        calc = np.zeros(d.shape[0])
        res = Result()
        try:
            check(_capi.load().lcb_light_curve(_ctx(), self._h, d.ctypes.data, d.shape[0], int(bool(scale)),
                                               int(rdata), dptr(calc), C.byref(res)))
        except LcbError as e:
            if e.code in (2, 3, 4, 8):
                raise ValueError(str(e)) from None
            raise
        return LcResult(d["time"], calc, res)

    def chisq_batch(self, data, names, values, scale=True) -> np.ndarray:
        """Chi-squared for N parameter sets (python/src/lib.rs:696-734; orchestration.rs:329-357)."""
        d = data if isinstance(data, np.ndarray) else read_data(data)
        d = np.ascontiguousarray(d, dtype=DATUM_DTYPE)
        values = np.ascontiguousarray(np.atleast_2d(np.asarray(values, dtype=np.float64)))
        nsets, ncols = values.shape
        if ncols != len(names):
            raise ValueError(f"values has {ncols} columns but {len(names)} names were given")
        arr = (C.c_char_p * len(names))(*[n.encode() for n in names])
        out = np.zeros(nsets)
        check(_capi.load().lcb_chisq_batch(_ctx(), self._h, d.ctypes.data, d.shape[0], arr, len(names),
                                           dptr(values), nsets, int(bool(scale)), dptr(out)))
        return out

    GRIDS = {"star1f": 0, "star2f": 1, "star1c": 2, "star2c": 3, "disc": 4, "edge": 5, "spot": 6}

    def grid(self, which: str) -> dict:
        """Elements of one grid as built on the GPU (posn, dirn, area, gravity, flux, ecl pairs)."""
        L = _capi.load()
        w = self.GRIDS[which]
        n = C.c_int64()
        check(L.lcb_model_grid(_ctx(), self._h, w, C.byref(n), None, None, None, None, None, None))
        k = n.value
        posn, dirn, ecl = np.zeros((k, 3)), np.zeros((k, 3)), np.zeros((k, 8))
        area, grav, flux = np.zeros(k, np.float32), np.zeros(k, np.float32), np.zeros(k, np.float32)
        fp = C.POINTER(C.c_float)
        if k:
            check(L.lcb_model_grid(_ctx(), self._h, w, C.byref(n), dptr(posn), dptr(dirn), area.ctypes.data_as(fp),
                                   grav.ctypes.data_as(fp), flux.ctypes.data_as(fp), dptr(ecl)))
        return dict(posn=posn, dirn=dirn, area=area, gravity=grav, flux=flux, ecl=ecl)

    def __repr__(self):
        return (f"Model(q={self.q}, iangle={self.iangle}, r1={self.r1}, r2={self.r2}, t1={self.t1}, "
                f"t2={self.t2})")


def chisq_batch_ragged(models, data: np.ndarray, offsets, scale=False, want_calc=False):
    """Ragged batch: model i on data[offsets[i]:offsets[i+1]]. Returns (chisq, calc or None, results)."""
    data = np.ascontiguousarray(data, dtype=DATUM_DTYPE)
    offs = np.ascontiguousarray(offsets, dtype=np.int64)
    n = len(models)
    arr = (C.c_void_p * n)(*[m._h.value for m in models])
    chisq = np.zeros(n)
    calc = np.zeros(data.shape[0]) if want_calc else None
    res = (Result * n)()
    check(_capi.load().lcb_chisq_batch_ragged(_ctx(), arr, n, data.ctypes.data, i64ptr(offs), int(bool(scale)),
                                              dptr(chisq), dptr(calc) if want_calc else None, res))
    return chisq, calc, list(res)


class Batch:
    """A resident batch: data uploaded once, parameters updated per step, the
    launch sequence replayed as a CUDA graph (lcb_batch_* in lcurve_b200.h)."""

    def __init__(self, models, data: np.ndarray, offsets):
        self._data = np.ascontiguousarray(data, dtype=DATUM_DTYPE)
        self._offs = np.ascontiguousarray(offsets, dtype=np.int64)
        self.n = len(models)
        arr = (C.c_void_p * self.n)(*[m._h.value for m in models])
        self._h = C.c_void_p()
        check(_capi.load().lcb_batch_create(_ctx(), arr, self.n, self._data.ctypes.data, i64ptr(self._offs),
                                            C.byref(self._h)))

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(_capi, "_lib", None) if _capi is not None else None  # None at interpreter exit
        if h and lib is not None:
            lib.lcb_batch_destroy(h)
            self._h = None

    def set_params(self, names, values) -> None:
        values = np.ascontiguousarray(np.asarray(values, dtype=np.float64).reshape(self.n, len(names)))
        key = tuple(names)
        if getattr(self, "_names_key", None) != key:  # the C array of names, kept across calls
            self._names_key, self._names_arr = key, (C.c_char_p * len(names))(*[n.encode() for n in names])
        check(_capi.load().lcb_batch_set_params(self._h, self._names_arr, len(names), dptr(values)))

    def run(self, scale=False) -> None:
        check(_capi.load().lcb_batch_run(self._h, int(bool(scale))))

    def set_tuning(self, flux_chunks: int = 0, roche_split: int = 0, flux_blocks_per_sm: int = 0) -> None:
        """Launch-shape choices (lcb_batch_set_tuning); 0 = the planner's heuristic."""
        check(_capi.load().lcb_batch_set_tuning(self._h, int(flux_chunks), int(roche_split), int(flux_blocks_per_sm)))

    def tuning(self) -> dict:
        """The launch-shape choices in effect (lcb_batch_get_tuning)."""
        a = (C.c_int * 3)()
        check(_capi.load().lcb_batch_get_tuning(self._h, a))
        return dict(flux_chunks=a[0], roche_split=a[1], flux_blocks_per_sm=a[2])

    def search_counts(self) -> dict:
        a = np.zeros(5, dtype=np.int64)
        check(_capi.load().lcb_batch_search_counts(self._h, i64ptr(a)))
        return dict(pot_evals=int(a[0]), dpot_evals=int(a[1]), searches=int(a[2]), bound_nodes=int(a[3]),
                    proven_misses=int(a[4]))

    def profile(self, scale=False) -> dict:
        """Run once with direct launches and CUDA events between stages; returns stage_ms()."""
        check(_capi.load().lcb_batch_profile(self._h, int(bool(scale))))
        return self.stage_ms()

    def chisq(self) -> np.ndarray:
        """The last run's chi-squared per model (NaN for a failed model), without the
        other result fields."""
        out = np.empty(self.n)
        check(_capi.load().lcb_batch_results(self._h, dptr(out), None, None))
        return out

    def results(self, want_calc=False):
        chisq = np.zeros(self.n)
        calc = np.zeros(self._data.shape[0]) if want_calc else None
        res = (Result * self.n)()
        check(_capi.load().lcb_batch_results(self._h, dptr(chisq), dptr(calc) if want_calc else None, res))
        return chisq, calc, list(res)

    def stats(self) -> dict:
        a = np.zeros(8, dtype=np.int64)
        check(_capi.load().lcb_batch_stats(self._h, i64ptr(a)))
        return dict(models=int(a[0]), elements=int(a[1]), subphases=int(a[2]), element_evals=int(a[3]),
                    flux_units=int(a[4]), roche_elements=int(a[5]), pot_evals=int(a[6]), dpot_evals=int(a[7]))

    def stage_ms(self) -> dict:
        a = np.zeros(6)
        check(_capi.load().lcb_batch_stage_ms(self._h, dptr(a)))
        return dict(phase=a[0], elements=a[1], roche=a[2], aux=a[3], flux=a[4], epilogue=a[5])
