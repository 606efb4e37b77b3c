"""ctypes binding of the CPU oracle (oracle/liblcurve_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.  The oracle is an
FP64 restatement of the reference's CPU path; see lcurve_oracle.cpp for the
per-function citations of scope-ml/lcurve-rs.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "liblcurve_oracle.so"

# Datum layout shared with the product C ABI (lcb_datum): 5 doubles + 2 int32.
DATUM_DTYPE = np.dtype([("time", "<f8"), ("expose", "<f8"), ("flux", "<f8"), ("ferr", "<f8"),
                        ("weight", "<f8"), ("ndiv", "<i4"), ("pad", "<i4")])

GRID_NAMES = {"star1f": 0, "star2f": 1, "star1c": 2, "star2c": 3, "disc": 4, "edge": 5, "spot": 6}

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def host_cpu() -> str:
    """Model name of this host's CPU (/proc/cpuinfo)."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def use_native() -> str:
    """Switches this process to the oracle built for the host's own CPU
    (-O3 -march=native, no FMA contraction: the same results), building it on
    first use; the timed CPU baseline runs it.  Must come before the first
    lib() call.  Returns the library path."""
    global LIB_PATH
    if _lib is not None:
        raise RuntimeError("use_native() must be called before the oracle is loaded")
    import hashlib
    flags = ""
    try:
        flags = next((ln for ln in open("/proc/cpuinfo") if ln.startswith("flags")), "")
    except OSError:
        pass
    key = hashlib.sha1((host_cpu() + flags).encode()).hexdigest()[:12]
    so = HERE / "_native" / f"liblcurve_oracle_{key}.so"
    # make rebuilds it when the source is newer
    subprocess.run(["make", "-s", "-C", str(HERE), "native", f"NATIVE_SO=_native/{so.name}"], check=True)
    LIB_PATH = so
    return str(so)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        build()
    L = C.CDLL(str(LIB_PATH))
    vp, cp, dp, ip = C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.c_int
    L.orc_model_load.argtypes = [cp, C.POINTER(vp), cp, ip]
    L.orc_model_parse.argtypes = [cp, C.POINTER(vp), cp, ip]
    L.orc_model_free.argtypes = [vp]
    L.orc_model_clone.argtypes = [vp]
    L.orc_model_clone.restype = vp
    L.orc_model_set.argtypes = [vp, cp, C.c_double]
    L.orc_model_get.argtypes = [vp, cp, dp]
    L.orc_model_set_comp.argtypes = [vp, cp, C.c_double]
    L.orc_model_set_defined.argtypes = [vp, cp, ip]
    L.orc_light_curve.argtypes = [vp, vp, ip, ip, ip, ip, dp, dp, cp, ip]
    L.orc_chisq_batch.argtypes = [vp, vp, ip, C.POINTER(cp), ip, dp, ip, ip, ip, dp]
    L.orc_chisq_ragged.argtypes = [C.POINTER(vp), ip, vp, C.POINTER(C.c_int64), ip, ip, dp]
    L.orc_grids_build.argtypes = [vp, C.POINTER(vp), cp, ip]
    L.orc_grids_free.argtypes = [vp]
    L.orc_grids_count.argtypes = [vp, ip]
    L.orc_grids_count.restype = C.c_int64
    L.orc_grids_fetch.argtypes = [vp, ip, dp, dp, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                  C.POINTER(C.c_float), C.POINTER(C.c_int), dp]
    L.orc_grids_info.argtypes = [vp, dp]
    L.orc_grids_light_curve.argtypes = [vp, vp, vp, ip, ip, ip, ip, dp, dp, cp, ip]
    L.orc_set_grid_threads.argtypes = [ip]
    L.orc_grids_set.argtypes = [vp, ip, C.c_int64, dp, dp, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                C.POINTER(C.c_float), C.POINTER(C.c_int), dp]
    for f in ("orc_xl1",):
        getattr(L, f).argtypes = [C.c_double]
        getattr(L, f).restype = C.c_double
    for f in ("orc_xl11", "orc_xl12", "orc_planck", "orc_dlpdlt"):
        getattr(L, f).argtypes = [C.c_double, C.c_double]
        getattr(L, f).restype = C.c_double
    L.orc_numface.argtypes = [ip]
    L.orc_numface.restype = C.c_int64
    L.orc_stream_spot.argtypes = [C.c_double, C.c_double, dp]
    L.orc_svd_scale.argtypes = [dp, dp, dp, ip, dp, ip, dp]
    L.orc_rpot.argtypes = [C.c_double] * 4
    L.orc_rpot.restype = C.c_double
    L.orc_drpot1.argtypes = [C.c_double] * 5 + [dp]
    L.orc_set_earth.argtypes = [C.c_double, C.c_double, dp]
    L.orc_strinit.argtypes = [C.c_double, dp, dp]
    L.orc_gsint_step.argtypes = [C.c_double, C.c_double, C.c_double, dp, dp]
    L.orc_ref_sphere.argtypes = [C.c_double, ip, C.c_double, C.c_double, dp]
    L.orc_face.argtypes = [C.c_double, ip, C.c_double, C.c_double, dp, C.c_double, dp, dp, dp]
    L.orc_dbrent_quadratic.argtypes = [dp]
    L.orc_bsstep_exp.argtypes = [dp]
    L.orc_star_eclipse.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, dp,
                                   C.c_double, ip, ip, dp, dp]
    L.orc_counters.argtypes = [C.POINTER(C.c_longlong)]
    _lib = L
    return L


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class OracleError(RuntimeError):
    pass


def _lc_dict(calc, sc):
    keys = ["wdwarf", "chisq", "wnok", "logg1", "logg2", "rv1", "rv2"]
    out = {k: sc[i] for i, k in enumerate(keys)}
    out["sfac"] = sc[7:12].copy()
    out["calc"] = calc
    return out


def make_data(times, expose=0.001, ndiv=1, flux=0.0, ferr=1.0, weight=1.0) -> np.ndarray:
    times = np.asarray(times, dtype=np.float64)
    d = np.zeros(times.shape[0], dtype=DATUM_DTYPE)
    d["time"] = times
    d["expose"] = expose
    d["flux"] = flux
    d["ferr"] = ferr
    d["weight"] = weight
    d["ndiv"] = ndiv
    return d


class Model:
    """Oracle model handle (parsed from the reference's .dat format)."""

    def __init__(self, path: str | os.PathLike | None = None, *, text: str | None = None, _handle=None):
        L = lib()
        self._h = C.c_void_p()
        err = C.create_string_buffer(512)
        if _handle is not None:
            self._h = C.c_void_p(_handle)
        elif text is not None:
            if L.orc_model_parse(text.encode(), C.byref(self._h), err, 512) != 0:
                raise OracleError(err.value.decode())
        else:
            if L.orc_model_load(str(path).encode(), C.byref(self._h), err, 512) != 0:
                raise OracleError(err.value.decode())

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_model_free(self._h)
            self._h = None

    def clone(self) -> "Model":
        return Model(_handle=lib().orc_model_clone(self._h))

    def set(self, name: str, value: float) -> bool:
        return bool(lib().orc_model_set(self._h, name.encode(), float(value)))

    def get(self, name: str) -> float:
        v = C.c_double()
        if not lib().orc_model_get(self._h, name.encode(), C.byref(v)):
            raise KeyError(name)
        return v.value

    def set_comp(self, name: str, value) -> None:
        if not lib().orc_model_set_comp(self._h, name.encode(), float(value)):
            raise KeyError(name)

    def set_defined(self, name: str, defined: bool) -> None:
        if not lib().orc_model_set_defined(self._h, name.encode(), int(bool(defined))):
            raise KeyError(name)

    def light_curve(self, data: np.ndarray, scale=False, rdata=False, nthreads=1):
        data = np.ascontiguousarray(data, dtype=DATUM_DTYPE)
        n = data.shape[0]
        calc = np.zeros(n)
        sc = np.zeros(12)
        err = C.create_string_buffer(512)
        rc = lib().orc_light_curve(self._h, data.ctypes.data, n, int(scale), int(rdata), int(nthreads),
                                   _dp(calc), _dp(sc), err, 512)
        if rc != 0:
            raise OracleError(err.value.decode())
        return _lc_dict(calc, sc)

    def chisq_batch(self, data: np.ndarray, names, values, scale=False, nthreads=1) -> np.ndarray:
        data = np.ascontiguousarray(data, dtype=DATUM_DTYPE)
        values = np.ascontiguousarray(values, dtype=np.float64)
        ndim = len(names)
        nsets = values.size // ndim
        arr = (C.c_char_p * ndim)(*[n.encode() for n in names])
        out = np.zeros(nsets)
        lib().orc_chisq_batch(self._h, data.ctypes.data, data.shape[0], arr, ndim, _dp(values), nsets,
                              int(scale), int(nthreads), _dp(out))
        return out

    def grids(self):
        return self.built_grids().fetch_all()

    def built_grids(self, threads: int = 1) -> "Grids":
        """The model's grids (orchestration.rs:36-170), kept for fetching and for
        light curves on them.  threads > 1 computes the elements' eclipse
        intervals with that many threads (same values; for large grids)."""
        return Grids(self, threads)


class Grids:
    """Handle of the oracle's grids of one model (built once)."""

    def __init__(self, model: Model, threads: int = 1):
        self.model = model
        self._g = C.c_void_p()
        err = C.create_string_buffer(512)
        lib().orc_set_grid_threads(int(threads))
        try:
            rc = lib().orc_grids_build(model._h, C.byref(self._g), err, 512)
        finally:
            lib().orc_set_grid_threads(1)
        if rc != 0:
            raise OracleError(err.value.decode())

    def __del__(self):
        if getattr(self, "_g", None) and _lib is not None:
            _lib.orc_grids_free(self._g)
            self._g = None

    def fetch(self, name: str):
        g, w = self._g, GRID_NAMES[name]
        n = lib().orc_grids_count(g, w)
        posn = np.zeros((n, 3)); dirn = np.zeros((n, 3))
        area = np.zeros(n, np.float32); grav = np.zeros(n, np.float32); flux = np.zeros(n, np.float32)
        necl = np.zeros(n, np.int32); ecl = np.zeros((n, 8))
        lib().orc_grids_fetch(g, w, _dp(posn), _dp(dirn),
                              area.ctypes.data_as(C.POINTER(C.c_float)),
                              grav.ctypes.data_as(C.POINTER(C.c_float)),
                              flux.ctypes.data_as(C.POINTER(C.c_float)),
                              necl.ctypes.data_as(C.POINTER(C.c_int)), _dp(ecl))
        return dict(posn=posn, dirn=dirn, area=area, gravity=grav, flux=flux, necl=necl, ecl=ecl)

    def store(self, name: str, g: dict) -> None:
        """Replaces grid `name` with the arrays of `g` (the layout fetch returns)."""
        n = g["posn"].shape[0]
        fp = C.POINTER(C.c_float)
        arr = {k: np.ascontiguousarray(g[k]) for k in ("posn", "dirn", "ecl")}
        f32 = {k: np.ascontiguousarray(g[k], dtype=np.float32) for k in ("area", "gravity", "flux")}
        necl = np.ascontiguousarray(g["necl"], dtype=np.int32)
        if lib().orc_grids_set(self._g, GRID_NAMES[name], n, _dp(arr["posn"]), _dp(arr["dirn"]),
                               f32["area"].ctypes.data_as(fp), f32["gravity"].ctypes.data_as(fp),
                               f32["flux"].ctypes.data_as(fp), necl.ctypes.data_as(C.POINTER(C.c_int)),
                               _dp(arr["ecl"])) != 0:
            raise OracleError("bad grid name")

    def info(self):
        info = np.zeros(10)
        lib().orc_grids_info(self._g, _dp(info))
        return dict(phase1=info[0], phase2=info[1], scale11=info[2], scale12=info[3],
                    scale21=info[4], scale22=info[5], rlens1=info[6], bspot=info[7:10].copy())

    def fetch_all(self):
        out = {name: self.fetch(name) for name in GRID_NAMES}
        out["info"] = self.info()
        return out

    def light_curve(self, data: np.ndarray, scale=False, rdata=False, nthreads=1):
        """light_curve on these grids (the time loop onwards, orchestration.rs:171-318)."""
        data = np.ascontiguousarray(data, dtype=DATUM_DTYPE)
        n = data.shape[0]
        calc = np.zeros(n)
        sc = np.zeros(12)
        err = C.create_string_buffer(512)
        rc = lib().orc_grids_light_curve(self._g, self.model._h, data.ctypes.data, n, int(scale), int(rdata),
                                         int(nthreads), _dp(calc), _dp(sc), err, 512)
        if rc != 0:
            raise OracleError(err.value.decode())
        return _lc_dict(calc, sc)


def chisq_ragged(models, data: np.ndarray, offsets, scale=False, nthreads=1) -> np.ndarray:
    data = np.ascontiguousarray(data, dtype=DATUM_DTYPE)
    offs = np.ascontiguousarray(offsets, dtype=np.int64)
    arr = (C.c_void_p * len(models))(*[m._h.value for m in models])
    out = np.zeros(len(models))
    lib().orc_chisq_ragged(arr, len(models), data.ctypes.data, offs.ctypes.data_as(C.POINTER(C.c_int64)),
                           int(scale), int(nthreads), _dp(out))
    return out


def counters():
    a = (C.c_longlong * 3)()
    lib().orc_counters(a)
    return dict(fblink=a[0], rpot=a[1], drpot=a[2])


def counters_reset():
    lib().orc_counters_reset()
