"""The reference's own CUDA flux kernel, run on this GPU as a comparator.

TEST INFRASTRUCTURE ONLY (imported by tests/, never by the product package).

crates/lcurve-cuda/kernels/flux_kernel.cu of the reference is compiled
unmodified for sm_100a into oracle/_ref/libref_flux.so by `make -C oracle ref
REF_ROOT=...` (the reference's build.rs stops at sm_90 and ships no PTX, so
as shipped it has no B200 image).  This module feeds it what the reference's
Rust host code prepares for it (crates/lcurve-cuda/src/batch.rs:390-500,
transfer.rs:1-160):

  * the grids, flattened to GpuPoint: f32 normal, position and flux, at most
    MAX_ECL = 3 eclipse pairs in f32 (transfer.rs:5, 138-141) -- here the
    oracle's grids, the restatement of the reference's CPU grid code;
  * GpuFluxParams: iangle.to_radians() cos/sin, q/(1+q), velocity factor,
    limb darkening, beaming, spins, disc limb darkening, lensing radius,
    ginterp phases and scale factors, grid sizes;
  * per datum the phase (4 Newton steps of the quadratic ephemeris + Roemer
    term), exposure in phase units and ndiv; per datum slfac and third;

and runs lcuda_flux_eval_stream (one block of 256 threads per datum) through
the reference's C ABI.  Its known defects (f32 phases, 3 eclipse pairs) make
it a timing comparator, not a parity reference: the reference's own GPU test
allows 1e-3 (crates/lcurve-cuda/tests/gpu_correctness.rs:90-94, 110-114).
"""
from __future__ import annotations

import ctypes as C
import math
import pathlib

import numpy as np

from . import oracle as O

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libref_flux.so"

MAX_ECL = 3
GPU_POINT = np.dtype([("dirn", "<f4", 3), ("posn", "<f4", 3), ("flux", "<f4"), ("n_ecl", "<i4"),
                      ("ecl_ing", "<f4", MAX_ECL), ("ecl_eg", "<f4", MAX_ECL)])
GPU_PARAMS = np.dtype([
    ("cosi", "<f8"), ("sini", "<f8"), ("xcofm", "<f8"), ("vfac", "<f8"),
    ("ldc1", "<f8", 4), ("mucrit1", "<f8"), ("ltype1", "<i4"),
    ("ldc2", "<f8", 4), ("mucrit2", "<f8"), ("ltype2", "<i4"),
    ("beam_factor1", "<f8"), ("beam_factor2", "<f8"), ("spin1", "<f8"), ("spin2", "<f8"),
    ("lin_limb_disc", "<f8"), ("quad_limb_disc", "<f8"),
    ("has_glens", "<i4"), ("rlens1", "<f8"),
    ("gint", "<f8", 6),
    ("n", "<i4", 7), ("_pad", "<i4", 1)], align=True)
GPU_DATUM = np.dtype([("phase", "<f8"), ("expose", "<f8"), ("flux_obs", "<f8"), ("ferr", "<f8"),
                      ("weight", "<f8"), ("ndiv", "<i4"), ("_pad", "<i4")])
GPU_FUDGE = np.dtype([("slfac", "<f8"), ("third", "<f8")])
assert GPU_POINT.itemsize == 56 and GPU_PARAMS.itemsize == 272 and GPU_DATUM.itemsize == 48
GRID_ORDER = ("star1f", "star1c", "star2f", "star2c", "disc", "edge", "spot")  # flux_kernel.cu:397-403
C_LIGHT = 2.99792458e8

_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(str(LIB_PATH))
        vp, sz = C.c_void_p, C.c_size_t
        L.lcuda_malloc.argtypes = [C.POINTER(vp), sz]
        L.lcuda_free.argtypes = [vp]
        L.lcuda_memcpy_h2d.argtypes = [vp, vp, sz]
        L.lcuda_memcpy_d2h.argtypes = [vp, vp, sz]
        L.lcuda_flux_eval_stream.argtypes = [vp, vp, vp, vp, vp, C.c_int, vp]
        L.lcuda_stream_sync.argtypes = [vp]
        _lib = L
    return _lib


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: cudaError {rc}")


def model_values(text: str) -> dict:
    """The first value of every `name = value ...` line of a model file."""
    out = {}
    for line in text.splitlines():
        if "=" not in line or line.lstrip().startswith("#"):
            continue
        k, v = line.split("=", 1)
        out[k.strip()] = v.split()[0]
    return out


def flatten(g: dict) -> np.ndarray:
    """transfer.rs:132-160 flatten_points: f32 fields, the first MAX_ECL pairs."""
    n = g["posn"].shape[0]
    p = np.zeros(n, dtype=GPU_POINT)
    p["dirn"] = g["dirn"].astype(np.float32)
    p["posn"] = g["posn"].astype(np.float32)
    p["flux"] = g["flux"]
    k = np.minimum(g["necl"], MAX_ECL)
    p["n_ecl"] = k
    for j in range(MAX_ECL):
        use = k > j
        p["ecl_ing"][use, j] = g["ecl"][use, 2 * j].astype(np.float32)
        p["ecl_eg"][use, j] = g["ecl"][use, 2 * j + 1].astype(np.float32)
    return p


def prepare(text: str, times, expose, ndiv, grids: "O.Grids") -> tuple:
    """(points, params, data, fudge) as batch.rs:390-500 builds them."""
    v = model_values(text)
    f = lambda k: float(v[k])  # noqa: E731
    g = {name: grids.fetch(name) for name in GRID_ORDER}
    info = grids.info()
    pts = np.concatenate([flatten(g[name]) for name in GRID_ORDER])
    ri = f("iangle") * (math.pi / 180.0)
    P = np.zeros(1, dtype=GPU_PARAMS)
    P["cosi"], P["sini"] = math.cos(ri), math.sin(ri)
    P["xcofm"] = f("q") / (1.0 + f("q"))
    P["vfac"] = f("velocity_scale") / (C_LIGHT / 1e3)
    P["ldc1"] = [f(f"ldc1_{k}") for k in range(1, 5)]
    P["ldc2"] = [f(f"ldc2_{k}") for k in range(1, 5)]
    P["mucrit1"], P["mucrit2"] = f("mucrit1"), f("mucrit2")
    P["ltype1"] = 0 if v["limb1"] == "Poly" else 1
    P["ltype2"] = 0 if v["limb2"] == "Poly" else 1
    P["beam_factor1"], P["beam_factor2"] = f("beam_factor1"), f("beam_factor2")
    P["spin1"], P["spin2"] = f("spin1"), f("spin2")
    P["lin_limb_disc"], P["quad_limb_disc"] = f("lin_limb_disc"), f("quad_limb_disc")
    P["has_glens"] = int(v.get("glens1", "0") in ("1", "true"))
    P["rlens1"] = info["rlens1"]
    P["gint"] = [info[k] for k in ("phase1", "phase2", "scale11", "scale12", "scale21", "scale22")]
    P["n"] = [g[name]["posn"].shape[0] for name in GRID_ORDER]
    t = np.asarray(times, dtype=np.float64)
    t0, period, pdot, deltat = f("t0"), f("period"), float(v.get("pdot", 0.0)), f("deltat")
    phase = (t - t0) / period
    for _ in range(4):
        phase -= (t0 + phase * (period + pdot * phase) - t) / (period + 2.0 * pdot * phase)
    phase += deltat / period / 2.0 * (np.cos(2.0 * math.pi * phase) - 1.0)
    D = np.zeros(t.size, dtype=GPU_DATUM)
    D["phase"], D["expose"], D["ndiv"], D["ferr"], D["weight"] = phase, expose / period, ndiv, 1.0, 1.0
    middle, rng = (t.min() + t.max()) / 2.0, (t.max() - t.min()) / 2.0
    frac = (t - middle) / rng if rng > 0 else np.zeros_like(t)
    Fd = np.zeros(t.size, dtype=GPU_FUDGE)
    Fd["slfac"] = 1.0 + frac * (f("slope") + frac * (f("quad") + frac * f("cube")))
    Fd["third"] = f("third")
    return pts, P, D, Fd


class Run:
    """Device copies of one prepared model; run(stream) launches the reference kernel."""

    def __init__(self, pts, params, data, fudge):
        L = lib()
        self.n = data.size
        self.bufs = []
        for a in (data, fudge, pts, params, np.zeros(self.n)):
            p = C.c_void_p()
            _check(L.lcuda_malloc(C.byref(p), max(a.nbytes, 16)), "lcuda_malloc")
            _check(L.lcuda_memcpy_h2d(p, a.ctypes.data, a.nbytes), "lcuda_memcpy_h2d")
            self.bufs.append(p)

    def launch(self, stream: int = 0) -> None:
        d, fu, pt, pa, out = self.bufs
        _check(lib().lcuda_flux_eval_stream(d, fu, pt, pa, out, self.n, C.c_void_p(stream)), "lcuda_flux_eval_stream")

    def result(self) -> np.ndarray:
        out = np.zeros(self.n)
        _check(lib().lcuda_memcpy_d2h(out.ctypes.data, self.bufs[4], out.nbytes), "lcuda_memcpy_d2h")
        return out

    def free(self) -> None:
        for p in self.bufs:
            lib().lcuda_free(p)
        self.bufs = []
