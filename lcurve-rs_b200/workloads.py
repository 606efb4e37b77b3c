"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset exists for this path; every input is generated here from a
base model in the reference's .dat format (the fields and values of the
reference's test_data/test_model.dat) plus per-workload overrides:

  single_small  500 times, Claret WD + Roche-filling secondary, 15,926 elements
  single_large  nlat 200/400 + opaque disc (nrad 200) + rim + bright spot,
                irradiation, 10,000 times x 5 exposure sub-divisions
  single_huge   nlat 400/800, disc nrad 1000 with rim, two star spots on star 2,
                lensing, 100,000 times x 11 sub-divisions
  batch_1024    1024 models, uniform q, iangle, r1, t1, t2 and per-model grid
                sizes and time counts; data = the single_small curve at each
                model's times + 1% Gaussian noise
"""
from __future__ import annotations

import numpy as np

BASE_MODEL = """\
q                    = 0.5 0.1 0.01 0
iangle               = 82.0 2.0 0.1 0
r1                   = 0.015 0.005 0.001 0
r2                   = -1 0.01 0.001 0
cphi3                = 0.015 0.001 0.001 0
cphi4                = 0.017 0.001 0.001 0
t1                   = 15000 500 100 0
t2                   = 3500 200 50 0
spin1                = 1 0.001 0.001 0
spin2                = 1 0.001 0.001 0
ldc1_1               = 0.4 0.01 0.01 0
ldc1_2               = 0.0 0.01 0.01 0
ldc1_3               = 0.0 0.01 0.01 0
ldc1_4               = 0.0 0.01 0.01 0
ldc2_1               = 0.6 0.01 0.01 0
ldc2_2               = 0.0 0.01 0.01 0
ldc2_3               = 0.0 0.01 0.01 0
ldc2_4               = 0.0 0.01 0.01 0
velocity_scale       = 0 1 1 0
beam_factor1         = 0 0.1 0.02 0
beam_factor2         = 0 0.1 0.002 0
deltat               = 0 0.001 0.001 0
t0                   = 0.0 0.0001 1e-05 0
period               = 1.0 1e-06 1e-06 0
gravity_dark1        = 0.25 0.0001 0.0001 0
gravity_dark2        = 0.08 0.0001 0.0001 0
absorb               = 0.5 0.001 0.001 0
slope                = 0 0.01 1e-05 0
quad                 = 0 0.01 1e-05 0
cube                 = 0 0.01 1e-05 0
third                = 0 0.01 1e-05 0
rdisc1               = 0.05 0.01 0.0001 0
rdisc2               = 0.35 0.01 0.02 0
height_disc          = 0.1 0.01 1e-05 0
beta_disc            = 1.5 0.01 1e-05 0
temp_disc            = 3000 50 40 0
texp_disc            = -1.8 0.2 0.001 0
lin_limb_disc        = 0.3 0.02 0.0001 0
quad_limb_disc       = 0 0.02 0.0001 0
radius_spot          = 0.35 0.005 0.01 0
length_spot          = 0.02 0.002 0.005 0
height_spot          = 0.05 0.005 1e-05 0
expon_spot           = 0 0.2 0.1 0
epow_spot            = 1 0.1 0.1 0
angle_spot           = 140 2 2 0
yaw_spot             = 0 2 2 0
temp_spot            = 15000 400 200 0
tilt_spot            = 90 5 2 0
cfrac_spot           = 0.2 0.02 0.008 0
delta_phase          = 1e-07
nlat1f               = 20
nlat2f               = 40
nlat1c               = 10
nlat2c               = 20
npole                = 0
nlatfill             = 0
nlngfill             = 0
lfudge               = 0.05
llo                  = 0
lhi                  = -50
phase1               = 0.05
phase2               = 0.45
wavelength           = 550
roche1               = 0
roche2               = 1
eclipse1             = 1
eclipse2             = 1
glens1               = 0
tperiod              = 0.15
gdark_bolom1         = 1
gdark_bolom2         = 1
mucrit1              = 0
mucrit2              = 0
limb1                = Poly
limb2                = Poly
use_radii            = 1
mirror               = 0
add_disc             = 0
nrad                 = 40
opaque               = 0
add_spot             = 0
nspot                = 100
iscale               = 0
"""


def model_text(**overrides) -> str:
    """BASE_MODEL with `key = value` overrides (physical values get the default
    range/step/vary fields; pass a full string to set them all)."""
    lines = BASE_MODEL.splitlines()
    keys = [ln.split("=")[0].strip() for ln in lines]
    for k, v in overrides.items():
        if isinstance(v, (int, float)) and k not in COMP_KEYS:
            v = f"{v!r} 0.01 0.001 0"
        entry = f"{k:<20} = {v}"
        if k in keys:
            lines[keys.index(k)] = entry
        else:
            lines.append(entry)
            keys.append(k)
    return "\n".join(lines) + "\n"


COMP_KEYS = {"delta_phase", "nlat1f", "nlat2f", "nlat1c", "nlat2c", "npole", "nlatfill", "nlngfill", "lfudge",
             "llo", "lhi", "phase1", "phase2", "wavelength", "roche1", "roche2", "eclipse1", "eclipse2", "glens1",
             "use_radii", "tperiod", "gdark_bolom1", "gdark_bolom2", "mucrit1", "mucrit2", "limb1", "limb2",
             "mirror", "add_disc", "nrad", "opaque", "add_spot", "nspot", "iscale"}

SMALL = dict(q=0.5, iangle=82.0, r1=0.015, r2=-1.0, roche1=0, roche2=1, t1=15000.0, t2=3500.0,
             limb1="Claret", ldc1_1=0.5, ldc1_2=-0.2, ldc1_3=0.3, ldc1_4=-0.1,
             limb2="Poly", ldc2_1=0.6, ldc2_2=0.0, ldc2_3=0.0, ldc2_4=0.0,
             gravity_dark1=0.08, gravity_dark2=0.08, nlat1f=50, nlat1c=50, nlat2f=100, nlat2c=100,
             add_disc=0, add_spot=0, absorb=0.0, period=1.0, t0=0.0)


def single_small():
    """500 times in [-0.2, 0.8], expose 0.001, ndiv 1."""
    return model_text(**SMALL), np.linspace(-0.2, 0.8, 500), 0.001, 1


def single_large(nlat1=200, nlat2=400, ntime=10000, nrad=200, nspot=100):
    o = dict(SMALL)
    o.update(nlat1f=nlat1, nlat1c=nlat1, nlat2f=nlat2, nlat2c=nlat2, add_disc=1, opaque=1, rdisc1=0.02,
             rdisc2=0.3, texp_disc=-0.75, nrad=nrad, add_spot=1, temp_spot=12000.0, length_spot=0.05,
             expon_spot=0.0, epow_spot=2.0, nspot=nspot, absorb=0.5)
    return model_text(**o), np.linspace(-0.2, 1.2, ntime), 0.01, 5


def single_huge(nlat1=400, nlat2=800, ntime=100000, nrad=1000, seed=7):
    rng = np.random.default_rng(seed)
    o = dict(SMALL)
    o.update(nlat1f=nlat1, nlat1c=nlat1, nlat2f=nlat2, nlat2c=nlat2, add_disc=1, opaque=1, rdisc1=0.02,
             rdisc2=0.3, texp_disc=-0.75, nrad=nrad, absorb=0.5, glens1=1, velocity_scale=400.0, tperiod=0.1)
    for k, sign in (("21", 1.0), ("22", -1.0)):
        o[f"stsp{k}_long"] = float(rng.uniform(0.0, 360.0))
        o[f"stsp{k}_lat"] = float(rng.uniform(-90.0, 90.0))
        o[f"stsp{k}_fwhm"] = 10.0
        o[f"stsp{k}_tcen"] = 3500.0 + sign * 500.0
    return model_text(**o), np.linspace(-0.2, 1.2, ntime), 0.01, 11


def batch_models(n=1024, seed=1234, nlat1=(30, 300), nlat2=(30, 500), ntime=(200, 5000)):
    """Per-model (text, times) for the uneven batch; times uniform in [-0.2, 0.8]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        o = dict(SMALL)
        n1 = int(rng.integers(nlat1[0], nlat1[1] + 1))
        n2 = int(rng.integers(nlat2[0], nlat2[1] + 1))
        nt = int(rng.integers(ntime[0], ntime[1] + 1))
        o.update(q=float(rng.uniform(0.05, 1.0)), iangle=float(rng.uniform(75.0, 90.0)),
                 r1=float(rng.uniform(0.005, 0.03)), t1=float(rng.uniform(8000.0, 40000.0)),
                 t2=float(rng.uniform(2500.0, 5000.0)), nlat1f=n1, nlat1c=n1, nlat2f=n2, nlat2c=n2)
        out.append((model_text(**o), np.linspace(-0.2, 0.8, nt)))
    return out


def workload_key(specs) -> str:
    """SHA-1 of a batch's model texts and time grids (identifies a batch_models draw)."""
    import hashlib  # noqa: PLC0415
    h = hashlib.sha1()
    for text, t in specs:
        h.update(text.encode())
        h.update(np.ascontiguousarray(t, dtype=np.float64).tobytes())
    return h.hexdigest()


def batch_noise(fid_flux, seed):
    """The batch's observed fluxes and errors: the fiducial (single_small) curve
    at every model's times plus N(0, (0.01 flux)^2), from default_rng(seed + 99)."""
    rng = np.random.default_rng(seed + 99)
    fid_flux = np.asarray(fid_flux, dtype=np.float64)
    sig = 0.01 * np.abs(fid_flux)
    return fid_flux + sig * rng.standard_normal(fid_flux.shape), sig


def noisy_data(times, flux, expose, ndiv, seed, frac=0.01):
    """Data records: flux + N(0, (frac*flux)^2), ferr = frac*flux, weight 1."""
    from . import make_data  # noqa: PLC0415
    rng = np.random.default_rng(seed)
    flux = np.asarray(flux, dtype=np.float64)
    sig = frac * np.abs(flux)
    d = make_data(times, expose=expose, ndiv=ndiv, flux=flux + sig * rng.standard_normal(flux.shape), ferr=sig,
                  weight=1.0)
    return d


def roche_lobe_eggleton(q_donor: float) -> float:
    """Eggleton (1983) volume-equivalent Roche-lobe radius, in units of the
    separation, of a star of mass ratio q_donor = M_star / M_companion."""
    a, b = q_donor ** (2.0 / 3.0), q_donor ** (1.0 / 3.0)
    return 0.49 * a / (0.6 * a + np.log(1.0 + b))


SWEEP_KINDS = ("roche_secondary", "sphere_secondary", "eclipse_flags", "gravity_darkening", "limb_laws",
               "disc", "bright_spot", "disc_spot_gd", "edge")


def model_sweep(n=100, seed=42):
    """Seeded models across the path's physical options, for parity sweeps at
    small grids (the base model's nlat 20/40, disc nrad 40): Roche-filling and
    spherical secondaries, eclipse flags on and off, gravity darkening with
    bolometric or band exponents, polynomial and Claret limb darkening, discs
    (opaque or not), bright spots, and edge cases (low inclination, q = 1,
    negative t2, mirror irradiation, a Roche-distorted primary).  Returns
    [(kind, text)]."""
    rng = np.random.default_rng(seed)
    u = lambda lo, hi: float(rng.uniform(lo, hi))  # noqa: E731
    out = []
    for i in range(n):
        kind = SWEEP_KINDS[i * len(SWEEP_KINDS) // n]
        o = dict(q=u(0.1, 0.9), iangle=u(66.0, 88.0), r1=u(0.008, 0.035), t1=u(9000.0, 28000.0),
                 t2=u(2800.0, 5500.0))
        if kind == "roche_secondary":
            o["absorb"] = u(0.0, 1.0)
        elif kind == "sphere_secondary":
            o.update(roche2=0, r2=u(0.1, min(0.4, 0.9 * roche_lobe_eggleton(o["q"]))))
        elif kind == "eclipse_flags":
            o.update(eclipse1=i % 2, eclipse2=(i // 2) % 2)
        elif kind == "gravity_darkening":
            o.update(gravity_dark1=u(0.08, 0.32), gravity_dark2=u(0.08, 0.32), absorb=u(0.0, 1.0),
                     gdark_bolom1=int(rng.integers(0, 2)), gdark_bolom2=int(rng.integers(0, 2)))
        elif kind == "limb_laws":
            for s in ("1", "2"):
                o[f"limb{s}"] = "Claret" if rng.integers(0, 2) else "Poly"
                for k, (lo, hi) in enumerate(((0.1, 0.8), (-0.5, 0.5), (-0.3, 0.3), (-0.2, 0.2)), start=1):
                    o[f"ldc{s}_{k}"] = u(lo, hi)
        if kind in ("disc", "bright_spot", "disc_spot_gd"):
            rl1 = roche_lobe_eggleton(1.0 / o["q"])
            rdisc2 = u(0.2, min(0.45, 0.9 * rl1))
            o.update(add_disc=1, opaque=int(rng.integers(0, 2)), rdisc1=o["r1"] + u(0.01, 0.03), rdisc2=rdisc2,
                     height_disc=u(0.02, 0.15), beta_disc=u(1.0, 2.0), temp_disc=u(2000.0, 8000.0),
                     texp_disc=u(-2.5, -0.5), lin_limb_disc=u(0.1, 0.6), quad_limb_disc=u(-0.2, 0.3))
        if kind in ("bright_spot", "disc_spot_gd"):
            o.update(add_spot=1, radius_spot=o["rdisc2"] * u(0.8, 1.0), length_spot=u(0.01, 0.05),
                     height_spot=u(0.02, 0.1), expon_spot=u(0.0, 2.0), epow_spot=u(0.5, 2.0),
                     angle_spot=u(100.0, 180.0), yaw_spot=u(-20.0, 20.0), temp_spot=u(8000.0, 25000.0),
                     tilt_spot=u(60.0, 120.0), cfrac_spot=u(0.05, 0.5))
        if kind == "disc_spot_gd":
            o.update(gravity_dark1=u(0.08, 0.32), gravity_dark2=u(0.08, 0.32))
        if kind == "edge":
            case = i % 5
            if case == 0:
                o.update(iangle=30.0)                     # no eclipses
            elif case == 1:
                o.update(q=1.0, iangle=80.0, r1=0.01)     # equal masses
            elif case == 2:
                o.update(t2=-0.3, iangle=78.0)            # t2 < 0: the secondary's temperature by irradiation
            elif case == 3:
                o.update(q=0.4, iangle=82.0, mirror=1)    # mirror irradiation term
            else:
                o.update(q=0.6, iangle=80.0, r1=0.02, roche1=1)  # Roche-distorted primary
        out.append((kind, model_text(**o)))
    return out
