"""C-ABI checks that need no GPU: exported symbols, parser, parameters, data files."""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


def header_symbols():
    text = "".join(h.read_text() for h in sorted((ROOT / "include").glob("*.h")))
    return sorted(set(re.findall(r"\b(lcb_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(lcb):
    L = lcb._capi.load()
    syms = header_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(lcb._capi.SYMBOLS)


def header_prototypes():
    """name -> (return type, parameter count) of every lcb_* prototype in include/*.h."""
    text = "".join(h.read_text() for h in sorted((ROOT / "include").glob("*.h")))
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    out = {}
    for m in re.finditer(r"(const\s+char\s*\*|void|int)\s+(lcb_[a-z_0-9]+)\s*\(([^;{]*?)\)\s*;", text):
        params = " ".join(m.group(3).split())
        n = 0 if params in ("", "void") else params.count(",") + 1
        out[m.group(2)] = (" ".join(m.group(1).split()), n)
    return out


def test_ctypes_signatures_match_the_headers(lcb):
    """Every declared function has as many ctypes argument types as the C
    prototype has parameters, and the matching return type."""
    L = lcb._capi.load()
    protos = header_prototypes()
    assert set(protos) == set(header_symbols())
    want_res = {"int": C.c_int, "void": None, "const char *": C.c_char_p, "const char*": C.c_char_p}
    for name, (ret, n) in protos.items():
        f = getattr(L, name)
        assert f.argtypes is not None and len(f.argtypes) == n, (name, n, f.argtypes)
        assert f.restype is want_res[ret], (name, ret, f.restype)


def test_version_and_errors(lcb):
    L = lcb._capi.load()
    assert b"sm_100a" in L.lcb_version()
    h = C.c_void_p()
    rc = L.lcb_model_load(b"/nonexistent/model.dat", C.byref(h))
    assert rc == 3 and b"cannot open" in L.lcb_last_error()


def test_model_parse_matches_oracle(lcb, oracle, test_model_path):
    m = lcb.Model(test_model_path)
    o = oracle.Model(test_model_path)
    i = 0
    while True:
        n = lcb._capi.load().lcb_param_name(i)
        if n is None:
            break
        name = n.decode()
        assert m.get_param(name) == o.get(name), name
        i += 1
    assert i == 77
    assert m.get_comp("nlat2f") == "40" and m.get_comp("limb1") == "Poly"
    assert m.get_comp("delta_phase") == "0.0000001"
    p = m.get_pparam("pdot")  # optional, defaulted (model.rs:262-271)
    assert p["value"] == 0.0 and p["defined"] is False


def test_model_errors_mirror_reference(lcb):
    text = (GOLDEN / "test_model.dat").read_text()
    for bad in (text + "\nbogus = 1\n",
                text.replace("limb1                = Poly", "limb1 = Linear"),
                text + "\nstsp11_long = 10 1 1 0\n",
                text.replace("glens1               = 0", "glens1 = 1").replace("roche1               = 0", "roche1 = 1"),
                text.replace("nlat1f               = 20", "nlat1f = 2.5"),
                text.replace("q                    = 0.5 0.1 0.01 0", "q = 0.5 0.1")):
        with pytest.raises(lcb.LcbError) as e:
            lcb.Model(text=bad)
        assert e.value.code == 2
    # comment stripping with an escaped hash (model.rs:299-309)
    m = lcb.Model(text=text.replace("q                    = 0.5 0.1 0.01 0", "q = 0.25 0.1 0.01 0 # mass ratio"))
    assert m.q == 0.25


def test_set_get_and_unknown_param(lcb, test_model_path):
    m = lcb.Model(test_model_path)
    m.set_param("iangle", 85.5)
    assert m.get_param("iangle") == 85.5 and m.iangle == 85.5
    m.q = 0.42
    assert m.get_pparam("q")["range"] == 0.1
    with pytest.raises(ValueError):
        m.set_param("nonexistent", 1.0)
    with pytest.raises(ValueError):
        m.get_param("")
    c = m.copy()
    c.q = 0.1
    assert m.q == 0.42
    m.set_comp("nlat1f", "33")
    assert m.get_comp("nlat1f") == "33"
    with pytest.raises(lcb.LcbError):
        m.set_comp("roche1", "1") if m.get_comp("glens1") == "1" else m.set_comp("nonexistent", "1")


def test_read_data_rules(lcb, tmp_path):
    p = tmp_path / "d.dat"
    p.write_text("# comment\n\n0.1 0.01 1.5 0.2 1 3\n0.2 0.01 1.6 -0.3 2 1\nshort line 1\n")
    d = lcb.read_data(p)
    assert d.shape == (2,)
    assert d["ndiv"].tolist() == [3, 1]
    # ferr < 0 -> |ferr| and weight 0 (types.rs:247-250)
    assert d["ferr"][1] == 0.3 and d["weight"][1] == 0.0
    p.write_text("0.1 0.01 x 0.2 1 3\n")
    with pytest.raises(lcb.LcbError):
        lcb.read_data(p)


def test_cpu_only_device_choice_fails_loudly(lcb):
    with pytest.raises(ValueError):
        lcb.set_device("cpu")
    lcb.set_device("cuda:0")
    assert lcb.get_device() == "cuda:0"
