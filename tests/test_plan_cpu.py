"""The host planner (lcb_plan.cpp: plan_batch) on CPU: the invariants every
device launch relies on, checked by a small driver compiled from the
library's host sources, on a batch that mixes the golden model, disc + rim +
bright-spot models, coarse/fine grids, exposure sub-divisions and one
physically invalid model (r2 = 0.99, orchestration.rs:350-354 -> NaN).

* segments: each model's elements are one contiguous range, in model order;
* data: per-datum model index and first sub-phase follow ndiv;
* flux units: every (element, sub-phase) pair of every planned model is in
  exactly one unit, units are ordered largest first, and slots are grouped
  by component (star 1, star 2, disc, rim, bright spot);
* element / Roche / aux blocks cover their segments;
* an invalid model is marked failed and owns no elements;
* re-planning into the same (reused) storage reproduces the plan exactly, and
  so does planning from four host threads at once (shared worker pool and
  bright-spot memo).

And the planner's FP64 helpers (L1 points, the bright-spot stream, grid
element counts) against the oracle's separate restatements.
"""
import shutil
import subprocess

import pytest

from conftest import GOLDEN, ROOT

DRIVER = r"""
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <thread>
#include <vector>
#include "lcb_plan.h"
using namespace lcb;
static int fails = 0;
#define CHECK(c, ...) do { if (!(c)) { ++fails; std::printf("FAIL " __VA_ARGS__); std::printf("\n"); } } while (0)
static int grp(int kind) { return kind == SEG_STAR1 ? 0 : kind == SEG_STAR2 ? 1 : kind == SEG_DISC ? 2 : kind == SEG_EDGE ? 3 : 4; }
template <class V> static bool same(const V& a, const V& b) {
    return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(a[0])) == 0);
}
int main(int argc, char** argv) {
    std::ifstream f(argv[1], std::ios::binary);
    std::string cur; int c; std::vector<Model> ms;
    while ((c = f.get()) != EOF) { if (c == 0x1e) { ms.push_back(parse_model_text(cur)); cur.clear(); } else cur += (char)c; }
    const int64_t n = (int64_t)ms.size();
    std::vector<const Model*> mp; for (auto& m : ms) mp.push_back(&m);
    std::vector<lcb_datum> data; std::vector<int64_t> st, cnt;
    for (int64_t i = 0; i < n; ++i) {
        st.push_back((int64_t)data.size());
        const int nt = 40 + (int)(i * 37 % 700);
        cnt.push_back(nt);
        for (int k = 0; k < nt; ++k) {
            lcb_datum d{}; d.time = -0.2 + 1.4 * k / (nt - 1); d.expose = 0.002; d.ferr = 0.01; d.weight = 1.0;
            d.ndiv = (k + (int)i) % 4 == 0 ? 3 : 1; data.push_back(d);
        }
    }
    PlanTuning tune;
    if (argc > 4) { tune.flux_chunks = std::atoi(argv[2]); tune.roche_split = std::atoi(argv[3]); tune.flux_blocks_per_sm = std::atoi(argv[4]); }
    Plan P;
    plan_batch(mp.data(), n, data.data(), st.data(), cnt.data(), 148, P, tune);
    if (tune.flux_chunks > 0) CHECK(P.flux_chunks == tune.flux_chunks, "flux_chunks %d", P.flux_chunks);
    if (tune.roche_split > 0 && P.roche_elems > 0) CHECK(P.roche_split == tune.roche_split, "roche_split %d", P.roche_split);
    CHECK(P.flux_blocks_per_sm == tune.flux_blocks_per_sm, "flux_blocks_per_sm");
    // segments: contiguous per model, in order
    int64_t e = 0;
    std::vector<int64_t> mfirst(n, -1), mcount(n, 0);
    for (const SegDesc& s : P.segs) {
        CHECK(s.first == e, "segment first %lld != %lld", (long long)s.first, (long long)e);
        CHECK(s.model >= 0 && s.model < n, "segment model %d", s.model);
        if (mfirst[s.model] < 0) mfirst[s.model] = s.first;
        CHECK(s.first == mfirst[s.model] + mcount[s.model], "model %d elements not contiguous", s.model);
        mcount[s.model] += s.count;
        e += s.count;
    }
    CHECK(e == P.nelem, "nelem %lld != %lld", (long long)P.nelem, (long long)e);
    // data: model index and first sub-phase
    int64_t sub = 0;
    for (int64_t i = 0; i < n; ++i) {
        const ModelDev& D = P.models[i];
        CHECK(D.sub_begin == sub || !P.model_ok[i], "model %lld sub_begin", (long long)i);
        for (int64_t k = 0; k < D.ndatum; ++k) {
            const int64_t dd = D.datum_begin + k;
            CHECK(P.datum_model[dd] == i, "datum %lld model", (long long)dd);
            CHECK(P.datum_sub0[dd] == sub, "datum %lld sub0 %lld != %lld", (long long)dd, (long long)P.datum_sub0[dd], (long long)sub);
            if (P.model_ok[i]) sub += data[st[i] + k].ndiv;
        }
        CHECK(!P.model_ok[i] || D.nsub == sub - D.sub_begin, "model %lld nsub", (long long)i);
    }
    CHECK(sub == P.nsub, "nsub");
    // flux units: exact cover, order, slot groups
    std::map<std::pair<int64_t, int32_t>, std::vector<std::pair<int32_t, int32_t>>> tiles;  // (e0, ne) -> (t0, nt)
    int64_t evals = 0, prev = INT64_MAX;
    for (const FluxUnit& u : P.units) {
        const int64_t sz = (int64_t)u.ne * u.nt;
        CHECK(sz <= prev, "units not largest first");
        prev = sz;
        evals += sz;
        tiles[{u.e0, u.ne}].push_back({u.t0, u.nt});
        const ModelDev& D = P.models[u.model];
        const int32_t lo[5] = {0, D.g1_end, D.g2_end, D.gd_end, D.ge_end};
        const int32_t hi[5] = {D.g1_end, D.g2_end, D.gd_end, D.ge_end, D.nslots};
        const SegDesc* seg = nullptr;
        for (const SegDesc& s : P.segs)
            if (u.e0 >= s.first && u.e0 < s.first + s.count) seg = &s;
        CHECK(seg && seg->model == u.model && u.e0 + u.ne <= seg->first + seg->count, "unit outside its segment");
        if (seg) { int g = grp(seg->kind); CHECK(u.slot >= lo[g] && u.slot < hi[g], "slot %d outside group %d", u.slot, g); }
    }
    CHECK(evals == P.evals, "evals %lld != %lld", (long long)evals, (long long)P.evals);
    for (auto& kv : tiles) {
        auto v = kv.second;
        std::sort(v.begin(), v.end());
        int64_t t = 0;
        for (auto& p : v) { CHECK(p.first == t, "sub-phase tiles overlap or leave a gap"); t += p.second; }
        const FluxUnit* any = nullptr;
        for (const FluxUnit& u : P.units) if (u.e0 == kv.first.first) { any = &u; break; }
        CHECK(any && t == P.models[any->model].nsub, "tiles of an element range do not cover the sub-phases");
    }
    for (const SegDesc& s : P.segs) {
        if (!P.model_ok[s.model] || P.models[s.model].nsub == 0) continue;
        int64_t covered = 0;
        for (auto& kv : tiles) if (kv.first.first >= s.first && kv.first.first < s.first + s.count) covered += kv.first.second;
        CHECK(covered == s.count, "segment elements covered %lld of %lld", (long long)covered, (long long)s.count);
    }
    // element, Roche and aux blocks
    std::vector<int64_t> eb(P.segs.size(), 0), ab(P.segs.size(), 0);
    for (const ElemBlock& b : P.eblocks) { CHECK(b.offset % kElemThreads == 0 && b.offset < P.segs[b.seg].count, "eblock"); eb[b.seg]++; }
    for (const ElemBlock& b : P.ablocks) { ab[b.seg]++; }
    for (size_t s = 0; s < P.segs.size(); ++s) {
        const int64_t want = (P.segs[s].count + kElemThreads - 1) / kElemThreads;
        CHECK(eb[s] == want, "segment %zu element blocks", s);
        const bool star = P.segs[s].kind == SEG_STAR1 || P.segs[s].kind == SEG_STAR2;
        CHECK(ab[s] == (star ? want : 0), "segment %zu aux blocks", s);
    }
    int64_t roche = 0;
    for (const ElemBlock& b : P.rblocks) {
        CHECK((b.by == 1 || b.by == 2) && b.offset % kRocheBlock == 0 && b.offset < P.segs[b.seg].count, "rblock");
        if (b.offset == 0) roche += P.segs[b.seg].count;
    }
    CHECK(roche == P.roche_elems, "roche elements %lld != %lld", (long long)roche, (long long)P.roche_elems);
    // failed models own nothing
    int failed = 0;
    for (int64_t i = 0; i < n; ++i)
        if (!P.model_ok[i]) { ++failed; CHECK(mcount[i] == 0 && !P.model_err[i].empty(), "failed model %lld", (long long)i); }
    // re-planning into the same storage
    Plan Q = P;
    plan_batch(mp.data(), n, data.data(), st.data(), cnt.data(), 148, P, tune);
    CHECK(same(P.segs, Q.segs) && same(P.bands, Q.bands) && same(P.rings, Q.rings) && same(P.units, Q.units) &&
          same(P.eblocks, Q.eblocks) && same(P.rblocks, Q.rblocks) && same(P.ablocks, Q.ablocks) &&
          same(P.models, Q.models) && same(P.datum_sub0, Q.datum_sub0) && P.shape_key == Q.shape_key,
          "re-planned batch differs");
    // planning from several host threads at once (they share the host's worker pool and
    // the bright-spot memo): every thread's plan equals the one above
    {
        const int nt = 4;
        std::vector<Plan> R(nt);
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t)
            th.emplace_back([&, t] {
                for (int rep = 0; rep < 3; ++rep)
                    plan_batch(mp.data(), n, data.data(), st.data(), cnt.data(), 148, R[t], tune);
            });
        for (auto& x : th) x.join();
        for (int t = 0; t < nt; ++t)
            CHECK(same(R[t].segs, Q.segs) && same(R[t].bands, Q.bands) && same(R[t].units, Q.units) &&
                  same(R[t].models, Q.models) && same(R[t].rblocks, Q.rblocks) && R[t].shape_key == Q.shape_key,
                  "plan of concurrent thread %d differs", t);
    }
    std::printf("models %lld failed %d elements %lld units %zu roche %lld fails %d\n", (long long)n, failed,
                (long long)P.nelem, P.units.size(), (long long)P.roche_elems, fails);
    return fails ? 1 : 0;
}
"""


def _set(text, name, value):
    out = []
    for line in text.splitlines():
        if line.split("=")[0].strip() == name:
            rest = line.split("=", 1)[1].split()
            rest[0] = str(value)
            line = f"{name} = {' '.join(rest)}"
        out.append(line)
    return "\n".join(out) + "\n"


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("plan")
    (d / "d.cpp").write_text(DRIVER)
    src = ROOT / "lcurve-rs_b200" / "csrc"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I/usr/local/cuda/include", f"-I{src}", str(d / "d.cpp"),
                    str(src / "lcb_plan.cpp"), str(src / "lcb_model.cpp"), "-o", str(d / "d"), "-lpthread"],
                   check=True)
    return d


def test_plan_invariants(driver):
    import importlib
    W = importlib.import_module("lcurve-rs_b200.workloads")
    gold = (GOLDEN / "test_model.dat").read_text()
    large, *_ = W.single_large(nlat1=30, nlat2=50, ntime=10, nrad=40, nspot=30)
    texts = [gold, large, W.model_text(**W.SMALL), _set(gold, "r2", 0.99), _set(large, "q", 0.3),
             _set(gold, "nlat1c", 20), _set(W.model_text(**W.SMALL), "iangle", 89.0)]
    (driver / "models.bin").write_text("\x1e".join(texts) + "\x1e")
    r = subprocess.run([str(driver / "d"), str(driver / "models.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "failed 1 " in r.stdout, r.stdout
    # the same invariants under every launch-shape choice an autotuner may set
    for tune in ((1, 1, 1), (16, 16, 4), (4, 2, 0), (2, 0, 3)):
        r = subprocess.run([str(driver / "d"), str(driver / "models.bin")] + [str(v) for v in tune],
                           capture_output=True, text=True)
        assert r.returncode == 0, (tune, r.stdout + r.stderr)


HELPERS = r"""
#include <cstdio>
#include <cstdlib>
#include "lcb_plan.h"
int main(int argc, char** argv) {
    // argv: q spin rad nlat, one case per 4 arguments
    for (int i = 1; i + 3 < argc; i += 4) {
        const double q = std::atof(argv[i]), spin = std::atof(argv[i + 1]), rad = std::atof(argv[i + 2]);
        const int nlat = std::atoi(argv[i + 3]);
        double s[3];
        lcb::host_stream_spot(q, rad, s);
        std::printf("%.17g %.17g %.17g %.17g %.17g %.17g %lld\n", lcb::host_xl1(q), lcb::host_xl11(q, spin),
                    lcb::host_xl12(q, spin), s[0], s[1], s[2], (long long)lcb::host_numface(nlat));
    }
}
"""


def test_host_geometry_helpers_match_the_oracle(driver, oracle):
    """The planner's own FP64 helpers (L1 points, the bright-spot stream
    integration, star-grid element counts) against the oracle's separate
    restatements (lagrange.rs, stream.rs:82-145, grid.rs:8-46)."""
    import ctypes as C
    (driver / "h.cpp").write_text(HELPERS)
    src = ROOT / "lcurve-rs_b200" / "csrc"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I/usr/local/cuda/include", f"-I{src}", str(driver / "h.cpp"),
                    str(src / "lcb_plan.cpp"), str(src / "lcb_model.cpp"), "-o", str(driver / "h"), "-lpthread"],
                   check=True)
    L = oracle.lib()
    # spot radii the stream crosses on its way in from L1 (fractions of the L1 distance)
    cases = [(q, spin, round(frac * L.orc_xl1(q), 6), nlat) for q in (0.08, 0.3, 0.7, 1.0)
             for spin, frac, nlat in ((1.0, 0.35, 20), (0.8, 0.55, 57), (1.2, 0.8, 300))]
    args = [str(v) for c in cases for v in c]
    out = subprocess.run([str(driver / "h")] + args, capture_output=True, text=True, check=True).stdout.splitlines()
    for (q, spin, rad, nlat), line in zip(cases, out):
        f = line.split()
        xl1, xl11, xl12, sx, sy, sz = (float(x) for x in f[:6])
        assert abs(xl1 - L.orc_xl1(q)) < 1e-12
        assert abs(xl11 - L.orc_xl11(q, spin)) < 1e-12 and abs(xl12 - L.orc_xl12(q, spin)) < 1e-12
        ref = (C.c_double * 3)()
        L.orc_stream_spot(q, rad, ref)
        assert max(abs(sx - ref[0]), abs(sy - ref[1]), abs(sz - ref[2])) < 1e-10, (q, rad)
        assert int(f[6]) == L.orc_numface(nlat)
