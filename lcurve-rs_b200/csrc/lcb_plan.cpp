// lcb_plan.cpp — host-side per-model set-up and batch decomposition.
//
// Per model this computes, in FP64 on the host, the handful of scalars that
// the reference recomputes inside its element loops: Lagrange points
// (crates/roche/src/lagrange.rs:89-142), reference spheres (surface.rs:14-39),
// reference gravities (grid.rs:166-181), the bright-spot position from the
// gas-stream integration (stream.rs:82-145 with bsstep.rs:159-324), Planck
// constants of the continuum (brightness.rs) and the lensing radius
// (orchestration.rs:52-58).  It then lays out band/ring tables for the
// element kernel and splits the flux sum into (element range x sub-phase
// tile) work units for the persistent flux kernel.
#include "lcb_plan.h"
#include "lcb_stream.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <cmath>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>

namespace lcb {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kC = 2.99792458e8;       // constants.rs:5
constexpr double kH = 6.6262e-34;         // constants.rs:11
constexpr double kK = 1.3806e-23;         // constants.rs:14
constexpr double kDay = 86400.0;          // constants.rs:65
constexpr double kEfac = 1.0000001;       // grid.rs:337, 396

inline double sq(double x) { return x * x; }
inline double deg2rad(double d) { return d * (kPi / 180.0); }
inline double cube(double x) { return (x * x) * x; }

Error model_err(const std::string& m) { return Error(LCB_ERR_MODEL, m); }

// `as i32` from f64: saturating, NaN -> 0.
int64_t sat_i32(double x) {
    if (std::isnan(x)) return 0;
    if (x >= 2147483647.0) return 2147483647;
    if (x <= -2147483648.0) return -2147483648LL;
    return (int64_t)x;
}

// Newton iteration of the quintic for the inner Lagrange point (lagrange.rs:8-142).
double l1_newton(double q, double a3, double a4, double a5, double a6, const char* who) {
    if (q <= 0.0) throw model_err(std::string(who) + ": q <= 0");
    double mu = q / (1.0 + q);
    double a1 = -1.0 + mu, a2 = 2.0 - 2.0 * mu;
    double d1 = a2, d2 = 2.0 * a3, d3 = 3.0 * a4, d4 = 4.0 * a5, d5 = 5.0 * a6;
    double x = 1.0 / (1.0 + q);
    for (int it = 0; it < 1000; ++it) {
        double xo = x;
        double f = x * (x * (x * (x * (x * a6 + a5) + a4) + a3) + a2) + a1;
        double df = x * (x * (x * (x * d5 + d4) + d3) + d2) + d1;
        x -= f / df;
        if (std::fabs(x - xo) <= 1.0e-12 * std::fabs(x)) return x;
    }
    throw model_err(std::string(who) + ": exceeded maximum iterations");
}

struct V3 { double x, y, z; };
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 scale(double s, V3 v) { return {s * v.x, s * v.y, s * v.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }

// Asynchronous Roche potentials and gradients (potential.rs:22-106).
double pot(bool primary, double q, double spin, V3 p) {
    double mu = q / (1.0 + q), comp = 1.0 - mu;
    double x2y2 = sq(p.x) + sq(p.y);
    double r1sq = x2y2 + sq(p.z);
    double r1 = std::sqrt(r1sq), r2 = std::sqrt(r1sq + 1.0 - 2.0 * p.x);
    if (primary) return -comp / r1 - mu / r2 - sq(spin) * x2y2 / 2.0 + mu * p.x;
    return -comp / r1 - mu / r2 - sq(spin) * (0.5 + 0.5 * x2y2 - p.x) - comp * p.x;
}
V3 dpot(bool primary, double q, double spin, V3 p) {
    double r1sq = norm2(p), r2sq = r1sq + 1.0 - 2.0 * p.x;
    double r1 = std::sqrt(r1sq), r2 = std::sqrt(r2sq);
    double mu = q / (1.0 + q);
    double mu1 = mu / r2 / r2sq, comp = (1.0 - mu) / r1 / r1sq, ssq = sq(spin);
    if (primary)
        return {comp * p.x + mu1 * (p.x - 1.0) - ssq * p.x + mu, comp * p.y + mu1 * p.y - ssq * p.y,
                comp * p.z + mu1 * p.z};
    return {comp * p.x + mu1 * (p.x - 1.0) - ssq * (p.x - 1.0) + mu - 1.0, comp * p.y + mu1 * p.y - ssq * p.y,
            comp * p.z + mu1 * p.z};
}

void ref_sphere(bool primary, double q, double spin, double ffac, double& rref, double& pref) {
    double rl = primary ? host_xl11(q, spin) : 1.0 - host_xl12(q, spin);
    double surf = ffac * rl;
    V3 p = primary ? V3{surf, 0.0, 0.0} : V3{1.0 - surf, 0.0, 0.0};
    pref = pot(primary, q, spin, p);
    rref = std::fmin(1.001 * ffac, 1.0) * rl;
}

// Surface point and gravity along a direction (surface.rs:54-121); returns gravity.
double face_gravity(bool primary, double q, double spin, V3 dirn, double rref, double pref, double acc) {
    V3 cofm = primary ? V3{0, 0, 0} : V3{1.0, 0.0, 0.0};
    auto f = [&](double r) { return pot(primary, q, spin, add(cofm, scale(r, dirn))); };
    double lo = rref / 2.0, hi = rref, t = pref + 1.0;
    for (int i = 0; i < 30 && t > pref; ++i) {
        lo = hi / 2.0;
        t = f(lo);
        if (t > pref) hi = lo;
    }
    for (int i = 0; i < 100 && hi - lo > acc; ++i) {
        double mid = (lo + hi) / 2.0;
        if (f(mid) < pref) lo = mid; else hi = mid;
    }
    double r = (lo + hi) / 2.0;
    return std::sqrt(norm2(dpot(primary, q, spin, add(cofm, scale(r, dirn)))));
}

// Planck function and its log-derivative (planck.rs:4-44).
const double kFac1 = 2.0e27 * kH * kC;
const double kFac2 = 1.0e9 * kH * kC / kK;
double planck(double wave, double temp) {
    double e = kFac2 / (wave * temp);
    if (e > 40.0) return kFac1 * std::exp(-e) / (wave * sq(wave));
    return kFac1 / (std::exp(e) - 1.0) / (wave * sq(wave));
}
double dlpdlt(double wave, double temp) {
    double e = kFac2 / (wave * temp);
    return e / (1.0 - std::exp(-e));
}

// ---- gas stream (lcb_stream.h: the same source runs on the device) ----------
void stream_to_radius_uncached(double q, double rad, double out[3]) {
    const int rc = stream::stream_to_radius_core(q, host_xl1(q), rad, out);
    if (rc == stream::kStreamChopFailed) throw model_err("stradv: binary chop failed to converge");
    if (rc != stream::kStreamOk) throw model_err("stradv: took too long without crossing radius=" + std::to_string(rad));
}

// stream_to_radius_uncached memoised on (q, rad), process-wide: the integration is ~20,000
// serial right-hand-side evaluations (the reference's 1e-3 step cap), and fits, batches and
// repeated light curves mostly revisit the same geometry.  The result is a function of (q, rad)
// alone, so a hit returns exactly what the integration would; failures are not cached.  The
// table holds the last kSpotMemo distinct pairs, enough for every model of a large batch
// (plan_batch integrates a batch's new pairs in parallel first, then every model hits).
constexpr size_t kSpotMemo = 8192;
struct SpotKey {
    uint64_t q, rad;
    bool operator==(const SpotKey& o) const { return q == o.q && rad == o.rad; }
};
struct SpotKeyHash {
    size_t operator()(const SpotKey& k) const { return (size_t)(k.q * 0x9E3779B97F4A7C15ull ^ (k.rad + (k.q >> 7))); }
};
static std::mutex g_spot_mu;
static std::unordered_map<SpotKey, std::array<double, 3>, SpotKeyHash> g_spot_memo;
static std::deque<SpotKey> g_spot_order;

static SpotKey spot_key(double q, double rad) {
    SpotKey k;
    std::memcpy(&k.q, &q, 8);
    std::memcpy(&k.rad, &rad, 8);
    return k;
}

static bool spot_cached(double q, double rad, double out[3]) {
    std::lock_guard<std::mutex> g(g_spot_mu);
    auto it = g_spot_memo.find(spot_key(q, rad));
    if (it == g_spot_memo.end()) return false;
    out[0] = it->second[0]; out[1] = it->second[1]; out[2] = it->second[2];
    return true;
}

static void spot_store(double q, double rad, const double out[3]) {
    std::lock_guard<std::mutex> g(g_spot_mu);
    const SpotKey k = spot_key(q, rad);
    if (g_spot_memo.emplace(k, std::array<double, 3>{out[0], out[1], out[2]}).second) {
        g_spot_order.push_back(k);
        if (g_spot_order.size() > kSpotMemo) {
            g_spot_memo.erase(g_spot_order.front());
            g_spot_order.pop_front();
        }
    }
}

static std::atomic<StreamDeviceFn> g_stream_device{nullptr};

void stream_to_radius(double q, double rad, double out[3]) {
    if (spot_cached(q, rad, out)) return;
    stream_to_radius_uncached(q, rad, out);
    spot_store(q, rad, out);
}

// Latitude bands of one star grid (grid.rs:157-322) appended to `bands`;
// returns the element count.
int64_t star_bands(const Model& m, bool primary, int nlat, bool infill, double thelo, double thehi, int nlatfill,
                   int nlngfill, std::vector<Band>& bands) {
    double dtheta = kPi / (double)nlat;
    int64_t count = 0;
    auto run = [&](double tlo, double thi, int nf, int ng) {
        bool fill = nf > 0 || ng > 0;
        int64_t n1 = 0, n2 = 0, n;
        if (fill) {
            n1 = sat_i32(std::ceil((double)(1 + nf) * (thi - tlo) / dtheta));
            n2 = sat_i32(std::ceil((thi - tlo) / dtheta));
            n = n1 + n2;
        } else {
            n = sat_i32(std::ceil((thi - tlo) / dtheta));
        }
        for (int64_t nt = 0; nt < n; ++nt) {
            double theta, p1, p2;
            int64_t nphi, nl;
            if (fill) {
                if (nt < n1) {
                    theta = tlo + (thi - tlo) * ((double)nt + 0.5) / (double)n1;
                    nphi = std::max<int64_t>(8, sat_i32(kPi * std::sin(theta) * (double)(1 + ng) / dtheta));
                    nl = n1;
                    p1 = primary ? -kPi / 2.0 : kPi / 2.0;
                    p2 = primary ? kPi / 2.0 : 3.0 * kPi / 2.0;
                } else {
                    theta = tlo + (thi - tlo) * ((double)(nt - n1) + 0.5) / (double)n2;
                    nphi = std::max<int64_t>(8, sat_i32(kPi * std::sin(theta) / dtheta));
                    nl = n2;
                    p1 = primary ? kPi / 2.0 : -kPi / 2.0;
                    p2 = primary ? 3.0 * kPi / 2.0 : kPi / 2.0;
                }
            } else {
                theta = tlo + (thi - tlo) * ((double)nt + 0.5) / (double)n;
                nphi = std::max<int64_t>(16, sat_i32(kTwoPi * std::sin(theta) / dtheta));
                nl = n;
                p1 = 0.0;
                p2 = kTwoPi;
            }
            Band b;
            b.first = count;
            b.nphi = nphi;
            b.sint = std::sin(theta);
            b.cost = std::cos(theta);
            b.phi1 = p1;
            b.phi2 = p2;
            b.aphi = (p2 - p1) / (double)nphi;
            b.ath = (thi - tlo) / (double)nl;
            bands.push_back(b);
            count += nphi;
        }
    };
    if (infill) {
        run(0.0, thelo, 0, 0);
        run(thelo, thehi, nlatfill, nlngfill);
        run(thehi, kPi, 0, 0);
    } else {
        run(0.0, kPi, 0, 0);
    }
    (void)m;
    return count;
}

// Infill latitude limits of the secondary's fine grid (grid.rs:112-151).
// Returns false when the grid falls back to no infill.
bool infill_limits(const Model& m, double r1, double r2, double& thelo, double& thehi) {
    double rangle = deg2rad(m.v(P_IANGLE));
    double cosi = std::cos(rangle);
    auto envelope = [&](double lam, double& x, double& y) {  // grid.rs:324-333
        double si = std::sin(rangle), ci = std::cos(rangle), sl = std::sin(lam), cl = std::cos(lam);
        double nrm = std::sqrt(ci * ci + si * si * cl * cl);
        x = sl + r1 * ci * sl / nrm;
        y = -ci * cl - r1 * cl / nrm;
    };
    thelo = 0.0;
    thehi = 0.0;
    if ((cosi + r1) / r2 >= 1.0) {
        thehi = kPi / 2.0 + rangle;
    } else {
        double lo = 0.0, hi = kPi / 2.0, x, y;
        while (hi > lo + 1e-7) {
            double mid = (lo + hi) / 2.0;
            envelope(mid, x, y);
            if (x * x + y * y < r2 * r2) lo = mid; else hi = mid;
        }
        envelope((lo + hi) / 2.0, x, y);
        thehi = std::fmax(kPi / 2.0 - deg2rad(m.llo),
                          std::fmin(kPi / 2.0 + rangle, std::acos(y * std::sin(rangle) / r2) + deg2rad(m.lfudge)));
    }
    double ratio2 = (cosi - r1) / r2;
    if (ratio2 >= 1.0) return false;
    if (ratio2 <= -1.0) thelo = 0.0;
    else thelo = std::fmin(kPi / 2.0 - deg2rad(m.lhi), std::fmax(kPi / 2.0 - std::acos(ratio2) + rangle - deg2rad(m.lfudge), 0.0));
    return true;
}

int grid_type(double phase, double p1, double p2) {  // types.rs:191-202
    double pn = phase - std::floor(phase);
    if (pn <= p1 || pn >= 1.0 - p1) return 1;
    if ((pn > p1 && pn < p2) || (pn > 1.0 - p2 && pn < 1.0 - p1)) return 2;
    return 3;
}

int highest_nonzero(const double* c) {
    int n = 1;
    for (int i = 0; i < 4; ++i)
        if (c[i] != 0.0) n = i + 1;
    return n;
}

struct ModelLayout {
    ModelDev dev;
    std::vector<SegDesc> segs;   // first = model-relative element offset
    std::vector<Band> bands;     // SegDesc.table model-relative
    std::vector<Ring> rings;
    int64_t nelem = 0;
};

// Everything orchestration.rs:36-170 computes before the time loop, reduced
// to per-model constants and element tables.
void prepare_model(const Model& m, const lcb_datum* data, int64_t ndata, ModelLayout& L) {
    ModelDev& D = L.dev;
    std::memset(&D, 0, sizeof D);
    const double q = m.v(P_Q);
    const double spin1 = m.v(P_SPIN1), spin2 = m.v(P_SPIN2);
    double r1raw, r2raw;
    get_r1r2(m, r1raw, r2raw);

    // light_curve_comp (orchestration.rs:42-46)
    double rl2_lc = 1.0 - host_xl12(q, spin2);
    double r2_lc = r2raw;
    if (r2_lc < 0.0) r2_lc = rl2_lc;
    else if (r2_lc > rl2_lc) throw model_err("light_curve_comp: secondary larger than Roche lobe");
    // set_star_grid (grid.rs:98-105)
    double rl1 = host_xl11(q, spin1), rl2 = 1.0 - host_xl12(q, spin2);
    double r1 = r1raw, r2 = r2raw;
    if (r1 < 0.0) r1 = rl1;
    else if (r1 > rl1) throw model_err("set_star_grid: primary star larger than Roche lobe");
    if (r2 < 0.0) r2 = rl2;
    else if (r2 > rl2) throw model_err("set_star_grid: secondary star larger than Roche lobe");

    D.q = q;
    D.xcofm = q / (1.0 + q);
    double ri = deg2rad(m.v(P_IANGLE));
    D.cosi_e = std::cos(ri); D.sini_e = std::sin(ri);
    D.cosi_l = std::cos(kTwoPi * m.v(P_IANGLE) / 360.0); D.sini_l = std::sin(kTwoPi * m.v(P_IANGLE) / 360.0);
    double rd = m.v(P_IANGLE) * kPi / 180.0;
    D.cosi_d = std::cos(rd); D.sini_d = std::sin(rd);
    D.r1 = r1; D.r2 = r2; D.spin1 = spin1; D.spin2 = spin2;
    D.ffac1 = r1 / rl1; D.ffac2 = r2 / rl2;
    ref_sphere(true, q, spin1, D.ffac1, D.rref1, D.pref1);
    ref_sphere(false, q, spin2, D.ffac2, D.rref2, D.pref2);
    D.delta = m.delta_phase;
    D.acc_face = m.delta_phase / 10.0;
    D.gref1 = m.roche1 ? face_gravity(true, q, spin1, {-1.0, 0.0, 0.0}, D.rref1, D.pref1, D.acc_face) : 1.0;
    D.gref2 = m.roche2 ? face_gravity(false, q, spin2, {1.0, 0.0, 0.0}, D.rref2, D.pref2, D.acc_face) : 1.0;
    double mu = q / (1.0 + q);
    D.ecl1 = RocheEcl{mu, 1.0 - mu, sq(spin1), D.rref1, D.pref1, 0.0, 1, 0};
    D.ecl2 = RocheEcl{mu, 1.0 - mu, sq(spin2), D.rref2, D.pref2, 1.0, 0, 0};
    D.roche1 = m.roche1; D.roche2 = m.roche2; D.eclipse1 = m.eclipse1; D.eclipse2 = m.eclipse2;
    D.npole = m.npole; D.glens1 = m.glens1;
    D.add_disc = m.add_disc; D.opaque = m.opaque; D.add_spot = m.add_spot; D.iscale = m.iscale;

    // continuum (brightness.rs:13-147)
    double xl1s = host_xl1(q);
    D.r1c = r1raw < 0.0 ? xl1s : r1raw;
    D.r2c = r2raw < 0.0 ? 1.0 - xl1s : r2raw;
    D.wavelength = m.wavelength;
    D.t1 = m.v(P_T1); D.t2 = m.v(P_T2); D.absorb = m.v(P_ABSORB);
    D.gdcbol1 = m.gdark_bolom1 ? m.v(P_GRAVITY_DARK1) : m.v(P_GRAVITY_DARK1) / dlpdlt(m.wavelength, m.v(P_T1));
    D.gdcbol2 = m.gdark_bolom2 ? m.v(P_GRAVITY_DARK2)
                               : m.v(P_GRAVITY_DARK2) / dlpdlt(m.wavelength, std::fabs(m.v(P_T2)));
    D.mirror = m.mirror;
    D.planck_t2abs = planck(m.wavelength, std::fabs(m.v(P_T2)));
    D.planck_t1 = planck(m.wavelength, m.v(P_T1));
    auto spot = [&](int base, SpotDev& s) {  // brightness.rs:187-201
        std::memset(&s, 0, sizeof s);
        for (int k = 0; k < 4; ++k)
            if (!m.p[base + k].defined) return;
        double lo = deg2rad(m.v(base)), la = deg2rad(m.v(base + 1));
        s.dx = std::cos(la) * std::cos(lo); s.dy = std::cos(la) * std::sin(lo); s.dz = std::sin(la);
        s.fwhm = m.v(base + 2); s.tcen = m.v(base + 3); s.on = 1;
    };
    spot(P_STSP11_LONG, D.spot1[0]); spot(P_STSP12_LONG, D.spot1[1]); spot(P_STSP13_LONG, D.spot1[2]);
    spot(P_STSP21_LONG, D.spot2[0]); spot(P_STSP22_LONG, D.spot2[1]);
    D.uesp_on = m.p[P_UESP_LONG1].defined && m.p[P_UESP_LONG2].defined && m.p[P_UESP_LATHW].defined &&
                m.p[P_UESP_TAPER].defined && m.p[P_UESP_TEMP].defined;
    if (D.uesp_on) {
        D.uesp_longhw = (m.v(P_UESP_LONG2) - m.v(P_UESP_LONG1)) / 2.0;
        double lc = deg2rad((m.v(P_UESP_LONG1) + m.v(P_UESP_LONG2)) / 2.0);
        D.uesp_dx = std::cos(lc); D.uesp_dy = std::sin(lc);
        D.uesp_lathw = m.v(P_UESP_LATHW); D.uesp_taper = m.v(P_UESP_TAPER); D.uesp_temp = m.v(P_UESP_TEMP);
    }

    // flux constants (flux.rs:7-111)
    for (int k = 0; k < 4; ++k) {
        D.ld1[k] = m.v(P_LDC1_1 + k); D.ld2[k] = m.v(P_LDC2_1 + k);
        D.ld1f[k] = (float)D.ld1[k]; D.ld2f[k] = (float)D.ld2[k];
    }
    D.ltype1 = m.limb1; D.ltype2 = m.limb2;
    D.npoly1 = highest_nonzero(D.ld1); D.npoly2 = highest_nonzero(D.ld2);
    D.mucrit1 = m.mucrit1; D.mucrit2 = m.mucrit2;
    D.mucrit1f = (float)m.mucrit1; D.mucrit2f = (float)m.mucrit2;
    D.beam1 = m.v(P_BEAM_FACTOR1); D.beam2 = m.v(P_BEAM_FACTOR2);
    D.vfac = (double)(float)m.v(P_VELOCITY_SCALE) / (kC / 1e3);
    D.beam1f = (float)D.beam1; D.beam2f = (float)D.beam2; D.vfacf = (float)D.vfac;
    D.spin1f = (float)spin1; D.spin2f = (float)spin2; D.xcofmf = (float)D.xcofm;
    D.lin_ld = m.v(P_LIN_LIMB_DISC); D.quad_ld = m.v(P_QUAD_LIMB_DISC);
    D.lin_ldf = (float)D.lin_ld; D.quad_ldf = (float)D.quad_ld;
    if (m.glens1) {  // orchestration.rs:52-58
        double gm = cube(1000.0 * m.v(P_VELOCITY_SCALE)) * m.tperiod * kDay / kTwoPi;
        double a = std::pow(gm / sq(kTwoPi / kDay / m.tperiod), 1.0 / 3.0);
        D.rlens1 = 4.0 * gm / (1.0 + q) / a / sq(kC);
    }
    D.rlens1f = (float)D.rlens1;

    // star grids (grid.rs:76-198) and their coarse copies (orchestration.rs:66-83)
    D.copy1 = m.nlat1f == m.nlat1c;
    D.copy2 = m.nlat2f == m.nlat2c && (!m.npole || r1raw >= r2_lc || (m.nlatfill == 0 && m.nlngfill == 0));
    auto add_star = [&](bool primary, bool fine, int role) {
        int nlat = primary ? (fine ? m.nlat1f : m.nlat1c) : (fine ? m.nlat2f : m.nlat2c);
        int nf = (!primary && fine) ? m.nlatfill : 0, ng = (!primary && fine) ? m.nlngfill : 0;
        bool infill = m.npole && !primary && (nf > 0 || ng > 0) && r2 > r1;
        double thelo = 0.0, thehi = 0.0;
        if (infill && !infill_limits(m, r1, r2, thelo, thehi)) { infill = false; nf = ng = 0; }
        SegDesc s{};
        s.first = L.nelem;
        s.kind = primary ? SEG_STAR1 : SEG_STAR2;
        s.role = role;
        s.table = (int32_t)L.bands.size();
        s.count = star_bands(m, primary, nlat, infill, thelo, thehi, nf, ng, L.bands);
        s.ntable = (int32_t)L.bands.size() - s.table;
        s.fine_star = fine;
        L.nelem += s.count;
        L.segs.push_back(s);
    };
    add_star(true, true, D.copy1 ? ROLE_BOTH : ROLE_FINE);
    if (!D.copy1) add_star(true, false, ROLE_COARSE);
    add_star(false, true, D.copy2 ? ROLE_BOTH : ROLE_FINE);
    if (!D.copy2) add_star(false, false, ROLE_COARSE);

    // disc, rim and bright spot
    D.rdisc1_g = m.v(P_RDISC1) > 0.0 ? m.v(P_RDISC1) : r1;
    D.rdisc1_l = m.v(P_RDISC1) > 0.0 ? m.v(P_RDISC1) : r1raw;
    D.rdisc2 = m.v(P_RDISC2) > 0.0 ? m.v(P_RDISC2) : m.v(P_RADIUS_SPOT);
    D.beta = m.v(P_BETA_DISC); D.height = m.v(P_HEIGHT_DISC);
    if (m.add_disc) {
        // set_disc_grid (grid.rs:336-392)
        SegDesc s{};
        s.first = L.nelem; s.kind = SEG_DISC; s.table = (int32_t)L.rings.size();
        double drad = (D.rdisc2 - D.rdisc1_g) / (double)m.nrad, drrad = D.rdisc2 / (double)m.nrad;
        int64_t cnt = 0;
        for (int i = 0; i < m.nrad; ++i) {
            Ring g;
            g.rad = D.rdisc1_g + (D.rdisc2 - D.rdisc1_g) * ((double)i + 0.5) / (double)m.nrad;
            g.ntheta = std::max<int64_t>(8, sat_i32(std::ceil(kTwoPi * g.rad / drrad)));
            g.h = kEfac * D.height * std::pow(g.rad, D.beta);
            double tanp = D.beta * g.h / g.rad;
            g.cosp = 1.0 / std::sqrt(1.0 + sq(tanp));
            g.sinp = tanp * g.cosp;
            g.area = kTwoPi / (double)g.ntheta * g.rad * drad;
            g.first = cnt;
            cnt += g.ntheta;
            L.rings.push_back(g);
        }
        s.count = cnt; s.ntable = (int32_t)L.rings.size() - s.table;
        L.nelem += cnt;
        L.segs.push_back(s);
        // set_disc_edge(outer = true) (grid.rs:395-481)
        double size = D.rdisc2 / (double)m.nrad;
        D.edge_rad = D.rdisc2;
        D.edge_h = D.height * std::pow(D.edge_rad, D.beta);
        D.edge_nout = sat_i32(2.0 * D.edge_h / size) + 2;
        D.edge_ntheta = std::max<int64_t>(8, sat_i32(std::ceil(kTwoPi * D.edge_rad / size)));
        D.edge_area = kTwoPi / (double)D.edge_ntheta * D.edge_rad * 2.0 * D.edge_h / (double)(D.edge_nout - 1);
        SegDesc e{};
        e.first = L.nelem; e.kind = SEG_EDGE;
        e.count = D.edge_ntheta * std::max<int64_t>(D.edge_nout, 0);
        L.nelem += e.count;
        L.segs.push_back(e);
        // continuum constants (brightness.rs:204-239; orchestration.rs:159-165)
        D.disc_bright = planck(m.wavelength, m.v(P_TEMP_DISC));
        D.texp_disc = m.v(P_TEXP_DISC);
        D.tedge = m.v(P_TEMP_EDGE); D.r2e = r2_lc; D.t2abs = std::fabs(m.v(P_T2)); D.absorb_edge = m.v(P_ABSORB_EDGE);
    }
    if (m.add_spot) {  // set_bright_spot_grid (grid.rs:484-553)
        double bs[3];
        stream_to_radius(q, m.v(P_RADIUS_SPOT), bs);
        double theta = std::atan2(bs[1], bs[0]) + kTwoPi / 4.0 + deg2rad(m.v(P_ANGLE_SPOT));
        double alpha = deg2rad(m.v(P_YAW_SPOT)), tilt = deg2rad(m.v(P_TILT_SPOT));
        for (int k = 0; k < 3; ++k) D.bspot[k] = bs[k];
        D.bvec[0] = std::cos(theta); D.bvec[1] = std::sin(theta); D.bvec[2] = 0.0;
        D.tvec[0] = std::sin(tilt) * std::sin(theta + alpha);
        D.tvec[1] = -std::sin(tilt) * std::cos(theta + alpha);
        D.tvec[2] = std::cos(tilt);
        D.expon_spot = m.v(P_EXPON_SPOT); D.epow_spot = m.v(P_EPOW_SPOT);
        D.bmax = std::pow(D.expon_spot / D.epow_spot, 1.0 / D.epow_spot);
        D.sfac_spot = 20.0 + D.bmax;
        D.length_spot = m.v(P_LENGTH_SPOT);
        D.area_spot = D.sfac_spot * D.length_spot * m.v(P_HEIGHT_SPOT) / (double)(m.nspot - 1);
        D.bright_ref = planck(m.wavelength, m.v(P_TEMP_SPOT));
        D.cfrac_spot = m.v(P_CFRAC_SPOT);
        D.nspot = m.nspot;
        SegDesc s{};
        s.first = L.nelem; s.kind = SEG_SPOT; s.count = 2 * (int64_t)std::max(m.nspot, 0);
        L.nelem += s.count;
        L.segs.push_back(s);
    }

    // ginterp and the special phases of comp_star1/2 (orchestration.rs:86-131, 255-259)
    D.phase1 = m.phase1; D.phase2 = m.phase2;
    D.nspec = 0;
    auto add_spec = [&](double phase, int star, int ecl_only) {
        SpecPhase& s = D.spec[D.nspec];
        s.phase = phase;
        s.phi = phase - std::floor(phase);
        double ph = kTwoPi * phase;
        s.ex = D.sini_e * std::cos(ph); s.ey = -D.sini_e * std::sin(ph); s.ez = D.cosi_e;
        s.star = star;
        int t = grid_type(phase, m.phase1, m.phase2);
        s.fine = star == 1 ? (t == 1) : (t == 3);
        s.star_ecl_only = ecl_only;
        return D.nspec++;
    };
    for (int k = 0; k < 2; ++k) { D.spec_g11[k] = D.spec_g12[k] = D.spec_g21[k] = D.spec_g22[k] = -1; }
    if (!D.copy1) {
        D.spec_g11[0] = add_spec(0.9999999999 * m.phase1, 1, 1);
        D.spec_g11[1] = add_spec(1.0000000001 * m.phase1, 1, 1);
        D.spec_g12[0] = add_spec(1.0 - 0.9999999999 * m.phase1, 1, 1);
        D.spec_g12[1] = add_spec(1.0 - 1.0000000001 * m.phase1, 1, 1);
    }
    if (!D.copy2) {
        D.spec_g21[0] = add_spec(1.0 - 1.0000000001 * m.phase2, 2, 1);
        D.spec_g21[1] = add_spec(1.0 - 0.9999999999 * m.phase2, 2, 1);
        D.spec_g22[0] = add_spec(1.0000000001 * m.phase2, 2, 1);
        D.spec_g22[1] = add_spec(0.9999999999 * m.phase2, 2, 1);
    }
    D.spec_wd = add_spec(0.5, 1, 0);

    // ephemeris and polynomial fudge (orchestration.rs:173-179, 231-241)
    D.t0 = m.v(P_T0); D.period = m.v(P_PERIOD); D.pdot = m.v(P_PDOT); D.deltat = m.v(P_DELTAT);
    D.slope = m.v(P_SLOPE); D.quad = m.v(P_QUAD); D.cube = m.v(P_CUBE); D.third = m.v(P_THIRD);
    double xmin = data[0].time, xmax = data[0].time;
    for (int64_t i = 1; i < ndata; ++i) {
        if (data[i].time < xmin) xmin = data[i].time;
        if (data[i].time > xmax) xmax = data[i].time;
    }
    D.middle = (xmin + xmax) / 2.0;
    D.range = (xmax - xmin) / 2.0;

    // log g reference terms (flux.rs:288-322)
    {
        double gm = cube(1000.0 * m.v(P_VELOCITY_SCALE)) * m.tperiod * kDay / kTwoPi;
        double a = std::pow(gm / sq(kTwoPi / kDay / m.tperiod), 1.0 / 3.0);
        double gscale = 100.0 * gm / sq(a);
        double acc = m.delta_phase / 10.0;
        double rlx;
        try { rlx = host_xl12(q, spin1); } catch (const Error&) { rlx = 0.5; }
        if (m.roche1) {
            double rr, pr;
            ref_sphere(true, q, spin1, r1raw / rlx, rr, pr);
            D.glogg1 = face_gravity(true, q, spin1, {-1.0, 0.0, 0.0}, rr, pr, acc) * gscale;
        } else {
            D.glogg1 = gscale / (1.0 + q) / sq(r1raw);
        }
        try { rlx = 1.0 - host_xl12(q, spin2); } catch (const Error&) { rlx = 0.5; }
        if (m.roche2) {
            double rr, pr;
            ref_sphere(false, q, spin2, r2raw / rlx, rr, pr);
            D.glogg2 = face_gravity(false, q, spin2, {1.0, 0.0, 0.0}, rr, pr, acc) * gscale;
        } else {
            D.glogg2 = gscale * q / (1.0 + q) / sq(r2raw);
        }
    }
}

}  // namespace

double host_xl1(double q) { return l1_newton(q, -1.0 + q / (1.0 + q), 1.0 + 2.0 * (q / (1.0 + q)), -2.0 - q / (1.0 + q), 1.0, "xl1"); }
double host_xl11(double q, double spin) {
    double mu = q / (1.0 + q), s = spin * spin;
    return l1_newton(q, -1.0 + mu, s + 2.0 * mu, -2.0 * s - mu, s, "xl11");
}
double host_xl12(double q, double spin) {
    double mu = q / (1.0 + q), s = spin * spin;
    return l1_newton(q, -s + mu, 3.0 * s + 2.0 * mu - 2.0, 1.0 - mu - 3.0 * s, s, "xl12");
}
void host_stream_spot(double q, double radius, double out[3]) { stream_to_radius(q, radius, out); }
void set_stream_device(StreamDeviceFn fn) { g_stream_device.store(fn); }
bool spot_memo_get(double q, double radius, double out[3]) { return spot_cached(q, radius, out); }
void spot_memo_put(double q, double radius, const double out[3]) { spot_store(q, radius, out); }
int64_t host_numface(int nlat) {
    std::vector<Band> b;
    Model m;
    return star_bands(m, true, nlat, false, 0, 0, 0, 0, b);
}

// A process-wide pool of host threads for the planner: a parallel loop
// publishes its index range as a job, the calling thread works on it too, and
// idle workers take indices from any open job, so small batches (an MCMC step
// plans a few models) pay no thread start-up per call.  Several contexts may
// plan at once: jobs are independent.
class HostPool {
    struct Job {
        const std::function<void(int64_t)>* f = nullptr;
        int64_t n = 0;
        std::atomic<int64_t> next{0}, done{0};
        int helpers = 0, users = 0;  // workers allowed / working on it (under the pool mutex)
    };
    std::mutex mu_;
    std::condition_variable work_cv_;  // workers wait here for a job with items left
    std::condition_variable done_cv_;  // callers of run() wait here for their job's end
    std::vector<Job*> open_;

    Job* pick() {
        for (Job* j : open_)
            if (j->users < j->helpers && j->next.load() < j->n) { ++j->users; return j; }
        return nullptr;
    }
    void work(Job* j) {
        for (int64_t i; (i = j->next.fetch_add(1)) < j->n;) {
            (*j->f)(i);
            if (j->done.fetch_add(1) + 1 == j->n) {
                std::lock_guard<std::mutex> g(mu_);
                done_cv_.notify_all();
            }
        }
    }

public:
    const int size;
    explicit HostPool(int workers) : size(workers) {
        for (int t = 0; t < workers; ++t)
            std::thread([this] {
                for (;;) {
                    Job* j = nullptr;
                    {
                        std::unique_lock<std::mutex> lk(mu_);
                        work_cv_.wait(lk, [&] { return (j = pick()) != nullptr; });
                    }
                    work(j);
                    std::lock_guard<std::mutex> g(mu_);
                    if (--j->users == 0) done_cv_.notify_all();
                }
            }).detach();  // process-lifetime workers
    }
    static HostPool& get() {
        static HostPool* p = new HostPool((int)std::max(1u, std::thread::hardware_concurrency()) - 1);
        return *p;
    }
    void run(int64_t n, int helpers, const std::function<void(int64_t)>& f) {
        Job j;
        j.f = &f;
        j.n = n;
        j.helpers = helpers;
        {
            std::lock_guard<std::mutex> g(mu_);
            open_.push_back(&j);
        }
        // wake only as many workers as can take an item (the caller works too)
        for (int64_t k = 0; k < std::min<int64_t>(helpers, n - 1); ++k) work_cv_.notify_one();
        work(&j);
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return j.done.load() == n; });
        open_.erase(std::find(open_.begin(), open_.end(), &j));
        done_cv_.wait(lk, [&] { return j.users == 0; });
    }
};

// Runs f(0..n) on the host's cores (items of `grain` or more per thread).
// f must not throw.
template <class F>
void parallel_for(int64_t n, int64_t grain, F&& f) {
    const int64_t nthreads =
        std::min<int64_t>(std::max(1u, std::thread::hardware_concurrency()), (n + grain - 1) / std::max<int64_t>(grain, 1));
    if (nthreads <= 1) {
        for (int64_t i = 0; i < n; ++i) f(i);
        return;
    }
    const std::function<void(int64_t)> fn = [&](int64_t i) { f(i); };
    HostPool::get().run(n, (int)nthreads - 1, fn);
}

void plan_batch(const Model* const* models, int64_t n, const lcb_datum* data, const int64_t* start,
                const int64_t* count, int num_sms, Plan& P, const PlanTuning& tune) {
    P.reset();
    P.models.resize(n);
    P.model_ok.assign(n, 0);
    P.model_err.assign(n, std::string());
    std::vector<ModelLayout> lay(n);
    auto prep = [&](int64_t i) {
        int64_t nd = count[i];
        try {
            if (nd <= 0) throw Error(LCB_ERR_EMPTY, "no data points");
            prepare_model(*models[i], data + start[i], nd, lay[i]);
            P.model_ok[i] = 1;
        } catch (const std::exception& e) {
            P.model_err[i] = e.what();
            lay[i] = ModelLayout();
            std::memset(&lay[i].dev, 0, sizeof(ModelDev));
            lay[i].dev.status = -1;
        }
    };
    // a bright spot's stream integration (~0.7 ms) outweighs the rest of a model's planning:
    // the batch's pairs (q, radius_spot) missing from the memo are integrated first, one per
    // thread, so that a small batch (an MCMC step over q) does not run them eight to a thread
    {
        std::vector<std::pair<double, double>> need;
        for (int64_t i = 0; i < n; ++i) {
            const Model& m = *models[i];
            double o[3];
            if (m.add_spot && count[i] > 0 && !spot_cached(m.v(P_Q), m.v(P_RADIUS_SPOT), o))
                need.emplace_back(m.v(P_Q), m.v(P_RADIUS_SPOT));
        }
        std::sort(need.begin(), need.end());
        need.erase(std::unique(need.begin(), need.end()), need.end());
        // many new pairs: one GPU thread each (a host core integrates one in ~0.7 ms, a GPU
        // thread in a few; the GPU wins once the host would run more than four per thread)
        const StreamDeviceFn dev = g_stream_device.load();
        const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
        if (dev && (int64_t)need.size() > 4 * hw) {
            std::vector<double> in, res(3 * need.size());
            std::vector<int> st(need.size(), -1);
            std::vector<size_t> which;
            for (size_t k = 0; k < need.size(); ++k) {
                try {
                    const double rl1 = host_xl1(need[k].first);
                    in.insert(in.end(), {need[k].first, rl1, need[k].second});
                    which.push_back(k);
                } catch (const std::exception&) {  // the model's own planning reports it
                }
            }
            if (!which.empty() && dev(in.data(), (int)which.size(), res.data(), st.data())) {
                std::vector<std::pair<double, double>> rest;
                for (size_t j = 0; j < which.size(); ++j) {
                    if (st[j] == stream::kStreamOk) spot_store(need[which[j]].first, need[which[j]].second, &res[3 * j]);
                    else rest.push_back(need[which[j]]);  // failures: the host path reports them
                }
                need.swap(rest);
            }
        }
        parallel_for((int64_t)need.size(), 1, [&](int64_t k) {
            double o[3];
            try {
                stream_to_radius(need[k].first, need[k].second, o);
            } catch (const std::exception&) {  // the model's own planning reports it
            }
        });
    }
    // models are independent: prepare them on the host's cores, 16 at least per thread
    // (one takes ~10 us, so waking helper threads only pays off for larger batches)
    parallel_for(n, 16, prep);
    // sub-phases and data: per-model sums, prefix offsets, then the per-datum
    // arrays of each model filled in parallel
    std::vector<int64_t> dbeg(n + 1, 0), sbeg(n + 1, 0);
    for (int64_t i = 0; i < n; ++i) dbeg[i + 1] = dbeg[i] + std::max<int64_t>(count[i], 0);
    P.ndatum = dbeg[n];
    parallel_for(n, 64, [&](int64_t i) {
        int64_t ns = 0;
        if (P.model_ok[i])
            for (int64_t k = 0; k < dbeg[i + 1] - dbeg[i]; ++k) ns += std::max(data[start[i] + k].ndiv, 0);
        sbeg[i + 1] = ns;
    });
    for (int64_t i = 0; i < n; ++i) {
        if (sbeg[i + 1] > INT32_MAX / 2) throw Error(LCB_ERR_INVALID, "too many sub-phases in one model");
        sbeg[i + 1] += sbeg[i];
    }
    P.datum_model.resize(P.ndatum);
    P.datum_sub0.resize(P.ndatum);
    P.datum_src.resize(P.ndatum);
    parallel_for(n, 64, [&](int64_t i) {
        ModelDev& D = lay[i].dev;
        D.datum_begin = dbeg[i];
        D.ndatum = dbeg[i + 1] - dbeg[i];
        D.sub_begin = sbeg[i];
        D.nsub = sbeg[i + 1] - sbeg[i];
        int64_t sub = sbeg[i];
        for (int64_t k = 0, dd = dbeg[i]; k < D.ndatum; ++k, ++dd) {
            const int64_t src = start[i] + k;
            P.datum_model[dd] = (int32_t)i;
            P.datum_sub0[dd] = sub;
            P.datum_src[dd] = src;
            if (P.model_ok[i]) sub += std::max(data[src].ndiv, 0);
        }
    });
    P.nsub = sbeg[n];
    P.datum_contiguous = true;
    for (int64_t i = 1; i < n && P.datum_contiguous; ++i)
        P.datum_contiguous = start[i] == start[i - 1] + std::max<int64_t>(count[i - 1], 0);

    // global element / table layout (a model's segments are contiguous): offsets of each model's
    // segments, bands, rings and elements, then the tables filled in parallel
    std::vector<size_t> seg_begin(n + 1, 0), band_begin(n + 1, 0), ring_begin(n + 1, 0);
    std::vector<int64_t> elem_begin(n + 1, 0);
    for (int64_t i = 0; i < n; ++i) {
        seg_begin[i + 1] = seg_begin[i] + lay[i].segs.size();
        band_begin[i + 1] = band_begin[i] + lay[i].bands.size();
        ring_begin[i + 1] = ring_begin[i] + lay[i].rings.size();
        elem_begin[i + 1] = elem_begin[i] + lay[i].nelem;
    }
    P.segs.resize(seg_begin[n]);
    P.bands.resize(band_begin[n]);
    P.rings.resize(ring_begin[n]);
    P.nelem = elem_begin[n];
    parallel_for(n, 64, [&](int64_t i) {
        const ModelLayout& L = lay[i];
        std::copy(L.bands.begin(), L.bands.end(), P.bands.begin() + band_begin[i]);
        std::copy(L.rings.begin(), L.rings.end(), P.rings.begin() + ring_begin[i]);
        size_t k = seg_begin[i];
        for (SegDesc s : L.segs) {
            s.first += elem_begin[i];
            s.model = (int32_t)i;
            if (s.kind == SEG_STAR1 || s.kind == SEG_STAR2) s.table += (int32_t)band_begin[i];
            if (s.kind == SEG_DISC) s.table += (int32_t)ring_begin[i];
            P.segs[k++] = s;
        }
    });
    if (P.nelem > ((int64_t)1 << 34)) throw Error(LCB_ERR_INVALID, "batch too large (elements)");

    // element-kernel blocks; Roche ray-march blocks (one per eclipsing Roche star); star-grid aux blocks:
    // counts per segment, prefix offsets, then each segment's blocks written in parallel
    const int64_t nseg = (int64_t)P.segs.size();
    auto roche_by = [&](const SegDesc& g, int by) {
        const ModelDev& D = lay[g.model].dev;
        bool roche = by == 1 ? D.roche1 : D.roche2;
        bool ecl;
        if (g.kind == SEG_STAR1) ecl = by == 2 && D.eclipse1;
        else if (g.kind == SEG_STAR2) ecl = by == 1 && D.eclipse2;
        else ecl = by == 1 ? D.eclipse1 : D.eclipse2;
        return roche && ecl;
    };
    std::vector<int64_t> eb(nseg + 1, 0), ab(nseg + 1, 0), rb(nseg + 1, 0);
    for (int64_t s = 0; s < nseg; ++s) {
        const SegDesc& g = P.segs[s];
        const int64_t ne = (g.count + kElemThreads - 1) / kElemThreads;
        eb[s + 1] = eb[s] + ne;
        ab[s + 1] = ab[s] + ((g.kind == SEG_STAR1 || g.kind == SEG_STAR2) ? ne : 0);
        int64_t nr = 0;
        for (int by = 1; by <= 2; ++by)
            if (roche_by(g, by)) {
                P.roche_elems += g.count;
                nr += (g.count + kRocheBlock - 1) / kRocheBlock;
            }
        rb[s + 1] = rb[s] + nr;
    }
    P.eblocks.resize(eb[nseg]);
    P.ablocks.resize(ab[nseg]);
    P.rblocks.resize(rb[nseg]);
    parallel_for(nseg, 64, [&](int64_t s) {
        const SegDesc& g = P.segs[s];
        int64_t k = eb[s];
        for (int64_t off = 0; off < g.count; off += kElemThreads) P.eblocks[k++] = ElemBlock{(int32_t)s, 0, off};
        k = ab[s];
        if (g.kind == SEG_STAR1 || g.kind == SEG_STAR2)
            for (int64_t off = 0; off < g.count; off += kElemThreads) P.ablocks[k++] = ElemBlock{(int32_t)s, 0, off};
        k = rb[s];
        for (int by = 1; by <= 2; ++by)
            if (roche_by(g, by))
                for (int64_t off = 0; off < g.count; off += kRocheBlock) P.rblocks[k++] = ElemBlock{(int32_t)s, by, off};
    });

    // small batches: spread each element's phase scan over several threads, a power
    // of two up to 16, until about sixteen waves of scan threads fill the GPU (the
    // choices an autotuning of 8..128-model batches made; large batches keep one
    // thread per element, where the scan proves blocks of steps at once)
    {
        const int64_t threads = (int64_t)P.rblocks.size() * kRocheBlock;
        const int64_t target = (int64_t)std::max(num_sms, 1) * 640 * 16;
        int split = 1;
        while (threads > 0 && split < 16 && (int64_t)(2 * split) * threads <= target) split *= 2;
        P.roche_split = split;
        if (tune.roche_split > 0 && threads > 0) P.roche_split = std::min(std::max(tune.roche_split, 1), 16);
    }

    // flux work units: choose the element range so there are a few units per resident block
    int64_t total = 0;
    for (const SegDesc& g : P.segs) total += g.count * lay[g.model].dev.nsub;
    P.evals = total;
    const int64_t resident = (int64_t)std::max(num_sms, 1) * 4;
    int64_t per_unit = std::max<int64_t>(total / (resident * 8), 1);
    int64_t erange = per_unit / kFluxTile;
    erange = std::min<int64_t>(std::max<int64_t>(erange, kFluxChunk), 16 * kFluxChunk);
    erange = (erange + kFluxChunk - 1) / kFluxChunk * kFluxChunk;
    if (tune.flux_chunks > 0) erange = (int64_t)std::min(std::max(tune.flux_chunks, 1), 16) * kFluxChunk;
    P.flux_chunks = (int)(erange / kFluxChunk);
    P.flux_blocks_per_sm = std::max(tune.flux_blocks_per_sm, 0);

    thread_local std::vector<std::pair<int64_t, FluxUnit>> fu;  // scratch kept across calls
    fu.clear();
    int64_t pbase = 0;
    for (int64_t i = 0; i < n; ++i) {
        ModelDev& D = lay[i].dev;
        D.pbase = pbase;
        if (!P.model_ok[i] || D.nsub == 0) { D.nslots = D.g1_end = D.g2_end = D.gd_end = D.ge_end = 0; continue; }
        int32_t slot = 0;
        auto kind_of = [&](const SegDesc& g) {
            if (g.kind == SEG_DISC || g.kind == SEG_EDGE) return (int32_t)UK_DISC;
            if (g.kind == SEG_SPOT) return (int32_t)UK_SPOT;
            bool s1 = g.kind == SEG_STAR1;
            bool generic = s1 ? D.beam1 != 0.0 : (D.beam2 != 0.0 || D.glens1);
            if (generic) return (int32_t)UK_STAR_GENERIC;
            int lt = s1 ? D.ltype1 : D.ltype2;
            if (lt == LIMB_CLARET) return (int32_t)UK_STAR_CLARET;
            int np = s1 ? D.npoly1 : D.npoly2;
            return (int32_t)(UK_STAR_POLY1 + (np - 1));
        };
        // slots grouped by component: star 1, star 2, disc, rim, bright spot
        // (the per-component sums of iscale read them as contiguous ranges)
        for (int pass = 0; pass < 5; ++pass) {
            for (size_t s = seg_begin[i]; s < seg_begin[i + 1]; ++s) {
                const SegDesc& g = P.segs[s];
                int grp = g.kind == SEG_STAR1 ? 0 : g.kind == SEG_STAR2 ? 1 : g.kind == SEG_DISC ? 2
                          : g.kind == SEG_EDGE ? 3 : 4;
                if (grp != pass) continue;
                for (int64_t e = 0; e < g.count; e += erange) {
                    int32_t ne = (int32_t)std::min<int64_t>(erange, g.count - e);
                    for (int64_t t = 0; t < D.nsub; t += kFluxTile) {
                        FluxUnit u{};
                        u.e0 = g.first + e;
                        u.ne = ne;
                        u.model = (int32_t)i;
                        u.t0 = (int32_t)t;
                        u.nt = (int32_t)std::min<int64_t>(kFluxTile, D.nsub - t);
                        u.slot = slot;
                        u.kind = kind_of(g);
                        u.star = g.kind == SEG_STAR1 ? 1 : g.kind == SEG_STAR2 ? 2 : 0;
                        u.role = g.role;
                        fu.push_back({(int64_t)ne * u.nt, u});
                    }
                    ++slot;
                }
            }
            if (pass == 0) D.g1_end = slot;
            if (pass == 1) D.g2_end = slot;
            if (pass == 2) D.gd_end = slot;
            if (pass == 3) D.ge_end = slot;
        }
        D.nslots = slot;
        pbase += (int64_t)slot * D.nsub;
    }
    P.npartial = pbase;
    // largest units first, ties in generation order: a stable LSD radix sort of the keys
    // largest - size (11-bit digits, keys carried with the indices; unit sizes are at most
    // 16 chunks x one tile = 2^21 element-evals, so two passes)
    thread_local std::vector<uint32_t> key, idx, ktmp, itmp;
    const size_t nu = fu.size();
    int64_t largest = 0;
    for (size_t k = 0; k < nu; ++k) largest = std::max(largest, std::min<int64_t>(fu[k].first, INT32_MAX));
    key.resize(nu);
    idx.resize(nu);
    ktmp.resize(nu);
    itmp.resize(nu);
    for (size_t k = 0; k < nu; ++k) {
        key[k] = (uint32_t)(largest - std::min<int64_t>(fu[k].first, INT32_MAX));
        idx[k] = (uint32_t)k;
    }
    for (int shift = 0; shift < 32 && (largest >> shift) > 0; shift += 11) {
        uint32_t count[2049] = {0};
        for (size_t k = 0; k < nu; ++k) ++count[((key[k] >> shift) & 2047u) + 1];
        for (int b = 1; b <= 2048; ++b) count[b] += count[b - 1];
        for (size_t k = 0; k < nu; ++k) {
            const uint32_t pos = count[(key[k] >> shift) & 2047u]++;
            ktmp[pos] = key[k];
            itmp[pos] = idx[k];
        }
        key.swap(ktmp);
        idx.swap(itmp);
    }
    P.units.resize(nu);
    for (size_t k = 0; k < nu; ++k) P.units[k] = fu[idx[k]].second;

    for (int64_t i = 0; i < n; ++i) {
        P.models[i] = lay[i].dev;
        P.any_iscale = P.any_iscale || (P.model_ok[i] && lay[i].dev.iscale);
    }

    // shape key: what the device buffers and the captured graph depend on
    P.shape_key = {n, P.nelem, P.nsub, P.ndatum, P.npartial, (int64_t)P.units.size(), (int64_t)P.eblocks.size(),
                   (int64_t)P.rblocks.size(), (int64_t)P.ablocks.size(), (int64_t)P.segs.size(),
                   (int64_t)P.bands.size(), (int64_t)P.rings.size(), (int64_t)P.roche_split,
                   (int64_t)P.flux_blocks_per_sm};
}

}  // namespace lcb
