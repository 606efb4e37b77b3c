// lcurve_oracle.cpp — FP64 CPU restatement of the lcurve-rs light-curve path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: tests/, the
// smoke check in __graft_entry__.py and the CPU-baseline leg of bench.py may
// load it; the product library (lcurve-rs_b200/) never does.
//
// Every function below restates one function of the reference (scope-ml/
// lcurve-rs) and cites it as crate/path:line.  Arithmetic is written in the
// same evaluation order as the reference so that, compiled with
// -ffp-contract=off (no FMA contraction, as rustc/LLVM does not contract),
// results reproduce the reference's FP64 values.  Storage precision follows
// the reference too: Point.area / gravity / flux are f32 (crates/lcurve/src/
// types.rs:14-20), so values are rounded through float where it does.
//
// Parity pin: tests/test_oracle_golden.py checks light_curve() on the
// reference's test_data/test_model.dat against test_data/test_lc.dat (500
// fluxes written by the original C++ lroche) at max relative error < 1e-6,
// the reference's own bound (tests/regression.rs:84-88).
//
// Parallelism mirrors the reference's Rayon loops: over times inside one
// light curve (crates/lcurve/src/orchestration.rs:229), over models in
// chisq_batch (orchestration.rs:343) and over elements in the continuum
// (brightness.rs:50,119).  The loops nest as Rayon's do: threads that run out
// of models help with the time loops of the models still running.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <condition_variable>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace orc {

// ---------------------------------------------------------------------------
// constants — crates/subs/src/constants.rs:5-95
// ---------------------------------------------------------------------------
static const double C_LIGHT = 2.99792458e8;   // constants.rs:5
static const double H_PLANCK = 6.6262e-34;    // constants.rs:11
static const double K_BOLTZ = 1.3806e-23;     // constants.rs:14
static const double DAY = 86400.0;            // constants.rs:65
static const double PI = 3.14159265358979323846;  // constants.rs:80 (f64 PI)
static const double TWOPI = 2.0 * PI;         // constants.rs:83

static inline double sqr(double x) { return x * x; }  // subs/src/lib.rs:11-14
static inline double sign(double a, double b) { return b >= 0.0 ? std::fabs(a) : -std::fabs(a); }  // lib.rs:17-20
// Rust f64::to_radians / to_degrees (core::f64): x * (PI/180), x * (180/PI).
static inline double to_rad(double x) { return x * (PI / 180.0); }
static inline double to_deg(double x) { return x * (180.0 / PI); }
// Rust powi(3) / powi(4) lower to repeated multiplication.
static inline double powi3(double x) { return (x * x) * x; }
static inline double powi4(double x) { double x2 = x * x; return x2 * x2; }
// Rust `as i32` / `as usize` from f64 saturate (NaN -> 0).
static inline int64_t sat_i32(double x) {
    if (std::isnan(x)) return 0;
    if (x >= 2147483647.0) return 2147483647;
    if (x <= -2147483648.0) return -2147483648LL;
    return (int64_t)x;
}
static inline int64_t sat_usize(double x) {
    if (std::isnan(x) || x <= 0.0) return 0;
    if (x >= 9.2e18) return INT64_MAX;
    return (int64_t)x;
}

struct RocheError : std::runtime_error { using std::runtime_error::runtime_error; };

// ---------------------------------------------------------------------------
// Vec3 — crates/subs/src/vec3.rs:7-120
// ---------------------------------------------------------------------------
struct Vec3 {
    double x = 0, y = 0, z = 0;
    Vec3() {}
    Vec3(double a, double b, double c) : x(a), y(b), z(c) {}
    double sqr() const { return x * x + y * y + z * z; }       // vec3.rs:29-31
    double length() const { return std::sqrt(sqr()); }        // vec3.rs:34-36
    static double dot(const Vec3& a, const Vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }  // vec3.rs:80-82
    bool unit() {                                              // vec3.rs:39-50
        double norm = sqr();
        if (norm > 0.0) { norm = std::sqrt(norm); x /= norm; y /= norm; z /= norm; return true; }
        return false;
    }
};
static inline Vec3 operator+(const Vec3& a, const Vec3& b) { return Vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline Vec3 operator-(const Vec3& a, const Vec3& b) { return Vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline Vec3 operator*(double s, const Vec3& v) { return Vec3(s * v.x, s * v.y, s * v.z); }

// ---------------------------------------------------------------------------
// Instrumentation: counts of the eclipse search's potential evaluations.
// ---------------------------------------------------------------------------
static std::atomic<long long> g_fblink_calls{0}, g_rpot_evals{0}, g_drpot_evals{0};
static thread_local long long t_fblink = 0, t_rpot = 0, t_drpot = 0;
static void flush_counters() {
    g_fblink_calls += t_fblink; g_rpot_evals += t_rpot; g_drpot_evals += t_drpot;
    t_fblink = t_rpot = t_drpot = 0;
}

// ---------------------------------------------------------------------------
// planck — crates/subs/src/planck.rs:4-44
// ---------------------------------------------------------------------------
static const double FAC1 = 2.0e27 * H_PLANCK * C_LIGHT;            // planck.rs:5
static const double FAC2 = 1.0e9 * H_PLANCK * C_LIGHT / K_BOLTZ;   // planck.rs:8
double planck(double wave, double temp) {                          // planck.rs:16-23
    double efac = FAC2 / (wave * temp);
    if (efac > 40.0) return FAC1 * std::exp(-efac) / (wave * sqr(wave));
    return FAC1 / (std::exp(efac) - 1.0) / (wave * sqr(wave));
}
double dlpdlt(double wave, double temp) {                          // planck.rs:40-43
    double efac = FAC2 / (wave * temp);
    return efac / (1.0 - std::exp(-efac));
}

// ---------------------------------------------------------------------------
// Lagrangian points — crates/roche/src/lagrange.rs
// ---------------------------------------------------------------------------
static const int LAG_NMAX = 1000;    // lagrange.rs:3
static const double LAG_EPS = 1.0e-12;  // lagrange.rs:4
static double lag_newton(double x, double a1, double a2, double a3, double a4, double a5, double a6, const char* who) {
    double d1 = a2, d2 = 2.0 * a3, d3 = 3.0 * a4, d4 = 4.0 * a5, d5 = 5.0 * a6;
    for (int i = 0; i < LAG_NMAX; ++i) {
        double xold = x;
        double f = x * (x * (x * (x * (x * a6 + a5) + a4) + a3) + a2) + a1;
        double df = x * (x * (x * (x * d5 + d4) + d3) + d2) + d1;
        x -= f / df;
        if (std::fabs(x - xold) <= LAG_EPS * std::fabs(x)) return x;
    }
    throw RocheError(std::string(who) + ": exceeded maximum iterations");
}
double xl1(double q) {                                  // lagrange.rs:8-32
    if (q <= 0.0) throw RocheError("xl1: q <= 0");
    double mu = q / (1.0 + q);
    return lag_newton(1.0 / (1.0 + q), -1.0 + mu, 2.0 - 2.0 * mu, -1.0 + mu, 1.0 + 2.0 * mu, -2.0 - mu, 1.0, "xl1");
}
double xl11(double q, double spin) {                    // lagrange.rs:89-114
    if (q <= 0.0) throw RocheError("xl11: q <= 0");
    double ssq = spin * spin;
    double mu = q / (1.0 + q);
    return lag_newton(1.0 / (1.0 + q), -1.0 + mu, 2.0 - 2.0 * mu, -1.0 + mu, ssq + 2.0 * mu, -2.0 * ssq - mu, ssq, "xl11");
}
double xl12(double q, double spin) {                    // lagrange.rs:117-142
    if (q <= 0.0) throw RocheError("xl12: q <= 0");
    double ssq = spin * spin;
    double mu = q / (1.0 + q);
    return lag_newton(1.0 / (1.0 + q), -1.0 + mu, 2.0 - 2.0 * mu, -ssq + mu, 3.0 * ssq + 2.0 * mu - 2.0,
                      1.0 - mu - 3.0 * ssq, ssq, "xl12");
}

// ---------------------------------------------------------------------------
// Roche potentials — crates/roche/src/potential.rs
// ---------------------------------------------------------------------------
enum Star { PRIMARY = 0, SECONDARY = 1 };

double rpot(double q, const Vec3& p) {                  // potential.rs:8-19
    if (q <= 0.0) throw RocheError("rpot: q <= 0");
    double mu = q / (1.0 + q);
    double comp = 1.0 - mu;
    double x2y2 = sqr(p.x) + sqr(p.y);
    double r1sq = x2y2 + sqr(p.z);
    double r1 = std::sqrt(r1sq);
    double r2 = std::sqrt(r1sq + 1.0 - 2.0 * p.x);
    return -comp / r1 - mu / r2 - (x2y2 + mu * (mu - 2.0 * p.x)) / 2.0;
}
double rpot1(double q, double spin, const Vec3& p) {    // potential.rs:22-33
    if (q <= 0.0) throw RocheError("rpot1: q <= 0");
    double mu = q / (1.0 + q);
    double comp = 1.0 - mu;
    double x2y2 = sqr(p.x) + sqr(p.y);
    double r1sq = x2y2 + sqr(p.z);
    double r1 = std::sqrt(r1sq);
    double r2 = std::sqrt(r1sq + 1.0 - 2.0 * p.x);
    return -comp / r1 - mu / r2 - sqr(spin) * x2y2 / 2.0 + mu * p.x;
}
double rpot2(double q, double spin, const Vec3& p) {    // potential.rs:36-47
    if (q <= 0.0) throw RocheError("rpot2: q <= 0");
    double mu = q / (1.0 + q);
    double comp = 1.0 - mu;
    double x2y2 = sqr(p.x) + sqr(p.y);
    double r1sq = x2y2 + sqr(p.z);
    double r1 = std::sqrt(r1sq);
    double r2 = std::sqrt(r1sq + 1.0 - 2.0 * p.x);
    return -comp / r1 - mu / r2 - sqr(spin) * (0.5 + 0.5 * x2y2 - p.x) - comp * p.x;
}
Vec3 drpot1(double q, double spin, const Vec3& p) {     // potential.rs:69-86
    if (q <= 0.0) throw RocheError("drpot1: q <= 0");
    double r1sq = p.sqr();
    double r2sq = r1sq + 1.0 - 2.0 * p.x;
    double r1 = std::sqrt(r1sq);
    double r2 = std::sqrt(r2sq);
    double mu = q / (1.0 + q);
    double mu1 = mu / r2 / r2sq;
    double comp = (1.0 - mu) / r1 / r1sq;
    double ssq = sqr(spin);
    return Vec3(comp * p.x + mu1 * (p.x - 1.0) - ssq * p.x + mu,
                comp * p.y + mu1 * p.y - ssq * p.y,
                comp * p.z + mu1 * p.z);
}
Vec3 drpot2(double q, double spin, const Vec3& p) {     // potential.rs:89-106
    if (q <= 0.0) throw RocheError("drpot2: q <= 0");
    double r1sq = p.sqr();
    double r2sq = r1sq + 1.0 - 2.0 * p.x;
    double r1 = std::sqrt(r1sq);
    double r2 = std::sqrt(r2sq);
    double mu = q / (1.0 + q);
    double mu1 = mu / r2 / r2sq;
    double comp = (1.0 - mu) / r1 / r1sq;
    double ssq = sqr(spin);
    return Vec3(comp * p.x + mu1 * (p.x - 1.0) - ssq * (p.x - 1.0) + mu - 1.0,
                comp * p.y + mu1 * p.y - ssq * p.y,
                comp * p.z + mu1 * p.z);
}
// potential.rs:110-117 (errors map to 0.0 via unwrap_or)
static double rpot_along_los(double q, Star star, double spin, const Vec3& earth, const Vec3& p, double lam) {
    ++t_rpot;
    Vec3 point = p + lam * earth;
    try {
        return star == PRIMARY ? rpot1(q, spin, point) : rpot2(q, spin, point);
    } catch (const RocheError&) { return 0.0; }
}
// potential.rs:120-127
static double drpot_along_los(double q, Star star, double spin, const Vec3& earth, const Vec3& p, double lam) {
    ++t_drpot;
    Vec3 point = p + lam * earth;
    Vec3 grad;
    try {
        grad = star == PRIMARY ? drpot1(q, spin, point) : drpot2(q, spin, point);
    } catch (const RocheError&) { grad = Vec3(); }
    return Vec3::dot(grad, earth);
}

// ---------------------------------------------------------------------------
// surface — crates/roche/src/surface.rs
// ---------------------------------------------------------------------------
// surface.rs:14-39 -> (rref, pref)
void ref_sphere(double q, Star star, double spin, double ffac, double& rref, double& pref) {
    double rl1 = star == PRIMARY ? xl11(q, spin) : 1.0 - xl12(q, spin);
    double tref = rl1;
    double surf_r = ffac * tref;
    Vec3 p = star == PRIMARY ? Vec3(surf_r, 0.0, 0.0) : Vec3(1.0 - surf_r, 0.0, 0.0);
    pref = star == PRIMARY ? rpot1(q, spin, p) : rpot2(q, spin, p);
    rref = std::fmin(1.001 * ffac, 1.0) * tref;
}
// surface.rs:54-121 -> posn, dirn (unit normal), radius, gravity
void face(double q, Star star, double spin, const Vec3& dirn, double rref, double pref, double acc,
          Vec3& pvec, Vec3& dvec, double& radius, double& gravity) {
    Vec3 cofm = star == PRIMARY ? Vec3() : Vec3(1.0, 0.0, 0.0);
    auto pot_fn = [&](double r) {
        Vec3 p = cofm + r * dirn;
        return star == PRIMARY ? rpot1(q, spin, p) : rpot2(q, spin, p);
    };
    double lo = rref / 2.0, hi = rref, tref = pref + 1.0;
    for (int i = 0; i < 30; ++i) {
        if (tref <= pref) break;
        lo = hi / 2.0;
        tref = pot_fn(lo);
        if (tref > pref) hi = lo;
    }
    for (int i = 0; i < 100; ++i) {
        if (hi - lo <= acc) break;
        double mid = (lo + hi) / 2.0;
        double pot_mid = pot_fn(mid);
        if (pot_mid < pref) lo = mid; else hi = mid;
    }
    radius = (lo + hi) / 2.0;
    pvec = cofm + radius * dirn;
    Vec3 grad = star == PRIMARY ? drpot1(q, spin, pvec) : drpot2(q, spin, pvec);
    gravity = grad.length();
    dvec = grad;
    dvec.unit();
}

// ---------------------------------------------------------------------------
// dbrent — crates/subs/src/numerical/dbrent.rs:20-165 (ITMAX = 100, line 3)
// Returns false when the iteration cap is reached (the reference's Err).
// ---------------------------------------------------------------------------
template <class F, class D>
static bool dbrent(double ax, double bx, double cx, F&& func, D&& dfunc, double acc, bool stopfast,
                   double fref, double& fmin_out, double& xmin_out) {
    double a = std::fmin(ax, cx), b = std::fmax(ax, cx);
    double x = bx, w = bx, v = bx;
    double fx = func(x), fw = fx, fv = fx;
    if (stopfast && fx < fref) { fmin_out = fx; xmin_out = x; return true; }
    double dx = dfunc(x), dw = dx, dv = dx;
    double e = 0.0, d = 0.0;
    for (int it = 0; it < 100; ++it) {
        double xm = 0.5 * (a + b);
        double tol1 = acc;
        double tol2 = 2.0 * tol1;
        if (std::fabs(x - xm) <= tol2 - 0.5 * (b - a)) { fmin_out = fx; xmin_out = x; return true; }
        if (std::fabs(e) > tol1) {
            double d1 = 2.0 * (b - a), d2 = d1;
            if (dw != dx) d1 = (w - x) * dx / (dx - dw);
            if (dv != dx) d2 = (v - x) * dx / (dx - dv);
            double u1 = x + d1, u2 = x + d2;
            bool ok1 = (a - u1) * (u1 - b) > 0.0 && dx * d1 <= 0.0;
            bool ok2 = (a - u2) * (u2 - b) > 0.0 && dx * d2 <= 0.0;
            double olde = e;
            e = d;
            if (ok1 || ok2) {
                if (ok1 && ok2) d = std::fabs(d1) < std::fabs(d2) ? d1 : d2;
                else if (ok1) d = d1;
                else d = d2;
                if (std::fabs(d) <= std::fabs(0.5 * olde)) {
                    double u = x + d;
                    if (u - a < tol2 || b - u < tol2) d = sign(tol1, xm - x);
                } else {
                    e = dx >= 0.0 ? a - x : b - x;
                    d = 0.5 * e;
                }
            } else {
                e = dx >= 0.0 ? a - x : b - x;
                d = 0.5 * e;
            }
        } else {
            e = dx >= 0.0 ? a - x : b - x;
            d = 0.5 * e;
        }
        double u, fu;
        if (std::fabs(d) >= tol1) {
            u = x + d;
            fu = func(u);
            if (stopfast && fu < fref) { fmin_out = fu; xmin_out = u; return true; }
        } else {
            u = x + sign(tol1, d);
            fu = func(u);
            if (stopfast && fu < fref) { fmin_out = fu; xmin_out = u; return true; }
            if (fu > fx) { fmin_out = fx; xmin_out = x; return true; }
        }
        double du = dfunc(u);
        if (fu <= fx) {
            if (u >= x) a = x; else b = x;
            v = w; fv = fw; dv = dw;
            w = x; fw = fx; dw = dx;
            x = u; fx = fu; dx = du;
        } else {
            if (u < x) a = u; else b = u;
            if (fu <= fw || w == x) {
                v = w; fv = fw; dv = dw;
                w = u; fw = fu; dw = du;
            } else if (fu < fv || v == x || v == w) {
                v = u; fv = fu; dv = du;
            }
        }
    }
    return false;
}

// ---------------------------------------------------------------------------
// eclipse — crates/roche/src/eclipse.rs
// ---------------------------------------------------------------------------
// misc.rs:42-45
static inline Vec3 set_earth_cosi_sini(double cosi, double sini, double phase) {
    double phi = TWOPI * phase;
    return Vec3(sini * std::cos(phi), -sini * std::sin(phi), cosi);
}
// eclipse.rs:202-224
static bool sphere_eclipse_los(const Vec3& earth, const Vec3& r, const Vec3& c, double rsphere,
                               double& lam1, double& lam2) {
    Vec3 d = r - c;
    double bquad = Vec3::dot(earth, d);
    if (bquad >= 0.0) return false;
    double cquad = d.sqr() - sqr(rsphere);
    double fac = sqr(bquad) - cquad;
    if (fac <= 0.0) return false;
    fac = std::sqrt(fac);
    lam2 = -bquad + fac;
    lam1 = std::fmax(cquad / lam2, 0.0);
    return true;
}
// eclipse.rs:229-265
bool sphere_eclipse_phase(double cosi, double sini, const Vec3& r, const Vec3& c, double rsphere,
                          double& phi1, double& phi2, double& lam1, double& lam2) {
    Vec3 d = r - c;
    double pdist = std::sqrt(sqr(d.x) + sqr(d.y));
    double bquad = d.z * cosi - pdist * sini;
    if (bquad >= 0.0) return false;
    double cquad = d.sqr() - sqr(rsphere);
    double fac = sqr(bquad) - cquad;
    if (fac <= 0.0) return false;
    fac = std::sqrt(fac);
    lam2 = -bquad + fac;
    lam1 = std::fmax(cquad / lam2, 0.0);
    if (cquad < 0.0) {
        phi1 = 0.0; phi2 = 1.0;
    } else {
        double delta = std::acos((cosi * d.z + std::sqrt(cquad)) / (sini * pdist));
        double phi = std::atan2(d.y, -d.x);
        double p1 = (phi - delta) / TWOPI;
        p1 -= std::floor(p1);
        phi1 = p1;
        phi2 = p1 + 2.0 * delta / TWOPI;
    }
    return true;
}

// Per-star Roche constants that the reference recomputes inside every fblink
// call (eclipse.rs:132, 279); they are pure functions of (q, star, spin, ffac).
struct RocheStar {
    double q, spin, ffac, rref, pref;
    Star star;
    Vec3 cofm;
};
static RocheStar make_roche_star(double q, Star star, double spin, double ffac) {
    RocheStar rs;
    rs.q = q; rs.star = star; rs.spin = spin; rs.ffac = ffac;
    ref_sphere(q, star, spin, ffac, rs.rref, rs.pref);
    rs.cofm = star == PRIMARY ? Vec3() : Vec3(1.0, 0.0, 0.0);
    return rs;
}

// eclipse.rs:123-197
static bool fblink(const RocheStar& rs, double acc, const Vec3& earth, const Vec3& p) {
    ++t_fblink;
    double lam1, lam2;
    if (!sphere_eclipse_los(earth, p, rs.cofm, rs.rref, lam1, lam2)) return false;
    if (lam1 == 0.0) return true;
    const double pref = rs.pref;
    auto func = [&](double lam) { return rpot_along_los(rs.q, rs.star, rs.spin, earth, p, lam); };
    size_t nstep = 1;
    double step_size = lam2 - lam1;
    double f1 = 0.0, f2 = 0.0, flam = 1.0, lam = lam1;
    while (step_size > acc) {
        lam = lam1 + step_size / 2.0;
        bool bracketted = false;
        for (size_t n = 0; n < nstep; ++n) {
            flam = func(lam + (double)n * step_size);
            if (flam <= pref) return true;
            if (nstep == 1) { f1 = func(lam1); f2 = func(lam2); }
            if (flam < f1 && flam < f2) {
                lam = lam + (double)n * step_size;
                bracketted = true;
                break;
            }
        }
        if (bracketted) break;
        step_size /= 2.0;
        nstep *= 2;
    }
    if (flam < f1 && flam < f2) {
        double fmin, xmin;
        auto dfunc = [&](double x) { return drpot_along_los(rs.q, rs.star, rs.spin, earth, p, x); };
        if (dbrent(lam1, lam, lam2, func, dfunc, acc, true, pref, fmin, xmin)) return fmin < pref;
        return false;
    }
    return false;
}

// eclipse.rs:347-373
static bool pot_min_search(const RocheStar& rs, double cosi, double sini, const Vec3& r,
                           double phi1, double phi2, double acc, double& phi_out) {
    int64_t nsteps = sat_usize(std::ceil((phi2 - phi1) / (acc / TWOPI)));
    nsteps = std::min<int64_t>(std::max<int64_t>(nsteps, 10), 1000);
    double dphi = (phi2 - phi1) / (double)nsteps;
    for (int64_t i = 0; i <= nsteps; ++i) {
        double phi = phi1 + (double)i * dphi;
        Vec3 earth = set_earth_cosi_sini(cosi, sini, phi);
        if (fblink(rs, acc, earth, r)) { phi_out = phi; return true; }
    }
    return false;
}

// eclipse.rs:270-338
static bool ingress_egress(const RocheStar& rs, double iangle, double delta, const Vec3& r,
                           double& ingress_out, double& egress_out) {
    double irad = to_rad(iangle);
    double cosi = std::cos(irad), sini = std::sin(irad);
    double phi1, phi2, lam1, lam2;
    if (!sphere_eclipse_phase(cosi, sini, r, rs.cofm, rs.rref, phi1, phi2, lam1, lam2)) return false;
    double acc = 2.0 * std::sqrt(2.0 * TWOPI * (lam2 - lam1) * delta);
    double phi;
    if (!pot_min_search(rs, cosi, sini, r, phi1, phi2, acc, phi)) return false;
    double pin = phi, pout = phi1;
    while (std::fabs(pin - pout) > delta) {
        double pmid = (pin + pout) / 2.0;
        Vec3 earth = set_earth_cosi_sini(cosi, sini, pmid);
        if (fblink(rs, acc, earth, r)) pin = pmid; else pout = pmid;
    }
    double ingress = (pin + pout) / 2.0;
    ingress -= std::floor(ingress);
    pin = phi; pout = phi2;
    while (std::fabs(pin - pout) > delta) {
        double pmid = (pin + pout) / 2.0;
        Vec3 earth = set_earth_cosi_sini(cosi, sini, pmid);
        if (fblink(rs, acc, earth, r)) pin = pmid; else pout = pmid;
    }
    double egress = (pin + pout) / 2.0;
    egress -= std::floor(egress);
    if (egress < ingress) egress += 1.0;
    ingress_out = ingress; egress_out = egress;
    return true;
}

// ---------------------------------------------------------------------------
// disc eclipse — crates/roche/src/disc_eclipse.rs
// ---------------------------------------------------------------------------
enum Circle { C_ABOVE, C_INSIDE, C_OUTSIDE, C_SEPARATE, C_CROSSING };
static double cut_phase(double rxy, double rcone, double radius) {  // disc_eclipse.rs:29-32
    double cos_val = (sqr(rxy) + sqr(rcone) - sqr(radius)) / (2.0 * rcone * rxy);
    return std::acos(std::fmin(std::fmax(cos_val, -1.0), 1.0)) / TWOPI;
}
static Circle circle_eclipse(double rxy, double z, double zcirc, double radius, double tani, double& phase) {  // 44-70
    phase = 0.0;
    if (z >= zcirc) return C_ABOVE;
    double rcone = tani * (zcirc - z);
    if (rcone >= rxy + radius) return C_OUTSIDE;
    if (rxy >= rcone + radius) return C_SEPARATE;
    if (rxy + rcone <= radius) return C_INSIDE;
    phase = cut_phase(rxy, rcone, radius);
    return C_CROSSING;
}
typedef std::vector<std::pair<double, double>> EclipseVec;
// disc_eclipse.rs:84-330
EclipseVec disc_eclipse(double iangle, double rdisc1, double rdisc2, double beta, double height, const Vec3& r) {
    EclipseVec temp;
    double hout = height * std::pow(rdisc2, beta);
    if (r.z >= hout) return temp;
    double irad = iangle * PI / 180.0;
    double sini = std::sin(irad), cosi = std::cos(irad);
    if (cosi == 0.0) {
        if (std::fabs(r.z) < hout) {
            double rxy = std::sqrt(sqr(r.x) + sqr(r.y));
            if (rxy <= rdisc2) {
                temp.push_back({0.0, 1.0});
            } else {
                double subtend = std::asin(rdisc2 / rxy) / TWOPI;
                double pcen = std::atan2(r.y, -r.x) / TWOPI;
                double ingress = pcen - subtend;
                ingress = ingress - std::floor(ingress);
                temp.push_back({ingress, ingress + 2.0 * subtend});
            }
        }
        return temp;
    }
    double rxy = std::sqrt(sqr(r.x) + sqr(r.y));
    if (rdisc1 < rxy && rxy < rdisc2 && std::fabs(r.z) < height * std::pow(rxy, beta)) {
        temp.push_back({0.0, 1.1});
        return temp;
    }
    double tani = sini / cosi;
    if (rxy < rdisc2 && r.z >= height * std::pow(std::fmax(rdisc1, rxy), beta)) {
        double phase;
        Circle result = circle_eclipse(rxy, r.z, hout, rdisc2, tani, phase);
        if (result == C_OUTSIDE) {
            temp.push_back({0.0, 1.1});
        } else if (result == C_CROSSING) {
            double phi0 = std::atan2(r.y, -r.x) / TWOPI;
            double ingress = phi0 + phase;
            ingress = ingress - std::floor(ingress);
            temp.push_back({ingress, ingress + 1.0 - 2.0 * phase});
        }
        return temp;
    }
    double rcone_lo = std::fmax(tani * (-hout - r.z), 0.0);
    if (rcone_lo >= rxy + rdisc2) return temp;
    double rcone_hi = tani * (hout - r.z);
    if (rxy >= rcone_hi + rdisc2) return temp;
    double eclipse_phase;
    if (rxy + rcone_lo <= rdisc2) {
        eclipse_phase = 0.5;
    } else if (rxy <= rdisc2) {
        eclipse_phase = cut_phase(rxy, rcone_lo, rdisc2);
    } else {
        if (sqr(rcone_hi) + sqr(rdisc2) >= sqr(rxy) && sqr(rcone_lo) + sqr(rdisc2) <= sqr(rxy)) {
            eclipse_phase = std::asin(rdisc2 / rxy) / TWOPI;
        } else if (sqr(rcone_hi) + sqr(rdisc2) < sqr(rxy)) {
            eclipse_phase = cut_phase(rxy, rcone_hi, rdisc2);
        } else {
            eclipse_phase = cut_phase(rxy, rcone_lo, rdisc2);
        }
    }
    double hin = height * std::pow(rdisc1, beta);
    double appear_phase = -1.0;
    auto step = [&](double zc, double rad) {
        double phase;
        Circle result = circle_eclipse(rxy, r.z, zc, rad, tani, phase);
        if (result == C_CROSSING) appear_phase = std::fmin(appear_phase, phase);
        else if (result != C_INSIDE) appear_phase = -1.0;
    };
    auto first = [&](double zc, double rad) {
        double phase;
        Circle result = circle_eclipse(rxy, r.z, zc, rad, tani, phase);
        if (result == C_INSIDE) appear_phase = 0.5;
        else if (result == C_CROSSING) appear_phase = phase;
    };
    if (r.z < -hout) {
        first(-hout, rdisc2);
        if (appear_phase > 0.0) step(-hin, rdisc1);
        if (appear_phase > 0.0) step(hin, rdisc1);
        if (appear_phase > 0.0) step(hout, rdisc2);
    } else if (rxy < rdisc1) {
        if (r.z < -hin) {
            first(-hin, rdisc1);
            if (appear_phase > 0.0) step(hin, rdisc1);
            if (appear_phase > 0.0) step(hout, rdisc2);
        } else if (r.z < hin) {
            first(hin, rdisc1);
            if (appear_phase > 0.0) step(hout, rdisc2);
        }
    }
    double phi0 = std::atan2(r.y, -r.x) / TWOPI;
    if (appear_phase <= 0.0) {
        double ingress = phi0 - eclipse_phase;
        ingress = ingress - std::floor(ingress);
        temp.push_back({ingress, ingress + 2.0 * eclipse_phase});
    } else if (appear_phase < eclipse_phase) {
        double ingress = phi0 - eclipse_phase;
        ingress = ingress - std::floor(ingress);
        temp.push_back({ingress, ingress + (eclipse_phase - appear_phase)});
        ingress = phi0 + appear_phase;
        ingress = ingress - std::floor(ingress);
        temp.push_back({ingress, ingress + (eclipse_phase - appear_phase)});
    }
    return temp;
}

// ---------------------------------------------------------------------------
// Bulirsch-Stoer — crates/subs/src/numerical/bsstep.rs:1-324
// ---------------------------------------------------------------------------
static const int KMAXX = 8, IMAXX = KMAXX + 1;
static const int NSEQ[IMAXX] = {2, 4, 6, 8, 10, 12, 14, 16, 18};
static const double SAFE1 = 0.25, SAFE2 = 0.7, REDMAX = 1.0e-5, REDMIN = 0.7, TINY = 1.0e-30, SCALMX = 0.1;
struct BsState {                                          // bsstep.rs:15-48
    bool first = true;
    int kmax = 0, kopt = 0;
    double epsold = -1.0, xnew = -1.0e29;
    double a[IMAXX] = {0};
    double alf[KMAXX][KMAXX] = {{0}};
};
typedef std::function<void(double, const double*, double*)> Derivs;
static void mmid(const double* y, const double* dydx, int nv, double xs, double htot, int nstep, double* yout,
                 const Derivs& derivs) {                  // bsstep.rs:57-93
    double h = htot / (double)nstep;
    double ym[8], yn[8];
    for (int i = 0; i < nv; ++i) { ym[i] = y[i]; yn[i] = y[i] + h * dydx[i]; }
    double x = xs + h;
    derivs(x, yn, yout);
    double h2 = 2.0 * h;
    for (int s = 1; s < nstep; ++s) {
        for (int i = 0; i < nv; ++i) { double swap = ym[i] + h2 * yout[i]; ym[i] = yn[i]; yn[i] = swap; }
        x += h;
        derivs(x, yn, yout);
    }
    for (int i = 0; i < nv; ++i) yout[i] = 0.5 * (ym[i] + yn[i] + h * yout[i]);
}
static void pzextr(int iest, double xest, const double* yest, double* yz, double* dy, int nv,
                   double d_tab[][KMAXX + 1], double* x_tab) {   // bsstep.rs:96-149
    x_tab[iest] = xest;
    for (int j = 0; j < nv; ++j) { dy[j] = yest[j]; yz[j] = yest[j]; }
    if (iest == 0) {
        for (int j = 0; j < nv; ++j) d_tab[j][0] = yest[j];
    } else {
        double c[8];
        for (int j = 0; j < nv; ++j) c[j] = yest[j];
        for (int k1 = 0; k1 < iest; ++k1) {
            double delta = 1.0 / (x_tab[iest - k1 - 1] - xest);
            double f1 = xest * delta;
            double f2 = x_tab[iest - k1 - 1] * delta;
            for (int j = 0; j < nv; ++j) {
                double qv = d_tab[j][k1];
                d_tab[j][k1] = dy[j];
                double delta_val = c[j] - qv;
                dy[j] = f1 * delta_val;
                c[j] = f2 * delta_val;
                yz[j] += dy[j];
            }
        }
        for (int j = 0; j < nv; ++j) d_tab[j][iest] = dy[j];
    }
}
// bsstep.rs:159-324; returns (hdid, hnext)
static void bsstep(double* y, const double* dydx, int nv, double& xx, double htry, double eps,
                   const double* yscal, BsState& st, const Derivs& derivs, double& hdid_out, double& hnext_out) {
    double yerr[8], ysav[8], yseq[8];
    double err[KMAXX] = {0};
    double d_tab[8][KMAXX + 1];
    double x_tab[KMAXX + 1];
    for (int i = 0; i < 8; ++i) for (int j = 0; j <= KMAXX; ++j) d_tab[i][j] = 0.0;
    for (int j = 0; j <= KMAXX; ++j) x_tab[j] = 0.0;
    if (eps != st.epsold) {
        st.xnew = -1.0e29;
        double eps1 = SAFE1 * eps;
        st.a[0] = NSEQ[0] + 1.0;
        for (int k = 0; k < KMAXX; ++k) st.a[k + 1] = st.a[k] + (double)NSEQ[k + 1];
        for (int iq = 1; iq < KMAXX; ++iq)
            for (int k = 0; k < iq; ++k)
                st.alf[k][iq] = std::pow(eps1, (st.a[k + 1] - st.a[iq + 1]) /
                                                   ((st.a[iq + 1] - st.a[0] + 1.0) * (double)(2 * k + 3)));
        st.epsold = eps;
        st.kopt = 1;
        for (int kopt = 1; kopt < KMAXX - 1; ++kopt) {
            if (st.a[kopt + 1] > st.a[kopt] * st.alf[kopt - 1][kopt]) { st.kopt = kopt; break; }
            st.kopt = kopt;
        }
        st.kmax = st.kopt;
    }
    double h = htry;
    for (int i = 0; i < nv; ++i) ysav[i] = y[i];
    if (xx != st.xnew || h != st.xnew) { st.first = true; st.kopt = st.kmax; }
    bool reduct = false;
    int km = 0;
    for (;;) {
        bool exitflag = false;
        for (int k = 0; k <= st.kmax; ++k) {
            st.xnew = xx + h;
            if (st.xnew == xx) { hdid_out = 0.0; hnext_out = 0.0; return; }
            mmid(ysav, dydx, nv, xx, h, NSEQ[k], yseq, derivs);
            double xest = sqr(h / (double)NSEQ[k]);
            pzextr(k, xest, yseq, y, yerr, nv, d_tab, x_tab);
            if (k != 0) {
                double errmax = TINY;
                for (int i = 0; i < nv; ++i) errmax = std::fmax(errmax, std::fabs(yerr[i] / yscal[i]));
                errmax /= eps;
                km = k - 1;
                err[km] = std::pow(errmax / SAFE1, 1.0 / (double)(2 * km + 3));
            }
            int koptm1 = st.kopt > 0 ? st.kopt - 1 : 0;
            if (k != 0 && (k >= koptm1 || st.first)) {
                if (err[km] != 0.0) {
                    double errmax = TINY;
                    for (int i = 0; i < nv; ++i) errmax = std::fmax(errmax, std::fabs(yerr[i] / yscal[i]));
                    errmax /= eps;
                    if (errmax < 1.0) { exitflag = true; break; }
                }
                if (k == st.kmax || k == st.kopt + 1) break;
                else if (k == st.kopt && st.alf[st.kopt - 1][st.kopt] < err[km]) break;
                else if (st.kopt == st.kmax && st.alf[km][st.kmax - 1] < err[km]) break;
                else if (st.alf[km][st.kopt] < err[km]) break;
            }
        }
        if (exitflag) break;
        double red;
        if (err[km] > 0.0) { red = SAFE2 / err[km]; red = std::fmin(std::fmax(red, REDMAX), REDMIN); }
        else red = REDMIN;
        h *= red;
        reduct = true;
    }
    xx = st.xnew;
    double hdid = h;
    st.first = false;
    double wrkmin = 1.0e35, scale = 1.0;
    for (int kk = 0; kk <= km; ++kk) {
        double fact = std::fmax(err[kk], SCALMX);
        double work = fact * st.a[kk + 1];
        if (work < wrkmin) { scale = fact; wrkmin = work; st.kopt = kk + 1; }
    }
    double hnext = h / scale;
    int k_final = km + 1;
    if (st.kopt >= k_final && st.kopt != st.kmax && !reduct) {
        double fact = std::fmax(scale / st.alf[st.kopt - 1][st.kopt], SCALMX);
        if (st.a[st.kopt + 1] * fact <= wrkmin) { hnext = h / fact; st.kopt += 1; }
    }
    hdid_out = hdid; hnext_out = hnext;
}

// ---------------------------------------------------------------------------
// gas stream — crates/roche/src/stream.rs, misc.rs:4-19
// ---------------------------------------------------------------------------
static Vec3 rocacc(double q, const Vec3& r, const Vec3& v) {   // misc.rs:4-19
    double f1 = 1.0 / (1.0 + q);
    double f2 = f1 * q;
    double yzsq = sqr(r.y) + sqr(r.z);
    double r1sq = sqr(r.x) + yzsq;
    double r2sq = sqr(r.x - 1.0) + yzsq;
    double fm1 = f1 / (r1sq * std::sqrt(r1sq));
    double fm2 = f2 / (r2sq * std::sqrt(r2sq));
    double fm3 = fm1 + fm2;
    return Vec3(-fm3 * r.x + fm2 + 2.0 * v.y + r.x - f2, -fm3 * r.y - 2.0 * v.x + r.y, -fm3 * r.z);
}
static void rocder(double q, double, const double* y, double* dydt) {  // stream.rs:65-77
    Vec3 r(y[0], y[1], y[2]), v(y[3], y[4], y[5]);
    dydt[0] = v.x; dydt[1] = v.y; dydt[2] = v.z;
    Vec3 a = rocacc(q, r, v);
    dydt[3] = a.x; dydt[4] = a.y; dydt[5] = a.z;
}
void strinit(double q, Vec3& r, Vec3& v) {                      // stream.rs:8-20
    const double SMALL = 1.0e-5;
    double rl1 = xl1(q);
    double mu = q / (1.0 + q);
    double a = (1.0 - mu) / powi3(rl1) + mu / powi3(1.0 - rl1);
    double lambda1 = std::sqrt(((a - 2.0) + std::sqrt(a * (9.0 * a - 8.0))) / 2.0);
    double m1 = (lambda1 * lambda1 - 2.0 * a - 1.0) / (2.0 * lambda1);
    r = Vec3(rl1 - SMALL, -m1 * SMALL, 0.0);
    v = Vec3(-lambda1 * SMALL, -lambda1 * m1 * SMALL, 0.0);
}
static void gsint(double q, Vec3& r, Vec3& v, double ttry, double& time, double eps, BsState& st,
                  double& tdid, double& tnext) {                // stream.rs:26-62
    double y[6] = {r.x, r.y, r.z, v.x, v.y, v.z};
    double dydt[6];
    rocder(q, time, y, dydt);
    double yscal[6] = {1, 1, 1, 1, 1, 1};
    Derivs d = [q](double t, const double* yi, double* dy) { rocder(q, t, yi, dy); };
    bsstep(y, dydt, 6, time, ttry, eps, yscal, st, d, tdid, tnext);
    r = Vec3(y[0], y[1], y[2]);
    v = Vec3(y[3], y[4], y[5]);
}
double stradv(double q, Vec3& r, Vec3& v, double rad, double acc, double smax) {  // stream.rs:82-145
    const double EPS = 1.0e-8, TMAX = 10.0;
    BsState st;
    double rinit = r.length(), rnow = rinit, time = 0.0, tnext = 1.0e-2;
    for (;;) {
        Vec3 ro = r, vo = v;
        double ttry = std::fmin(tnext, smax);
        double tdid, tn;
        gsint(q, r, v, ttry, time, EPS, st, tdid, tn);
        tnext = tn;
        rnow = r.length();
        if ((rinit > rad && rnow <= rad) || (rinit < rad && rnow >= rad)) {
            double lo = 0.0, hi = tdid, rlo = ro.length(), rhi = rnow;
            double to = time - tdid;
            int guard = 0;
            while (std::fabs(rhi - rlo) > acc) {
                double tmid = (lo + hi) / 2.0;
                r = ro; v = vo;
                double t = to;
                BsState st2;
                double a1, a2;
                gsint(q, r, v, tmid, t, EPS, st2, a1, a2);
                rnow = r.length();
                if ((rhi > rad && rnow > rad) || (rhi < rad && rnow < rad)) { rhi = rnow; hi = tmid; }
                else { rlo = rnow; lo = tmid; }
                if (++guard > 100000) throw RocheError("stradv: binary chop failed to converge");
            }
            return time;
        }
        if (time > TMAX) throw RocheError("stradv: took too long without crossing radius");
    }
}

// ---------------------------------------------------------------------------
// Model — crates/lcurve/src/model.rs
// ---------------------------------------------------------------------------
struct Pparam { double value = 0, range = 0, dstep = 0; bool vary = false, defined = false; };  // model.rs:7-19

// Physical parameter names in the reference's declaration order (model.rs:66-137).
static const char* PHYS_NAMES[] = {
    "q", "iangle", "r1", "r2", "cphi3", "cphi4", "spin1", "spin2",
    "t1", "t2", "ldc1_1", "ldc1_2", "ldc1_3", "ldc1_4",
    "ldc2_1", "ldc2_2", "ldc2_3", "ldc2_4",
    "velocity_scale", "beam_factor1", "beam_factor2",
    "t0", "period", "pdot", "deltat",
    "gravity_dark1", "gravity_dark2", "absorb",
    "slope", "quad", "cube", "third",
    "rdisc1", "rdisc2", "height_disc", "beta_disc",
    "temp_disc", "texp_disc", "lin_limb_disc", "quad_limb_disc",
    "temp_edge", "absorb_edge",
    "radius_spot", "length_spot", "height_spot",
    "expon_spot", "epow_spot", "angle_spot", "yaw_spot",
    "temp_spot", "tilt_spot", "cfrac_spot",
    "stsp11_long", "stsp11_lat", "stsp11_fwhm", "stsp11_tcen",
    "stsp12_long", "stsp12_lat", "stsp12_fwhm", "stsp12_tcen",
    "stsp13_long", "stsp13_lat", "stsp13_fwhm", "stsp13_tcen",
    "stsp21_long", "stsp21_lat", "stsp21_fwhm", "stsp21_tcen",
    "stsp22_long", "stsp22_lat", "stsp22_fwhm", "stsp22_tcen",
    "uesp_long1", "uesp_long2", "uesp_lathw", "uesp_taper", "uesp_temp",
};
static const int NPHYS = sizeof(PHYS_NAMES) / sizeof(PHYS_NAMES[0]);
enum P {
    Q, IANGLE, R1, R2, CPHI3, CPHI4, SPIN1, SPIN2, T1, T2, LDC1_1, LDC1_2, LDC1_3, LDC1_4,
    LDC2_1, LDC2_2, LDC2_3, LDC2_4, VELOCITY_SCALE, BEAM_FACTOR1, BEAM_FACTOR2,
    T0, PERIOD, PDOT, DELTAT, GRAVITY_DARK1, GRAVITY_DARK2, ABSORB, SLOPE, QUAD, CUBE, THIRD,
    RDISC1, RDISC2, HEIGHT_DISC, BETA_DISC, TEMP_DISC, TEXP_DISC, LIN_LIMB_DISC, QUAD_LIMB_DISC,
    TEMP_EDGE, ABSORB_EDGE, RADIUS_SPOT, LENGTH_SPOT, HEIGHT_SPOT, EXPON_SPOT, EPOW_SPOT, ANGLE_SPOT,
    YAW_SPOT, TEMP_SPOT, TILT_SPOT, CFRAC_SPOT,
    STSP11_LONG, STSP11_LAT, STSP11_FWHM, STSP11_TCEN, STSP12_LONG, STSP12_LAT, STSP12_FWHM, STSP12_TCEN,
    STSP13_LONG, STSP13_LAT, STSP13_FWHM, STSP13_TCEN, STSP21_LONG, STSP21_LAT, STSP21_FWHM, STSP21_TCEN,
    STSP22_LONG, STSP22_LAT, STSP22_FWHM, STSP22_TCEN, UESP_LONG1, UESP_LONG2, UESP_LATHW, UESP_TAPER, UESP_TEMP,
};
static const char* COMP_NAMES[] = {  // model.rs:228-234
    "delta_phase", "nlat1f", "nlat2f", "nlat1c", "nlat2c",
    "npole", "nlatfill", "nlngfill", "lfudge", "llo", "lhi",
    "phase1", "phase2", "wavelength",
    "roche1", "roche2", "eclipse1", "eclipse2", "glens1",
    "use_radii", "tperiod", "gdark_bolom1", "gdark_bolom2",
    "mucrit1", "mucrit2", "limb1", "limb2",
    "mirror", "add_disc", "nrad", "opaque", "add_spot", "nspot", "iscale",
};
static const int NCOMP = sizeof(COMP_NAMES) / sizeof(COMP_NAMES[0]);

struct Model {                                             // model.rs:66-182
    Pparam p[NPHYS];
    double delta_phase = 0, lfudge = 0, llo = 0, lhi = 0, phase1 = 0, phase2 = 0, wavelength = 0, tperiod = 0;
    double mucrit1 = 0, mucrit2 = 0;
    int nlat1f = 0, nlat2f = 0, nlat1c = 0, nlat2c = 0, nlatfill = 0, nlngfill = 0, nrad = 0, nspot = 0;
    bool npole = false, roche1 = false, roche2 = false, eclipse1 = false, eclipse2 = false, glens1 = false;
    bool use_radii = false, gdark_bolom1 = false, gdark_bolom2 = false, mirror = false, add_disc = false;
    bool opaque = false, add_spot = false, iscale = false;
    int limb1 = 0, limb2 = 0;  // 0 = Poly, 1 = Claret (types.rs:62-68)
    double v(int i) const { return p[i].value; }
};

struct ParseError : std::runtime_error { using std::runtime_error::runtime_error; };

static std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n\v\f");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n\v\f");
    return s.substr(a, b - a + 1);
}
static std::vector<std::string> split_ws(const std::string& s) {
    std::vector<std::string> out;
    std::istringstream is(s);
    std::string t;
    while (is >> t) out.push_back(t);
    return out;
}
// Rust's f64::from_str: decimal / exponent forms, inf / nan words; no hex, no whitespace.
static bool rust_parse_f64(const std::string& s, double& out) {
    if (s.empty()) return false;
    std::string t = s;
    size_t i = (t[0] == '+' || t[0] == '-') ? 1 : 0;
    std::string body = t.substr(i);
    std::string low;
    for (char c : body) low += (char)std::tolower((unsigned char)c);
    if (low == "inf" || low == "infinity") { out = (t[0] == '-') ? -INFINITY : INFINITY; return true; }
    if (low == "nan") { out = NAN; return true; }
    for (char c : body) if (!(std::isdigit((unsigned char)c) || c == '.' || c == 'e' || c == 'E' || c == '+' || c == '-')) return false;
    char* end = nullptr;
    out = std::strtod(t.c_str(), &end);
    return end && *end == '\0' && end != t.c_str();
}
static double parse_double(const std::string& s) {        // model.rs:55-57
    double v;
    if (!rust_parse_f64(trim(s), v)) throw ParseError("bad double: '" + s + "'");
    return v;
}
static int parse_int(const std::string& s) {              // model.rs:59-61
    std::string t = trim(s);
    if (t.empty()) throw ParseError("bad int: '" + s + "'");
    size_t i = (t[0] == '+' || t[0] == '-') ? 1 : 0;
    if (i == t.size()) throw ParseError("bad int: '" + s + "'");
    for (size_t k = i; k < t.size(); ++k) if (!std::isdigit((unsigned char)t[k])) throw ParseError("bad int: '" + s + "'");
    long long v = std::strtoll(t.c_str(), nullptr, 10);
    if (v > 2147483647LL || v < -2147483648LL) throw ParseError("bad int: '" + s + "'");
    return (int)v;
}
static bool parse_bool(const std::string& s) {            // model.rs:48-53
    std::string t = trim(s);
    if (t == "1" || t == "true" || t == "yes") return true;
    if (t == "0" || t == "false" || t == "no") return false;
    throw ParseError("bad bool: '" + s + "'");
}
static Pparam parse_pparam(const std::string& s) {        // model.rs:23-38
    auto parts = split_ws(s);
    if (parts.size() < 4) throw ParseError("Pparam: too few fields in '" + s + "'");
    Pparam p;
    if (!rust_parse_f64(parts[0], p.value)) throw ParseError("bad value: " + parts[0]);
    if (!rust_parse_f64(parts[1], p.range)) throw ParseError("bad range: " + parts[1]);
    if (!rust_parse_f64(parts[2], p.dstep)) throw ParseError("bad dstep: " + parts[2]);
    p.vary = parse_bool(parts[3]);
    p.defined = parts.size() > 4 ? parse_bool(parts[4]) : true;
    return p;
}

// model.rs:186-442
Model model_from_string(const std::string& contents) {
    std::map<std::string, std::string> pv;
    std::map<std::string, bool> found;
    for (int i = 0; i < NPHYS; ++i) found[PHYS_NAMES[i]] = false;
    for (int i = 0; i < NCOMP; ++i) found[COMP_NAMES[i]] = false;
    std::istringstream is(contents);
    std::string line;
    int line_num = 0;
    while (std::getline(is, line)) {
        ++line_num;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        std::string trimmed = trim(line);
        if (trimmed.empty() || trimmed[0] == '#') continue;
        size_t eq = trimmed.find('=');
        if (eq == std::string::npos) continue;
        std::string param = trim(trimmed.substr(0, eq));
        std::string value = trimmed.substr(eq + 1);
        size_t nhash = 0;
        for (;;) {
            size_t pos = value.find('#', nhash);
            if (pos == std::string::npos) break;
            if (pos > 0 && value[pos - 1] == '\\') { nhash = pos + 1; continue; }
            value.resize(pos);
            break;
        }
        value = trim(value);
        if (!found.count(param))
            throw ParseError("Parameter '" + param + "' on line " + std::to_string(line_num) + " was not recognised");
        found[param] = true;
        pv[param] = value;
    }
    static const char* optional_defaults[] = {"pdot", "third", "temp_edge", "absorb_edge"};
    for (auto& kv : found) {
        if (kv.second) continue;
        bool opt = false;
        for (auto* o : optional_defaults) if (kv.first == o) opt = true;
        if (opt) pv[kv.first] = "0 1.e-10 1.e-10 0 0";
        else if (kv.first.rfind("stsp", 0) != 0 && kv.first.rfind("uesp", 0) != 0)
            throw ParseError("Parameter '" + kv.first + "' was not defined");
    }
    static const char* groups[5][4] = {
        {"stsp11_long", "stsp11_lat", "stsp11_fwhm", "stsp11_tcen"},
        {"stsp12_long", "stsp12_lat", "stsp12_fwhm", "stsp12_tcen"},
        {"stsp13_long", "stsp13_lat", "stsp13_fwhm", "stsp13_tcen"},
        {"stsp21_long", "stsp21_lat", "stsp21_fwhm", "stsp21_tcen"},
        {"stsp22_long", "stsp22_lat", "stsp22_fwhm", "stsp22_tcen"},
    };
    for (auto& g : groups) {
        bool any = false, all = true;
        for (auto* n : g) { bool f = found[n]; any = any || f; all = all && f; }
        if (any && !all) throw ParseError(std::string("One or more of ") + std::string(g[0]).substr(0, 6) + " parameters were not initialised");
    }
    {
        const char* ug[] = {"uesp_long1", "uesp_long2", "uesp_lathw", "uesp_taper", "uesp_temp"};
        bool any = false, all = true;
        for (auto* n : ug) { bool f = found[n]; any = any || f; all = all && f; }
        if (any && !all) throw ParseError("One or more uniform equatorial spot parameters were not initialised");
    }
    Model m;
    auto lim = [&](const char* key) {
        const std::string& s = pv.at(key);
        if (s == "Poly") return 0;
        if (s == "Claret") return 1;
        throw ParseError(std::string("bad ") + key + ": '" + s + "'");
    };
    m.limb1 = lim("limb1");
    m.limb2 = lim("limb2");
    m.roche1 = parse_bool(pv.at("roche1"));
    m.glens1 = parse_bool(pv.at("glens1"));
    if (m.glens1 && m.roche1) throw ParseError("glens1=1 and roche1=1 are not simultaneously allowed");
    for (int i = 0; i < NPHYS; ++i) {
        auto it = pv.find(PHYS_NAMES[i]);
        if (it != pv.end()) m.p[i] = parse_pparam(it->second);
        else m.p[i] = Pparam();
    }
    m.delta_phase = parse_double(pv.at("delta_phase"));
    m.nlat1f = parse_int(pv.at("nlat1f"));
    m.nlat2f = parse_int(pv.at("nlat2f"));
    m.nlat1c = parse_int(pv.at("nlat1c"));
    m.nlat2c = parse_int(pv.at("nlat2c"));
    m.npole = parse_bool(pv.at("npole"));
    m.nlatfill = parse_int(pv.at("nlatfill"));
    m.nlngfill = parse_int(pv.at("nlngfill"));
    m.lfudge = parse_double(pv.at("lfudge"));
    m.llo = parse_double(pv.at("llo"));
    m.lhi = parse_double(pv.at("lhi"));
    m.phase1 = parse_double(pv.at("phase1"));
    m.phase2 = parse_double(pv.at("phase2"));
    m.wavelength = parse_double(pv.at("wavelength"));
    m.roche2 = parse_bool(pv.at("roche2"));
    m.eclipse1 = parse_bool(pv.at("eclipse1"));
    m.eclipse2 = parse_bool(pv.at("eclipse2"));
    m.use_radii = parse_bool(pv.at("use_radii"));
    m.tperiod = parse_double(pv.at("tperiod"));
    m.gdark_bolom1 = parse_bool(pv.at("gdark_bolom1"));
    m.gdark_bolom2 = parse_bool(pv.at("gdark_bolom2"));
    m.mucrit1 = parse_double(pv.at("mucrit1"));
    m.mucrit2 = parse_double(pv.at("mucrit2"));
    m.mirror = parse_bool(pv.at("mirror"));
    m.add_disc = parse_bool(pv.at("add_disc"));
    m.nrad = parse_int(pv.at("nrad"));
    m.opaque = parse_bool(pv.at("opaque"));
    m.add_spot = parse_bool(pv.at("add_spot"));
    m.nspot = parse_int(pv.at("nspot"));
    m.iscale = parse_bool(pv.at("iscale"));
    return m;
}

// model.rs:445-454
static void get_r1r2(const Model& m, double& r1, double& r2) {
    if (m.use_radii) { r1 = m.v(R1); r2 = m.v(R2); return; }
    double sini = std::sin(to_rad(m.v(IANGLE)));
    double a = sini * std::cos(2.0 * PI * m.v(CPHI4));
    double b = sini * std::cos(2.0 * PI * m.v(CPHI3));
    double r2pr1 = std::sqrt(1.0 - a * a);
    double r2mr1 = std::sqrt(1.0 - b * b);
    r1 = (r2pr1 - r2mr1) / 2.0;
    r2 = (r2pr1 + r2mr1) / 2.0;
}
static int phys_index(const char* name) {
    for (int i = 0; i < NPHYS; ++i) if (std::strcmp(PHYS_NAMES[i], name) == 0) return i;
    return -1;
}

// ---------------------------------------------------------------------------
// Point / LDC / Ginterp — crates/lcurve/src/types.rs
// ---------------------------------------------------------------------------
struct Point {                                             // types.rs:8-46
    Vec3 posn, dirn;
    float area = 0.0f, gravity = 1.0f;
    EclipseVec eclipse;
    float flux = 0.0f;
    bool visible(double phase) const {                     // types.rs:50-58
        double phi = phase - std::floor(phase);
        for (auto& e : eclipse)
            if ((phi >= e.first && phi <= e.second) || phi <= e.second - 1.0) return false;
        return true;
    }
};
static Point make_point(const Vec3& posn, const Vec3& dirn, double area, double gravity, const EclipseVec& ecl) {
    Point p;
    p.posn = posn; p.dirn = dirn; p.area = (float)area; p.gravity = (float)gravity; p.eclipse = ecl;
    return p;
}
struct LDC {                                               // types.rs:71-126
    double l1 = 0, l2 = 0, l3 = 0, l4 = 0, mucrit = 0;
    int ltype = 0;
    double imu(double mu) const {
        if (mu <= 0.0) return 0.0;
        mu = std::fmin(mu, 1.0);
        double ommu = 1.0 - mu;
        double im = 1.0;
        if (ltype == 0) {
            im -= ommu * (l1 + ommu * (l2 + ommu * (l3 + ommu * l4)));
        } else {
            im -= l1 + l2 + l3 + l4;
            double msq = std::sqrt(mu);
            im += msq * (l1 + msq * (l2 + msq * (l3 + msq * l4)));
        }
        return im;
    }
    bool see(double mu) const { return mu > mucrit; }
};
static LDC get_ldc1(const Model& m) {  // model.rs:535-540
    LDC l; l.l1 = m.v(LDC1_1); l.l2 = m.v(LDC1_2); l.l3 = m.v(LDC1_3); l.l4 = m.v(LDC1_4);
    l.mucrit = m.mucrit1; l.ltype = m.limb1; return l;
}
static LDC get_ldc2(const Model& m) {  // model.rs:543-548
    LDC l; l.l1 = m.v(LDC2_1); l.l2 = m.v(LDC2_2); l.l3 = m.v(LDC2_3); l.l4 = m.v(LDC2_4);
    l.mucrit = m.mucrit2; l.ltype = m.limb2; return l;
}
struct Ginterp {                                           // types.rs:130-202
    double phase1 = 0.05, phase2 = 0.45, scale11 = 1, scale12 = 1, scale21 = 1, scale22 = 1;
    double scale1(double phase) const {
        double pnorm = phase - std::floor(phase);
        if (pnorm <= phase1 || pnorm >= 1.0 - phase1) return 1.0;
        return (scale11 * (1.0 - phase1 - pnorm) + scale12 * (pnorm - phase1)) / (1.0 - 2.0 * phase1);
    }
    double scale2(double phase) const {
        double pnorm = phase - std::floor(phase);
        if (pnorm >= phase2 && pnorm <= 1.0 - phase2) return 1.0;
        if (pnorm < 0.5) return (scale22 * (phase2 - pnorm) + scale21 * (pnorm + phase2)) / (2.0 * phase2);
        return (scale21 * (1.0 + phase2 - pnorm) + scale22 * (pnorm - 1.0 + phase2)) / (2.0 * phase2);
    }
    int grid_type(double phase) const {
        double pnorm = phase - std::floor(phase);
        if (pnorm <= phase1 || pnorm >= 1.0 - phase1) return 1;
        if ((pnorm > phase1 && pnorm < phase2) || (pnorm > 1.0 - phase2 && pnorm < 1.0 - phase1)) return 2;
        return 3;
    }
};
struct Datum { double time, expose, flux, ferr, weight; int32_t ndiv; int32_t pad; };  // types.rs:207-220

// ---------------------------------------------------------------------------
// grid — crates/lcurve/src/grid.rs
// ---------------------------------------------------------------------------
// grid.rs:8-46
int64_t numface(int nlat, bool infill, double thelo, double thehi, int nlatfill, int nlngfill) {
    int64_t nface = 0;
    double dtheta = PI / (double)nlat;
    if (infill) {
        int64_t nl1 = sat_i32(std::ceil(thelo / dtheta));
        for (int64_t i = 0; i < nl1; ++i) {
            double theta = thelo * ((double)i + 0.5) / (double)nl1;
            double dphi = dtheta / std::sin(theta);
            nface += std::max<int64_t>(16, sat_usize(TWOPI / dphi));
        }
        int64_t nl2 = sat_i32(std::ceil(((double)(1 + nlatfill) * (thehi - thelo)) / dtheta));
        for (int64_t i = 0; i < nl2; ++i) {
            double theta = thelo + (thehi - thelo) * ((double)i + 0.5) / (double)nl2;
            double dphi = dtheta / std::sin(theta) / (double)(1 + nlngfill);
            nface += std::max<int64_t>(8, sat_usize(PI / dphi));
        }
        int64_t nl3 = sat_i32(std::ceil((thehi - thelo) / dtheta));
        for (int64_t i = 0; i < nl3; ++i) {
            double theta = thelo + (thehi - thelo) * ((double)i + 0.5) / (double)nl3;
            double dphi = dtheta / std::sin(theta);
            nface += std::max<int64_t>(8, sat_usize(PI / dphi));
        }
        int64_t nl4 = sat_i32(std::ceil((PI - thehi) / dtheta));
        for (int64_t i = 0; i < nl4; ++i) {
            double theta = thehi + (PI - thehi) * ((double)i + 0.5) / (double)nl4;
            double dphi = dtheta / std::sin(theta);
            nface += std::max<int64_t>(16, sat_usize(TWOPI / dphi));
        }
    } else {
        int64_t nl = sat_i32(std::ceil(PI / dtheta));
        for (int64_t i = 0; i < nl; ++i) {
            double theta = PI * ((double)i + 0.5) / (double)nl;
            double dphi = dtheta / std::sin(theta);
            nface += std::max<int64_t>(16, sat_usize(TWOPI / dphi));
        }
    }
    return nface;
}

struct GridCtx {
    // Roche stars for eclipse tests (lazily built so that sphere-only models
    // never call ref_sphere with an out-of-range filling factor).
    std::unique_ptr<RocheStar> rs1, rs2;
};

// grid.rs:49-73
static void star_eclipse(double q, double r, double spin, double ffac, double iangle, const Vec3& posn,
                         double delta, bool roche, Star star, EclipseVec& eclipses) {
    double ri = to_rad(iangle);
    double cosi = std::cos(ri), sini = std::sin(ri);
    Vec3 cofm = star == PRIMARY ? Vec3() : Vec3(1.0, 0.0, 0.0);
    if (roche) {
        RocheStar rs = make_roche_star(q, star, spin, ffac);
        double ing, eg;
        if (ingress_egress(rs, iangle, delta, posn, ing, eg)) eclipses.push_back({ing, eg});
    } else {
        double phi1, phi2, l1, l2;
        if (sphere_eclipse_phase(cosi, sini, posn, cofm, r, phi1, phi2, l1, l2)) eclipses.push_back({phi1, phi2});
    }
}

static Vec3 envelope_xy(double rangle, double lambda, double r1) {  // grid.rs:324-333 (x, y)
    double sini = std::sin(rangle), cosi = std::cos(rangle);
    double sinl = std::sin(lambda), cosl = std::cos(lambda);
    double norm = std::sqrt(cosi * cosi + sini * sini * cosl * cosl);
    double x = sinl + r1 * cosi * sinl / norm;
    double y = -cosi * cosl - r1 * cosl / norm;
    return Vec3(x, y, 0.0);
}

struct GridArgs {
    double r1, r2, rref1, pref1, rref2, pref2, ffac1, ffac2, gref, acc;
    bool eclipse;
    Star which;
};

// An element's eclipse intervals are a function of its position alone.  The
// builders below compute them element by element, as the reference does
// (grid.rs:227-320: serial per star), unless orc_set_grid_threads(n > 1) was
// called: then each builder computes them after its loop, n threads over its
// elements -- the same function of the same inputs, so the same grid, built
// faster.  Only the full-size parity tests use that.
static int g_grid_threads = 1;
template <class F>
static void parallel_for(int64_t n, int nthreads, F&& f);
template <class F>
static void grid_eclipses(std::vector<Point>& pts, size_t first, F&& ecl_of) {
    parallel_for((int64_t)(pts.size() - first), g_grid_threads, [&](int64_t i) {
        Point& p = pts[first + (size_t)i];
        ecl_of(p.posn, p.eclipse);
    });
}

// grid.rs:201-322
static void add_faces(std::vector<Point>& star, double tlo, double thi, double dtheta, int nlatfill, int nlngfill,
                      const Model& mdl, const GridArgs& g) {
    Vec3 cofm1(0, 0, 0), cofm2(1.0, 0.0, 0.0);
    bool infill = nlatfill > 0 || nlngfill > 0;
    int64_t nlat, nlat1 = 0, nlat2 = 0;
    if (infill) {
        nlat1 = sat_i32(std::ceil((double)(1 + nlatfill) * (thi - tlo) / dtheta));
        nlat2 = sat_i32(std::ceil((thi - tlo) / dtheta));
        nlat = nlat1 + nlat2;
    } else {
        nlat = sat_i32(std::ceil((thi - tlo) / dtheta));
    }
    const double q = mdl.v(Q);
    const size_t first = star.size();
    const bool defer = g_grid_threads > 1;
    auto ecl_of = [&](const Vec3& posn, EclipseVec& eclipses) {
        if (!g.eclipse) return;
        if (g.which == PRIMARY)
            star_eclipse(q, g.r2, mdl.v(SPIN2), g.ffac2, mdl.v(IANGLE), posn, mdl.delta_phase, mdl.roche2,
                         SECONDARY, eclipses);
        else
            star_eclipse(q, g.r1, mdl.v(SPIN1), g.ffac1, mdl.v(IANGLE), posn, mdl.delta_phase, mdl.roche1,
                         PRIMARY, eclipses);
    };
    for (int64_t nt = 0; nt < nlat; ++nt) {
        double theta, phi1, phi2;
        int64_t nphi, nl;
        if (infill) {
            if (nt < nlat1) {
                theta = tlo + (thi - tlo) * ((double)nt + 0.5) / (double)nlat1;
                double sint = std::sin(theta);
                nphi = std::max<int64_t>(8, sat_i32(PI * sint * (double)(1 + nlngfill) / dtheta));
                nl = nlat1;
                if (g.which == PRIMARY) { phi1 = -PI / 2.0; phi2 = PI / 2.0; }
                else { phi1 = PI / 2.0; phi2 = 3.0 * PI / 2.0; }
            } else {
                theta = tlo + (thi - tlo) * ((double)(nt - nlat1) + 0.5) / (double)nlat2;
                double sint = std::sin(theta);
                nphi = std::max<int64_t>(8, sat_i32(PI * sint / dtheta));
                nl = nlat2;
                if (g.which == PRIMARY) { phi1 = PI / 2.0; phi2 = 3.0 * PI / 2.0; }
                else { phi1 = -PI / 2.0; phi2 = PI / 2.0; }
            }
        } else {
            theta = tlo + (thi - tlo) * ((double)nt + 0.5) / (double)nlat;
            double sint = std::sin(theta);
            nphi = std::max<int64_t>(16, sat_i32(TWOPI * sint / dtheta));
            nl = nlat;
            phi1 = 0.0;
            phi2 = TWOPI;
        }
        double sint = std::sin(theta), cost = std::cos(theta);
        for (int64_t np = 0; np < nphi; ++np) {
            double phi = phi1 + (phi2 - phi1) * ((double)np + 0.5) / (double)nphi;
            double sinp = std::sin(phi), cosp = std::cos(phi);
            Vec3 dirn = mdl.npole ? Vec3(sint * cosp, sint * sinp, cost) : Vec3(cost, sint * cosp, sint * sinp);
            Vec3 posn, dvec;
            double rad, gravity;
            if (g.which == PRIMARY && mdl.roche1) {
                face(q, PRIMARY, mdl.v(SPIN1), dirn, g.rref1, g.pref1, g.acc, posn, dvec, rad, gravity);
            } else if (g.which == SECONDARY && mdl.roche2) {
                face(q, SECONDARY, mdl.v(SPIN2), dirn, g.rref2, g.pref2, g.acc, posn, dvec, rad, gravity);
            } else if (g.which == PRIMARY) {
                rad = g.r1; posn = cofm1 + rad * dirn; dvec = dirn; gravity = 1.0;
            } else {
                rad = g.r2; posn = cofm2 + rad * dirn; dvec = dirn; gravity = 1.0;
            }
            double area = ((phi2 - phi1) / (double)nphi * rad * sint) * ((thi - tlo) / (double)nl * rad) /
                          Vec3::dot(dirn, dvec);
            EclipseVec eclipses;
            if (!defer) ecl_of(posn, eclipses);
            star.push_back(make_point(posn, dvec, area, gravity / g.gref, eclipses));
        }
    }
    if (defer) grid_eclipses(star, first, ecl_of);
}

static std::vector<Point> set_star_grid_inner(const Model& mdl, Star which, GridArgs g, int nlat, bool infill,
                                              double thelo, double thehi, int nlatfill, int nlngfill) {  // grid.rs:157-198
    g.acc = mdl.delta_phase / 10.0;
    double dtheta = PI / (double)nlat;
    const double q = mdl.v(Q);
    g.gref = 1.0;
    Vec3 pv, dv; double rr, gg;
    if (which == PRIMARY && mdl.roche1) {
        face(q, PRIMARY, mdl.v(SPIN1), Vec3(-1.0, 0.0, 0.0), g.rref1, g.pref1, g.acc, pv, dv, rr, gg);
        g.gref = gg;
    } else if (which == SECONDARY && mdl.roche2) {
        face(q, SECONDARY, mdl.v(SPIN2), Vec3(1.0, 0.0, 0.0), g.rref2, g.pref2, g.acc, pv, dv, rr, gg);
        g.gref = gg;
    }
    std::vector<Point> star;
    if (infill) {
        add_faces(star, 0.0, thelo, dtheta, 0, 0, mdl, g);
        add_faces(star, thelo, thehi, dtheta, nlatfill, nlngfill, mdl, g);
        add_faces(star, thehi, PI, dtheta, 0, 0, mdl, g);
    } else {
        add_faces(star, 0.0, PI, dtheta, 0, 0, mdl, g);
    }
    return star;
}

// grid.rs:76-155
std::vector<Point> set_star_grid(const Model& mdl, Star which, bool fine) {
    double r1, r2;
    get_r1r2(mdl, r1, r2);
    GridArgs g{};
    g.which = which;
    g.eclipse = which == PRIMARY ? mdl.eclipse1 : mdl.eclipse2;
    int nlat = which == PRIMARY ? (fine ? mdl.nlat1f : mdl.nlat1c) : (fine ? mdl.nlat2f : mdl.nlat2c);
    int nlatfill = which == PRIMARY ? 0 : (fine ? mdl.nlatfill : 0);
    int nlngfill = which == PRIMARY ? 0 : (fine ? mdl.nlngfill : 0);
    const double q = mdl.v(Q);
    double rl1 = xl11(q, mdl.v(SPIN1));
    if (r1 < 0.0) r1 = rl1;
    else if (r1 > rl1) throw RocheError("set_star_grid: primary star larger than Roche lobe");
    double rl2 = 1.0 - xl12(q, mdl.v(SPIN2));
    if (r2 < 0.0) r2 = rl2;
    else if (r2 > rl2) throw RocheError("set_star_grid: secondary star larger than Roche lobe");
    g.r1 = r1; g.r2 = r2;
    g.ffac1 = r1 / rl1;
    ref_sphere(q, PRIMARY, mdl.v(SPIN1), g.ffac1, g.rref1, g.pref1);
    g.ffac2 = r2 / rl2;
    ref_sphere(q, SECONDARY, mdl.v(SPIN2), g.ffac2, g.rref2, g.pref2);
    bool infill = mdl.npole && which == SECONDARY && (nlatfill > 0 || nlngfill > 0) && r2 > r1;
    double thelo = 0.0, thehi = 0.0;
    if (infill) {
        double rangle = to_rad(mdl.v(IANGLE));
        double cosi = std::cos(rangle);
        double ratio = (cosi + r1) / r2;
        if (ratio >= 1.0) {
            thehi = PI / 2.0 + rangle;
        } else {
            double llo_val = 0.0, lhi_val = PI / 2.0;
            while (lhi_val > llo_val + 1e-7) {
                double lmid = (llo_val + lhi_val) / 2.0;
                Vec3 xy = envelope_xy(rangle, lmid, r1);
                if (xy.x * xy.x + xy.y * xy.y < r2 * r2) llo_val = lmid; else lhi_val = lmid;
            }
            double sini = std::sin(rangle);
            Vec3 xy = envelope_xy(rangle, (llo_val + lhi_val) / 2.0, r1);
            thehi = std::fmax(PI / 2.0 - to_rad(mdl.llo),
                              std::fmin(PI / 2.0 + rangle, std::acos(xy.y * sini / r2) + to_rad(mdl.lfudge)));
        }
        double ratio2 = (cosi - r1) / r2;
        if (ratio2 >= 1.0) {
            return set_star_grid_inner(mdl, which, g, nlat, false, 0.0, 0.0, 0, 0);
        } else if (ratio2 <= -1.0) {
            thelo = 0.0;
        } else {
            thelo = std::fmin(PI / 2.0 - to_rad(mdl.lhi),
                              std::fmax(PI / 2.0 - std::acos(ratio2) + rangle - to_rad(mdl.lfudge), 0.0));
        }
    }
    return set_star_grid_inner(mdl, which, g, nlat, infill, thelo, thehi, nlatfill, nlngfill);
}

// grid.rs:336-392
std::vector<Point> set_disc_grid(const Model& mdl) {
    const double EFAC = 1.0000001;
    double r1, r2;
    get_r1r2(mdl, r1, r2);
    const double q = mdl.v(Q);
    double rl1 = xl11(q, mdl.v(SPIN1));
    if (r1 < 0.0) r1 = rl1;
    double rl2 = 1.0 - xl12(q, mdl.v(SPIN2));
    if (r2 < 0.0) r2 = rl2;
    double rdisc1 = mdl.v(RDISC1) > 0.0 ? mdl.v(RDISC1) : r1;
    double rdisc2 = mdl.v(RDISC2) > 0.0 ? mdl.v(RDISC2) : mdl.v(RADIUS_SPOT);
    double ffac1 = r1 / rl1, ffac2 = r2 / rl2;
    double drad = (rdisc2 - rdisc1) / (double)mdl.nrad;
    double drrad = rdisc2 / (double)mdl.nrad;
    std::vector<Point> disc;
    const bool defer = g_grid_threads > 1;
    auto ecl_of = [&](const Vec3& posn, EclipseVec& ecl) {
        if (mdl.opaque) ecl = disc_eclipse(mdl.v(IANGLE), rdisc1, rdisc2, mdl.v(BETA_DISC), mdl.v(HEIGHT_DISC), posn);
        if (mdl.eclipse1) star_eclipse(q, r1, mdl.v(SPIN1), ffac1, mdl.v(IANGLE), posn, mdl.delta_phase, mdl.roche1, PRIMARY, ecl);
        if (mdl.eclipse2) star_eclipse(q, r2, mdl.v(SPIN2), ffac2, mdl.v(IANGLE), posn, mdl.delta_phase, mdl.roche2, SECONDARY, ecl);
    };
    for (int i = 0; i < mdl.nrad; ++i) {
        double rad = rdisc1 + (rdisc2 - rdisc1) * ((double)i + 0.5) / (double)mdl.nrad;
        int64_t ntheta = std::max<int64_t>(8, sat_i32(std::ceil(TWOPI * rad / drrad)));
        double h = EFAC * mdl.v(HEIGHT_DISC) * std::pow(rad, mdl.v(BETA_DISC));
        double tanp = mdl.v(BETA_DISC) * h / rad;
        double cosp = 1.0 / std::sqrt(1.0 + sqr(tanp));
        double sinp = tanp * cosp;
        double area = TWOPI / (double)ntheta * rad * drad;
        for (int64_t j = 0; j < ntheta; ++j) {
            double theta = TWOPI * (double)j / (double)ntheta;
            double sint = std::sin(theta), cost = std::cos(theta);
            Vec3 posn(rad * cost, rad * sint, h);
            Vec3 dirn(-cost * sinp, -sint * sinp, cosp);
            EclipseVec ecl;
            if (!defer) ecl_of(posn, ecl);
            disc.push_back(make_point(posn, dirn, area, 1.0, ecl));
        }
    }
    if (defer) grid_eclipses(disc, 0, ecl_of);
    return disc;
}

// grid.rs:395-481
std::vector<Point> set_disc_edge(const Model& mdl, bool outer) {
    const double EFAC = 1.0000001;
    double r1, r2;
    get_r1r2(mdl, r1, r2);
    const double q = mdl.v(Q);
    double rl1 = xl11(q, mdl.v(SPIN1));
    if (r1 < 0.0) r1 = rl1;
    double rl2 = 1.0 - xl12(q, mdl.v(SPIN2));
    if (r2 < 0.0) r2 = rl2;
    double rdisc1 = mdl.v(RDISC1) > 0.0 ? mdl.v(RDISC1) : r1;
    double rdisc2 = mdl.v(RDISC2) > 0.0 ? mdl.v(RDISC2) : mdl.v(RADIUS_SPOT);
    double size = rdisc2 / (double)mdl.nrad;
    double ffac1 = r1 / rl1, ffac2 = r2 / rl2;
    double rad_val = outer ? rdisc2 : rdisc1;
    double h = mdl.v(HEIGHT_DISC) * std::pow(rad_val, mdl.v(BETA_DISC));
    int64_t nout = sat_i32(2.0 * h / size) + 2;
    int64_t ntheta = std::max<int64_t>(8, sat_i32(std::ceil(TWOPI * rad_val / size)));
    double area = TWOPI / (double)ntheta * rad_val * 2.0 * h / (double)(nout - 1);
    std::vector<Point> edge;
    const bool defer = g_grid_threads > 1;
    auto ecl_of = [&](const Vec3& posn, EclipseVec& ecl) {
        if (mdl.opaque) ecl = disc_eclipse(mdl.v(IANGLE), rdisc1, rdisc2, mdl.v(BETA_DISC), mdl.v(HEIGHT_DISC), posn);
        if (mdl.eclipse1) {
            try { star_eclipse(q, r1, mdl.v(SPIN1), ffac1, mdl.v(IANGLE), posn, mdl.delta_phase, mdl.roche1, PRIMARY, ecl); }
            catch (const RocheError&) {}
        }
        if (mdl.eclipse2) star_eclipse(q, r2, mdl.v(SPIN2), ffac2, mdl.v(IANGLE), posn, mdl.delta_phase, mdl.roche2, SECONDARY, ecl);
    };
    auto eclipses_for = [&](const Vec3& posn) {
        EclipseVec ecl;
        if (!defer) ecl_of(posn, ecl);
        return ecl;
    };
    for (int64_t i = 0; i < ntheta; ++i) {
        double theta = TWOPI * (double)i / (double)ntheta;
        double sint = std::sin(theta), cost = std::cos(theta);
        Vec3 posn = outer ? Vec3(EFAC * rad_val * cost, EFAC * rad_val * sint, EFAC * h)
                          : Vec3(rad_val * cost / EFAC, rad_val * sint / EFAC, EFAC * h);
        Vec3 dirn(cost, sint, 0.0);
        edge.push_back(make_point(posn, dirn, area / 2.0, 1.0, eclipses_for(posn)));
        for (int64_t j = 0; j < nout - 1; ++j) {
            double z = -h + 2.0 * h * (double)j / (double)(nout - 1);
            Vec3 p2, d2;
            if (outer) { p2 = Vec3(EFAC * rad_val * cost, EFAC * rad_val * sint, z); d2 = Vec3(cost, sint, 0.0); }
            else { p2 = Vec3(rad_val * cost / EFAC, rad_val * sint / EFAC, z); d2 = Vec3(-cost, -sint, 0.0); }
            edge.push_back(make_point(p2, d2, area, 1.0, eclipses_for(p2)));
        }
    }
    if (defer) grid_eclipses(edge, 0, ecl_of);
    return edge;
}

// grid.rs:484-553
std::vector<Point> set_bright_spot_grid(const Model& mdl, Vec3* bspot_out = nullptr) {
    double r1, r2;
    get_r1r2(mdl, r1, r2);
    const double q = mdl.v(Q);
    double rl1 = xl11(q, mdl.v(SPIN1));
    if (r1 < 0.0) r1 = rl1;
    else if (r1 > rl1) throw RocheError("set_bright_spot_grid: primary larger than Roche lobe");
    double rl2 = 1.0 - xl12(q, mdl.v(SPIN2));
    if (r2 < 0.0) r2 = rl2;
    else if (r2 > rl2) throw RocheError("set_bright_spot_grid: secondary larger than Roche lobe");
    double ffac1 = r1 / rl1, ffac2 = r2 / rl2;
    Vec3 bspot, vel;
    strinit(q, bspot, vel);
    stradv(q, bspot, vel, mdl.v(RADIUS_SPOT), 1e-10, 1e-3);
    if (bspot_out) *bspot_out = bspot;
    double theta = std::atan2(bspot.y, bspot.x) + TWOPI / 4.0 + to_rad(mdl.v(ANGLE_SPOT));
    double alpha = to_rad(mdl.v(YAW_SPOT));
    double tilt = to_rad(mdl.v(TILT_SPOT));
    Vec3 bvec(std::cos(theta), std::sin(theta), 0.0);
    Vec3 pvec(0.0, 0.0, 1.0);
    Vec3 tvec(std::sin(tilt) * std::sin(theta + alpha), -std::sin(tilt) * std::cos(theta + alpha), std::cos(tilt));
    double bmax = std::pow(mdl.v(EXPON_SPOT) / mdl.v(EPOW_SPOT), 1.0 / mdl.v(EPOW_SPOT));
    double sfac = 20.0 + bmax;
    double area = sfac * mdl.v(LENGTH_SPOT) * mdl.v(HEIGHT_SPOT) / (double)(mdl.nspot - 1);
    double bright_ref = planck(mdl.wavelength, mdl.v(TEMP_SPOT));
    std::vector<Point> spot;
    const bool defer = g_grid_threads > 1;
    auto ecl_of = [&](const Vec3& posn, EclipseVec& ecl) {
        if (mdl.eclipse1) star_eclipse(q, r1, mdl.v(SPIN1), ffac1, mdl.v(IANGLE), posn, mdl.delta_phase, mdl.roche1, PRIMARY, ecl);
        if (mdl.eclipse2) star_eclipse(q, r2, mdl.v(SPIN2), ffac2, mdl.v(IANGLE), posn, mdl.delta_phase, mdl.roche2, SECONDARY, ecl);
    };
    for (int i = 0; i < mdl.nspot; ++i) {
        double dist = sfac * (double)i / (double)(mdl.nspot - 1);
        Vec3 posn = bspot + (mdl.v(LENGTH_SPOT) * (dist - bmax)) * bvec;
        EclipseVec ecl;
        if (!defer) ecl_of(posn, ecl);
        double bright = bright_ref * std::pow(dist / bmax, mdl.v(EXPON_SPOT)) *
                        std::exp(mdl.v(EXPON_SPOT) / mdl.v(EPOW_SPOT) - std::pow(dist, mdl.v(EPOW_SPOT)));
        Point pt = make_point(posn, tvec, area, 1.0, ecl);
        pt.flux = (float)(bright * (1.0 - mdl.v(CFRAC_SPOT)) * area);
        spot.push_back(pt);
        Point pp = make_point(posn, pvec, area, 1.0, ecl);
        pp.flux = (float)(bright * mdl.v(CFRAC_SPOT) * area);
        spot.push_back(pp);
    }
    if (defer) grid_eclipses(spot, 0, ecl_of);
    return spot;
}

// ---------------------------------------------------------------------------
// brightness — crates/lcurve/src/brightness.rs
// ---------------------------------------------------------------------------
static const double FWHM_EFAC = 2.3548200450309493;  // brightness.rs:8
struct SpotInfo { bool on = false; Vec3 dir; double fwhm = 0, tcen = 0; };
static SpotInfo spot_info(const Pparam& lo, const Pparam& la, const Pparam& fw, const Pparam& tc) {  // 187-201
    SpotInfo s;
    if (!lo.defined || !la.defined || !fw.defined || !tc.defined) return s;
    double clong = std::cos(to_rad(lo.value)), slong = std::sin(to_rad(lo.value));
    double clat = std::cos(to_rad(la.value)), slat = std::sin(to_rad(la.value));
    s.on = true; s.dir = Vec3(clat * clong, clat * slong, slat); s.fwhm = fw.value; s.tcen = tc.value;
    return s;
}
static double angular_dist(const Vec3& posn, const Vec3& dir, double len) {  // 177-183
    if (len <= 0.0) return 180.0;
    double c = std::fmin(std::fmax(Vec3::dot(posn, dir) / len, -1.0), 1.0);
    return to_deg(std::acos(c));
}
// brightness.rs:150-174 -> (geom, temp)
static void irradiation(double t_base, double gravity, double gdcbol, double absorb, double t_irr, double mu, double r,
                        double r_irr, double& geom, double& temp) {
    double t_grav = t_base * std::pow(gravity, gdcbol);
    if (mu >= r_irr) {
        geom = sqr(r_irr / r) * mu;
        temp = std::pow(powi4(t_grav) + absorb * powi4(t_irr) * geom, 0.25);
    } else if (mu > -r_irr) {
        double x0 = -mu / r_irr;
        geom = sqr(r_irr / r) * r_irr * (std::sqrt(1.0 - x0 * x0) * (2.0 + x0 * x0) / 3.0 - x0 * (PI / 2.0 - std::asin(x0))) / PI;
        temp = std::pow(powi4(t_grav) + absorb * powi4(t_irr) * geom, 0.25);
    } else {
        geom = 0.0; temp = t_grav;
    }
}

template <class F>
static void parallel_for(int64_t n, int nthreads, F&& f);

// brightness.rs:13-147
void set_star_continuum(const Model& mdl, std::vector<Point>& star1, std::vector<Point>& star2, int nthreads) {
    double r1, r2;
    get_r1r2(mdl, r1, r2);
    double rl1 = xl1(mdl.v(Q));
    if (r1 < 0.0) r1 = rl1;
    double rl2 = 1.0 - rl1;
    if (r2 < 0.0) r2 = rl2;
    Vec3 cofm2(1.0, 0.0, 0.0);
    double gdcbol1 = mdl.gdark_bolom1 ? mdl.v(GRAVITY_DARK1) : mdl.v(GRAVITY_DARK1) / dlpdlt(mdl.wavelength, mdl.v(T1));
    SpotInfo s11 = spot_info(mdl.p[STSP11_LONG], mdl.p[STSP11_LAT], mdl.p[STSP11_FWHM], mdl.p[STSP11_TCEN]);
    SpotInfo s12 = spot_info(mdl.p[STSP12_LONG], mdl.p[STSP12_LAT], mdl.p[STSP12_FWHM], mdl.p[STSP12_TCEN]);
    SpotInfo s13 = spot_info(mdl.p[STSP13_LONG], mdl.p[STSP13_LAT], mdl.p[STSP13_FWHM], mdl.p[STSP13_TCEN]);
    bool is_uespot = mdl.p[UESP_LONG1].defined && mdl.p[UESP_LONG2].defined && mdl.p[UESP_LATHW].defined &&
                     mdl.p[UESP_TAPER].defined && mdl.p[UESP_TEMP].defined;
    Vec3 uespot_dir;
    double longhw = 0.0;
    if (is_uespot) {
        longhw = (mdl.v(UESP_LONG2) - mdl.v(UESP_LONG1)) / 2.0;
        double lcen = to_rad((mdl.v(UESP_LONG1) + mdl.v(UESP_LONG2)) / 2.0);
        uespot_dir = Vec3(std::cos(lcen), std::sin(lcen), 0.0);
    }
    const double t1v = mdl.v(T1);
    parallel_for((int64_t)star1.size(), nthreads, [&](int64_t i) {
        Point& pt = star1[i];
        Vec3 vec = cofm2 - pt.posn;
        double r = vec.length();
        double mu = Vec3::dot(pt.dirn, vec) / r;
        double t1 = t1v;
        for (const SpotInfo* s : {&s11, &s12, &s13}) {
            if (!s->on) continue;
            double dist = angular_dist(pt.posn, s->dir, pt.posn.length());
            t1 += (s->tcen - t1v) * std::exp(-sqr(dist / (s->fwhm / FWHM_EFAC)) / 2.0);
        }
        if (is_uespot) {
            Vec3 evec(pt.posn.x, pt.posn.y, 0.0);
            double evecl = evec.length();
            if (evecl > 0.0) {
                double rd = pt.posn.length();
                double clat = std::fmin(std::fmax(Vec3::dot(pt.posn, evec) / evecl / rd, -1.0), 1.0);
                double dlat = to_deg(std::acos(clat));
                double clong = std::fmin(std::fmax(Vec3::dot(uespot_dir, evec) / evecl, -1.0), 1.0);
                double dlong = to_deg(std::acos(clong));
                double lathw = mdl.v(UESP_LATHW), taper = mdl.v(UESP_TAPER), utemp = mdl.v(UESP_TEMP);
                if (dlat <= lathw && dlong <= longhw) t1 = utemp;
                else if (dlat <= lathw) t1 += (utemp - t1v) * std::exp(-(dlong - longhw) / taper);
                else if (dlong <= longhw) t1 += (utemp - t1v) * std::exp(-(dlat - lathw) / taper);
                else t1 += (utemp - t1v) * std::exp(-(dlat - lathw) / taper) * std::exp(-(dlong - longhw) / taper);
            }
        }
        double geom, temp;
        irradiation(t1, (double)pt.gravity, gdcbol1, mdl.v(ABSORB), mdl.v(T2), mu, r, r2, geom, temp);
        pt.flux = (float)((double)pt.area * planck(mdl.wavelength, temp));
        if (mdl.mirror) pt.flux += (float)((double)pt.area * geom * planck(mdl.wavelength, std::fabs(mdl.v(T2))));
    });
    Vec3 cofm1(0, 0, 0);
    double t2_abs = std::fabs(mdl.v(T2));
    double gdcbol2 = mdl.gdark_bolom2 ? mdl.v(GRAVITY_DARK2) : mdl.v(GRAVITY_DARK2) / dlpdlt(mdl.wavelength, t2_abs);
    SpotInfo s21 = spot_info(mdl.p[STSP21_LONG], mdl.p[STSP21_LAT], mdl.p[STSP21_FWHM], mdl.p[STSP21_TCEN]);
    SpotInfo s22 = spot_info(mdl.p[STSP22_LONG], mdl.p[STSP22_LAT], mdl.p[STSP22_FWHM], mdl.p[STSP22_TCEN]);
    parallel_for((int64_t)star2.size(), nthreads, [&](int64_t i) {
        Point& pt = star2[i];
        Vec3 vec = cofm1 - pt.posn;
        double r = vec.length();
        double mu = Vec3::dot(pt.dirn, vec) / r;
        double t2 = t2_abs;
        for (const SpotInfo* s : {&s21, &s22}) {
            if (!s->on) continue;
            Vec3 off = pt.posn - cofm2;
            double dist = angular_dist(off, s->dir, off.length());
            t2 += (s->tcen - t2) * std::exp(-sqr(dist / (s->fwhm / FWHM_EFAC)) / 2.0);
        }
        double geom, temp;
        irradiation(t2, (double)pt.gravity, gdcbol2, mdl.v(ABSORB), mdl.v(T1), mu, r, r1, geom, temp);
        pt.flux = (float)((double)pt.area * planck(mdl.wavelength, temp));
        if (mdl.mirror) pt.flux += (float)((double)pt.area * geom * planck(mdl.wavelength, mdl.v(T1)));
    });
}
// brightness.rs:204-212
void set_disc_continuum(double rdisc, double tdisc, double texp, double wave, std::vector<Point>& disc) {
    double bright = planck(wave, tdisc);
    for (auto& pt : disc) {
        double r = pt.posn.length();
        pt.flux = (float)(bright * std::pow(r / rdisc, texp) * (double)pt.area);
    }
}
// brightness.rs:215-239
void set_edge_continuum(double tedge, double r2, double t2, double absorb, double wave, std::vector<Point>& edge) {
    Vec3 cofm2(1.0, 0.0, 0.0);
    for (auto& pt : edge) {
        Vec3 vec = cofm2 - pt.posn;
        double r = vec.length();
        double mu = Vec3::dot(pt.dirn, vec) / r;
        double temp;
        if (mu >= r2) {
            double geom = sqr(r2 / r) * mu;
            temp = std::pow(powi4(tedge) + absorb * powi4(t2) * geom, 0.25);
        } else if (mu > -r2) {
            double x0 = -mu / r2;
            double geom = sqr(r2 / r) * r2 * (std::sqrt(1.0 - x0 * x0) * (2.0 + x0 * x0) / 3.0 - x0 * (PI / 2.0 - std::asin(x0))) / PI;
            temp = std::pow(powi4(tedge) + absorb * powi4(t2) * geom, 0.25);
        } else {
            temp = tedge;
        }
        pt.flux = (float)((double)pt.area * planck(wave, temp));
    }
}

// ---------------------------------------------------------------------------
// flux — crates/lcurve/src/flux.rs
// ---------------------------------------------------------------------------
static inline void exposure_weight(double phase, double expose, int nd, int ndiv, double& phi, double& wgt) {  // 379-387
    if (ndiv == 1) { phi = phase; wgt = 1.0; return; }
    phi = phase + expose * ((double)nd - (double)(ndiv - 1) / 2.0) / (double)(ndiv - 1);
    wgt = (nd == 0 || nd == ndiv - 1) ? 0.5 : 1.0;
}
static double lensing_mag(const Vec3& s, const Vec3& earth, double rlens1) {  // flux.rs:390-406
    double d = -Vec3::dot(s, earth);
    if (d <= 0.0) return 1.0;
    double p = (s + d * earth).length();
    double ph = p / 2.0;
    double phsq = ph * ph;
    double rd = rlens1 * d;
    double pd = phsq > 25.0 * rd ? p + rd / p : ph + std::sqrt(phsq + rd);
    return pd * pd / (pd - ph) / ph / 4.0;
}
typedef std::vector<Point> Pts;

struct FluxArgs {
    double iangle; LDC ldc1, ldc2; double lin_limb_disc, quad_limb_disc; double q, beam1, beam2, spin1, spin2;
    float vscale; bool glens1; double rlens1; Ginterp gint;
};

// flux.rs:7-111
double comp_light(const FluxArgs& a, double phase, double expose, int ndiv,
                  const Pts& star1f, const Pts& star2f, const Pts& star1c, const Pts& star2c,
                  const Pts& disc, const Pts& edge, const Pts& spot) {
    double xcofm = a.q / (1.0 + a.q);
    double cosi = std::cos(TWOPI * a.iangle / 360.0);
    double sini = std::sin(TWOPI * a.iangle / 360.0);
    double vfac = (double)a.vscale / (C_LIGHT / 1e3);
    double sum = 0.0;
    for (int nd = 0; nd < ndiv; ++nd) {
        double phi, wgt;
        exposure_weight(phase, expose, nd, ndiv, phi, wgt);
        Vec3 earth = set_earth_cosi_sini(cosi, sini, phi);
        int ptype = a.gint.grid_type(phi);
        const Pts& star1 = ptype == 1 ? star1f : star1c;
        const Pts& star2 = ptype == 3 ? star2f : star2c;
        double ssum = 0.0;
        for (const auto& pt : star1) {
            if (!pt.visible(phi)) continue;
            double mu = Vec3::dot(earth, pt.dirn);
            if (!a.ldc1.see(mu)) continue;
            if (a.beam1 != 0.0) {
                double vx = -vfac * a.spin1 * pt.posn.y;
                double vy = vfac * (a.spin1 * pt.posn.x - xcofm);
                double vr = -(earth.x * vx + earth.y * vy);
                double vn = pt.dirn.x * vx + pt.dirn.y * vy;
                double mud = mu - mu * vr - vn;
                ssum += mu * (double)pt.flux * (1.0 - a.beam1 * vr) * a.ldc1.imu(mud);
            } else {
                ssum += mu * (double)pt.flux * a.ldc1.imu(mu);
            }
        }
        ssum *= a.gint.scale1(phi);
        double ssum2 = 0.0;
        for (const auto& pt : star2) {
            if (!pt.visible(phi)) continue;
            double mu = Vec3::dot(earth, pt.dirn);
            if (!a.ldc2.see(mu)) continue;
            double mag = a.glens1 ? lensing_mag(pt.posn, earth, a.rlens1) : 1.0;
            if (a.beam2 != 0.0) {
                double vx = -vfac * a.spin2 * pt.posn.y;
                double vy = vfac * (a.spin2 * (pt.posn.x - 1.0) + 1.0 - xcofm);
                double vr = -(earth.x * vx + earth.y * vy);
                double vn = pt.dirn.x * vx + pt.dirn.y * vy;
                double mud = mu - mu * vr - vn;
                ssum2 += mu * mag * (double)pt.flux * (1.0 - a.beam2 * vr) * a.ldc2.imu(mud);
            } else {
                ssum2 += mu * mag * (double)pt.flux * a.ldc2.imu(mu);
            }
        }
        ssum += a.gint.scale2(phi) * ssum2;
        for (const Pts* comp : {&disc, &edge}) {
            for (const auto& pt : *comp) {
                double mu = Vec3::dot(earth, pt.dirn);
                if (mu > 0.0 && pt.visible(phi)) {
                    double ommu = 1.0 - mu;
                    ssum += mu * (double)pt.flux * (1.0 - ommu * (a.lin_limb_disc + a.quad_limb_disc * ommu));
                }
            }
        }
        for (const auto& pt : spot) {
            double mu = Vec3::dot(earth, pt.dirn);
            if (mu > 0.0 && pt.visible(phi)) ssum += mu * (double)pt.flux;
        }
        sum += wgt * ssum;
    }
    return sum / (double)std::max(1, ndiv - 1);
}

// flux.rs:115-159
double comp_star1(const FluxArgs& a, double phase, double expose, int ndiv, const Pts& star1f, const Pts& star1c) {
    double xcofm = a.q / (1.0 + a.q);
    double ri = to_rad(a.iangle);
    double cosi = std::cos(ri), sini = std::sin(ri);
    double vfac = (double)a.vscale / (C_LIGHT / 1e3);
    double sum = 0.0;
    for (int nd = 0; nd < ndiv; ++nd) {
        double phi, wgt;
        exposure_weight(phase, expose, nd, ndiv, phi, wgt);
        Vec3 earth = set_earth_cosi_sini(cosi, sini, phi);
        const Pts& star1 = a.gint.grid_type(phi) == 1 ? star1f : star1c;
        double ssum = 0.0;
        for (const auto& pt : star1) {
            if (!pt.visible(phi)) continue;
            double mu = Vec3::dot(earth, pt.dirn);
            if (!a.ldc1.see(mu)) continue;
            if (a.beam1 != 0.0) {
                double vx = -vfac * pt.posn.y;
                double vy = vfac * (pt.posn.x - xcofm);
                double vr = -(earth.x * vx + earth.y * vy);
                double vn = pt.dirn.x * vx + pt.dirn.y * vy;
                double mud = mu - mu * vr - vn;
                ssum += mu * (double)pt.flux * (1.0 - a.beam1 * vr) * a.ldc1.imu(mud);
            } else {
                double vr = vfac * (earth.x * pt.posn.y - earth.y * (pt.posn.x - xcofm));
                ssum += mu * (double)pt.flux * (1.0 - a.beam1 * vr) * a.ldc1.imu(mu);
            }
        }
        sum += wgt * a.gint.scale1(phase) * ssum;
    }
    return sum / (double)std::max(1, ndiv - 1);
}

// flux.rs:162-206
double comp_star2(const FluxArgs& a, double phase, double expose, int ndiv, const Pts& star2f, const Pts& star2c) {
    double xcofm = a.q / (1.0 + a.q);
    double ri = to_rad(a.iangle);
    double cosi = std::cos(ri), sini = std::sin(ri);
    double vfac = (double)a.vscale / (C_LIGHT / 1e3);
    double sum = 0.0;
    for (int nd = 0; nd < ndiv; ++nd) {
        double phi, wgt;
        exposure_weight(phase, expose, nd, ndiv, phi, wgt);
        Vec3 earth = set_earth_cosi_sini(cosi, sini, phi);
        const Pts& star2 = a.gint.grid_type(phi) == 3 ? star2f : star2c;
        double ssum = 0.0;
        for (const auto& pt : star2) {
            if (!pt.visible(phi)) continue;
            double mu = Vec3::dot(earth, pt.dirn);
            if (!a.ldc2.see(mu)) continue;
            double mag = a.glens1 ? lensing_mag(pt.posn, earth, a.rlens1) : 1.0;
            if (a.beam2 != 0.0) {
                double vx = -vfac * pt.posn.y;
                double vy = vfac * (pt.posn.x - xcofm);
                double vr = -(earth.x * vx + earth.y * vy);
                double vn = pt.dirn.x * vx + pt.dirn.y * vy;
                double mud = mu - mu * vr - vn;
                ssum += mu * mag * (double)pt.flux * (1.0 - a.beam2 * vr) * a.ldc2.imu(mud);
            } else {
                double vr = vfac * (earth.x * pt.posn.y - earth.y * (pt.posn.x - xcofm));
                ssum += mu * mag * (double)pt.flux * (1.0 - a.beam2 * vr) * a.ldc2.imu(mu);
            }
        }
        sum += wgt * a.gint.scale2(phi) * ssum;
    }
    return sum / (double)std::max(1, ndiv - 1);
}

// flux.rs:209-285 (comp_disc / comp_edge / comp_spot share one form)
static double comp_simple(const FluxArgs& a, double phase, double expose, int ndiv, const Pts& pts, bool ld) {
    double ri = to_rad(a.iangle);
    double cosi = std::cos(ri), sini = std::sin(ri);
    double sum = 0.0;
    for (int nd = 0; nd < ndiv; ++nd) {
        double phi, wgt;
        exposure_weight(phase, expose, nd, ndiv, phi, wgt);
        Vec3 earth = set_earth_cosi_sini(cosi, sini, phi);
        double ssum = 0.0;
        for (const auto& pt : pts) {
            double mu = Vec3::dot(earth, pt.dirn);
            if (mu > 0.0 && pt.visible(phi)) {
                if (ld) {
                    double ommu = 1.0 - mu;
                    ssum += mu * (double)pt.flux * (1.0 - ommu * (a.lin_limb_disc + a.quad_limb_disc * ommu));
                } else {
                    ssum += mu * (double)pt.flux;
                }
            }
        }
        sum += wgt * ssum;
    }
    return sum / (double)std::max(1, ndiv - 1);
}

// flux.rs:288-322
static double comp_gravity(const Model& mdl, const Pts& star, bool primary) {
    double gm = powi3(1000.0 * mdl.v(VELOCITY_SCALE)) * mdl.tperiod * DAY / TWOPI;
    double a = std::pow(gm / sqr(TWOPI / DAY / mdl.tperiod), 1.0 / 3.0);
    double gscale = 100.0 * gm / sqr(a);
    double r1, r2;
    get_r1r2(mdl, r1, r2);
    const double q = mdl.v(Q);
    double gref;
    if (primary) {
        double rl1;
        try { rl1 = xl12(q, mdl.v(SPIN1)); } catch (const RocheError&) { rl1 = 0.5; }
        if (mdl.roche1) {
            double acc = mdl.delta_phase / 10.0, ffac1 = r1 / rl1, rref, pref, rad, g;
            ref_sphere(q, PRIMARY, mdl.v(SPIN1), ffac1, rref, pref);
            Vec3 pv, dv;
            face(q, PRIMARY, mdl.v(SPIN1), Vec3(-1.0, 0.0, 0.0), rref, pref, acc, pv, dv, rad, g);
            gref = g * gscale;
        } else {
            gref = gscale / (1.0 + q) / sqr(r1);
        }
    } else {
        double rl2;
        try { rl2 = 1.0 - xl12(q, mdl.v(SPIN2)); } catch (const RocheError&) { rl2 = 1.0 - 0.5; }
        if (mdl.roche2) {
            double acc = mdl.delta_phase / 10.0, ffac2 = r2 / rl2, rref, pref, rad, g;
            ref_sphere(q, SECONDARY, mdl.v(SPIN2), ffac2, rref, pref);
            Vec3 pv, dv;
            face(q, SECONDARY, mdl.v(SPIN2), Vec3(1.0, 0.0, 0.0), rref, pref, acc, pv, dv, rad, g);
            gref = g * gscale;
        } else {
            gref = gscale * q / (1.0 + q) / sqr(r2);
        }
    }
    double sumfg = 0.0, sumf = 0.0;
    for (const auto& pt : star) { sumfg += (double)pt.flux * (double)pt.gravity; sumf += (double)pt.flux; }
    if (gref > 0.0 && sumfg > 0.0 && sumf > 0.0) return std::log10(gref * sumfg / sumf);
    return 0.0;
}
// flux.rs:347-373
static double comp_radius(const Pts& star, const Vec3& cofm) {
    double sumsa = 0.0, sumvol = 0.0;
    for (const auto& pt : star) {
        Vec3 vec = pt.posn - cofm;
        double r = vec.length();
        double rcosa = Vec3::dot(pt.dirn, vec);
        sumsa += (double)pt.area * rcosa / powi3(r);
        sumvol += (double)pt.area * rcosa;
    }
    return std::pow(sumvol / sumsa, 1.0 / 3.0);
}

// ---------------------------------------------------------------------------
// thread pool (stands in for Rayon's work-stealing into_par_iter)
//
// A parallel loop publishes its index range as a job.  Idle workers take
// chunks of indices from the newest open job, and a thread that waits for its
// own loop to finish helps jobs opened after its own (loops nested inside
// other threads' iterations) instead of sleeping.  Loops therefore nest as
// Rayon's do: in chisq_batch (orchestration.rs:343) threads that run out of
// models help with the time loops (orchestration.rs:229) of the models still
// running.  One pool of nthreads - 1 workers exists per thread count.
// ---------------------------------------------------------------------------
class Pool {
    struct Job {
        const std::function<void(int64_t)>* fn = nullptr;
        int64_t n = 0, chunk = 1;
        std::atomic<int64_t> next{0}, done{0};
        int users = 0;  // threads inside work() on this job (guarded by the pool mutex)
        uint64_t seq = 0;
        std::exception_ptr err;
    };
    std::mutex mu_;
    std::condition_variable cv_;  // new job, job finished, job released
    std::vector<Job*> open_;
    uint64_t seq_ = 0;
    std::vector<std::thread> workers_;

    // Newest open job with unclaimed indices (and, for a waiting caller, newer than `after`).
    Job* pick(uint64_t after) {
        for (size_t k = open_.size(); k-- > 0;) {
            Job* j = open_[k];
            if (j->seq > after && j->next.load() < j->n) { ++j->users; return j; }
        }
        return nullptr;
    }
    void work(Job* j) {
        for (;;) {
            int64_t i0 = j->next.fetch_add(j->chunk);
            if (i0 >= j->n) break;
            int64_t i1 = std::min(j->n, i0 + j->chunk);
            for (int64_t i = i0; i < i1; ++i) {
                try { (*j->fn)(i); }
                catch (...) {
                    std::lock_guard<std::mutex> g(mu_);
                    if (!j->err) j->err = std::current_exception();
                }
            }
            flush_counters();
            if (j->done.fetch_add(i1 - i0) + (i1 - i0) == j->n) {
                std::lock_guard<std::mutex> g(mu_);
                cv_.notify_all();
            }
        }
        std::lock_guard<std::mutex> g(mu_);
        if (--j->users == 0) cv_.notify_all();
    }

public:
    explicit Pool(int nthreads) {
        for (int t = 1; t < nthreads; ++t)
            workers_.emplace_back([this] {
                for (;;) {
                    Job* j = nullptr;
                    {
                        std::unique_lock<std::mutex> lk(mu_);
                        cv_.wait(lk, [&] { return (j = pick(0)) != nullptr; });
                    }
                    work(j);
                }
            });
        for (auto& w : workers_) w.detach();  // process-lifetime pool
    }
    static Pool& get(int nthreads) {
        static std::mutex m;
        static std::map<int, Pool*> pools;
        std::lock_guard<std::mutex> g(m);
        Pool*& p = pools[nthreads];
        if (!p) p = new Pool(nthreads);
        return *p;
    }
    void run(int64_t n, int nthreads, const std::function<void(int64_t)>& fn) {
        Job j;
        j.fn = &fn;
        j.n = n;
        j.chunk = std::max<int64_t>(1, n / (64 * (int64_t)nthreads));
        {
            std::lock_guard<std::mutex> g(mu_);
            j.seq = ++seq_;
            j.users = 1;
            open_.push_back(&j);
            cv_.notify_all();
        }
        work(&j);
        std::unique_lock<std::mutex> lk(mu_);
        while (j.done.load() < n) {
            Job* other = pick(j.seq);
            if (!other) { cv_.wait(lk); continue; }
            lk.unlock();
            work(other);
            lk.lock();
        }
        open_.erase(std::find(open_.begin(), open_.end(), &j));
        cv_.wait(lk, [&] { return j.users == 0; });
        if (j.err) std::rethrow_exception(j.err);
    }
};

template <class F>
static void parallel_for(int64_t n, int nthreads, F&& f) {
    if (nthreads <= 1 || n < 2) {
        for (int64_t i = 0; i < n; ++i) f(i);
        return;
    }
    const std::function<void(int64_t)> fn = [&](int64_t i) { f(i); };
    Pool::get(nthreads).run(n, nthreads, fn);
}

// ---------------------------------------------------------------------------
// orchestration — crates/lcurve/src/orchestration.rs
// ---------------------------------------------------------------------------
struct LcResult {                                              // orchestration.rs:9-28
    std::vector<double> calc;
    double wdwarf = 0, chisq = 0, wnok = 0, logg1 = 0, logg2 = 0, rv1 = 0, rv2 = 0;
    double sfac[5] = {1, 1, 1, 1, 1};
};
struct Grids {
    Pts star1f, star2f, star1c, star2c, disc, edge, spot;
    Ginterp gint;
    double rlens1 = 0.0;
    Vec3 bspot;
};

static FluxArgs make_flux_args(const Model& mdl, const Ginterp& gint, double rlens1) {
    FluxArgs a;
    a.iangle = mdl.v(IANGLE); a.ldc1 = get_ldc1(mdl); a.ldc2 = get_ldc2(mdl);
    a.lin_limb_disc = mdl.v(LIN_LIMB_DISC); a.quad_limb_disc = mdl.v(QUAD_LIMB_DISC);
    a.q = mdl.v(Q); a.beam1 = mdl.v(BEAM_FACTOR1); a.beam2 = mdl.v(BEAM_FACTOR2);
    a.spin1 = mdl.v(SPIN1); a.spin2 = mdl.v(SPIN2); a.vscale = (float)mdl.v(VELOCITY_SCALE);
    a.glens1 = mdl.glens1; a.rlens1 = rlens1; a.gint = gint;
    return a;
}

// orchestration.rs:36-170 (everything before the time loop)
void build_grids(const Model& mdl, Grids& G, int nthreads) {
    double r1, r2;
    get_r1r2(mdl, r1, r2);
    double rl2 = 1.0 - xl12(mdl.v(Q), mdl.v(SPIN2));
    if (r2 < 0.0) r2 = rl2;
    else if (r2 > rl2) throw RocheError("light_curve_comp: secondary larger than Roche lobe");
    LDC ldc1 = get_ldc1(mdl), ldc2 = get_ldc2(mdl);
    G.rlens1 = 0.0;
    if (mdl.glens1) {
        double gm = powi3(1000.0 * mdl.v(VELOCITY_SCALE)) * mdl.tperiod * DAY / TWOPI;
        double a = std::pow(gm / sqr(TWOPI / DAY / mdl.tperiod), 1.0 / 3.0);
        G.rlens1 = 4.0 * gm / (1.0 + mdl.v(Q)) / a / sqr(C_LIGHT);
    }
    G.star1f = set_star_grid(mdl, PRIMARY, true);
    G.star2f = set_star_grid(mdl, SECONDARY, true);
    set_star_continuum(mdl, G.star1f, G.star2f, nthreads);
    G.star1c = mdl.nlat1f == mdl.nlat1c ? G.star1f : set_star_grid(mdl, PRIMARY, false);
    bool copy2 = mdl.nlat2f == mdl.nlat2c && (!mdl.npole || r1 >= r2 || (mdl.nlatfill == 0 && mdl.nlngfill == 0));
    G.star2c = copy2 ? G.star2f : set_star_grid(mdl, SECONDARY, false);
    if (mdl.nlat1c != mdl.nlat1f || !copy2) set_star_continuum(mdl, G.star1c, G.star2c, nthreads);
    G.gint = Ginterp();
    G.gint.phase1 = mdl.phase1; G.gint.phase2 = mdl.phase2;
    // The reference hands the live Ginterp to comp_star1/2 (orchestration.rs:94-130), so each
    // later ratio already sees the scale factors assigned before it; FluxArgs is rebuilt per call.
    auto fa = [&]() { return make_flux_args(mdl, G.gint, G.rlens1); };
    if (mdl.nlat1c != mdl.nlat1f) {
        double ff = comp_star1(fa(), 0.9999999999 * mdl.phase1, 0.0, 1, G.star1f, G.star1c);
        double fc = comp_star1(fa(), 1.0000000001 * mdl.phase1, 0.0, 1, G.star1f, G.star1c);
        G.gint.scale11 = ff / fc;
        ff = comp_star1(fa(), 1.0 - 0.9999999999 * mdl.phase1, 0.0, 1, G.star1f, G.star1c);
        fc = comp_star1(fa(), 1.0 - 1.0000000001 * mdl.phase1, 0.0, 1, G.star1f, G.star1c);
        G.gint.scale12 = ff / fc;
    }
    if (!copy2) {
        double ff = comp_star2(fa(), 1.0 - 1.0000000001 * mdl.phase2, 0.0, 1, G.star2f, G.star2c);
        double fc = comp_star2(fa(), 1.0 - 0.9999999999 * mdl.phase2, 0.0, 1, G.star2f, G.star2c);
        G.gint.scale21 = ff / fc;
        ff = comp_star2(fa(), 1.0000000001 * mdl.phase2, 0.0, 1, G.star2f, G.star2c);
        fc = comp_star2(fa(), 0.9999999999 * mdl.phase2, 0.0, 1, G.star2f, G.star2c);
        G.gint.scale22 = ff / fc;
    }
    (void)ldc1; (void)ldc2;
    if (mdl.add_disc) {
        G.disc = set_disc_grid(mdl);
        G.edge = set_disc_edge(mdl, true);
        double rdisc1 = mdl.v(RDISC1) > 0.0 ? mdl.v(RDISC1) : r1;
        double rdisc2 = mdl.v(RDISC2) > 0.0 ? mdl.v(RDISC2) : mdl.v(RADIUS_SPOT);
        if (mdl.opaque) {
            for (Pts* grid : {&G.star1f, &G.star1c, &G.star2f, &G.star2c}) {
                Pts& gr = *grid;
                parallel_for((int64_t)gr.size(), nthreads, [&](int64_t i) {
                    auto e = disc_eclipse(mdl.v(IANGLE), rdisc1, rdisc2, mdl.v(BETA_DISC), mdl.v(HEIGHT_DISC), gr[i].posn);
                    for (auto& x : e) gr[i].eclipse.push_back(x);
                });
            }
        }
        set_disc_continuum(rdisc2, mdl.v(TEMP_DISC), mdl.v(TEXP_DISC), mdl.wavelength, G.disc);
        set_edge_continuum(mdl.v(TEMP_EDGE), r2, std::fabs(mdl.v(T2)), mdl.v(ABSORB_EDGE), mdl.wavelength, G.edge);
    }
    if (mdl.add_spot) G.spot = set_bright_spot_grid(mdl, &G.bspot);
}

// orchestration.rs:361-388
static void re_scale(const std::vector<Datum>& data, std::vector<double>& fit, double& scale, double& chisq, double& wnok) {
    double sdy = 0.0, syy = 0.0;
    wnok = 0.0;
    for (size_t i = 0; i < data.size(); ++i) {
        const Datum& d = data[i];
        if (d.weight > 0.0) {
            double wgt = d.weight / sqr(d.ferr);
            sdy += wgt * d.flux * fit[i];
            syy += wgt * fit[i] * fit[i];
            wnok += d.weight;
        }
    }
    if (wnok > 0.0 && syy > 0.0) {
        scale = sdy / syy;
        for (auto& f : fit) f *= scale;
        chisq = 0.0;
        for (size_t i = 0; i < data.size(); ++i)
            if (data[i].weight > 0.0) chisq += data[i].weight * sqr((data[i].flux - fit[i]) / data[i].ferr);
    } else {
        scale = 1.0; chisq = 0.0; wnok = 0.0;
    }
}
// orchestration.rs:391-401
static void compute_chisq(const std::vector<Datum>& data, const std::vector<double>& calc, double& chisq, double& wnok) {
    chisq = 0.0; wnok = 0.0;
    for (size_t i = 0; i < data.size(); ++i) {
        if (data[i].weight > 0.0) {
            wnok += data[i].weight;
            chisq += data[i].weight * sqr((data[i].flux - calc[i]) / data[i].ferr);
        }
    }
}
// orchestration.rs:405-436 — least squares by one-sided Jacobi SVD (nalgebra's
// SVD is the reference; its solve treats singular values below 1e-12 as zero).
static std::vector<double> svd_scale(const std::vector<Datum>& data, const std::vector<std::vector<double>>& fcomp, int ncol) {
    int nok = 0;
    for (auto& d : data) if (d.weight > 0.0) ++nok;
    if (nok < ncol || nok == 0) return std::vector<double>(ncol, 1.0);
    std::vector<double> A((size_t)nok * ncol), b(nok);
    int row = 0;
    for (size_t i = 0; i < data.size(); ++i) {
        if (data[i].weight > 0.0) {
            double w = std::sqrt(data[i].weight) / data[i].ferr;
            for (int j = 0; j < ncol; ++j) A[(size_t)row * ncol + j] = fcomp[i][j] * w;
            b[row] = data[i].flux * w;
            ++row;
        }
    }
    // One-sided Jacobi on columns: A = U S V^T
    std::vector<double> V((size_t)ncol * ncol, 0.0);
    for (int j = 0; j < ncol; ++j) V[(size_t)j * ncol + j] = 1.0;
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < ncol; ++p) for (int qc = p + 1; qc < ncol; ++qc) {
            double alpha = 0, beta = 0, gamma = 0;
            for (int i = 0; i < nok; ++i) {
                double ap = A[(size_t)i * ncol + p], aq = A[(size_t)i * ncol + qc];
                alpha += ap * ap; beta += aq * aq; gamma += ap * aq;
            }
            if (gamma == 0.0) continue;
            off = std::fmax(off, std::fabs(gamma) / std::sqrt(alpha * beta));
            double zeta = (beta - alpha) / (2.0 * gamma);
            double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
            double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
            for (int i = 0; i < nok; ++i) {
                double ap = A[(size_t)i * ncol + p], aq = A[(size_t)i * ncol + qc];
                A[(size_t)i * ncol + p] = c * ap - s * aq;
                A[(size_t)i * ncol + qc] = s * ap + c * aq;
            }
            for (int i = 0; i < ncol; ++i) {
                double vp = V[(size_t)i * ncol + p], vq = V[(size_t)i * ncol + qc];
                V[(size_t)i * ncol + p] = c * vp - s * vq;
                V[(size_t)i * ncol + qc] = s * vp + c * vq;
            }
        }
        if (off < 1e-15) break;
    }
    std::vector<double> x(ncol, 0.0);
    for (int j = 0; j < ncol; ++j) {
        double sj = 0.0;
        for (int i = 0; i < nok; ++i) sj += sqr(A[(size_t)i * ncol + j]);
        sj = std::sqrt(sj);
        if (!(sj > 1e-12)) continue;
        double ub = 0.0;
        for (int i = 0; i < nok; ++i) ub += A[(size_t)i * ncol + j] / sj * b[i];
        for (int k = 0; k < ncol; ++k) x[k] += V[(size_t)k * ncol + j] * ub / sj;
    }
    for (double v : x) if (!std::isfinite(v)) return std::vector<double>(ncol, 1.0);
    return x;
}

static inline double datum_phase(const Model& mdl, double time) {  // orchestration.rs:231-237
    double t0 = mdl.v(T0), period = mdl.v(PERIOD), pdot = mdl.v(PDOT);
    double phase = (time - t0) / period;
    for (int k = 0; k < 4; ++k)
        phase -= (t0 + phase * (period + pdot * phase) - time) / (period + 2.0 * pdot * phase);
    phase += mdl.v(DELTAT) / period / 2.0 * (std::cos(2.0 * PI * phase) - 1.0);
    return phase;
}

// orchestration.rs:171-318: the time loop, scaling and the per-star sums, on grids
// already built by build_grids.
LcResult light_curve_on(const Model& mdl, const Grids& G, const std::vector<Datum>& data, bool scale, bool rdata,
                        int nthreads) {
    if (data.empty()) throw std::runtime_error("light_curve_comp: no data");
    size_t n = data.size();
    LcResult res;
    res.calc.assign(n, 0.0);
    double xmin = data[0].time, xmax = data[0].time;
    for (size_t i = 1; i < n; ++i) { if (data[i].time < xmin) xmin = data[i].time; if (data[i].time > xmax) xmax = data[i].time; }
    double middle = (xmin + xmax) / 2.0, range = (xmax - xmin) / 2.0;
    int ncol = mdl.v(T2) > 0.0 ? 5 : 4;
    std::vector<std::vector<double>> fcomp;
    FluxArgs fa = make_flux_args(mdl, G.gint, G.rlens1);
    auto prep = [&](size_t np, double& phase, double& expose, double& slfac) {
        phase = datum_phase(mdl, data[np].time);
        expose = data[np].expose / mdl.v(PERIOD);
        double frac = (data[np].time - middle) / range;
        slfac = 1.0 + frac * (mdl.v(SLOPE) + frac * (mdl.v(QUAD) + frac * mdl.v(CUBE)));
    };
    if (mdl.iscale) {
        fcomp.assign(n, std::vector<double>(ncol, 0.0));
        parallel_for((int64_t)n, nthreads, [&](int64_t np) {
            double phase, expose, slfac;
            prep(np, phase, expose, slfac);
            int nd = data[np].ndiv;
            auto& row = fcomp[np];
            row[0] = slfac * comp_star1(fa, phase, expose, nd, G.star1f, G.star1c);
            row[1] = slfac * comp_simple(fa, phase, expose, nd, G.disc, true);
            row[2] = slfac * comp_simple(fa, phase, expose, nd, G.edge, true);
            row[3] = slfac * comp_simple(fa, phase, expose, nd, G.spot, false);
            if (mdl.v(T2) > 0.0) row[4] = slfac * comp_star2(fa, phase, expose, nd, G.star2f, G.star2c);
        });
    } else {
        parallel_for((int64_t)n, nthreads, [&](int64_t np) {
            double phase, expose, slfac;
            prep(np, phase, expose, slfac);
            res.calc[np] = slfac * comp_light(fa, phase, expose, data[np].ndiv, G.star1f, G.star2f, G.star1c, G.star2c,
                                              G.disc, G.edge, G.spot) + mdl.v(THIRD);
        });
    }
    res.wdwarf = comp_star1(fa, 0.5, 0.0, 1, G.star1f, G.star1c);
    double sfac[5] = {1, 1, 1, 1, 1};
    double chisq = 0.0, wnok = 0.0;
    if (scale) {
        if (mdl.iscale) {
            std::vector<double> s = svd_scale(data, fcomp, ncol);
            res.wdwarf *= s[0];
            for (int j = 0; j < 5; ++j) sfac[j] = j < ncol ? s[j] : 0.0;
            for (size_t np = 0; np < n; ++np) {
                res.calc[np] = sfac[0] * fcomp[np][0] + sfac[1] * fcomp[np][1] + sfac[2] * fcomp[np][2] + sfac[3] * fcomp[np][3];
                if (mdl.v(T2) > 0.0) res.calc[np] += sfac[4] * fcomp[np][4];
            }
            compute_chisq(data, res.calc, chisq, wnok);
        } else {
            double s;
            re_scale(data, res.calc, s, chisq, wnok);
            res.wdwarf *= s;
            for (int j = 0; j < 5; ++j) sfac[j] = s;
        }
    } else {
        res.wdwarf *= sfac[0];
        if (mdl.iscale) {
            for (size_t np = 0; np < n; ++np) {
                res.calc[np] = sfac[0] * fcomp[np][0] + sfac[1] * fcomp[np][1] + sfac[2] * fcomp[np][2] + sfac[3] * fcomp[np][3];
                if (mdl.v(T2) > 0.0) res.calc[np] += sfac[4] * fcomp[np][4];
            }
        } else {
            for (auto& c : res.calc) c *= sfac[0];
        }
        if (rdata) compute_chisq(data, res.calc, chisq, wnok);
    }
    res.chisq = chisq; res.wnok = wnok;
    for (int j = 0; j < 5; ++j) res.sfac[j] = sfac[j];
    res.logg1 = comp_gravity(mdl, G.star1f, true);
    res.logg2 = comp_gravity(mdl, G.star2f, false);
    res.rv1 = comp_radius(G.star1f, Vec3());
    res.rv2 = comp_radius(G.star2f, Vec3(1.0, 0.0, 0.0));
    return res;
}

// orchestration.rs:36-318
LcResult light_curve_comp(const Model& mdl, const std::vector<Datum>& data, bool scale, bool rdata, int nthreads) {
    if (data.empty()) throw std::runtime_error("light_curve_comp: no data");
    Grids G;
    build_grids(mdl, G, nthreads);
    return light_curve_on(mdl, G, data, scale, rdata, nthreads);
}

}  // namespace orc

// ===========================================================================
// C ABI for the Python test harness (ctypes).
// ===========================================================================
using namespace orc;

struct OrcModel { Model m; };
struct OrcGrids { Grids g; };

static void set_err(char* err, int errlen, const std::string& msg) {
    if (err && errlen > 0) { std::snprintf(err, (size_t)errlen, "%s", msg.c_str()); }
}

extern "C" {

int orc_model_load(const char* path, void** out, char* err, int errlen) {
    try {
        std::ifstream f(path);
        if (!f) { set_err(err, errlen, std::string("cannot open ") + path); return 2; }
        std::stringstream ss; ss << f.rdbuf();
        auto* m = new OrcModel{model_from_string(ss.str())};
        *out = m;
        return 0;
    } catch (const std::exception& e) { set_err(err, errlen, e.what()); return 3; }
}
int orc_model_parse(const char* text, void** out, char* err, int errlen) {
    try { *out = new OrcModel{model_from_string(text)}; return 0; }
    catch (const std::exception& e) { set_err(err, errlen, e.what()); return 3; }
}
void orc_model_free(void* m) { delete (OrcModel*)m; }
void* orc_model_clone(void* m) { return new OrcModel(*(OrcModel*)m); }
// model.rs:459-493 — returns 1 if the name is a physical parameter.
int orc_model_set(void* m, const char* name, double v) {
    int i = phys_index(name);
    if (i < 0) return 0;
    ((OrcModel*)m)->m.p[i].value = v;
    return 1;
}
int orc_model_get(void* m, const char* name, double* v) {
    int i = phys_index(name);
    if (i < 0) return 0;
    *v = ((OrcModel*)m)->m.p[i].value;
    return 1;
}
// Computational parameters by name (integers / flags / doubles).
int orc_model_set_comp(void* mh, const char* name, double v) {
    Model& m = ((OrcModel*)mh)->m;
    std::string n(name);
#define SETI(k) if (n == #k) { m.k = (int)v; return 1; }
#define SETB(k) if (n == #k) { m.k = v != 0.0; return 1; }
#define SETD(k) if (n == #k) { m.k = v; return 1; }
    SETD(delta_phase) SETI(nlat1f) SETI(nlat2f) SETI(nlat1c) SETI(nlat2c) SETB(npole) SETI(nlatfill) SETI(nlngfill)
    SETD(lfudge) SETD(llo) SETD(lhi) SETD(phase1) SETD(phase2) SETD(wavelength) SETB(roche1) SETB(roche2)
    SETB(eclipse1) SETB(eclipse2) SETB(glens1) SETB(use_radii) SETD(tperiod) SETB(gdark_bolom1) SETB(gdark_bolom2)
    SETD(mucrit1) SETD(mucrit2) SETI(limb1) SETI(limb2) SETB(mirror) SETB(add_disc) SETI(nrad) SETB(opaque)
    SETB(add_spot) SETI(nspot) SETB(iscale)
#undef SETI
#undef SETB
#undef SETD
    return 0;
}
int orc_model_set_defined(void* mh, const char* name, int defined) {
    int i = phys_index(name);
    if (i < 0) return 0;
    ((OrcModel*)mh)->m.p[i].defined = defined != 0;
    return 1;
}

// scalars: wdwarf chisq wnok logg1 logg2 rv1 rv2 sfac[5] (12 doubles)
int orc_light_curve(void* mh, const Datum* data, int n, int scale, int rdata, int nthreads, double* calc,
                    double* scalars, char* err, int errlen) {
    try {
        std::vector<Datum> d(data, data + n);
        LcResult r = light_curve_comp(((OrcModel*)mh)->m, d, scale != 0, rdata != 0, nthreads);
        flush_counters();
        for (int i = 0; i < n; ++i) calc[i] = r.calc[i];
        double s[12] = {r.wdwarf, r.chisq, r.wnok, r.logg1, r.logg2, r.rv1, r.rv2,
                        r.sfac[0], r.sfac[1], r.sfac[2], r.sfac[3], r.sfac[4]};
        if (scalars) for (int i = 0; i < 12; ++i) scalars[i] = s[i];
        return 0;
    } catch (const std::exception& e) { flush_counters(); set_err(err, errlen, e.what()); return 1; }
}

// orchestration.rs:329-357: NaN for a model that fails.
int orc_chisq_batch(void* base, const Datum* data, int n, const char** names, int ndim, const double* values,
                    int nsets, int scale, int nthreads, double* out) {
    std::vector<Datum> d(data, data + n);
    const Model& b = ((OrcModel*)base)->m;
    parallel_for(nsets, nthreads, [&](int64_t i) {
        Model m = b;
        for (int j = 0; j < ndim; ++j) {
            int k = phys_index(names[j]);
            if (k >= 0) m.p[k].value = values[(size_t)i * ndim + j];
        }
        try { out[i] = light_curve_comp(m, d, scale != 0, true, nthreads).chisq; }
        catch (const std::exception&) { out[i] = NAN; }
    });
    flush_counters();
    return 0;
}

// Ragged batch: model i uses data[offsets[i] .. offsets[i+1]).
int orc_chisq_ragged(void** models, int nmodels, const Datum* data, const int64_t* offsets, int scale, int nthreads,
                     double* out) {
    parallel_for(nmodels, nthreads, [&](int64_t i) {
        std::vector<Datum> d(data + offsets[i], data + offsets[i + 1]);
        try { out[i] = light_curve_comp(((OrcModel*)models[i])->m, d, scale != 0, true, nthreads).chisq; }
        catch (const std::exception&) { out[i] = NAN; }
    });
    flush_counters();
    return 0;
}

// Threads the grid builders use for eclipse intervals (1 = element by element,
// as the reference); the full-size parity tests raise it.
void orc_set_grid_threads(int n) { g_grid_threads = n < 1 ? 1 : n; }

// Grid extraction for per-element parity tests.
int orc_grids_build(void* mh, void** out, char* err, int errlen) {
    try {
        auto* g = new OrcGrids();
        build_grids(((OrcModel*)mh)->m, g->g, g_grid_threads);
        flush_counters();
        *out = g;
        return 0;
    } catch (const std::exception& e) { flush_counters(); set_err(err, errlen, e.what()); return 1; }
}
void orc_grids_free(void* g) { delete (OrcGrids*)g; }
// The light curve of a model on grids already built for it by orc_grids_build
// (the time loop and everything after it, orchestration.rs:171-318).
int orc_grids_light_curve(void* gh, void* mh, const Datum* data, int n, int scale, int rdata, int nthreads,
                          double* calc, double* scalars, char* err, int errlen) {
    try {
        std::vector<Datum> d(data, data + n);
        LcResult r = light_curve_on(((OrcModel*)mh)->m, ((OrcGrids*)gh)->g, d, scale != 0, rdata != 0, nthreads);
        flush_counters();
        for (int i = 0; i < n; ++i) calc[i] = r.calc[i];
        double s[12] = {r.wdwarf, r.chisq, r.wnok, r.logg1, r.logg2, r.rv1, r.rv2,
                        r.sfac[0], r.sfac[1], r.sfac[2], r.sfac[3], r.sfac[4]};
        if (scalars) for (int i = 0; i < 12; ++i) scalars[i] = s[i];
        return 0;
    } catch (const std::exception& e) { flush_counters(); set_err(err, errlen, e.what()); return 1; }
}
static const Pts* grid_sel(OrcGrids* g, int which) {
    switch (which) {
        case 0: return &g->g.star1f; case 1: return &g->g.star2f; case 2: return &g->g.star1c; case 3: return &g->g.star2c;
        case 4: return &g->g.disc; case 5: return &g->g.edge; case 6: return &g->g.spot;
    }
    return nullptr;
}
int64_t orc_grids_count(void* gh, int which) {
    const Pts* p = grid_sel((OrcGrids*)gh, which);
    return p ? (int64_t)p->size() : -1;
}
// posn/dirn: 3n doubles; area/gravity/flux: n floats; necl: n ints; ecl: 8n doubles (4 pairs max)
int orc_grids_fetch(void* gh, int which, double* posn, double* dirn, float* area, float* gravity, float* flux,
                    int* necl, double* ecl) {
    const Pts* p = grid_sel((OrcGrids*)gh, which);
    if (!p) return 1;
    for (size_t i = 0; i < p->size(); ++i) {
        const Point& pt = (*p)[i];
        posn[3 * i] = pt.posn.x; posn[3 * i + 1] = pt.posn.y; posn[3 * i + 2] = pt.posn.z;
        dirn[3 * i] = pt.dirn.x; dirn[3 * i + 1] = pt.dirn.y; dirn[3 * i + 2] = pt.dirn.z;
        area[i] = pt.area; gravity[i] = pt.gravity; flux[i] = pt.flux;
        necl[i] = (int)pt.eclipse.size();
        for (int k = 0; k < 4; ++k) {
            bool have = k < (int)pt.eclipse.size();
            ecl[8 * i + 2 * k] = have ? pt.eclipse[k].first : 0.0;
            ecl[8 * i + 2 * k + 1] = have ? pt.eclipse[k].second : 0.0;
        }
    }
    return 0;
}
// Replaces the points of one grid (same arrays as orc_grids_fetch), for light curves on
// element sets assembled elsewhere (the slab-split tests).
int orc_grids_set(void* gh, int which, int64_t n, const double* posn, const double* dirn, const float* area,
                  const float* gravity, const float* flux, const int* necl, const double* ecl) {
    Pts* p = const_cast<Pts*>(grid_sel((OrcGrids*)gh, which));
    if (!p) return 1;
    p->assign((size_t)n, Point());
    for (int64_t i = 0; i < n; ++i) {
        Point& pt = (*p)[i];
        pt.posn = Vec3(posn[3 * i], posn[3 * i + 1], posn[3 * i + 2]);
        pt.dirn = Vec3(dirn[3 * i], dirn[3 * i + 1], dirn[3 * i + 2]);
        pt.area = area[i]; pt.gravity = gravity[i]; pt.flux = flux[i];
        for (int k = 0; k < necl[i] && k < 4; ++k) pt.eclipse.push_back({ecl[8 * i + 2 * k], ecl[8 * i + 2 * k + 1]});
    }
    return 0;
}
// gint scales, rlens1, bright-spot position: 10 doubles
void orc_grids_info(void* gh, double* out) {
    Grids& g = ((OrcGrids*)gh)->g;
    double v[10] = {g.gint.phase1, g.gint.phase2, g.gint.scale11, g.gint.scale12, g.gint.scale21, g.gint.scale22,
                    g.rlens1, g.bspot.x, g.bspot.y, g.bspot.z};
    for (int i = 0; i < 10; ++i) out[i] = v[i];
}

// Known-answer hooks for unit tests (lagrange.rs:148-185, potential.rs:145-150, misc.rs:58-69).
double orc_xl1(double q) { try { return xl1(q); } catch (...) { return NAN; } }
double orc_xl11(double q, double s) { try { return xl11(q, s); } catch (...) { return NAN; } }
double orc_xl12(double q, double s) { try { return xl12(q, s); } catch (...) { return NAN; } }
double orc_planck(double w, double t) { return planck(w, t); }
double orc_dlpdlt(double w, double t) { return dlpdlt(w, t); }
int64_t orc_numface(int nlat) { return numface(nlat, false, 0.0, 0.0, 0, 0); }
// Roche-geometry helpers of the reference's roche crate, for its unit-test known answers.
double orc_rpot(double q, double x, double y, double z) {
    try { return rpot(q, Vec3(x, y, z)); } catch (const std::exception&) { return NAN; }
}
void orc_drpot1(double q, double spin, double x, double y, double z, double* out3) {
    try {
        Vec3 g = drpot1(q, spin, Vec3(x, y, z));
        out3[0] = g.x; out3[1] = g.y; out3[2] = g.z;
    } catch (const std::exception&) {
        out3[0] = out3[1] = out3[2] = NAN;
    }
}
void orc_set_earth(double iangle, double phase, double* out3) {  // misc.rs:36-39
    const double irad = iangle * (PI / 180.0);  // f64::to_radians
    Vec3 e = set_earth_cosi_sini(std::cos(irad), std::sin(irad), phase);
    out3[0] = e.x; out3[1] = e.y; out3[2] = e.z;
}
void orc_strinit(double q, double* r3, double* v3) {
    try {
        Vec3 r, v;
        strinit(q, r, v);
        r3[0] = r.x; r3[1] = r.y; r3[2] = r.z; v3[0] = v.x; v3[1] = v.y; v3[2] = v.z;
    } catch (const std::exception&) {
        for (int k = 0; k < 3; ++k) r3[k] = v3[k] = NAN;
    }
}
// One gsint step of size ttry from strinit, for the Jacobi-constant check (stream.rs:292-309):
// the stream state before (rv0) and after (rv1) the step, 6 values each.
void orc_gsint_step(double q, double ttry, double eps, double* rv0, double* rv1) {
    try {
        Vec3 r, v;
        strinit(q, r, v);
        rv0[0] = r.x; rv0[1] = r.y; rv0[2] = r.z; rv0[3] = v.x; rv0[4] = v.y; rv0[5] = v.z;
        BsState st;
        double time = 0.0, tdid = 0.0, tnext = 0.0;
        gsint(q, r, v, ttry, time, eps, st, tdid, tnext);
        rv1[0] = r.x; rv1[1] = r.y; rv1[2] = r.z; rv1[3] = v.x; rv1[4] = v.y; rv1[5] = v.z;
    } catch (const std::exception&) {
        for (int k = 0; k < 6; ++k) rv0[k] = rv1[k] = NAN;
    }
}
void orc_ref_sphere(double q, int secondary, double spin, double ffac, double* rref_pref) {
    try {
        ref_sphere(q, secondary ? SECONDARY : PRIMARY, spin, ffac, rref_pref[0], rref_pref[1]);
    } catch (const std::exception&) {
        rref_pref[0] = rref_pref[1] = NAN;
    }
}
// face (surface.rs:54-121) of the star in direction dirn: point, normal, radius and gravity.
void orc_face(double q, int secondary, double spin, double ffac, const double* dirn, double acc, double* pvec3,
              double* dvec3, double* r_g) {
    try {
        double rref = 0.0, pref = 0.0;
        const Star star = secondary ? SECONDARY : PRIMARY;
        ref_sphere(q, star, spin, ffac, rref, pref);
        Vec3 pvec, dvec;
        face(q, star, spin, Vec3(dirn[0], dirn[1], dirn[2]), rref, pref, acc, pvec, dvec, r_g[0], r_g[1]);
        pvec3[0] = pvec.x; pvec3[1] = pvec.y; pvec3[2] = pvec.z;
        dvec3[0] = dvec.x; dvec3[1] = dvec.y; dvec3[2] = dvec.z;
    } catch (const std::exception&) {
        for (int k = 0; k < 3; ++k) pvec3[k] = dvec3[k] = NAN;
        r_g[0] = r_g[1] = NAN;
    }
}
// dbrent (dbrent.rs:20-169) on f(x) = (x - 3)^2 + 1 from the bracket (0, 2, 6) (dbrent.rs:172-181).
int orc_dbrent_quadratic(double* fmin_xmin) {
    auto f = [](double x) { return (x - 3.0) * (x - 3.0) + 1.0; };
    auto df = [](double x) { return 2.0 * (x - 3.0); };
    return dbrent(0.0, 2.0, 6.0, f, df, 1e-10, false, 0.0, fmin_xmin[0], fmin_xmin[1]) ? 1 : 0;
}
// One bsstep (bsstep.rs:159-326) of dy/dx = y from y(0) = 1 with htry = 1 (bsstep.rs:570-597):
// returns y and the x reached.
void orc_bsstep_exp(double* y_x) {
    double y[1] = {1.0}, dydx[1] = {1.0}, yscal[1] = {1.0}, xx = 0.0, hdid = 0.0, hnext = 0.0;
    BsState st;
    Derivs d = [](double, const double* yi, double* dy) { dy[0] = yi[0]; };
    bsstep(y, dydx, 1, xx, 1.0, 1e-10, yscal, st, d, hdid, hnext);
    y_x[0] = y[0];
    y_x[1] = xx;
}
// svd_scale (orchestration.rs:405-436) on caller-supplied component fluxes (fcomp: n x ncol,
// row-major), for checks of the least-squares restatement itself.
void orc_svd_scale(const double* flux, const double* ferr, const double* weight, int n, const double* fcomp,
                   int ncol, double* out) {
    std::vector<Datum> data(n);
    std::vector<std::vector<double>> fc(n, std::vector<double>(ncol));
    for (int i = 0; i < n; ++i) {
        data[i].flux = flux[i]; data[i].ferr = ferr[i]; data[i].weight = weight[i];
        for (int j = 0; j < ncol; ++j) fc[i][j] = fcomp[(size_t)i * ncol + j];
    }
    std::vector<double> x = svd_scale(data, fc, ncol);
    for (int j = 0; j < ncol; ++j) out[j] = x[j];
}
// The exports below return NaNs where the reference raises an error (an unreachable
// radius, an invalid q): an exception must not cross the C boundary.
void orc_stream_spot(double q, double rad, double* out3) {
    try {
        Vec3 r, v;
        strinit(q, r, v);
        stradv(q, r, v, rad, 1e-10, 1e-3);
        out3[0] = r.x; out3[1] = r.y; out3[2] = r.z;
    } catch (const std::exception&) {
        out3[0] = out3[1] = out3[2] = NAN;
    }
}
// Per-element star-eclipse interval (for parity of the eclipse kernel on arbitrary points).
int orc_star_eclipse(double q, double r, double spin, double ffac, double iangle, const double* posn, double delta,
                     int roche, int star, double* ing, double* eg) {
    EclipseVec e;
    star_eclipse(q, r, spin, ffac, iangle, Vec3(posn[0], posn[1], posn[2]), delta, roche != 0, star ? SECONDARY : PRIMARY, e);
    flush_counters();
    if (e.empty()) return 0;
    *ing = e[0].first; *eg = e[0].second;
    return 1;
}
void orc_counters(long long* out) {
    flush_counters();
    out[0] = g_fblink_calls.load(); out[1] = g_rpot_evals.load(); out[2] = g_drpot_evals.load();
}
void orc_counters_reset() {
    flush_counters();
    g_fblink_calls = 0; g_rpot_evals = 0; g_drpot_evals = 0;
}

}  // extern "C"
