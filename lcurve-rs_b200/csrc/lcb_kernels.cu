// lcb_kernels.cu — sm_100a kernels of the light-curve path, in launch order.
//
//   k_phase    : one thread per datum: ephemeris + Roemer phase and the
//                exposure sub-divisions (orchestration.rs:231-241,
//                flux.rs:379-387) with their earth vectors.
//   k_elements : one thread per grid element of every model in the batch.
//                Surface point (surface.rs:54-121) or sphere point, area,
//                gravity (grid.rs:201-322; disc/rim/spot grid.rs:336-553);
//                eclipse intervals by a spherical star (eclipse.rs:229-265)
//                and by an opaque disc (disc_eclipse.rs:84-330); continuum
//                flux (brightness.rs).  Elements eclipsed by a Roche-distorted
//                star keep that slot for k_roche.
//   k_roche    : one thread per element eclipsed by a Roche-distorted star:
//                the FP64 ray-march ingress_egress (eclipse.rs:270-373), the
//                phase scan with exact second-order miss proofs, then the two
//                bisections.  Small batches run k_roche_scan (the scan split
//                over several threads, first hit by atomicMin) and
//                k_roche_chop2 (the ingress and egress bisections from that
//                hit, one thread each) instead.
//   k_aux      : per star element, the per-model FP64 sums of ginterp,
//                wdwarf, log g and radii (flux.rs:115-206, 288-373).
//   k_flux     : persistent FP32 flux sum (flux.rs:7-111) over work units of
//                (element range x 512 sub-phases).  Element chunks arrive in
//                shared memory by cp.async.bulk (TMA) double buffering; a
//                classification pass lists each chunk's contributing
//                elements; each thread keeps 4 sub-phases in registers, in
//                pairs on the packed FP32x2 pipe, and accumulates in FP32
//                blocks of 32 elements folded into a two-sum pair.
//                Visibility is decided exactly in FP64 per (element, tile)
//                and per sub-phase only where an eclipse edge falls inside
//                the tile.
//   k_epilogue : one block per model: ginterp scale factors, exposure
//                smearing, slope/third, chi-squared / re_scale
//                (orchestration.rs:243-310, 361-401), and with iscale = 1 the
//                per-component fluxes and their one-sided Jacobi SVD scale
//                factors (405-436).
#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "lcb_kernels.cuh"
#include "lcb_stream.h"

namespace lcb {

namespace {

// LCURVE_DEBUG_BOUNDS build (make bounds): index checks that record
// kStatusBounds for the model and skip the access instead of reading or
// writing out of range; in the normal build they compile to nothing.
#ifdef LCURVE_DEBUG_BOUNDS
#define LCB_IN_BOUNDS(cond, status_word) ((cond) || (atomicOr((status_word), kStatusBounds), false))
#else
#define LCB_IN_BOUNDS(cond, status_word) true
#endif

constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kFac1 = 2.0e27 * 6.6262e-34 * 2.99792458e8;      // planck.rs:5
constexpr double kFac2 = 1.0e9 * 6.6262e-34 * 2.99792458e8 / 1.3806e-23;  // planck.rs:8
constexpr double kFwhmEfac = 2.3548200450309493;                  // brightness.rs:8
constexpr double kEfac = 1.0000001;                               // grid.rs:396
#ifndef LCB_ROCHE_MIN_BLOCKS
#define LCB_ROCHE_MIN_BLOCKS 5
#endif
#ifndef LCB_CERT_BUDGET
#define LCB_CERT_BUDGET 32
#endif
constexpr int kRocheMinBlocks = LCB_ROCHE_MIN_BLOCKS;  // k_roche blocks per SM (128 threads): register budget
#ifndef LCB_SCAN_MIN_BLOCKS
#define LCB_SCAN_MIN_BLOCKS LCB_ROCHE_MIN_BLOCKS
#endif
#ifndef LCB_CHOP_MIN_BLOCKS
#define LCB_CHOP_MIN_BLOCKS LCB_ROCHE_MIN_BLOCKS
#endif
constexpr int kScanMinBlocks = LCB_SCAN_MIN_BLOCKS;  // the same for the split scan (small batches)
constexpr int kChopMinBlocks = LCB_CHOP_MIN_BLOCKS;  // and for its bisection kernel
constexpr int kCertBudget = LCB_CERT_BUDGET;           // miss-proof nodes per line of sight before the full search
#ifndef LCB_TUBE_MAX
#define LCB_TUBE_MAX 8
#endif
constexpr int kTubeMax = LCB_TUBE_MAX;  // scan steps per phase-block miss proof (1: single steps only)
#ifndef LCB_FLUX_UNROLL
#define LCB_FLUX_UNROLL 4
#endif
constexpr int kFluxUnroll = LCB_FLUX_UNROLL;  // list elements per unrolled step of the flux loop
#ifndef LCB_SPLIT_TUBES
#define LCB_SPLIT_TUBES 0  // phase blocks in the split scan of small batches (slower there: 0)
#endif
#ifndef LCB_TUBE_BUDGET
#define LCB_TUBE_BUDGET 24
#endif
constexpr int kTubeBudget = LCB_TUBE_BUDGET;  // nodes of one phase-block proof
constexpr int kTubeCool = 8;  // single steps after a failed two-step block before the next block
#ifndef LCB_CHOP_BUDGET
#define LCB_CHOP_BUDGET 0
#endif
constexpr int kChopBudget = LCB_CHOP_BUDGET;           // the same in the bisections (0: no proofs there)

__device__ __forceinline__ double sq(double x) { return x * x; }
__device__ __forceinline__ double rad2deg(double r) { return r * (180.0 / kPi); }

__device__ __forceinline__ double planck_d(double wave, double temp) {  // planck.rs:16-23
    double e = kFac2 / (wave * temp);
    if (e > 40.0) return kFac1 * exp(-e) / (wave * sq(wave));
    return kFac1 / (exp(e) - 1.0) / (wave * sq(wave));
}

// ---------------------------------------------------------------------------
// Roche potentials
// ---------------------------------------------------------------------------
// Exact-rounding potential (surface.rs:54-121 builds the stars from it).
__device__ __forceinline__ double pot_exact(bool primary, double q, double ssq, double x, double y, double z) {
    double mu = q / (1.0 + q), comp = 1.0 - mu;
    double x2y2 = sq(x) + sq(y);
    double r1sq = x2y2 + sq(z);
    double r1 = sqrt(r1sq), r2 = sqrt(r1sq + 1.0 - 2.0 * x);
    if (primary) return -comp / r1 - mu / r2 - ssq * x2y2 / 2.0 + mu * x;
    return -comp / r1 - mu / r2 - ssq * (0.5 + 0.5 * x2y2 - x) - comp * x;
}
__device__ __forceinline__ void dpot_exact(bool primary, double q, double ssq, double x, double y, double z,
                                           double& gx, double& gy, double& gz) {
    double r1sq = x * x + y * y + z * z, r2sq = r1sq + 1.0 - 2.0 * x;
    double r1 = sqrt(r1sq), r2 = sqrt(r2sq);
    double mu = q / (1.0 + q);
    double mu1 = mu / r2 / r2sq, comp = (1.0 - mu) / r1 / r1sq;
    gx = comp * x + mu1 * (x - 1.0) - (primary ? ssq * x - mu : ssq * (x - 1.0) - mu + 1.0);
    gy = comp * y + mu1 * y - ssq * y;
    gz = comp * z + mu1 * z;
}

// Potential along a line of sight p + lam*e for the eclipse search
// (potential.rs:110-117).  1/r from rsqrt: decisions against pref differ
// from the divided form only within an ulp of the surface.
struct Los {
    double px, py, pz, ex, ey, ez;
};
__device__ __forceinline__ double los_pot(const RocheEcl& s, const Los& L, double lam) {
    double x = fma(lam, L.ex, L.px), y = fma(lam, L.ey, L.py), z = fma(lam, L.ez, L.pz);
    double x2y2 = x * x + y * y;
    double r1sq = x2y2 + z * z;
    double r2sq = r1sq + 1.0 - 2.0 * x;
    double v = -s.comp * rsqrt(r1sq) - s.mu * rsqrt(r2sq);
    if (s.primary) return v - s.ssq * x2y2 * 0.5 + s.mu * x;
    return v - s.ssq * (0.5 + 0.5 * x2y2 - x) - s.comp * x;
}
__device__ __forceinline__ double los_dpot(const RocheEcl& s, const Los& L, double lam) {  // potential.rs:120-127
    double x = fma(lam, L.ex, L.px), y = fma(lam, L.ey, L.py), z = fma(lam, L.ez, L.pz);
    double r1sq = x * x + y * y + z * z, r2sq = r1sq + 1.0 - 2.0 * x;
    double i1 = rsqrt(r1sq), i2 = rsqrt(r2sq);
    double comp = s.comp * (i1 * i1 * i1), mu1 = s.mu * (i2 * i2 * i2);
    double gx = comp * x + mu1 * (x - 1.0) - (s.primary ? s.ssq * x - s.mu : s.ssq * (x - 1.0) - s.mu + 1.0);
    double gy = comp * y + mu1 * y - s.ssq * y;
    double gz = comp * z + mu1 * z;
    return gx * L.ex + gy * L.ey + gz * L.ez;
}

// Work counters of the eclipse search (potential and gradient evaluations, fblink calls),
// and the bound on one line-of-sight search's potential evaluations (the reference has
// none; reaching it marks the model failed: kStatusIterCap).
struct EclCount {
    int pot = 0, dpot = 0, fbl = 0, cert = 0, skipped = 0;
    int cap = kFblinkEvalCap;
};

// dbrent with stop-fast (crates/subs/src/numerical/dbrent.rs:20-165).
// Returns 1 = bracketed minimum below fref, 0 = not below.
// `local` counts the search's evaluations so far; past cnt.cap the search stops
// and sets `capped` (the model then fails).
__device__ bool dbrent_below(const RocheEcl& s, const Los& L, double ax, double bx, double cx, double acc,
                             double fref, EclCount& cnt, int& local, bool& capped) {
    double a = fmin(ax, cx), b = fmax(ax, cx);
    double x = bx, w = bx, v = bx;
    if (local + 2 > cnt.cap) { capped = true; return false; }
    local += 2;
    double fx = los_pot(s, L, x), fw = fx, fv = fx;
    ++cnt.pot;
    if (fx < fref) return true;
    double dx = los_dpot(s, L, x), dw = dx, dv = dx;
    ++cnt.dpot;
    double e = 0.0, d = 0.0;
    for (int it = 0; it < 100; ++it) {
        double xm = 0.5 * (a + b);
        double tol1 = acc, tol2 = 2.0 * tol1;
        if (fabs(x - xm) <= tol2 - 0.5 * (b - a)) return fx < fref;
        if (fabs(e) > tol1) {
            double d1 = 2.0 * (b - a), d2 = d1;
            if (dw != dx) d1 = (w - x) * dx / (dx - dw);
            if (dv != dx) d2 = (v - x) * dx / (dx - dv);
            double u1 = x + d1, u2 = x + d2;
            bool ok1 = (a - u1) * (u1 - b) > 0.0 && dx * d1 <= 0.0;
            bool ok2 = (a - u2) * (u2 - b) > 0.0 && dx * d2 <= 0.0;
            double olde = e;
            e = d;
            if (ok1 || ok2) {
                d = (ok1 && ok2) ? (fabs(d1) < fabs(d2) ? d1 : d2) : (ok1 ? d1 : d2);
                if (fabs(d) <= fabs(0.5 * olde)) {
                    double u = x + d;
                    if (u - a < tol2 || b - u < tol2) d = (xm - x >= 0.0) ? fabs(tol1) : -fabs(tol1);
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
        if (local + 2 > cnt.cap) { capped = true; return false; }
        local += 2;
        if (fabs(d) >= tol1) {
            u = x + d;
            fu = los_pot(s, L, u);
            ++cnt.pot;
            if (fu < fref) return true;
        } else {
            u = x + (d >= 0.0 ? fabs(tol1) : -fabs(tol1));
            fu = los_pot(s, L, u);
            ++cnt.pot;
            if (fu < fref) return true;
            if (fu > fx) return fx < fref;
        }
        double du = los_dpot(s, L, u);
        ++cnt.dpot;
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
    return false;  // iteration cap: the reference maps its Err to "not eclipsed"
}

// Squared distances from the segment p + lam*e, lam in [a, b] (|e| = 1), to the
// two stars' centres (the primary at the origin, the secondary at (1, 0, 0)).
__device__ __forceinline__ void closest_sq(const Los& L, double a, double b, double& d1, double& d2) {
    double t1 = fmin(fmax(-(L.px * L.ex + L.py * L.ey + L.pz * L.ez), a), b);
    double x1 = fma(t1, L.ex, L.px), y1 = fma(t1, L.ey, L.py), z1 = fma(t1, L.ez, L.pz);
    d1 = x1 * x1 + y1 * y1 + z1 * z1;
    double qx = L.px - 1.0;
    double t2 = fmin(fmax(-(qx * L.ex + L.py * L.ey + L.pz * L.ez), a), b);
    double x2 = fma(t2, L.ex, qx), y2 = fma(t2, L.ey, L.py), z2 = fma(t2, L.ez, L.pz);
    d2 = x2 * x2 + y2 * y2 + z2 * z2;
}

#ifndef LCB_PROOF_FAST_RSQRT
#define LCB_PROOF_FAST_RSQRT 1
#endif
// 1/sqrt(x) for the miss proofs' nodes: a single-precision hardware estimate
// (rsqrtf, within 2 ulp of FP32, i.e. relative error e0 < 2^-22) refined by one
// Newton-Raphson step for the inverse square root in FP64, y1 = y0 (3 - x y0^2) / 2,
// whose relative error is 3/2 e0^2 + O(e0^3) < 2e-13 plus a few FP64 roundings.
// The proofs' 1e-9 relative margin above the surface value covers that many
// times over; the reference-path evaluations (los_pot, los_dpot) keep rsqrt.
// The squared distances to the two centres along a line of sight (a few
// separations long, in units of the separation) lie far inside FP32's normal
// range; at x = 0 the result is NaN, so the node's bound fails and the line of
// sight is left to the full search.
__device__ __forceinline__ double proof_rsqrt(double x) {
#if LCB_PROOF_FAST_RSQRT
    const double y = (double)rsqrtf((float)x);
    return y * fma(-0.5 * x, y * y, 1.5);
#else
    return rsqrt(x);
#endif
}

// The potential and its derivative along the line of sight at one point
// (los_pot and los_dpot sharing the two distances), and the gradient's norm
// when `grad` is not null.  For the miss proofs only (proof_rsqrt).
__device__ __forceinline__ void los_pot_dpot(const RocheEcl& s, const Los& L, double lam, double& f, double& df,
                                             double* grad = nullptr) {
    double x = fma(lam, L.ex, L.px), y = fma(lam, L.ey, L.py), z = fma(lam, L.ez, L.pz);
    double x2y2 = x * x + y * y;
    double r1sq = x2y2 + z * z, r2sq = r1sq + 1.0 - 2.0 * x;
    double i1 = proof_rsqrt(r1sq), i2 = proof_rsqrt(r2sq);
    double v = -s.comp * i1 - s.mu * i2;
    f = s.primary ? v - s.ssq * x2y2 * 0.5 + s.mu * x : v - s.ssq * (0.5 + 0.5 * x2y2 - x) - s.comp * x;
    double comp = s.comp * (i1 * i1 * i1), mu1 = s.mu * (i2 * i2 * i2);
    double gx = comp * x + mu1 * (x - 1.0) - (s.primary ? s.ssq * x - s.mu : s.ssq * (x - 1.0) - s.mu + 1.0);
    double gy = comp * y + mu1 * y - s.ssq * y;
    double gz = comp * z + mu1 * z;
    df = gx * L.ex + gy * L.ey + gz * L.ez;
    if (grad) {  // |grad| = n2 / sqrt(n2), to the same 2e-13 (n2 = 0: NaN, the node fails)
        const double n2 = gx * gx + gy * gy + gz * gz;
        *grad = n2 * proof_rsqrt(n2);
    }
}

// True when the potential provably stays above the surface value on the whole
// line-of-sight segment [a, b]: an adaptive march over sub-segments, each
// certified by a second-order bound.  Along a line the Roche potential's
// second derivative is at least -M, M = 2 comp / r1^3 + 2 mu / r2^3 + ssq with
// r1, r2 the segment's closest approaches to the two centres (each gravity
// term -c / r has second derivative c (r^2 - 3 s^2) / r^5 >= -2 c / r^3, s the
// distance along the line from the closest point; the centrifugal term
// -ssq (x^2 + y^2) / 2 contributes -ssq (ex^2 + ey^2) >= -ssq; the rest is
// linear), so on a sub-segment of length h around m
//   phi >= phi(m) - |phi'(m)| h / 2 - M h^2 / 8.
// The bound must clear the surface value by 1e-9 relative (far above the
// rounding of any evaluation).  False means "not proven".
//
// With w > 0 the segment stands for a fan of lines through p whose unit
// directions lie within w of L's: every point of the fan at parameter t is
// within |t| w of L's point at t.  The Hessian of the potential has norm at
// most H = 2 comp / r1^3 + 2 mu / r2^3 + ssq with r1, r2 now the closest
// approaches of that tube, so a point x within r of the sub-segment's point y
// has phi(x) >= phi(y) - |grad phi(y)| r - H r^2 / 2, and
// |grad phi(y)| <= |grad phi(m)| + H h / 2: each node subtracts
// (|grad phi(m)| + H h / 2) r + H r^2 / 2, r = (|m| + h / 2) w.
template <bool kTube>
__device__ __forceinline__ bool certify_miss(const RocheEcl& s, const Los& L, double a, double b, int budget,
                                             int& nodes, double w = 0.0) {
    const double thr = s.pref + 1e-9 * fmax(fabs(s.pref), 1.0);
    const double hmin = 1e-6 * (b - a);
    double d1, d2;
    closest_sq(L, a, b, d1, d2);
    const double i1 = rsqrt(d1), i2 = rsqrt(d2);
    const double curv = 2.0 * s.comp * (i1 * i1 * i1) + 2.0 * s.mu * (i2 * i2 * i2) + s.ssq;
    double hess = 0.0;
    if (kTube) {
        const double widen = fmax(fabs(a), fabs(b)) * w;
        const double r1 = sqrt(d1) - widen, r2 = sqrt(d2) - widen;
        if (!(r1 > 1e-3 && r2 > 1e-3)) return false;
        hess = 2.0 * s.comp / (r1 * r1 * r1) + 2.0 * s.mu / (r2 * r2 * r2) + s.ssq;
    }
    double t = a, h = b - a;
    for (int it = 0; it < budget; ++it) {
        if (t >= b) return true;
        double hh = fmin(h, b - t);
        ++nodes;
        const double m = t + 0.5 * hh;
        double f, df, g = 0.0;
        los_pot_dpot(s, L, m, f, df, kTube ? &g : nullptr);
        double bound = f - fabs(df) * (0.5 * hh) - curv * (0.125 * hh * hh);
        if (kTube) {
            const double r = (fabs(m) + 0.5 * hh) * w;
            bound -= (g + hess * (0.5 * hh)) * r + 0.5 * hess * r * r;
        }
        if (bound > thr) {
            t += hh;
            h = 2.0 * hh;
        } else {
            if (hh <= hmin) return false;
            h = 0.5 * hh;
        }
    }
    return t >= b;
}

// Is point p hidden from earth direction e by the Roche star? (eclipse.rs:123-197)
// With `prove` > 0 (a node budget), a line of sight whose first reference evaluation is not
// inside the star is first tested with the rigorous second-order bound: every point
// the reference search evaluates lies in [lam1 - acc, lam2 + acc] (dbrent.rs:116
// may step acc past an end), so a proven miss is exactly its "false".
// Not inlined: as a call, the search's working set does not add to the
// registers the surrounding scan/bisection loop keeps live, which lets the
// kernel run 5 blocks per SM (451 -> 350 ms on the 1024-model batch).
__device__ __noinline__ bool fblink(const RocheEcl& s, double acc, const Los& L, EclCount& cnt, bool& capped, int prove) {
    ++cnt.fbl;
    double dx = L.px - s.cofmx, dy = L.py, dz = L.pz;
    double bq = L.ex * dx + L.ey * dy + L.ez * dz;  // sphere_eclipse_los, eclipse.rs:202-224
    if (bq >= 0.0) return false;
    double cq = (dx * dx + dy * dy + dz * dz) - sq(s.rref);
    double fac = sq(bq) - cq;
    if (fac <= 0.0) return false;
    fac = sqrt(fac);
    double lam2 = -bq + fac, lam1 = fmax(cq / lam2, 0.0);
    if (lam1 == 0.0) return true;
    const double pref = s.pref;
    double step = lam2 - lam1;
    if (!(step > acc)) return false;  // no evaluation: flam = 1 > f1 = f2 = 0
    // the reference's first evaluation, at the middle of the chord
    const double lam0 = lam1 + step / 2.0;
    double flam = los_pot(s, L, lam0);
    ++cnt.pot;
    if (flam <= pref) return true;
    if (prove > 0) {  // prove: the miss-proof node budget (0: no proof)
        const double pad = 1.001 * acc + 1e-12;
        if (certify_miss<false>(s, L, lam1 - pad, lam2 + pad, prove, cnt.cert)) { ++cnt.skipped; return false; }
    }
    int nstep = 1;
    double f1 = los_pot(s, L, lam1), f2 = los_pot(s, L, lam2), lam = lam0;
    int local = 2;
    bool br = flam < f1 && flam < f2;
    if (!br) {
        step /= 2.0;
        nstep = 2;
        while (step > acc) {
            lam = lam1 + step / 2.0;
            for (int n = 0; n < nstep; ++n) {
                flam = los_pot(s, L, lam + (double)n * step);
                ++local;
                if (flam <= pref) { cnt.pot += local; return true; }
                if (flam < f1 && flam < f2) { lam = lam + (double)n * step; br = true; break; }
            }
            if (br) break;
            if (local > cnt.cap) { capped = true; cnt.pot += local; return false; }
            step /= 2.0;
            nstep *= 2;
        }
    }
    cnt.pot += local;
    if (br) return dbrent_below(s, L, lam1, lam, lam2, acc, pref, cnt, local, capped);
    return false;
}

// Phase-block miss proof: L is the middle line of a block of consecutive scan
// steps whose unit directions lie within tube_w of L's (all lines pass through
// p).  True when every step of the block provably misses, i.e. each step's own
// fblink would return false (see certify_miss).  A separate call from fblink:
// the single-step search keeps its own, smaller register allocation.
__device__ __noinline__ bool tube_miss(const RocheEcl& s, double acc, const Los& L, double tube_w, int budget,
                                       int& nodes) {
    const double dx = L.px - s.cofmx, dy = L.py, dz = L.pz;
    // every step's b = e.d lies within |d| tube_w of the middle line's; its chord of the
    // bounding sphere, where it has one, within [c / lam2max, lam2max] (lam2 = -b +
    // sqrt(b^2 - c) falls as b rises)
    const double dd = dx * dx + dy * dy + dz * dz;
    const double cq = dd - sq(s.rref);
    if (!(cq > 0.0)) return false;
    const double bmin = L.ex * dx + L.ey * dy + L.ez * dz - sqrt(dd) * tube_w;
    if (bmin >= 0.0) return true;  // every step: b >= 0, no chord
    const double fac = sq(bmin) - cq;
    if (fac <= 0.0) return true;   // every step misses the bounding sphere
    const double lam2 = -bmin + sqrt(fac), lam1 = cq / lam2;
    const double pad = 1.001 * acc + 1e-12;
    return certify_miss<true>(s, L, lam1 - pad, lam2 + pad, budget, nodes, tube_w);
}

__device__ __forceinline__ void earth_at(double cosi, double sini, double phase, double& ex, double& ey, double& ez) {
    double sn, cs;  // misc.rs:42-45
    sincos(kTwoPi * phase, &sn, &cs);
    ex = sini * cs;
    ey = -sini * sn;
    ez = cosi;
}

// Analytic sphere eclipse (eclipse.rs:229-265).
__device__ bool sphere_phase(double cosi, double sini, double px, double py, double pz, double cx, double rs,
                             double& phi1, double& phi2, double& lam1, double& lam2) {
    double dx = px - cx, dy = py, dz = pz;
    double pdist = sqrt(sq(dx) + sq(dy));
    double bq = dz * cosi - pdist * sini;
    if (bq >= 0.0) return false;
    double cq = (dx * dx + dy * dy + dz * dz) - sq(rs);
    double fac = sq(bq) - cq;
    if (fac <= 0.0) return false;
    fac = sqrt(fac);
    lam2 = -bq + fac;
    lam1 = fmax(cq / lam2, 0.0);
    if (cq < 0.0) {
        phi1 = 0.0;
        phi2 = 1.0;
    } else {
        double delta = acos((cosi * dz + sqrt(cq)) / (sini * pdist));
        double phi = atan2(dy, -dx);
        double p1 = (phi - delta) / kTwoPi;
        p1 -= floor(p1);
        phi1 = p1;
        phi2 = p1 + 2.0 * delta / kTwoPi;
    }
    return true;
}

// Ingress/egress of point p behind a Roche-distorted star (eclipse.rs:270-373).
// The phase scan of pot_min_search (eclipse.rs:347-373) and the two bisections
// (eclipse.rs:301-332) run as one loop with a single line-of-sight search call
// site: lanes of a warp in different stages reconverge inside the search, and
// the search code exists once.  Misses are proven (fblink's `prove`) only in the
// scan, where nearly all lines of sight miss by a wide margin.
// The phase scan of pot_min_search (eclipse.rs:347-373): phases phi1 + i dphi,
// i = 0 .. nsteps, and the search tolerance acc (eclipse.rs:297).
struct Scan {
    double phi1, phi2, acc, dphi;
    int nsteps;
};
__device__ __forceinline__ bool scan_setup(const RocheEcl& s, double cosi, double sini, double delta, double px,
                                           double py, double pz, Scan& sc) {
    double lam1, lam2;
    if (!sphere_phase(cosi, sini, px, py, pz, s.cofmx, s.rref, sc.phi1, sc.phi2, lam1, lam2)) return false;
    sc.acc = 2.0 * sqrt(2.0 * kTwoPi * (lam2 - lam1) * delta);
    double ns = ceil((sc.phi2 - sc.phi1) / (sc.acc / kTwoPi));
    sc.nsteps = (ns != ns || ns <= 10.0) ? 10 : (ns >= 1000.0 ? 1000 : (int)ns);
    sc.dphi = (sc.phi2 - sc.phi1) / (double)sc.nsteps;
    return true;
}

// Bound on |e(ph) - e(mid)| for phases within `half` of mid: the earth vector's
// xy part (length sini) turns by 2 pi (ph - mid), a chord of 2 sini sin(pi |ph - mid|).
__device__ __forceinline__ double tube_width(double sini, double half) {
    return 2.0 * sini * sin(fmin(kPi * half, 0.5 * kPi)) * (1.0 + 1e-12) + 1e-15;
}

constexpr int kNoHit = 0x7f7f7f7f;  // first-hit sentinel (the byte pattern a memset of 0x7f writes)

// `known_hit` >= 0: the scan's first hit is already known (split scan): go
// straight to the bisections from that phase; kNoHit: the point is not eclipsed.
// `only` = 1 or 2 runs just the ingress or just the egress bisection (the two are
// independent: both start from the first hit), leaving `ing` resp. the unwrapped
// `eg` set; the caller then applies egress < ingress -> egress + 1 itself.
// kScan = false compiles the bisections alone (a known first hit is then required).
template <bool kScan>
__device__ bool ingress_egress(const RocheEcl& s, double cosi, double sini, double delta, double px, double py,
                               double pz, double& ing, double& eg, bool& capped, EclCount& evals, int known_hit = -1,
                               int only = 0) {
    Scan sc;
    if (!scan_setup(s, cosi, sini, delta, px, py, pz, sc)) return false;
    if (known_hit == kNoHit) return false;
    const double phi1 = sc.phi1, phi2 = sc.phi2, acc = sc.acc, dphi = sc.dphi;
    const int nsteps = sc.nsteps;
    Los L{px, py, pz, 0.0, 0.0, 0.0};
    enum { SCAN, CHOP_IN, CHOP_EG };
    // blk: scan steps the next phase-block proof covers; after a failed two-step block,
    // kTubeCool single steps before the next (wait)
    int mode = SCAN, i = 0, it = 0, blk = kTubeMax, wait = 0, last = 0;
    double phi = 0.0, pin = 0.0, pout = 0.0;
    if (known_hit >= 0) {  // as the scan below sets up its first hit
        phi = phi1 + (double)known_hit * dphi;
        if (only == 2) { mode = CHOP_EG; pin = phi; pout = phi2; }
        else { mode = CHOP_IN; pin = phi; pout = phi1; }
    }
    for (;;) {
        double ph, tube = 0.0;
        if (kScan && mode == SCAN) {
            if (i > nsteps) return false;  // no eclipsed phase found
            last = wait > 0 ? i : min(i + blk - 1, nsteps);
            if (last > i) {  // steps i .. last at once: one phase-block proof
                ph = phi1 + 0.5 * (double)(i + last) * dphi;
                tube = tube_width(sini, 0.5 * (double)(last - i) * dphi);
            } else {
                ph = phi1 + (double)i * dphi;
            }
        } else {
            if (!(fabs(pin - pout) > delta) || it >= 200) {
                double r = (pin + pout) / 2.0;
                r -= floor(r);
                if (mode == CHOP_IN) {
                    ing = r;
                    if (only == 1) return true;
                    mode = CHOP_EG; pin = phi; pout = phi2; it = 0;
                    continue;
                }
                eg = r;
                if (only == 2) return true;
                if (eg < ing) eg += 1.0;
                return true;
            }
            ph = (pin + pout) / 2.0;
        }
        earth_at(cosi, sini, ph, L.ex, L.ey, L.ez);
        const bool hit = tube > 0.0 ? tube_miss(s, acc, L, tube, kTubeBudget, evals.cert)
                                    : fblink(s, acc, L, evals, capped, !(kScan && mode == SCAN) ? kChopBudget : kCertBudget);
        if (capped) return false;
        if (kScan && mode == SCAN) {
            if (tube > 0.0) {
                if (hit) {  // the block's steps are all misses: counted as the searches they stand for
                    evals.fbl += last - i + 1;
                    ++evals.skipped;  // one proof
                    i = last + 1;
                    blk = min(2 * blk, kTubeMax);
                } else {
                    blk >>= 1;
                    if (blk < 2) wait = kTubeCool;
                }
            } else if (hit) { phi = ph; mode = CHOP_IN; pin = phi; pout = phi1; it = 0; }
            else {
                ++i;
                if (wait > 0) --wait;
                if (wait == 0) blk = max(blk, min(2, kTubeMax));
            }
        } else {
            if (hit) pin = ph; else pout = ph;
            ++it;
        }
    }
}

// Disc occultation (disc_eclipse.rs:29-70, 84-330); returns the number of pairs (<= 2).
__device__ __forceinline__ double cut_phase(double rxy, double rcone, double radius) {
    double c = (sq(rxy) + sq(rcone) - sq(radius)) / (2.0 * rcone * rxy);
    return acos(fmin(fmax(c, -1.0), 1.0)) / kTwoPi;
}
enum { C_ABOVE, C_INSIDE, C_OUTSIDE, C_SEPARATE, C_CROSSING };
__device__ __forceinline__ int circle_ecl(double rxy, double z, double zc, double radius, double tani, double& ph) {
    ph = 0.0;
    if (z >= zc) return C_ABOVE;
    double rcone = tani * (zc - z);
    if (rcone >= rxy + radius) return C_OUTSIDE;
    if (rxy >= rcone + radius) return C_SEPARATE;
    if (rxy + rcone <= radius) return C_INSIDE;
    ph = cut_phase(rxy, rcone, radius);
    return C_CROSSING;
}
__device__ int disc_eclipse(const ModelDev& M, double rdisc1, double px, double py, double pz, double* ing,
                            double* eg) {
    const double rdisc2 = M.rdisc2, beta = M.beta, height = M.height;
    double hout = height * pow(rdisc2, beta);
    if (pz >= hout) return 0;
    double sini = M.sini_d, cosi = M.cosi_d;
    if (cosi == 0.0) {
        if (fabs(pz) < hout) {
            double rxy = sqrt(sq(px) + sq(py));
            if (rxy <= rdisc2) { ing[0] = 0.0; eg[0] = 1.0; return 1; }
            double subtend = asin(rdisc2 / rxy) / kTwoPi;
            double pc = atan2(py, -px) / kTwoPi;
            double i0 = pc - subtend;
            i0 -= floor(i0);
            ing[0] = i0; eg[0] = i0 + 2.0 * subtend;
            return 1;
        }
        return 0;
    }
    double rxy = sqrt(sq(px) + sq(py));
    if (rdisc1 < rxy && rxy < rdisc2 && fabs(pz) < height * pow(rxy, beta)) { ing[0] = 0.0; eg[0] = 1.1; return 1; }
    double tani = sini / cosi;
    if (rxy < rdisc2 && pz >= height * pow(fmax(rdisc1, rxy), beta)) {
        double ph;
        int r = circle_ecl(rxy, pz, hout, rdisc2, tani, ph);
        if (r == C_OUTSIDE) { ing[0] = 0.0; eg[0] = 1.1; return 1; }
        if (r == C_CROSSING) {
            double i0 = atan2(py, -px) / kTwoPi + ph;
            i0 -= floor(i0);
            ing[0] = i0; eg[0] = i0 + 1.0 - 2.0 * ph;
            return 1;
        }
        return 0;
    }
    double rlo = fmax(tani * (-hout - pz), 0.0);
    if (rlo >= rxy + rdisc2) return 0;
    double rhi = tani * (hout - pz);
    if (rxy >= rhi + rdisc2) return 0;
    double ecl;
    if (rxy + rlo <= rdisc2) ecl = 0.5;
    else if (rxy <= rdisc2) ecl = cut_phase(rxy, rlo, rdisc2);
    else if (sq(rhi) + sq(rdisc2) >= sq(rxy) && sq(rlo) + sq(rdisc2) <= sq(rxy)) ecl = asin(rdisc2 / rxy) / kTwoPi;
    else if (sq(rhi) + sq(rdisc2) < sq(rxy)) ecl = cut_phase(rxy, rhi, rdisc2);
    else ecl = cut_phase(rxy, rlo, rdisc2);
    double hin = height * pow(rdisc1, beta);
    double app = -1.0;
    auto first = [&](double zc, double rad) {
        double ph;
        int r = circle_ecl(rxy, pz, zc, rad, tani, ph);
        if (r == C_INSIDE) app = 0.5; else if (r == C_CROSSING) app = ph;
    };
    auto next = [&](double zc, double rad) {
        if (!(app > 0.0)) return;
        double ph;
        int r = circle_ecl(rxy, pz, zc, rad, tani, ph);
        if (r == C_CROSSING) app = fmin(app, ph); else if (r != C_INSIDE) app = -1.0;
    };
    if (pz < -hout) {
        first(-hout, rdisc2); next(-hin, rdisc1); next(hin, rdisc1); next(hout, rdisc2);
    } else if (rxy < rdisc1) {
        if (pz < -hin) { first(-hin, rdisc1); next(hin, rdisc1); next(hout, rdisc2); }
        else if (pz < hin) { first(hin, rdisc1); next(hout, rdisc2); }
    }
    double phi0 = atan2(py, -px) / kTwoPi;
    if (app <= 0.0) {
        double i0 = phi0 - ecl;
        i0 -= floor(i0);
        ing[0] = i0; eg[0] = i0 + 2.0 * ecl;
        return 1;
    }
    if (app < ecl) {
        double i0 = phi0 - ecl;
        i0 -= floor(i0);
        ing[0] = i0; eg[0] = i0 + (ecl - app);
        double i1 = phi0 + app;
        i1 -= floor(i1);
        ing[1] = i1; eg[1] = i1 + (ecl - app);
        return 2;
    }
    return 0;
}

// Irradiated temperature (brightness.rs:150-174) -> temp, geom.
__device__ __forceinline__ double irradiate(double tbase, double gravity, double gdcbol, double absorb, double tirr,
                                            double mu, double r, double rirr, double& geom) {
    double tg = tbase * pow(gravity, gdcbol);
    double tg4 = sq(tg) * sq(tg), ti4 = sq(tirr) * sq(tirr);
    if (mu >= rirr) {
        geom = sq(rirr / r) * mu;
        return pow(tg4 + absorb * ti4 * geom, 0.25);
    }
    if (mu > -rirr) {
        double x0 = -mu / rirr;
        geom = sq(rirr / r) * rirr * (sqrt(1.0 - x0 * x0) * (2.0 + x0 * x0) / 3.0 - x0 * (kPi / 2.0 - asin(x0))) / kPi;
        return pow(tg4 + absorb * ti4 * geom, 0.25);
    }
    geom = 0.0;
    return tg;
}

__device__ __forceinline__ double ang_dist(double px, double py, double pz, const SpotDev& s, double len) {
    if (len <= 0.0) return 180.0;  // brightness.rs:177-183
    double c = fmin(fmax((px * s.dx + py * s.dy + pz * s.dz) / len, -1.0), 1.0);
    return rad2deg(acos(c));
}

// LDC::imu in FP64 (types.rs:101-119)
__device__ __forceinline__ double imu_d(const double* l, int ltype, double mu) {
    if (mu <= 0.0) return 0.0;
    mu = fmin(mu, 1.0);
    double om = 1.0 - mu, im = 1.0;
    if (ltype == 0) {
        im -= om * (l[0] + om * (l[1] + om * (l[2] + om * l[3])));
    } else {
        im -= l[0] + l[1] + l[2] + l[3];
        double ms = sqrt(mu);
        im += ms * (l[0] + ms * (l[1] + ms * (l[2] + ms * l[3])));
    }
    return im;
}

__device__ __forceinline__ double lens_mag_d(double sx, double sy, double sz, double ex, double ey, double ez,
                                             double rl) {  // flux.rs:390-406
    double d = -(sx * ex + sy * ey + sz * ez);
    if (d <= 0.0) return 1.0;
    double ax = sx + d * ex, ay = sy + d * ey, az = sz + d * ez;
    double p = sqrt(ax * ax + ay * ay + az * az), ph = p / 2.0, phsq = ph * ph, rd = rl * d;
    double pd = phsq > 25.0 * rd ? p + rd / p : ph + sqrt(phsq + rd);
    return pd * pd / (pd - ph) / ph / 4.0;
}

// ---------------------------------------------------------------------------
// k_elements: grid, continuum, analytic eclipses
// ---------------------------------------------------------------------------
// Eclipse pair slots per element: star elements use slot 0 for the eclipse by
// the other star and slots 1-2 for the opaque disc; disc, rim and spot
// elements use slots 0-1 for the disc, 2 for star 1 and 3 for star 2.  A
// Roche-distorted eclipser leaves its slot empty here for k_roche to fill.
__device__ __forceinline__ int roche_slot(int kind, int by) {
    return (kind == SEG_STAR1 || kind == SEG_STAR2) ? 0 : (by == 1 ? 2 : 3);
}

__global__ void __launch_bounds__(kElemThreads) k_elements(ElemArgs A) {
    const ElemBlock blk = A.blocks[blockIdx.x];
    const SegDesc sg = A.segs[blk.seg];
    const ModelDev& M = A.models[sg.model];
    const int64_t i = blk.offset + threadIdx.x;
    if (i >= sg.count) return;

    double px = 0, py = 0, pz = 0, dx = 0, dy = 0, dz = 1;
    float area = 0.f, grav = 1.f, flux = 0.f;
    double2 ecl[kMaxEcl];
    for (int k = 0; k < kMaxEcl; ++k) ecl[k] = make_double2(INFINITY, -INFINITY);

    // analytic eclipse by a spherical star (grid.rs:49-73); Roche stars go to k_roche
    auto sphere_ecl = [&](int by, int slot) {
        if (by == 1 ? M.roche1 : M.roche2) return;
        double a, b, l1, l2;
        if (sphere_phase(M.cosi_e, M.sini_e, px, py, pz, by == 1 ? 0.0 : 1.0, by == 1 ? M.r1 : M.r2, a, b, l1, l2))
            ecl[slot] = make_double2(a, b);
    };
    auto disc_ecl = [&](double rdisc1, int slot) {
        double a[2], b[2];
        int n = disc_eclipse(M, rdisc1, px, py, pz, a, b);
        for (int k = 0; k < n; ++k) ecl[slot + k] = make_double2(a[k], b[k]);
    };

    if (sg.kind == SEG_STAR1 || sg.kind == SEG_STAR2) {
        const bool primary = sg.kind == SEG_STAR1;
        // band of element i (grid.rs:227-262)
        int lo = 0, hi = sg.ntable - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (A.bands[sg.table + mid].first <= i) lo = mid; else hi = mid - 1;
        }
        if (!LCB_IN_BOUNDS(sg.table + lo < A.sz.nbands && sg.first + i < A.sz.nelem, A.status + sg.model)) return;
        const Band b = A.bands[sg.table + lo];
        const int64_t np = i - b.first;
        double phi = b.phi1 + (b.phi2 - b.phi1) * ((double)np + 0.5) / (double)b.nphi;
        double sinp, cosp;
        sincos(phi, &sinp, &cosp);
        double ux, uy, uz;
        if (M.npole) { ux = b.sint * cosp; uy = b.sint * sinp; uz = b.cost; }
        else { ux = b.cost; uy = b.sint * cosp; uz = b.sint * sinp; }
        const bool roche = primary ? M.roche1 : M.roche2;
        const double cofm = primary ? 0.0 : 1.0;
        double rad, g;
        if (roche) {  // face (surface.rs:54-121)
            const double ssq = primary ? sq(M.spin1) : sq(M.spin2);
            const double rref = primary ? M.rref1 : M.rref2, pref = primary ? M.pref1 : M.pref2;
            double rlo = rref / 2.0, rhi = rref, t = pref + 1.0;
            for (int k = 0; k < 30 && t > pref; ++k) {
                rlo = rhi / 2.0;
                t = pot_exact(primary, M.q, ssq, cofm + rlo * ux, rlo * uy, rlo * uz);
                if (t > pref) rhi = rlo;
            }
            for (int k = 0; k < 100 && rhi - rlo > M.acc_face; ++k) {
                double mid = (rlo + rhi) / 2.0;
                if (pot_exact(primary, M.q, ssq, cofm + mid * ux, mid * uy, mid * uz) < pref) rlo = mid;
                else rhi = mid;
            }
            rad = (rlo + rhi) / 2.0;
            px = cofm + rad * ux; py = rad * uy; pz = rad * uz;
            double gx, gy, gz;
            dpot_exact(primary, M.q, ssq, px, py, pz, gx, gy, gz);
            double n2 = gx * gx + gy * gy + gz * gz;
            g = sqrt(n2);
            if (n2 > 0.0) { dx = gx / g; dy = gy / g; dz = gz / g; }
            else { dx = gx; dy = gy; dz = gz; }
        } else {
            rad = primary ? M.r1 : M.r2;
            px = cofm + rad * ux; py = rad * uy; pz = rad * uz;
            dx = ux; dy = uy; dz = uz;
            g = 1.0;
        }
        area = (float)(((b.aphi * rad) * b.sint) * (b.ath * rad) / (ux * dx + uy * dy + uz * dz));
        grav = (float)(g / (primary ? M.gref1 : M.gref2));
        if (primary ? M.eclipse1 : M.eclipse2) sphere_ecl(primary ? 2 : 1, 0);
        if (M.add_disc && M.opaque) disc_ecl(M.rdisc1_l, 1);  // orchestration.rs:145-157
        // continuum (brightness.rs:49-144)
        const double cx = primary ? 1.0 : 0.0;
        double vx = cx - px, vy = -py, vz = -pz;
        double r = sqrt(vx * vx + vy * vy + vz * vz);
        double mu = (dx * vx + dy * vy + dz * vz) / r;
        double geom, temp;
        if (primary) {
            double t1 = M.t1, plen = sqrt(px * px + py * py + pz * pz);
            for (int k = 0; k < 3; ++k) {
                const SpotDev& s = M.spot1[k];
                if (!s.on) continue;
                double dist = ang_dist(px, py, pz, s, plen);
                t1 += (s.tcen - M.t1) * exp(-sq(dist / (s.fwhm / kFwhmEfac)) / 2.0);
            }
            if (M.uesp_on) {
                double el = sqrt(px * px + py * py);
                if (el > 0.0) {
                    double clat = fmin(fmax((px * px + py * py) / el / plen, -1.0), 1.0);
                    double dlat = rad2deg(acos(clat));
                    double clong = fmin(fmax((M.uesp_dx * px + M.uesp_dy * py) / el, -1.0), 1.0);
                    double dlong = rad2deg(acos(clong));
                    double hw = M.uesp_lathw, lw = M.uesp_longhw, tp = M.uesp_taper, ut = M.uesp_temp;
                    if (dlat <= hw && dlong <= lw) t1 = ut;
                    else if (dlat <= hw) t1 += (ut - M.t1) * exp(-(dlong - lw) / tp);
                    else if (dlong <= lw) t1 += (ut - M.t1) * exp(-(dlat - hw) / tp);
                    else t1 += (ut - M.t1) * exp(-(dlat - hw) / tp) * exp(-(dlong - lw) / tp);
                }
            }
            temp = irradiate(t1, (double)grav, M.gdcbol1, M.absorb, M.t2, mu, r, M.r2c, geom);
            flux = (float)((double)area * planck_d(M.wavelength, temp));
            if (M.mirror) flux += (float)((double)area * geom * M.planck_t2abs);
        } else {
            double t2 = fabs(M.t2);
            for (int k = 0; k < 2; ++k) {
                const SpotDev& s = M.spot2[k];
                if (!s.on) continue;
                double ox = px - 1.0, oy = py, oz = pz;
                double dist = ang_dist(ox, oy, oz, s, sqrt(ox * ox + oy * oy + oz * oz));
                t2 += (s.tcen - t2) * exp(-sq(dist / (s.fwhm / kFwhmEfac)) / 2.0);
            }
            temp = irradiate(t2, (double)grav, M.gdcbol2, M.absorb, M.t1, mu, r, M.r1c, geom);
            flux = (float)((double)area * planck_d(M.wavelength, temp));
            if (M.mirror) flux += (float)((double)area * geom * M.planck_t1);
        }
    } else if (sg.kind == SEG_DISC) {  // grid.rs:356-390, brightness.rs:204-212
        int lo = 0, hi = sg.ntable - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (A.rings[sg.table + mid].first <= i) lo = mid; else hi = mid - 1;
        }
        if (!LCB_IN_BOUNDS(sg.table + lo < A.sz.nrings && sg.first + i < A.sz.nelem, A.status + sg.model)) return;
        const Ring g = A.rings[sg.table + lo];
        double th = kTwoPi * (double)(i - g.first) / (double)g.ntheta;
        double st, ct;
        sincos(th, &st, &ct);
        px = g.rad * ct; py = g.rad * st; pz = g.h;
        dx = -ct * g.sinp; dy = -st * g.sinp; dz = g.cosp;
        area = (float)g.area;
        if (M.opaque) disc_ecl(M.rdisc1_g, 0);
        if (M.eclipse1) sphere_ecl(1, 2);
        if (M.eclipse2) sphere_ecl(2, 3);
        double r = sqrt(px * px + py * py + pz * pz);
        flux = (float)(M.disc_bright * pow(r / M.rdisc2, M.texp_disc) * (double)area);
    } else if (sg.kind == SEG_EDGE) {  // grid.rs:411-478, brightness.rs:215-239
        const int64_t col = i / M.edge_nout, row = i - col * M.edge_nout;
        double th = kTwoPi * (double)col / (double)M.edge_ntheta;
        double st, ct;
        sincos(th, &st, &ct);
        const double rv = M.edge_rad, h = M.edge_h;
        if (row == 0) {
            px = kEfac * rv * ct; py = kEfac * rv * st; pz = kEfac * h;
            area = (float)(M.edge_area / 2.0);
        } else {
            pz = -h + 2.0 * h * (double)(row - 1) / (double)(M.edge_nout - 1);
            px = kEfac * rv * ct; py = kEfac * rv * st;
            area = (float)M.edge_area;
        }
        dx = ct; dy = st; dz = 0.0;
        if (M.opaque) disc_ecl(M.rdisc1_g, 0);
        if (M.eclipse1) sphere_ecl(1, 2);
        if (M.eclipse2) sphere_ecl(2, 3);
        double vx = 1.0 - px, vy = -py, vz = -pz;
        double r = sqrt(vx * vx + vy * vy + vz * vz);
        double mu = (dx * vx + dy * vy + dz * vz) / r;
        double temp, r2 = M.r2e, t4 = sq(M.tedge) * sq(M.tedge), i4 = sq(M.t2abs) * sq(M.t2abs);
        if (mu >= r2) {
            double geom = sq(r2 / r) * mu;
            temp = pow(t4 + M.absorb_edge * i4 * geom, 0.25);
        } else if (mu > -r2) {
            double x0 = -mu / r2;
            double geom = sq(r2 / r) * r2 * (sqrt(1.0 - x0 * x0) * (2.0 + x0 * x0) / 3.0 - x0 * (kPi / 2.0 - asin(x0))) / kPi;
            temp = pow(t4 + M.absorb_edge * i4 * geom, 0.25);
        } else {
            temp = M.tedge;
        }
        flux = (float)((double)area * planck_d(M.wavelength, temp));
    } else {  // SEG_SPOT: grid.rs:520-550
        const int64_t k = i >> 1;
        const bool tilted = (i & 1) == 0;
        double dist = M.sfac_spot * (double)k / (double)(M.nspot - 1);
        double f = M.length_spot * (dist - M.bmax);
        px = M.bspot[0] + f * M.bvec[0]; py = M.bspot[1] + f * M.bvec[1]; pz = M.bspot[2] + f * M.bvec[2];
        if (M.eclipse1) sphere_ecl(1, 2);
        if (M.eclipse2) sphere_ecl(2, 3);
        double bright = M.bright_ref * pow(dist / M.bmax, M.expon_spot) *
                        exp(M.expon_spot / M.epow_spot - pow(dist, M.epow_spot));
        area = (float)M.area_spot;
        if (tilted) { dx = M.tvec[0]; dy = M.tvec[1]; dz = M.tvec[2]; flux = (float)(bright * (1.0 - M.cfrac_spot) * M.area_spot); }
        else { dx = 0.0; dy = 0.0; dz = 1.0; flux = (float)(bright * M.cfrac_spot * M.area_spot); }
    }
    const int64_t e = sg.first + i;
    if (!LCB_IN_BOUNDS(e < A.sz.nelem, A.status + sg.model)) return;
    A.el_rec[e] = make_float4((float)dx, (float)dy, (float)dz, flux);
    A.el_pos[e] = make_float4((float)px, (float)py, (float)pz, 0.f);
    A.el_p64[e] = make_double4(px, py, pz, (double)area);
    A.el_d64[e] = make_double4(dx, dy, dz, (double)grav);
    unsigned used = 0;
    for (int k = 0; k < kMaxEcl; ++k) {
        A.el_ecl[k * A.sz.nelem + e] = ecl[k];
        if (ecl[k].x <= 2.0) used |= 1u << k;
    }
    if (used) atomicOr(A.ecl_grp + e / kEclGroup, used);
}

// ---------------------------------------------------------------------------
// k_roche: FP64 Roche ray-march of one element per thread (eclipse.rs:270-373)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void roche_counters(const ElemArgs& A, const EclCount& cnt);

// ORs each lane's slot bits into its element group's used-slot word with one
// atomic per distinct word of the warp (lanes hold consecutive elements, so a
// warp spans one or two words).  All 32 lanes call it; g < 0 or bits == 0: none.
__device__ __forceinline__ void group_or_warp(unsigned* grp, int64_t g, unsigned bits) {
    const bool mine = bits != 0u && g >= 0;
    unsigned pending = __ballot_sync(0xffffffffu, mine);
    while (pending) {
        const int src = __ffs(pending) - 1;
        const int64_t gs = __shfl_sync(0xffffffffu, g, src);
        const bool same = mine && g == gs;
        const unsigned all = __reduce_or_sync(0xffffffffu, same ? bits : 0u);
        if ((int)(threadIdx.x & 31) == src) atomicOr(grp + gs, all);
        pending &= ~__ballot_sync(0xffffffffu, same);
    }
}

__global__ void __launch_bounds__(kRocheBlock, kRocheMinBlocks) k_roche(ElemArgs A) {
    const ElemBlock blk = A.rblocks[blockIdx.x];
    const SegDesc sg = A.segs[blk.seg];
    const int64_t i = blk.offset + threadIdx.x;
    EclCount cnt;
    cnt.cap = A.fblink_cap;
    bool capped = false;
    int64_t g = -1;
    unsigned bits = 0u;
    if (i < sg.count && LCB_IN_BOUNDS(sg.first + i < A.sz.nelem, A.status + sg.model)) {
        const ModelDev& M = A.models[sg.model];
        const int by = blk.by;
        const int64_t e = sg.first + i;
        const double4 p = A.el_p64[e];
        double a, b;
        if (ingress_egress<true>(by == 1 ? M.ecl1 : M.ecl2, M.cosi_e, M.sini_e, M.delta, p.x, p.y, p.z, a, b, capped, cnt)) {
            const int slot = roche_slot(sg.kind, by);
            A.el_ecl[slot * A.sz.nelem + e] = make_double2(a, b);
            g = e / kEclGroup;
            bits = 1u << slot;
        }
        if (capped) atomicOr(A.status + sg.model, kStatusIterCap);
    }
    group_or_warp(A.ecl_grp, g, bits);
    roche_counters(A, cnt);
}

// One chunk of a split phase scan: scan indices [c L, (c+1) L) of 0 .. nsteps,
// L = ceil((nsteps+1)/K); the first hit is merged into *first with atomicMin,
// and a chunk stops once an earlier chunk has hit.  The minimum over chunks is
// the single scan's first hit, so the decision is the reference's.
__device__ void scan_chunk(const RocheEcl& s, double cosi, double sini, double delta, double px, double py,
                           double pz, int chunk, int split, int* first, bool& capped, EclCount& evals) {
    Scan sc;
    if (!scan_setup(s, cosi, sini, delta, px, py, pz, sc)) return;
    const int total = sc.nsteps + 1, len = (total + split - 1) / split;
    const int lo = chunk * len, hi = min(total, lo + len);
    Los L{px, py, pz, 0.0, 0.0, 0.0};
#if LCB_SPLIT_TUBES
    int blk = kTubeMax, wait = 0, n = 0;  // phase blocks as in ingress_egress
    for (int i = lo; i < hi; ++n) {
        if ((n & 7) == 0 && *(volatile int*)first < lo) return;
        const int last = wait > 0 ? i : min(i + blk - 1, hi - 1);
        if (last > i) {
            earth_at(cosi, sini, sc.phi1 + 0.5 * (double)(i + last) * sc.dphi, L.ex, L.ey, L.ez);
            if (tube_miss(s, sc.acc, L, tube_width(sini, 0.5 * (double)(last - i) * sc.dphi), kTubeBudget, evals.cert)) {
                ++evals.skipped;
                i = last + 1;
                blk = min(2 * blk, kTubeMax);
            } else {
                blk >>= 1;
                if (blk < 2) wait = kTubeCool;
            }
            continue;
        }
        earth_at(cosi, sini, sc.phi1 + (double)i * sc.dphi, L.ex, L.ey, L.ez);
        const bool hit = fblink(s, sc.acc, L, evals, capped, kCertBudget);
        if (capped) return;
        if (hit) {
            atomicMin(first, i);
            return;
        }
        ++i;
        if (wait > 0) --wait;
        if (wait == 0) blk = max(blk, min(2, kTubeMax));
    }
#else
    for (int i = lo; i < hi; ++i) {
        if (((i - lo) & 7) == 0 && *(volatile int*)first < lo) return;
        earth_at(cosi, sini, sc.phi1 + (double)i * sc.dphi, L.ex, L.ey, L.ez);
        const bool hit = fblink(s, sc.acc, L, evals, capped, kCertBudget);
        if (capped) return;
        if (hit) {
            atomicMin(first, i);
            return;
        }
    }
#endif
}

__device__ __forceinline__ void roche_counters(const ElemArgs& A, const EclCount& cnt) {
    if (!A.counters) return;  // eclipse-search work counters, one atomic per warp and counter
    unsigned long long v[5] = {(unsigned long long)cnt.pot, (unsigned long long)cnt.dpot, (unsigned long long)cnt.fbl,
                               (unsigned long long)cnt.cert, (unsigned long long)cnt.skipped};
    for (int k = 0; k < 5; ++k) {
        unsigned long long x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0 && x) atomicAdd(A.counters + k, x);
    }
}

// Split scan, first kernel: block b scans chunk b % split of the elements of
// Roche block b / split.  For small batches, whose time is otherwise the
// longest single scan, this spreads each scan over `split` threads.
__global__ void __launch_bounds__(kRocheBlock, kScanMinBlocks) k_roche_scan(ElemArgs A) {
    const int64_t rb = blockIdx.x / A.roche_split;
    const int chunk = (int)(blockIdx.x % A.roche_split);
    const ElemBlock blk = A.rblocks[rb];
    const SegDesc sg = A.segs[blk.seg];
    const int64_t i = blk.offset + threadIdx.x;
    EclCount cnt;
    cnt.cap = A.fblink_cap;
    bool capped = false;
    if (i < sg.count && LCB_IN_BOUNDS(sg.first + i < A.sz.nelem, A.status + sg.model)) {
        const ModelDev& M = A.models[sg.model];
        const double4 p = A.el_p64[sg.first + i];
        scan_chunk(blk.by == 1 ? M.ecl1 : M.ecl2, M.cosi_e, M.sini_e, M.delta, p.x, p.y, p.z, chunk, A.roche_split,
                   A.firsthit + rb * kRocheBlock + threadIdx.x, capped, cnt);
        if (capped) atomicOr(A.status + sg.model, kStatusIterCap);
    }
    cnt.fbl = 0;  // the second kernel counts the reference's scan searches
    roche_counters(A, cnt);
}

// Split scan, second kernel with two threads per element: adjacent lanes run
// the ingress and the egress bisection of one element at once (each from the
// first hit, eclipse.rs:301-332), halving the longest chain of line-of-sight
// searches; the ingress lane combines the pair.  Block b covers half of Roche
// block b / 2.
__global__ void __launch_bounds__(kRocheBlock, kChopMinBlocks) k_roche_chop2(ElemArgs A) {
    const int64_t rb = blockIdx.x >> 1;
    const int slot = (int)(blockIdx.x & 1) * (kRocheBlock / 2) + (int)(threadIdx.x >> 1);
    const int part = threadIdx.x & 1;  // 0: ingress, 1: egress
    const ElemBlock blk = A.rblocks[rb];
    const SegDesc sg = A.segs[blk.seg];
    const int64_t i = blk.offset + slot;
    EclCount cnt;
    cnt.cap = A.fblink_cap;
    bool capped = false, found = false;
    double a = 0.0, b = 0.0;
    int64_t e = 0;
    const bool valid = i < sg.count && LCB_IN_BOUNDS(sg.first + i < A.sz.nelem, A.status + sg.model);
    if (valid) {
        const ModelDev& M = A.models[sg.model];
        const RocheEcl& R = blk.by == 1 ? M.ecl1 : M.ecl2;
        e = sg.first + i;
        const double4 p = A.el_p64[e];
        const int first = A.firsthit[rb * kRocheBlock + slot];
        Scan sc;
        if (part == 0 && scan_setup(R, M.cosi_e, M.sini_e, M.delta, p.x, p.y, p.z, sc))
            cnt.fbl += first == kNoHit ? sc.nsteps + 1 : first + 1;  // the single scan's searches
        found = ingress_egress<false>(R, M.cosi_e, M.sini_e, M.delta, p.x, p.y, p.z, a, b, capped, cnt, first, part + 1);
    }
    const double egress = __shfl_xor_sync(0xffffffffu, b, 1);
    const bool found_eg = __shfl_xor_sync(0xffffffffu, (int)found, 1) != 0;
    const bool capped_eg = __shfl_xor_sync(0xffffffffu, (int)capped, 1) != 0;
    int64_t g = -1;
    unsigned bits = 0u;
    if (valid && part == 0) {
        if (found && found_eg) {
            const int slot = roche_slot(sg.kind, blk.by);
            A.el_ecl[slot * A.sz.nelem + e] = make_double2(a, egress < a ? egress + 1.0 : egress);
            g = e / kEclGroup;
            bits = 1u << slot;
        }
        if (capped || capped_eg) atomicOr(A.status + sg.model, kStatusIterCap);
    }
    group_or_warp(A.ecl_grp, g, bits);
    roche_counters(A, cnt);
}

// ---------------------------------------------------------------------------
// k_aux: per-model FP64 sums over the star grids -- comp_star1/2 at the ginterp
// and wdwarf phases (flux.rs:115-206), log g (flux.rs:288-322), radii (347-373)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kElemThreads) k_aux(ElemArgs A) {
    const ElemBlock blk = A.ablocks[blockIdx.x];
    const SegDesc sg = A.segs[blk.seg];
    const ModelDev& M = A.models[sg.model];
    const int64_t i = blk.offset + threadIdx.x;
    const bool valid = i < sg.count && LCB_IN_BOUNDS(sg.first + i < A.sz.nelem, A.status + sg.model);
    const int star = sg.kind == SEG_STAR1 ? 1 : 2;
    double px = 0, py = 0, pz = 0, dx = 0, dy = 0, dz = 0, area = 0, grav = 0, flux = 0;
    double2 ecl[kMaxEcl];
    if (valid) {
        const int64_t e = sg.first + i;
        double4 p = A.el_p64[e], d = A.el_d64[e];
        px = p.x; py = p.y; pz = p.z; area = p.w;
        dx = d.x; dy = d.y; dz = d.z; grav = d.w;
        flux = (double)A.el_rec[e].w;
        for (int k = 0; k < kMaxEcl; ++k) ecl[k] = A.el_ecl[k * A.sz.nelem + e];
    }
    double vals[16];
    int slot[16];
    int nv = 0;
    for (int s = 0; s < M.nspec; ++s) {
        const SpecPhase& sp = M.spec[s];
        if (sp.star != star) continue;
        bool match = sg.role == ROLE_BOTH || (sg.role == ROLE_FINE) == (sp.fine != 0);
        if (!match) continue;
        double c = 0.0;
        if (valid) {
            // the ginterp sums run before the opaque-disc pairs exist (orchestration.rs:93-157)
            const int ne = sp.star_ecl_only ? 1 : kMaxEcl;
            bool vis = true;
            for (int k = 0; k < ne; ++k)
                if ((sp.phi >= ecl[k].x && sp.phi <= ecl[k].y) || sp.phi <= ecl[k].y - 1.0) vis = false;
            double mu = sp.ex * dx + sp.ey * dy + sp.ez * dz;
            const double* ld = star == 1 ? M.ld1 : M.ld2;
            int lt = star == 1 ? M.ltype1 : M.ltype2;
            double beam = star == 1 ? M.beam1 : M.beam2;
            if (vis && mu > (star == 1 ? M.mucrit1 : M.mucrit2)) {
                double mag = (star == 2 && M.glens1) ? lens_mag_d(px, py, pz, sp.ex, sp.ey, sp.ez, M.rlens1) : 1.0;
                if (beam != 0.0) {
                    double vxx = -M.vfac * py, vyy = M.vfac * (px - M.xcofm);
                    double vr = -(sp.ex * vxx + sp.ey * vyy), vn = dx * vxx + dy * vyy;
                    double mud = mu - mu * vr - vn;
                    c = mu * mag * flux * (1.0 - beam * vr) * imu_d(ld, lt, mud);
                } else {
                    c = mu * mag * flux * imu_d(ld, lt, mu);
                }
            }
        }
        vals[nv] = c;
        slot[nv] = AUX_SPEC0 + s;
        ++nv;
    }
    if (sg.fine_star) {
        double sa = 0.0, vol = 0.0;
        if (valid) {
            double wx = px - (star == 1 ? 0.0 : 1.0), wy = py, wz = pz;
            double r = sqrt(wx * wx + wy * wy + wz * wz);
            double rc = dx * wx + dy * wy + dz * wz;
            sa = area * rc / ((r * r) * r);
            vol = area * rc;
        }
        vals[nv] = flux * grav; slot[nv++] = star == 1 ? AUX_FG1 : AUX_FG2;
        vals[nv] = flux; slot[nv++] = star == 1 ? AUX_F1 : AUX_F2;
        vals[nv] = sa; slot[nv++] = star == 1 ? AUX_SA1 : AUX_SA2;
        vals[nv] = vol; slot[nv++] = star == 1 ? AUX_VOL1 : AUX_VOL2;
    }
    if (nv == 0) return;
    __shared__ double red[16][kElemThreads / 32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < nv; ++k) {
        double v = vals[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double t = 0.0;
        for (int w = 0; w < kElemThreads / 32; ++w) t += red[threadIdx.x][w];
        atomicAdd(A.aux + (int64_t)sg.model * kNumAux + slot[threadIdx.x], t);
    }
}

// ---------------------------------------------------------------------------
// k_phase
// ---------------------------------------------------------------------------
__global__ void k_phase(PhaseArgs A) {
    for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < A.ndatum;
         d += (int64_t)gridDim.x * blockDim.x) {
        const ModelDev& M = A.models[A.dmodel[d]];
        if (M.status < 0) continue;
        const lcb_datum D = A.data[d];
        double phase = (D.time - M.t0) / M.period;
        for (int k = 0; k < 4; ++k)
            phase -= (M.t0 + phase * (M.period + M.pdot * phase) - D.time) / (M.period + 2.0 * M.pdot * phase);
        phase += M.deltat / M.period / 2.0 * (cos(2.0 * kPi * phase) - 1.0);
        double expose = D.expose / M.period;
        double frac = (D.time - M.middle) / M.range;
        A.d_slfac[d] = 1.0 + frac * (M.slope + frac * (M.quad + frac * M.cube));
        int64_t j = A.dsub0[d];
        for (int nd = 0; nd < D.ndiv; ++nd, ++j) {
            double phi = phase, w = 1.0;
            if (D.ndiv != 1) {
                phi = phase + expose * ((double)nd - (double)(D.ndiv - 1) / 2.0) / (double)(D.ndiv - 1);
                w = (nd == 0 || nd == D.ndiv - 1) ? 0.5 : 1.0;
            }
            double sn, cs;
            sincos(kTwoPi * phi, &sn, &cs);
            A.sp_e[j] = make_float4((float)(M.sini_l * cs), (float)(-M.sini_l * sn), (float)M.cosi_l, 0.f);
            double pn = phi - floor(phi);
            A.sp_phi[j] = pn;
            int t = (pn <= M.phase1 || pn >= 1.0 - M.phase1) ? 1
                    : (((pn > M.phase1 && pn < M.phase2) || (pn > 1.0 - M.phase2 && pn < 1.0 - M.phase1)) ? 2 : 3);
            A.sp_type[j] = (int8_t)t;
            A.sp_w[j] = w;
        }
    }
}

// ---------------------------------------------------------------------------
// k_flux
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
}
__device__ __forceinline__ void mbar_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}" : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after `limit` SM clock cycles (by default about 2 s);
// on time-out the caller records an error status instead of hanging.
constexpr long long kWaitLimit = 4000000000LL;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit = kWaitLimit) {
    if (mbar_test(bar, parity)) return true;
    long long t0 = clock64();
    while (!mbar_test(bar, parity)) {
        __nanosleep(64);
        if (clock64() - t0 > limit) return false;
    }
    return true;
}

// The bounded wait on an mbarrier that nothing completes (no copy, no arrival):
// it must give up after `limit` cycles and report kStatusTmaTimeout.
__global__ void k_wait_probe(long long limit, int* status, long long* waited) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const long long t0 = clock64();
    const bool ok = mbar_wait(&bar, 0u, limit);
    const long long t1 = clock64();
    if (threadIdx.x == 0) {
        *status = ok ? 0 : kStatusTmaTimeout;
        *waited = t1 - t0;
    }
}

enum { CLS_VIS = 0, CLS_MIX = 1, CLS_HID = 2 };
// used-slot words a flux unit spans (units hold at most 16 chunks of elements)
constexpr int kUnitGroups = 16 * kFluxChunk / kEclGroup + 2;

struct FluxSmem {
    float4 rec[2][kFluxChunk];
    double2 ecl[2][kMaxEcl][kFluxChunk];  // the slots the chunk uses, slot-major
    unsigned cmask[2];                    // which slots were staged
    unsigned gw[kUnitGroups];             // the unit's words of used-slot masks (ecl_grp)
    uint16_t list[kFluxChunk];   // contributing elements: index | pairs << 8 | (partly eclipsed << 15)
    int wtot[2][kFluxThreads / 32];
    uint64_t bar[2];
    int unit;
};
static_assert(kFluxChunk == 2 * kFluxThreads, "the classification pass gives each thread two elements");
static_assert(kFluxChunk <= 256 && kMaxEcl < 8, "list entries hold the element in 8 bits and its pairs in 3");

size_t flux_smem_bytes_impl() { return sizeof(FluxSmem); }

// Range classification of one eclipse pair against [lo, hi] (exact in FP64).
__device__ __forceinline__ int pair_cls(double ing, double eg, double lo, double hi) {
    if ((ing <= lo && hi <= eg) || hi <= eg - 1.0) return CLS_HID;
    if ((hi < ing || lo > eg) && lo > eg - 1.0) return CLS_VIS;
    return CLS_MIX;
}

// Classifies element e of a staged chunk against the tile's phase range from
// the chunk's staged slots `cm` (an unused slot, (inf, -inf), is neutral).
__device__ __forceinline__ int classify(const double2 (*ecl)[kFluxChunk], unsigned cm, int e, const double* rlo,
                                        const double* rhi) {
    int res = -1;
    for (int h = 0; h < 2; ++h) {
        if (!(rlo[h] <= rhi[h])) continue;  // empty half
        int c = CLS_VIS;
        for (unsigned m = cm; m; m &= m - 1u) {
            const double2 p = ecl[__ffs(m) - 1][e];
            const int pc = pair_cls(p.x, p.y, rlo[h], rhi[h]);
            if (pc == CLS_HID) { c = CLS_HID; break; }
            if (pc == CLS_MIX) c = CLS_MIX;
        }
        if (res < 0) res = c;
        else if (res != c) res = CLS_MIX;
    }
    return res < 0 ? CLS_HID : res;
}

// Moves element e's used pairs among the staged slots `cm` to slots 0, 1, ..
// (in place: a pair only moves to a lower slot); returns their number.
__device__ __forceinline__ int compact_pairs(double2 (*ecl)[kFluxChunk], unsigned cm, int e) {
    int n = 0;
    for (unsigned m = cm; m; m &= m - 1u) {
        const double2 p = ecl[__ffs(m) - 1][e];
        if (p.x <= 2.0) ecl[n++][e] = p;
    }
    return n;
}

// The earth vector of phase theta/2pi is (sini cos t, -sini sin t, cosi), so an
// element's mu over a phase arc is A cos t + B sin t + C.  The tile's active
// sub-phases lie on (at most) two arcs shorter than pi, one per half of [0, 1).
struct Arcs {
    float ca[2], sa[2], cb[2], sb[2];
    bool on[2];
};
// Largest mu of direction (dx, dy, dz) over the arcs (FP32; the caller keeps a margin).
__device__ __forceinline__ float max_mu(const Arcs& a, float si, float ci, float dx, float dy, float dz) {
    const float A = si * dx, B = -si * dy, C = ci * dz;
    float m = -2.f;
    for (int h = 0; h < 2; ++h) {
        if (!a.on[h]) continue;
        float in1 = a.ca[h] * B - a.sa[h] * A, in2 = A * a.sb[h] - B * a.cb[h];
        float v = (in1 >= 0.f && in2 >= 0.f) ? sqrtf(A * A + B * B)
                                              : fmaxf(A * a.ca[h] + B * a.sa[h], A * a.cb[h] + B * a.sb[h]);
        m = fmaxf(m, v + C);
    }
    return m;
}
constexpr float kFacingMargin = 2e-5f;  // far above the FP32 rounding of mu

// The thread's sub-phases (bit k: phase ph[k]) at which element e is behind one
// of its npair pairs (moved to slots 0 .. npair-1 by compact_pairs).
__device__ __forceinline__ unsigned hidden_mask(const double2 (*ecl)[kFluxChunk], int npair, int e,
                                                const double* ph) {
    unsigned h = 0u;
#pragma unroll 1
    for (int j = 0; j < npair; ++j) {
        const double2 p = ecl[j][e];
#pragma unroll
        for (int k = 0; k < kFluxR; ++k)
            h |= (((ph[k] >= p.x && ph[k] <= p.y) || ph[k] <= p.y - 1.0) ? 1u : 0u) << k;
    }
    return h;
}

// Per-kind contribution of one element at one sub-phase (FP32).
template <int KIND>
struct Contrib {
    float a0, a1, a2, a3, thr, sumc;  // LD coefficients, mu threshold, sum of Claret coefficients
    __device__ void setup(const ModelDev& M, int star) {
        const float* l = star == 1 ? M.ld1f : M.ld2f;
        a0 = l[0]; a1 = l[1]; a2 = l[2]; a3 = l[3];
        float mc = star == 1 ? M.mucrit1f : M.mucrit2f;
        thr = fmaxf(mc, 0.f);
        sumc = a0 + a1 + a2 + a3;
        if (KIND == UK_DISC) { a0 = M.lin_ldf; a1 = M.quad_ldf; thr = 0.f; }
        if (KIND == UK_SPOT) thr = 0.f;
    }
    __device__ __forceinline__ float operator()(float mu, float fl) const {
        if (KIND == UK_SPOT) return mu * fl;
        if (KIND == UK_DISC) {
            float om = 1.f - mu;
            return mu * fl * (1.f - om * (a0 + a1 * om));
        }
        if (KIND == UK_STAR_CLARET) {
            float m = fminf(mu, 1.f);
            float ms = m * rsqrtf(m);
            float im = (1.f - sumc) + ms * (a0 + ms * (a1 + ms * (a2 + ms * a3)));
            return mu * fl * im;
        }
        float om = 1.f - fminf(mu, 1.f);
        float p;
        if (KIND == UK_STAR_POLY1) p = a0;
        else if (KIND == UK_STAR_POLY2) p = a0 + om * a1;
        else if (KIND == UK_STAR_POLY3) p = a0 + om * (a1 + om * a2);
        else p = a0 + om * (a1 + om * (a2 + om * a3));
        return mu * fl * (1.f - om * p);
    }
    // Two sub-phases at once with the packed FP32x2 pipe (sm_100): the same
    // operations as operator(), each lane rounded as its scalar counterpart.
    __device__ __forceinline__ float2 pair(float2 mu, float fl) const {
        const float2 one = make_float2(1.f, 1.f), f2 = make_float2(fl, fl);
        const float2 mf = __fmul2_rn(mu, f2);
        if (KIND == UK_SPOT) return mf;
        if (KIND == UK_DISC) {
            const float2 om = __fadd2_rn(one, make_float2(-mu.x, -mu.y));
            const float2 q = __ffma2_rn(make_float2(a1, a1), om, make_float2(a0, a0));
            return __fmul2_rn(mf, __ffma2_rn(make_float2(-om.x, -om.y), q, one));
        }
        const float2 m = make_float2(fminf(mu.x, 1.f), fminf(mu.y, 1.f));
        if (KIND == UK_STAR_CLARET) {
            const float2 ms = __fmul2_rn(m, make_float2(rsqrtf(m.x), rsqrtf(m.y)));
            float2 h = __ffma2_rn(ms, make_float2(a3, a3), make_float2(a2, a2));
            h = __ffma2_rn(ms, h, make_float2(a1, a1));
            h = __ffma2_rn(ms, h, make_float2(a0, a0));
            const float2 im = __ffma2_rn(ms, h, make_float2(1.f - sumc, 1.f - sumc));
            return __fmul2_rn(mf, im);
        }
        const float2 om = __fadd2_rn(one, make_float2(-m.x, -m.y));
        float2 p;
        if (KIND == UK_STAR_POLY1) p = make_float2(a0, a0);
        else if (KIND == UK_STAR_POLY2) p = __ffma2_rn(om, make_float2(a1, a1), make_float2(a0, a0));
        else if (KIND == UK_STAR_POLY3) {
            p = __ffma2_rn(om, make_float2(a2, a2), make_float2(a1, a1));
            p = __ffma2_rn(om, p, make_float2(a0, a0));
        } else {
            p = __ffma2_rn(om, make_float2(a3, a3), make_float2(a2, a2));
            p = __ffma2_rn(om, p, make_float2(a1, a1));
            p = __ffma2_rn(om, p, make_float2(a0, a0));
        }
        return __fmul2_rn(mf, __ffma2_rn(make_float2(-om.x, -om.y), p, one));
    }
};

// FP32 LDC::imu for the beaming path (types.rs:101-119)
__device__ __forceinline__ float imu_f(const float* l, int lt, float mu) {
    if (mu <= 0.f) return 0.f;
    mu = fminf(mu, 1.f);
    float om = 1.f - mu;
    if (lt == 0) return 1.f - om * (l[0] + om * (l[1] + om * (l[2] + om * l[3])));
    float ms = mu * rsqrtf(mu);
    return (1.f - (l[0] + l[1] + l[2] + l[3])) + ms * (l[0] + ms * (l[1] + ms * (l[2] + ms * l[3])));
}

template <int KIND>
__device__ void flux_unit(const FluxArgs& A, const FluxUnit& U, FluxSmem& S, uint32_t* parity) {
    const ModelDev& M = A.models[U.model];
    const int tid = threadIdx.x;
    const int64_t sbase = M.sub_begin + U.t0;
    // ---- the tile's sub-phases in registers
    float ex[kFluxR], ey[kFluxR], ez[kFluxR];
    double ph[kFluxR];
    bool act[kFluxR];
    double dlo[2] = {2.0, 2.0}, dhi[2] = {-1.0, -1.0};
#pragma unroll
    for (int k = 0; k < kFluxR; ++k) {
        int j = tid + k * kFluxThreads;
        act[k] = false;
        ex[k] = ey[k] = ez[k] = 0.f;
        ph[k] = -1.0;
        if (j < U.nt) {
            int t = A.sp_type[sbase + j];
            bool a = true;
            if (U.star == 1) a = U.role == ROLE_BOTH || ((U.role == ROLE_FINE) == (t == 1));
            else if (U.star == 2) a = U.role == ROLE_BOTH || ((U.role == ROLE_FINE) == (t == 3));
            if (a) {
                float4 e = A.sp_e[sbase + j];
                ex[k] = e.x; ey[k] = e.y; ez[k] = e.z;
                ph[k] = A.sp_phi[sbase + j];
                act[k] = true;
                int h = ph[k] >= 0.5 ? 1 : 0;
                dlo[h] = fmin(dlo[h], ph[k]);
                dhi[h] = fmax(dhi[h], ph[k]);
            }
        }
    }
    // the unit's used-slot words, read once (issue() combines them per chunk)
    const int64_t g0 = U.e0 / kEclGroup;
    const int ngw = (int)((U.e0 + U.ne - 1) / kEclGroup - g0 + 1);
    for (int t = tid; t < ngw && t < kUnitGroups; t += kFluxThreads) S.gw[t] = A.ecl_grp[g0 + t];
    // block min/max of the two halves
    for (int h = 0; h < 2; ++h) {
        double a = dlo[h], b = dhi[h];
        for (int o = 16; o > 0; o >>= 1) {
            a = fmin(a, __shfl_xor_sync(0xffffffffu, a, o));
            b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
        }
        dlo[h] = a; dhi[h] = b;
    }
    __shared__ double s_lo[kFluxThreads / 32][2], s_hi[kFluxThreads / 32][2];
    if ((tid & 31) == 0) {
        s_lo[tid >> 5][0] = dlo[0]; s_lo[tid >> 5][1] = dlo[1];
        s_hi[tid >> 5][0] = dhi[0]; s_hi[tid >> 5][1] = dhi[1];
    }
    __syncthreads();
    double rlo[2] = {2.0, 2.0}, rhi[2] = {-1.0, -1.0};
    for (int w = 0; w < kFluxThreads / 32; ++w)
        for (int h = 0; h < 2; ++h) { rlo[h] = fmin(rlo[h], s_lo[w][h]); rhi[h] = fmax(rhi[h], s_hi[w][h]); }
    const bool any = rlo[0] <= rhi[0] || rlo[1] <= rhi[1];
    Arcs arcs;
    for (int h = 0; h < 2; ++h) {
        arcs.on[h] = rlo[h] <= rhi[h];
        float lo = arcs.on[h] ? (float)rlo[h] : 0.f, hi = arcs.on[h] ? (float)rhi[h] : 0.f;
        sincospif(2.f * lo, &arcs.sa[h], &arcs.ca[h]);
        sincospif(2.f * hi, &arcs.sb[h], &arcs.cb[h]);
    }
    const float sif = (float)M.sini_l, cif = (float)M.cosi_l;

    static_assert(kFluxR % 2 == 0, "sub-phases are processed in pairs");
    float2 ex2[kFluxR / 2], ey2[kFluxR / 2], ez2[kFluxR / 2];
#pragma unroll
    for (int k = 0; k < kFluxR; k += 2) {
        ex2[k / 2] = make_float2(ex[k], ex[k + 1]);
        ey2[k / 2] = make_float2(ey[k], ey[k + 1]);
        ez2[k / 2] = make_float2(ez[k], ez[k + 1]);
    }
    float acc_hi[kFluxR], acc_lo[kFluxR];
#pragma unroll
    for (int k = 0; k < kFluxR; ++k) acc_hi[k] = acc_lo[k] = 0.f;

    Contrib<KIND> C;
    C.setup(M, U.star);
    const float face_thr = (KIND == UK_STAR_GENERIC ? (U.star == 1 ? M.mucrit1f : M.mucrit2f) : C.thr) - kFacingMargin;
    // generic-path constants
    const float* ldg = U.star == 1 ? M.ld1f : M.ld2f;
    const int ltg = U.star == 1 ? M.ltype1 : M.ltype2;
    const float beam = U.star == 1 ? M.beam1f : M.beam2f;
    const float spin = U.star == 1 ? M.spin1f : M.spin2f;
    const float thrg = U.star == 1 ? M.mucrit1f : M.mucrit2f;  // see(mu) without the mu > 0 shortcut
    const bool lens = U.star == 2 && M.glens1;

    const int nchunks = any ? (U.ne + kFluxChunk - 1) / kFluxChunk : 0;
    auto issue = [&](int c) {
        int b = c & 1;
        int64_t e0 = U.e0 + (int64_t)c * kFluxChunk;
        int n = min(kFluxChunk, U.ne - c * kFluxChunk);
        // only the eclipse slots some element of the chunk uses
        unsigned cm = 0;
        for (int64_t g = e0 / kEclGroup; g <= (e0 + n - 1) / kEclGroup; ++g)
            cm |= g - g0 < kUnitGroups ? S.gw[g - g0] : A.ecl_grp[g];
        S.cmask[b] = cm;  // published to the waiting threads by the arrive below
        uint32_t bytes = (uint32_t)n * 16u * (1u + (uint32_t)__popc(cm));
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect(&S.bar[b], bytes);
        bulk_load(S.rec[b], A.el_rec + e0, (uint32_t)n * 16u, &S.bar[b]);
        for (int k = 0; k < kMaxEcl; ++k)
            if ((cm >> k) & 1u) bulk_load(S.ecl[b][k], A.el_ecl + k * A.sz.nelem + e0, (uint32_t)n * 16u, &S.bar[b]);
    };
    if (tid == 0) {
        if (nchunks > 0) issue(0);
        if (nchunks > 1) issue(1);
    }
    for (int c = 0; c < nchunks; ++c) {
        const int b = c & 1;
        const int n = min(kFluxChunk, U.ne - c * kFluxChunk);
        if (!mbar_wait(&S.bar[b], parity[b])) atomicOr(A.status + U.model, kStatusTmaTimeout);
        parity[b] ^= 1u;
        const unsigned cm = S.cmask[b];
        // classify every element of the chunk and list the contributing ones in
        // ascending order (ballot prefix sums): the loop below then runs over a
        // dense list without per-element branches
        const int lane = tid & 31, warp = tid >> 5;
        uint16_t ent[2];
        unsigned keep[2];
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
            const int e = tid + rr * kFluxThreads;
            int cl = CLS_HID;
            if (e < n) {
                cl = classify(S.ecl[b], cm, e, rlo, rhi);
                if (cl != CLS_HID) {  // never facing the observer on this tile: contributes exactly 0
                    const float4 r = S.rec[b][e];
                    if (max_mu(arcs, sif, cif, r.x, r.y, r.z) <= face_thr) cl = CLS_HID;
                }
            }
            // list entry: element | pairs << 8 | partly eclipsed << 15 (the pairs of a
            // partly eclipsed element are moved to the front for hidden_at)
            ent[rr] = (uint16_t)(cl == CLS_MIX ? (e | compact_pairs(S.ecl[b], cm, e) << 8 | 0x8000) : e);
            keep[rr] = __ballot_sync(0xffffffffu, cl != CLS_HID);
            if (lane == 0) S.wtot[rr][warp] = __popc(keep[rr]);
        }
        __syncthreads();
        int nlist = 0;
        {
            const unsigned below = (1u << lane) - 1u;
            int base = 0;
#pragma unroll
            for (int rr = 0; rr < 2; ++rr) {
                int off = base;
                for (int w = 0; w < kFluxThreads / 32; ++w) {
                    if (w == warp) off = base;
                    base += S.wtot[rr][w];
                }
                if ((keep[rr] >> lane) & 1u) S.list[off + __popc(keep[rr] & below)] = ent[rr];
            }
            nlist = base;
        }
        __syncthreads();
        for (int s0 = 0; s0 < nlist; s0 += 32) {
            float part[kFluxR];
#pragma unroll
            for (int k = 0; k < kFluxR; ++k) part[k] = 0.f;
            const int s1 = min(s0 + 32, nlist);
#pragma unroll kFluxUnroll
            for (int q = s0; q < s1; ++q) {
                const int ev = S.list[q];
                const int e = ev & 0xff;
                const float4 r = S.rec[b][e];
                // sub-phases behind one of a partly eclipsed element's pairs (bit k: sub-phase k)
                const unsigned hid = (ev & 0x8000) ? hidden_mask(S.ecl[b], (ev >> 8) & 7, e, ph) : 0u;
                if (KIND == UK_STAR_GENERIC) {
                    const float4 p = __ldg(A.el_pos + U.e0 + (int64_t)c * kFluxChunk + e);
                    float vx, vy;
                    if (U.star == 1) { vx = -M.vfacf * spin * p.y; vy = M.vfacf * (spin * p.x - M.xcofmf); }
                    else { vx = -M.vfacf * spin * p.y; vy = M.vfacf * (spin * (p.x - 1.f) + 1.f - M.xcofmf); }
                    const float vn = r.x * vx + r.y * vy;
#pragma unroll
                    for (int k = 0; k < kFluxR; ++k) {
                        float mu = ex[k] * r.x + ey[k] * r.y + ez[k] * r.z;
                        bool v = mu > thrg && !((hid >> k) & 1u);
                        if (v) {
                            float mag = 1.f;
                            if (lens) {
                                float d = -(p.x * ex[k] + p.y * ey[k] + p.z * ez[k]);
                                if (d > 0.f) {
                                    float ax = p.x + d * ex[k], ay = p.y + d * ey[k], az = p.z + d * ez[k];
                                    float pp = sqrtf(ax * ax + ay * ay + az * az), phh = pp * 0.5f, phsq = phh * phh;
                                    float rd = M.rlens1f * d;
                                    float pd = phsq > 25.f * rd ? pp + rd / pp : phh + sqrtf(phsq + rd);
                                    mag = pd * pd / (pd - phh) / phh * 0.25f;
                                }
                            }
                            if (beam != 0.f) {
                                float vr = -(ex[k] * vx + ey[k] * vy);
                                float mud = mu - mu * vr - vn;
                                part[k] += mu * mag * r.w * (1.f - beam * vr) * imu_f(ldg, ltg, mud);
                            } else {
                                part[k] += mu * mag * r.w * imu_f(ldg, ltg, mu);
                            }
                        }
                    }
                } else {
                    // sub-phases in pairs on the packed FP32x2 pipe
                    const float2 rx = make_float2(r.x, r.x), ry = make_float2(r.y, r.y), rz = make_float2(r.z, r.z);
#pragma unroll
                    for (int k = 0; k < kFluxR; k += 2) {
                        const float2 mu = __ffma2_rn(ez2[k / 2], rz, __ffma2_rn(ey2[k / 2], ry, __fmul2_rn(ex2[k / 2], rx)));
                        const float2 c = C.pair(mu, r.w);
                        if (mu.x > C.thr && !((hid >> k) & 1u)) part[k] += c.x;
                        if (mu.y > C.thr && !((hid >> (k + 1)) & 1u)) part[k + 1] += c.y;
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < kFluxR; ++k) {  // two-sum fold of the 32-element block
                float s = acc_hi[k] + part[k];
                float bb = s - acc_hi[k];
                float err = (acc_hi[k] - (s - bb)) + (part[k] - bb);
                acc_hi[k] = s;
                acc_lo[k] += err;
            }
        }
        __syncthreads();  // everyone is done with buffer b
        if (tid == 0 && c + 2 < nchunks) issue(c + 2);
    }
    // ---- write the partial sums of this (slot, tile)
    double* out = A.partial + M.pbase + (int64_t)U.slot * M.nsub + U.t0;
#pragma unroll
    for (int k = 0; k < kFluxR; ++k) {
        int j = tid + k * kFluxThreads;
        if (j < U.nt) out[j] = act[k] ? (double)acc_hi[k] + (double)acc_lo[k] : 0.0;
    }
}

__global__ void __launch_bounds__(kFluxThreads, 5) k_flux(FluxArgs A) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    FluxSmem& S = *reinterpret_cast<FluxSmem*>(smem_raw);
    if (threadIdx.x == 0) {
        mbar_init(&S.bar[0]);
        mbar_init(&S.bar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t parity[2] = {0u, 0u};
    for (;;) {
        if (threadIdx.x == 0) S.unit = atomicAdd(A.counter, 1);
        __syncthreads();
        const int64_t u = S.unit;
        __syncthreads();
        if (u >= A.nunits) break;
        const FluxUnit U = A.units[u];
        if (!LCB_IN_BOUNDS(U.e0 + U.ne <= A.sz.nelem &&
                               A.models[U.model].sub_begin + U.t0 + U.nt <= A.sz.nsub &&
                               A.models[U.model].pbase + (int64_t)(U.slot + 1) * A.models[U.model].nsub <=
                                   A.sz.npartial,
                           A.status + U.model))
            continue;  // the unit is skipped by the whole block
        switch (U.kind) {
            case UK_STAR_POLY1: flux_unit<UK_STAR_POLY1>(A, U, S, parity); break;
            case UK_STAR_POLY2: flux_unit<UK_STAR_POLY2>(A, U, S, parity); break;
            case UK_STAR_POLY3: flux_unit<UK_STAR_POLY3>(A, U, S, parity); break;
            case UK_STAR_POLY4: flux_unit<UK_STAR_POLY4>(A, U, S, parity); break;
            case UK_STAR_CLARET: flux_unit<UK_STAR_CLARET>(A, U, S, parity); break;
            case UK_STAR_GENERIC: flux_unit<UK_STAR_GENERIC>(A, U, S, parity); break;
            case UK_DISC: flux_unit<UK_DISC>(A, U, S, parity); break;
            default: flux_unit<UK_SPOT>(A, U, S, parity); break;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// k_epilogue
// ---------------------------------------------------------------------------
struct Gint {  // types.rs:130-202
    double p1, p2, s11, s12, s21, s22;
    __device__ double scale1(double phase) const {
        double pn = phase - floor(phase);
        if (pn <= p1 || pn >= 1.0 - p1) return 1.0;
        return (s11 * (1.0 - p1 - pn) + s12 * (pn - p1)) / (1.0 - 2.0 * p1);
    }
    __device__ double scale2(double phase) const {
        double pn = phase - floor(phase);
        if (pn >= p2 && pn <= 1.0 - p2) return 1.0;
        if (pn < 0.5) return (s22 * (p2 - pn) + s21 * (pn + p2)) / (2.0 * p2);
        return (s21 * (1.0 + p2 - pn) + s22 * (pn - 1.0 + p2)) / (2.0 * p2);
    }
};

constexpr int kEpiThreads = 256;

__device__ double block_sum(double v, double* red) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < kEpiThreads / 32; ++w) s += red[w];
    return s;
}

// Several block sums at once (one pair of barriers).
template <int N>
__device__ void block_sums(double (&v)[N], double (*red)[kEpiThreads / 32]) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < N; ++k) red[k][warp] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; ++k) {
        double s = 0.0;
        for (int w = 0; w < kEpiThreads / 32; ++w) s += red[k][w];
        v[k] = s;
    }
}

// iscale = 1 (orchestration.rs:185-227, 264-283, 405-436): the star-1, disc,
// rim, bright-spot and star-2 fluxes of each datum, and with scale the
// weighted least-squares scale factor of each, by one-sided Jacobi SVD of
// the design matrix (singular values at or below 1e-12 dropped), as the
// oracle restates nalgebra's solve.  No `third` term in this path.
// comp_star1/2 take the ginterp factor at the exposure's centre phase.
__device__ void epilogue_iscale(const EpiArgs& A, const ModelDev& M, const Gint& g, double s_wd, const double* aux,
                                double* res) {
    __shared__ double red[3][kEpiThreads / 32];
    const int ncol = M.t2 > 0.0 ? 5 : 4;
    const double* P = A.partial + M.pbase;
    double* F = A.fcomp + M.datum_begin * 5;
    double* X = A.svda + M.datum_begin * 5;
    for (int64_t d = threadIdx.x; d < M.ndatum; d += blockDim.x) {
        const int64_t gd = M.datum_begin + d;
        const lcb_datum D = A.data[gd];
        int64_t j = A.dsub0[gd] - M.sub_begin;
        const double centre = (D.ndiv > 0 ? A.sp_phi[M.sub_begin + j] : 0.0) +
                              (D.ndiv > 1 ? 0.5 * D.expose / M.period : 0.0);
        double f[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int nd = 0; nd < D.ndiv; ++nd, ++j) {
            const double w = A.sp_w[M.sub_begin + j];
            double c[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
            for (int s = 0; s < M.g1_end; ++s) c[0] += P[(int64_t)s * M.nsub + j];
            for (int s = M.g2_end; s < M.gd_end; ++s) c[1] += P[(int64_t)s * M.nsub + j];
            for (int s = M.gd_end; s < M.ge_end; ++s) c[2] += P[(int64_t)s * M.nsub + j];
            for (int s = M.ge_end; s < M.nslots; ++s) c[3] += P[(int64_t)s * M.nsub + j];
            for (int s = M.g1_end; s < M.g2_end; ++s) c[4] += P[(int64_t)s * M.nsub + j];
            f[0] += w * g.scale1(centre) * c[0];
            f[1] += w * c[1];
            f[2] += w * c[2];
            f[3] += w * c[3];
            f[4] += w * g.scale2(centre) * c[4];
        }
        const double den = (double)max(1, D.ndiv - 1), slf = A.d_slfac[gd];
        for (int k = 0; k < 5; ++k) F[d * 5 + k] = k < ncol ? slf * (f[k] / den) : 0.0;
    }
    double sf[5] = {1.0, 1.0, 1.0, 1.0, 1.0}, wdf = 1.0;
    if (A.scale) {
        // rows with weight > 0, scaled by sqrt(weight)/ferr; other rows are zero and add nothing
        double nok[1] = {0.0};
        for (int64_t d = threadIdx.x; d < M.ndatum; d += blockDim.x) {
            const lcb_datum D = A.data[M.datum_begin + d];
            const double w = D.weight > 0.0 ? sqrt(D.weight) / D.ferr : 0.0;
            if (D.weight > 0.0) nok[0] += 1.0;
            for (int k = 0; k < 5; ++k) X[d * 5 + k] = F[d * 5 + k] * w;
        }
        block_sums(nok, red);
        double x[5] = {1.0, 1.0, 1.0, 1.0, 1.0};
        if (nok[0] >= ncol && nok[0] > 0.0) {
            double V[5][5];
            for (int a = 0; a < 5; ++a)
                for (int b = 0; b < 5; ++b) V[a][b] = a == b ? 1.0 : 0.0;
            for (int sweep = 0; sweep < 60; ++sweep) {
                double off = 0.0;
                for (int p = 0; p < ncol; ++p)
                    for (int q = p + 1; q < ncol; ++q) {
                        double abg[3] = {0.0, 0.0, 0.0};
                        for (int64_t d = threadIdx.x; d < M.ndatum; d += blockDim.x) {
                            const double ap = X[d * 5 + p], aq = X[d * 5 + q];
                            abg[0] += ap * ap; abg[1] += aq * aq; abg[2] += ap * aq;
                        }
                        block_sums(abg, red);
                        const double alpha = abg[0], beta = abg[1], gamma = abg[2];
                        if (gamma == 0.0) continue;
                        off = fmax(off, fabs(gamma) / sqrt(alpha * beta));
                        const double zeta = (beta - alpha) / (2.0 * gamma);
                        const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                        const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
                        for (int64_t d = threadIdx.x; d < M.ndatum; d += blockDim.x) {
                            const double ap = X[d * 5 + p], aq = X[d * 5 + q];
                            X[d * 5 + p] = c * ap - s * aq;
                            X[d * 5 + q] = s * ap + c * aq;
                        }
                        for (int i = 0; i < ncol; ++i) {  // every thread keeps the same V
                            const double vp = V[i][p], vq = V[i][q];
                            V[i][p] = c * vp - s * vq;
                            V[i][q] = s * vp + c * vq;
                        }
                    }
                if (off < 1e-15) break;
            }
            double sol[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
            for (int jc = 0; jc < ncol; ++jc) {
                double su[2] = {0.0, 0.0};
                for (int64_t d = threadIdx.x; d < M.ndatum; d += blockDim.x) {
                    const lcb_datum D = A.data[M.datum_begin + d];
                    const double b = D.weight > 0.0 ? D.flux * sqrt(D.weight) / D.ferr : 0.0;
                    su[0] += X[d * 5 + jc] * X[d * 5 + jc];
                    su[1] += X[d * 5 + jc] * b;
                }
                block_sums(su, red);
                const double sj = sqrt(su[0]);
                if (!(sj > 1e-12)) continue;
                const double ub = su[1] / sj;
                for (int k = 0; k < ncol; ++k) sol[k] += V[k][jc] * ub / sj;
            }
            bool finite = true;
            for (int k = 0; k < ncol; ++k) finite = finite && isfinite(sol[k]);
            if (finite)
                for (int k = 0; k < ncol; ++k) x[k] = sol[k];
        }
        for (int k = 0; k < 5; ++k) sf[k] = k < ncol ? x[k] : 0.0;
        wdf = x[0];
    }
    double cw[2] = {0.0, 0.0};  // chi-squared, wnok
    for (int64_t d = threadIdx.x; d < M.ndatum; d += blockDim.x) {
        const int64_t gd = M.datum_begin + d;
        const lcb_datum D = A.data[gd];
        double c = sf[0] * F[d * 5 + 0] + sf[1] * F[d * 5 + 1] + sf[2] * F[d * 5 + 2] + sf[3] * F[d * 5 + 3];
        if (ncol == 5) c += sf[4] * F[d * 5 + 4];
        A.calc[gd] = c;
        if ((A.scale || A.rdata) && D.weight > 0.0) {
            cw[1] += D.weight;
            cw[0] += D.weight * sq((D.flux - c) / D.ferr);
        }
    }
    block_sums(cw, red);
    if (threadIdx.x == 0) {
        res[0] = s_wd * wdf;
        res[1] = cw[0];
        res[2] = cw[1];
        double fg1 = aux[AUX_FG1], f1 = aux[AUX_F1], fg2 = aux[AUX_FG2], f2 = aux[AUX_F2];
        res[3] = (M.glogg1 > 0.0 && fg1 > 0.0 && f1 > 0.0) ? log10(M.glogg1 * fg1 / f1) : 0.0;
        res[4] = (M.glogg2 > 0.0 && fg2 > 0.0 && f2 > 0.0) ? log10(M.glogg2 * fg2 / f2) : 0.0;
        res[5] = pow(aux[AUX_VOL1] / aux[AUX_SA1], 1.0 / 3.0);
        res[6] = pow(aux[AUX_VOL2] / aux[AUX_SA2], 1.0 / 3.0);
        for (int k = 0; k < 5; ++k) res[7 + k] = sf[k];
    }
}

__global__ void __launch_bounds__(kEpiThreads) k_epilogue(EpiArgs A) {
    const int64_t m = blockIdx.x;
    const ModelDev& M = A.models[m];
    double* res = A.results + m * 12;
    __shared__ double red[kEpiThreads / 32];
    __shared__ Gint G;
    __shared__ double s_wd;
    const bool in_range = LCB_IN_BOUNDS(M.pbase + (int64_t)M.nslots * M.nsub <= A.sz.npartial &&
                                            M.datum_begin + M.ndatum <= A.sz.ndatum && M.sub_begin + M.nsub <= A.sz.nsub,
                                        A.bad + m);
    if (M.status < 0 || A.status[m] != 0 || !in_range) {
        if (threadIdx.x == 0) {
            for (int k = 0; k < 12; ++k) res[k] = NAN;
        }
        for (int64_t d = threadIdx.x; d < M.ndatum; d += blockDim.x) A.calc[M.datum_begin + d] = NAN;
        return;
    }
    const double* aux = A.aux + m * kNumAux;
    if (threadIdx.x == 0) {  // orchestration.rs:86-131 with the live Ginterp
        Gint g{M.phase1, M.phase2, 1.0, 1.0, 1.0, 1.0};
        auto c1 = [&](int s) { return g.scale1(M.spec[s].phase) * aux[AUX_SPEC0 + s]; };
        auto c2 = [&](int s) { return g.scale2(M.spec[s].phase) * aux[AUX_SPEC0 + s]; };
        if (!M.copy1) {
            g.s11 = c1(M.spec_g11[0]) / c1(M.spec_g11[1]);
            g.s12 = c1(M.spec_g12[0]) / c1(M.spec_g12[1]);
        }
        if (!M.copy2) {
            g.s21 = c2(M.spec_g21[0]) / c2(M.spec_g21[1]);
            g.s22 = c2(M.spec_g22[0]) / c2(M.spec_g22[1]);
        }
        G = g;
        s_wd = g.scale1(0.5) * aux[AUX_SPEC0 + M.spec_wd];
    }
    __syncthreads();
    const Gint g = G;
    if (M.iscale) {
        epilogue_iscale(A, M, g, s_wd, aux, res);
        return;
    }
    const double* P = A.partial + M.pbase;
    double chi = 0.0, wnok = 0.0, sdy = 0.0, syy = 0.0;
    for (int64_t d = threadIdx.x; d < M.ndatum; d += blockDim.x) {
        const int64_t gd = M.datum_begin + d;
        const lcb_datum D = A.data[gd];
        int64_t j = A.dsub0[gd] - M.sub_begin;
        double sum = 0.0;
        for (int nd = 0; nd < D.ndiv; ++nd, ++j) {
            double pn = A.sp_phi[M.sub_begin + j];
            double s1 = 0.0, s2 = 0.0, s0 = 0.0;
            for (int s = 0; s < M.g1_end; ++s) s1 += P[(int64_t)s * M.nsub + j];
            for (int s = M.g1_end; s < M.g2_end; ++s) s2 += P[(int64_t)s * M.nsub + j];
            for (int s = M.g2_end; s < M.nslots; ++s) s0 += P[(int64_t)s * M.nsub + j];
            double ss = s1 * g.scale1(pn);
            ss += g.scale2(pn) * s2;
            ss += s0;
            sum += A.sp_w[M.sub_begin + j] * ss;
        }
        double c = A.d_slfac[gd] * (sum / (double)max(1, D.ndiv - 1)) + M.third;
        A.calc[gd] = c;
        if (D.weight > 0.0) {
            if (A.scale) {
                double w = D.weight / sq(D.ferr);
                sdy += w * D.flux * c;
                syy += w * c * c;
                wnok += D.weight;
            } else if (A.rdata) {
                wnok += D.weight;
                chi += D.weight * sq((D.flux - c) / D.ferr);
            }
        }
    }
    double sfac = 1.0;
    if (A.scale) {  // re_scale (orchestration.rs:361-388)
        sdy = block_sum(sdy, red);
        syy = block_sum(syy, red);
        wnok = block_sum(wnok, red);
        if (wnok > 0.0 && syy > 0.0) {
            sfac = sdy / syy;
            chi = 0.0;
            for (int64_t d = threadIdx.x; d < M.ndatum; d += blockDim.x) {
                const int64_t gd = M.datum_begin + d;
                const lcb_datum D = A.data[gd];
                double c = A.calc[gd] * sfac;
                A.calc[gd] = c;
                if (D.weight > 0.0) chi += D.weight * sq((D.flux - c) / D.ferr);
            }
            chi = block_sum(chi, red);
        } else {
            chi = 0.0;
            wnok = 0.0;
        }
    } else {
        chi = block_sum(chi, red);
        wnok = block_sum(wnok, red);
    }
    if (threadIdx.x == 0) {
        res[0] = s_wd * sfac;
        res[1] = chi;
        res[2] = wnok;
        double fg1 = aux[AUX_FG1], f1 = aux[AUX_F1], fg2 = aux[AUX_FG2], f2 = aux[AUX_F2];
        res[3] = (M.glogg1 > 0.0 && fg1 > 0.0 && f1 > 0.0) ? log10(M.glogg1 * fg1 / f1) : 0.0;
        res[4] = (M.glogg2 > 0.0 && fg2 > 0.0 && f2 > 0.0) ? log10(M.glogg2 * fg2 / f2) : 0.0;
        res[5] = pow(aux[AUX_VOL1] / aux[AUX_SA1], 1.0 / 3.0);
        res[6] = pow(aux[AUX_VOL2] / aux[AUX_SA2], 1.0 / 3.0);
        for (int k = 0; k < 5; ++k) res[7 + k] = sfac;
    }
}

// FMA throughput microbenchmark: 8 independent FMA chains per thread.
template <class T>
__global__ void __launch_bounds__(256) k_fma_peak(T* out, int iters, T seed) {
    T a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + (T)(threadIdx.x + k);
    const T b = (T)0.999999, c = (T)1e-7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = a[k] * b + c;
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == (T)-12345.0) out[0] = s;  // keeps the chains live
}

}  // namespace

cudaError_t measure_fma_peak(int fp64, int num_sms, cudaStream_t s, double* tflops) {
    void* out = nullptr;
    cudaError_t e = cudaMalloc(&out, 16);
    if (e != cudaSuccess) return e;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = num_sms * 8, threads = 256, iters = fp64 ? 4096 : 8192;
    double best = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(a, s);
        if (fp64) k_fma_peak<double><<<blocks, threads, 0, s>>>((double*)out, iters, 1.0);
        else k_fma_peak<float><<<blocks, threads, 0, s>>>((float*)out, iters, 1.0f);
        cudaEventRecord(b, s);
        e = cudaEventSynchronize(b);
        if (e != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
        if (rep > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    *tflops = best;
    return e != cudaSuccess ? e : cudaGetLastError();
}

__global__ void k_ecl_export(const double2* __restrict__ ecl, int64_t nelem, int64_t first, int64_t count,
                             double2* __restrict__ out) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // (element, slot), slot fastest
    if (j >= count * kMaxEcl) return;
    const int64_t i = j / kMaxEcl;
    const int k = (int)(j - i * kMaxEcl);
    out[j] = ecl[k * nelem + first + i];
}

__global__ void k_ecl_import(const double2* __restrict__ in, int64_t nelem, double2* __restrict__ ecl,
                             unsigned* __restrict__ grp) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nelem * kMaxEcl) return;
    const int64_t e = j / kMaxEcl;
    const int k = (int)(j - e * kMaxEcl);
    const double2 p = in[j];
    ecl[k * nelem + e] = p;
    if (p.x <= 2.0) atomicOr(grp + e / kEclGroup, 1u << k);
}

cudaError_t launch_ecl_export(const double2* ecl, int64_t nelem, int64_t first, int64_t count, double2* out,
                              cudaStream_t s) {
    const int64_t n = count * kMaxEcl;
    if (n > 0) k_ecl_export<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(ecl, nelem, first, count, out);
    return cudaGetLastError();
}

cudaError_t launch_ecl_import(const double2* in, int64_t nelem, double2* ecl, unsigned* ecl_grp, cudaStream_t s) {
    const int64_t n = nelem * kMaxEcl;
    if (n > 0) k_ecl_import<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in, nelem, ecl, ecl_grp);
    return cudaGetLastError();
}

// The bright spot's gas-stream end point for pair i (lcb_stream.h, the planner's
// host code compiled for the device): one thread per pair, each in a block of its
// own, since every integration is one long serial chain of FP64 operations and
// the pairs' step sequences differ (lanes of one warp would diverge).
__global__ void __launch_bounds__(1) k_stream(const double* __restrict__ in, int n, double* __restrict__ out,
                                              int* __restrict__ status) {
    const int i = blockIdx.x;
    if (i >= n) return;
    double o[3] = {0.0, 0.0, 0.0};
    status[i] = stream::stream_to_radius_core(in[3 * i], in[3 * i + 1], in[3 * i + 2], o);
    out[3 * i] = o[0]; out[3 * i + 1] = o[1]; out[3 * i + 2] = o[2];
}

cudaError_t launch_stream(const double* in, int n, double* out, int* status, cudaStream_t s) {
    if (n > 0) k_stream<<<(unsigned)n, 1, 0, s>>>(in, n, out, status);
    return cudaGetLastError();
}

cudaError_t launch_wait_probe(long long limit, int* status, long long* waited, cudaStream_t s) {
    k_wait_probe<<<1, 32, 0, s>>>(limit, status, waited);
    return cudaGetLastError();
}

size_t flux_smem_bytes() { return flux_smem_bytes_impl(); }

// The flux kernel's dynamic shared memory exceeds the 48 KB default; the
// attribute is set once per process (outside any stream capture).
cudaError_t configure_flux() {
    static cudaError_t status = cudaFuncSetAttribute(k_flux, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     (int)flux_smem_bytes());
    return status;
}

int flux_blocks_per_sm() {
    if (configure_flux() != cudaSuccess) return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_flux, kFluxThreads, flux_smem_bytes()) != cudaSuccess) return 0;
    return n;
}

cudaError_t launch_phase(const PhaseArgs& a, cudaStream_t s) {
    if (a.ndatum <= 0) return cudaSuccess;
    int64_t blocks = (a.ndatum + 255) / 256;
    if (blocks > 65535 * 8) blocks = 65535 * 8;
    k_phase<<<(unsigned)blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_elements(const ElemArgs& a, cudaStream_t s) {
    if (a.nblocks > 0) {
        k_elements<<<(unsigned)a.nblocks, kElemThreads, 0, s>>>(a);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_roche(const ElemArgs& a, cudaStream_t s) {
    if (a.nrblocks <= 0) return cudaSuccess;
    if (a.roche_split <= 1) {
        k_roche<<<(unsigned)a.nrblocks, kRocheBlock, 0, s>>>(a);
        return cudaGetLastError();
    }
    // firsthit starts at kNoHit (memset by the caller's launch sequence)
    k_roche_scan<<<(unsigned)(a.nrblocks * a.roche_split), kRocheBlock, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_roche_chop2<<<(unsigned)(2 * a.nrblocks), kRocheBlock, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_aux(const ElemArgs& a, cudaStream_t s) {
    if (a.nablocks <= 0) return cudaSuccess;
    k_aux<<<(unsigned)a.nablocks, kElemThreads, 0, s>>>(a);
    return cudaGetLastError();
}

int roche_block_size() { return kRocheBlock; }

cudaError_t launch_flux(const FluxArgs& a, int grid, cudaStream_t s) {
    if (a.nunits <= 0) return cudaSuccess;
    cudaError_t e = configure_flux();
    if (e != cudaSuccess) return e;
    k_flux<<<grid, kFluxThreads, flux_smem_bytes(), s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_epilogue(const EpiArgs& a, cudaStream_t s) {
    if (a.nmodels <= 0) return cudaSuccess;
    k_epilogue<<<(unsigned)a.nmodels, kEpiThreads, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace lcb
