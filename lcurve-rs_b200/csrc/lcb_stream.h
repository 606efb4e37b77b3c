// lcb_stream.h — the gas stream from L1 to a radius (the bright spot's position),
// compiled for the host (planner, g++) and for the device (k_stream, nvcc) from
// this one source.
//
// Bulirsch-Stoer with the reference's step control (crates/subs/src/numerical/
// bsstep.rs:13-324), the rotating-frame acceleration (crates/roche/src/misc.rs:4-19),
// one gsint step (crates/roche/src/stream.rs:26-62) and strinit + stradv(q, r, v,
// rad, 1e-10, 1e-3) (stream.rs:8-20, 82-145).  Plain C++ with no exceptions, no
// allocation and no library calls beyond sqrt / pow / fabs / fmax, so the host and
// the device run the same operations (pow may round differently in its last bit
// on the two, which moves the end point by rounding only).
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define LCB_HD __host__ __device__
#else
#define LCB_HD
#endif

namespace lcb {
namespace stream {

enum { kStreamOk = 0, kStreamChopFailed = 1, kStreamTooLong = 2 };

LCB_HD inline double sq(double x) { return x * x; }

class BulirschStoer {  // bsstep.rs:13-324
public:
    static constexpr int kK = 8;
    LCB_HD static int nseq(int k) { return 2 * (k + 1); }  // 2, 4, .., 18

    template <class F>  // F(y, dydx): the right-hand side
    LCB_HD void step(double* y, const double* dydx, double& x, double htry, double eps, double& hdid,
                     double& hnext, const F& f) {
        const double safe1 = 0.25, safe2 = 0.7, redmax = 1.0e-5, redmin = 0.7, tiny = 1.0e-30, scalmx = 0.1;
        double err[kK] = {0}, ysav[6], yseq[6], yerr[6];
        double tab[6][kK + 1] = {{0}}, xt[kK + 1] = {0};
        if (eps != epsold_) {
            xnew_ = -1.0e29;
            double eps1 = safe1 * eps;
            a_[0] = nseq(0) + 1.0;
            for (int k = 0; k < kK; ++k) a_[k + 1] = a_[k] + nseq(k + 1);
            for (int iq = 1; iq < kK; ++iq)
                for (int k = 0; k < iq; ++k)
                    alf_[k][iq] = pow(eps1, (a_[k + 1] - a_[iq + 1]) / ((a_[iq + 1] - a_[0] + 1.0) * (2 * k + 3)));
            epsold_ = eps;
            kopt_ = 1;
            for (int k = 1; k < kK - 1; ++k) {
                kopt_ = k;
                if (a_[k + 1] > a_[k] * alf_[k - 1][k]) break;
            }
            kmax_ = kopt_;
        }
        double h = htry;
        for (int i = 0; i < 6; ++i) ysav[i] = y[i];
        if (x != xnew_ || h != xnew_) { first_ = true; kopt_ = kmax_; }
        bool reduct = false;
        int km = 0;
        for (;;) {
            bool done = false;
            for (int k = 0; k <= kmax_; ++k) {
                xnew_ = x + h;
                if (xnew_ == x) { hdid = 0.0; hnext = 0.0; return; }
                midpoint(ysav, dydx, h, nseq(k), yseq, f);
                double xest = sq(h / nseq(k));
                extrapolate(k, xest, yseq, y, yerr, tab, xt);
                double errmax = 0.0;
                if (k != 0) {
                    errmax = tiny;
                    for (int i = 0; i < 6; ++i) errmax = fmax(errmax, fabs(yerr[i]));
                    errmax /= eps;
                    km = k - 1;
                    err[km] = pow(errmax / safe1, 1.0 / (2 * km + 3));
                }
                if (k != 0 && (k >= (kopt_ - 1 > 0 ? kopt_ - 1 : 0) || first_)) {
                    if (err[km] != 0.0 && errmax < 1.0) { done = true; break; }
                    if (k == kmax_ || k == kopt_ + 1) break;
                    if (k == kopt_ && alf_[kopt_ - 1][kopt_] < err[km]) break;
                    if (kopt_ == kmax_ && alf_[km][kmax_ - 1] < err[km]) break;
                    if (alf_[km][kopt_] < err[km]) break;
                }
            }
            if (done) break;
            double red = err[km] > 0.0 ? fmin(fmax(safe2 / err[km], redmax), redmin) : redmin;
            h *= red;
            reduct = true;
        }
        x = xnew_;
        hdid = h;
        first_ = false;
        double wrkmin = 1.0e35, fac = 1.0;
        for (int kk = 0; kk <= km; ++kk) {
            double f2 = fmax(err[kk], scalmx), work = f2 * a_[kk + 1];
            if (work < wrkmin) { fac = f2; wrkmin = work; kopt_ = kk + 1; }
        }
        hnext = h / fac;
        if (kopt_ >= km + 1 && kopt_ != kmax_ && !reduct) {
            double f2 = fmax(fac / alf_[kopt_ - 1][kopt_], scalmx);
            if (a_[kopt_ + 1] * f2 <= wrkmin) { hnext = h / f2; kopt_ += 1; }
        }
    }

private:
    template <class F>
    LCB_HD static void midpoint(const double* y, const double* dydx, double htot, int n, double* yout,
                                const F& f) {  // bsstep.rs:57-93
        double h = htot / n, ym[6], yn[6];
        for (int i = 0; i < 6; ++i) { ym[i] = y[i]; yn[i] = y[i] + h * dydx[i]; }
        f(yn, yout);
        for (int s = 1; s < n; ++s) {
            for (int i = 0; i < 6; ++i) { double t = ym[i] + 2.0 * h * yout[i]; ym[i] = yn[i]; yn[i] = t; }
            f(yn, yout);
        }
        for (int i = 0; i < 6; ++i) yout[i] = 0.5 * (ym[i] + yn[i] + h * yout[i]);
    }
    LCB_HD static void extrapolate(int iest, double xest, const double* yest, double* yz, double* dy,
                                   double tab[6][kK + 1], double* xt) {  // bsstep.rs:96-149
        xt[iest] = xest;
        for (int j = 0; j < 6; ++j) { dy[j] = yest[j]; yz[j] = yest[j]; }
        if (iest == 0) {
            for (int j = 0; j < 6; ++j) tab[j][0] = yest[j];
            return;
        }
        double c[6];
        for (int j = 0; j < 6; ++j) c[j] = yest[j];
        for (int k1 = 0; k1 < iest; ++k1) {
            double d = 1.0 / (xt[iest - k1 - 1] - xest);
            double f1 = xest * d, f2 = xt[iest - k1 - 1] * d;
            for (int j = 0; j < 6; ++j) {
                double qv = tab[j][k1];
                tab[j][k1] = dy[j];
                double dl = c[j] - qv;
                dy[j] = f1 * dl;
                c[j] = f2 * dl;
                yz[j] += dy[j];
            }
        }
        for (int j = 0; j < 6; ++j) tab[j][iest] = dy[j];
    }
    bool first_ = true;
    int kmax_ = 0, kopt_ = 0;
    double epsold_ = -1.0, xnew_ = -1.0e29, a_[kK + 1] = {0}, alf_[kK][kK] = {{0}};
};

// Acceleration in the rotating frame (misc.rs:4-19) as an ODE right-hand side.
struct RocheRhs {
    double q;
    LCB_HD void operator()(const double* y, double* d) const {
        double f1 = 1.0 / (1.0 + q), f2 = f1 * q;
        double yz = sq(y[1]) + sq(y[2]);
        double r1sq = sq(y[0]) + yz, r2sq = sq(y[0] - 1.0) + yz;
        double fm1 = f1 / (r1sq * sqrt(r1sq)), fm2 = f2 / (r2sq * sqrt(r2sq)), fm3 = fm1 + fm2;
        d[0] = y[3]; d[1] = y[4]; d[2] = y[5];
        d[3] = -fm3 * y[0] + fm2 + 2.0 * y[4] + y[0] - f2;
        d[4] = -fm3 * y[1] - 2.0 * y[3] + y[1];
        d[5] = -fm3 * y[2];
    }
};

// One gsint step (stream.rs:26-62).
LCB_HD inline void stream_step(double q, double* y, double& t, double htry, BulirschStoer& bs, double& hdid,
                               double& hnext) {
    const RocheRhs f{q};
    double d[6];
    f(y, d);
    bs.step(y, d, t, htry, 1.0e-8, hdid, hnext, f);
}

LCB_HD inline double radius3(const double* y) { return sqrt(sq(y[0]) + sq(y[1]) + sq(y[2])); }

// strinit + stradv(q, r, v, rad, 1e-10, 1e-3) (stream.rs:8-20, 82-145): the stream's
// position where its distance from the primary first crosses rad; rl1 is the L1
// distance of mass ratio q.  Returns kStreamOk, or kStreamChopFailed / kStreamTooLong
// (the reference's two errors).
LCB_HD inline int stream_to_radius_core(double q, double rl1, double rad, double out[3]) {
    const double small = 1.0e-5;
    double mu = q / (1.0 + q);
    double a = (1.0 - mu) / (rl1 * rl1 * rl1) + mu / ((1.0 - rl1) * (1.0 - rl1) * (1.0 - rl1));
    double lam = sqrt(((a - 2.0) + sqrt(a * (9.0 * a - 8.0))) / 2.0);
    double m1 = (lam * lam - 2.0 * a - 1.0) / (2.0 * lam);
    double y[6] = {rl1 - small, -m1 * small, 0.0, -lam * small, -lam * m1 * small, 0.0};
    BulirschStoer bs;
    double rinit = radius3(y), t = 0.0, tnext = 1.0e-2;
    // the reference stops at t > 10 (at least 10^4 steps of at most 1e-3); the step count
    // bound only ends a stream whose steps stop advancing t
    for (long nstep = 0;; ++nstep) {
        if (nstep > 4000000) return kStreamTooLong;
        double yo[6];
        for (int i = 0; i < 6; ++i) yo[i] = y[i];
        double hdid, hn;
        stream_step(q, y, t, fmin(tnext, 1.0e-3), bs, hdid, hn);
        tnext = hn;
        double rnow = radius3(y);
        if ((rinit > rad && rnow <= rad) || (rinit < rad && rnow >= rad)) {
            double lo = 0.0, hi = hdid, rlo = radius3(yo), rhi = rnow, t0 = t - hdid;
            for (int guard = 0; fabs(rhi - rlo) > 1e-10; ++guard) {
                if (guard > 100000) return kStreamChopFailed;
                double tm = (lo + hi) / 2.0;
                for (int i = 0; i < 6; ++i) y[i] = yo[i];
                double tt = t0, a1, a2;
                BulirschStoer bs2;
                stream_step(q, y, tt, tm, bs2, a1, a2);
                rnow = radius3(y);
                if ((rhi > rad && rnow > rad) || (rhi < rad && rnow < rad)) { rhi = rnow; hi = tm; }
                else { rlo = rnow; lo = tm; }
            }
            out[0] = y[0]; out[1] = y[1]; out[2] = y[2];
            return kStreamOk;
        }
        if (t > 10.0) return kStreamTooLong;
    }
}

}  // namespace stream
}  // namespace lcb
