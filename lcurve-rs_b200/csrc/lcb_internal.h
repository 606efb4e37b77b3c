// lcb_internal.h — data layout shared by the host planner and the sm_100a kernels.
//
// HBM layout of one planned batch (all models concatenated):
//   elements   : per element, el_rec float4 {dirn.xyz, flux}, el_pos float4
//                {posn.xyz, 0}, el_ecl double2[4] eclipse (ingress, egress)
//                pairs, unused pairs = (+inf, -inf) so they never hide.
//   sub-phases : per (datum, exposure sub-division), sp_e float4 earth vector,
//                sp_phi double phase in [0,1), sp_type int8 grid type (1..3),
//                sp_w double trapezoid weight.
//   partials   : per model, nslots x nsub doubles; slot = one element range of
//                one grid segment; each flux work unit owns one (slot, tile).
#pragma once

#include <cstdint>

namespace lcb {

constexpr int kMaxEcl = 4;        // eclipse pairs per element (star: 1 + 2 disc; disc: 2 + 2 stars)
// The eclipse pairs are stored slot-major (pair k of element e at k * nelem + e), and a
// word per group of kEclGroup consecutive elements records which slots any of them uses,
// so the flux kernel stages only the slots a chunk of elements has.
constexpr int kEclGroup = 64;
constexpr int kMaxSpec = 9;       // special phases: 4 star1 ginterp + 4 star2 ginterp + wdwarf
constexpr int kNumAux = 32;       // FP64 per-model accumulators

// Element segment kinds.
enum SegKind : int32_t { SEG_STAR1 = 0, SEG_STAR2 = 1, SEG_DISC = 2, SEG_EDGE = 3, SEG_SPOT = 4 };
// Which star grid(s) a star segment stands for (fine, coarse, or both when
// the coarse grid is a copy of the fine one: orchestration.rs:66-79).
enum GridRole : int32_t { ROLE_FINE = 1, ROLE_COARSE = 2, ROLE_BOTH = 3 };

// aux accumulator slots
enum AuxSlot : int32_t {
    AUX_SPEC0 = 0,           // 0..8: raw comp_star sums at the special phases
    AUX_FG1 = 9, AUX_F1 = 10, AUX_FG2 = 11, AUX_F2 = 12,   // logg sums (flux.rs:288-322)
    AUX_SA1 = 13, AUX_VOL1 = 14, AUX_SA2 = 15, AUX_VOL2 = 16,  // rv sums (flux.rs:347-373)
};

struct RocheEcl {          // constants of a Roche-distorted eclipsing star
    double mu, comp, ssq;  // q/(1+q), 1-mu, spin^2
    double rref, pref;     // reference sphere (surface.rs:14-39)
    double cofmx;          // 0 (primary) or 1 (secondary)
    int32_t primary;
    int32_t pad;
};

struct SpotDev {           // Gaussian star spot (brightness.rs:187-201)
    double dx, dy, dz, fwhm, tcen;
    int32_t on, pad;
};

struct SpecPhase {         // one phase at which comp_star1/2 is needed as a raw sum
    double phase, phi;     // phase and its fractional part
    double ex, ey, ez;     // earth vector (iangle.to_radians() form, flux.rs:120-125)
    int32_t star;          // 1 or 2
    int32_t fine;          // grid selected by grid_type(phase)
    int32_t star_ecl_only; // ginterp sums run before the opaque-disc eclipses are added
    int32_t pad;
};

struct ModelDev {
    // ---- geometry / eclipses (FP64)
    double q, xcofm;
    double cosi_e, sini_e;      // iangle.to_radians(): eclipse.rs:281-283, grid.rs:53-55
    double cosi_l, sini_l;      // (TWOPI*iangle/360): flux.rs:10-11 (comp_light)
    double cosi_d, sini_d;      // iangle*PI/180: disc_eclipse.rs:103-105
    double r1, r2;              // grid radii (negative -> Roche lobe)
    double spin1, spin2, ffac1, ffac2;
    double rref1, pref1, rref2, pref2, gref1, gref2;
    double delta, acc_face;     // delta_phase, delta_phase/10
    RocheEcl ecl1, ecl2;        // star 1 / star 2 as the eclipser
    int32_t roche1, roche2, eclipse1, eclipse2, npole, glens1;
    int32_t add_disc, opaque, add_spot, copy1, copy2, iscale;
    // ---- disc
    double rdisc1_g, rdisc1_l, rdisc2, beta, height;  // _g: set_disc_grid (r1 replaced); _l: light_curve_comp
    double edge_h, edge_area, edge_rad;
    int64_t edge_ntheta, edge_nout;
    // ---- continuum (brightness.rs)
    double wavelength, t1, t2, absorb, gdcbol1, gdcbol2, r1c, r2c;
    double planck_t2abs, planck_t1;   // mirror terms
    int32_t mirror, nspot1, nspot2, uesp_on;
    SpotDev spot1[3], spot2[2];
    double uesp_dx, uesp_dy, uesp_longhw, uesp_lathw, uesp_taper, uesp_temp;
    double disc_bright, texp_disc;
    double tedge, r2e, t2abs, absorb_edge;
    // ---- bright spot (grid.rs:484-553)
    double bspot[3], bvec[3], tvec[3];
    double length_spot, bmax, sfac_spot, area_spot, bright_ref, expon_spot, epow_spot, cfrac_spot;
    int64_t nspot;
    // ---- flux (double copies for the FP64 aux sums; float copies for the FP32 kernel)
    double ld1[4], ld2[4], mucrit1, mucrit2, beam1, beam2, vfac, rlens1, lin_ld, quad_ld;
    int32_t ltype1, ltype2, npoly1, npoly2;
    float ld1f[4], ld2f[4], mucrit1f, mucrit2f, beam1f, beam2f, vfacf, rlens1f, lin_ldf, quad_ldf;
    float spin1f, spin2f, xcofmf, padf;
    // ---- ginterp / ephemeris / data
    double phase1, phase2;
    double t0, period, pdot, deltat, slope, quad, cube, third, middle, range;
    int32_t nspec, pad0;
    SpecPhase spec[kMaxSpec];
    int32_t spec_g11[2], spec_g12[2], spec_g21[2], spec_g22[2], spec_wd;  // indices into spec
    int32_t pad1;
    double glogg1, glogg2;      // gref * gscale terms of comp_gravity1/2
    // ---- layout
    int64_t sub_begin, nsub;        // sub-phases
    int64_t datum_begin, ndatum;    // data
    int64_t pbase;                  // partial buffer offset
    int32_t nslots, g1_end, g2_end, status;  // slots: [0,g1_end) star1, [g1_end,g2_end) star2, rest
    int32_t gd_end, ge_end;                  // rest: [g2_end,gd_end) disc, [gd_end,ge_end) rim, [ge_end,nslots) spot
};

struct SegDesc {            // a contiguous run of elements of one model and kind
    int64_t first;          // global element index
    int64_t count;
    int32_t model;
    int32_t kind;           // SegKind
    int32_t role;           // GridRole (stars)
    int32_t table;          // first band (stars) / ring (disc)
    int32_t ntable;
    int32_t fine_star;      // 1 if this is the fine grid of its star (logg/rv sums)
};

struct Band {               // one latitude band of a star grid (grid.rs:227-262)
    int64_t first;          // element offset in the segment
    int64_t nphi;
    double sint, cost;
    double phi1, phi2;
    double aphi, ath;       // (phi2-phi1)/nphi, (thi-tlo)/nl
};

struct Ring {               // one disc annulus (grid.rs:356-364)
    int64_t first;
    int64_t ntheta;
    double rad, h, cosp, sinp, area;
};

struct ElemBlock {          // one block of an element kernel
    int32_t seg;
    int32_t by;             // k_roche: eclipsing star (1 or 2)
    int64_t offset;         // element offset within the segment
};

// Flux work unit kinds (one template instantiation each).
enum UnitKind : int32_t {
    UK_STAR_POLY1 = 0, UK_STAR_POLY2, UK_STAR_POLY3, UK_STAR_POLY4, UK_STAR_CLARET,
    UK_STAR_GENERIC,        // beaming and/or lensing
    UK_DISC, UK_SPOT, UK_COUNT
};

struct FluxUnit {
    int64_t e0;             // first global element
    int32_t ne;             // elements
    int32_t model;
    int32_t t0;             // first sub-phase (model-relative)
    int32_t nt;             // sub-phases in the tile
    int32_t slot;           // model-relative slot
    int32_t kind;           // UnitKind
    int32_t star;           // 1, 2, or 0 for disc/edge/spot
    int32_t role;           // GridRole for star units
    int32_t pad[2];
};

// Kernel geometry of the flux kernel.
constexpr int kFluxThreads = 128;
constexpr int kFluxR = 4;                          // sub-phases per thread
constexpr int kFluxTile = kFluxThreads * kFluxR;   // sub-phases per work unit
constexpr int kFluxChunk = 256;                    // elements staged per TMA chunk
constexpr int kElemThreads = 256;
#ifndef LCB_ROCHE_BLOCK
#define LCB_ROCHE_BLOCK 128
#endif
constexpr int kRocheBlock = LCB_ROCHE_BLOCK;       // elements per k_roche block

// Potential evaluations allowed in one line-of-sight search of the eclipse search
// (the reference has no such bound; a model that reaches it fails: kStatusIterCap).
constexpr int kFblinkEvalCap = 1 << 18;

// Device status bits (ModelDev.status / batch status word).
constexpr int kStatusIterCap = 1;     // an iteration cap without a reference counterpart tripped
constexpr int kStatusTmaTimeout = 2;  // a bounded mbarrier wait gave up
constexpr int kStatusBounds = 4;      // LCURVE_DEBUG_BOUNDS build: an index check failed (access skipped)

}  // namespace lcb
