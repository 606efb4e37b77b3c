// lcb_model.h — host-side model description, .dat parser and data reader.
//
// Same file format, parameter names, defaults and error behaviour as the
// reference (crates/lcurve/src/model.rs:186-442, types.rs:229-265).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/lcurve_b200.h"

namespace lcb {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

struct Pparam {  // model.rs:7-13
    double value = 0.0, range = 0.0, dstep = 0.0;
    bool vary = false, defined = false;
};

// Physical parameters in declaration order (model.rs:66-137).
enum Phys : int {
    P_Q, P_IANGLE, P_R1, P_R2, P_CPHI3, P_CPHI4, P_SPIN1, P_SPIN2, P_T1, P_T2,
    P_LDC1_1, P_LDC1_2, P_LDC1_3, P_LDC1_4, P_LDC2_1, P_LDC2_2, P_LDC2_3, P_LDC2_4,
    P_VELOCITY_SCALE, P_BEAM_FACTOR1, P_BEAM_FACTOR2, P_T0, P_PERIOD, P_PDOT, P_DELTAT,
    P_GRAVITY_DARK1, P_GRAVITY_DARK2, P_ABSORB, P_SLOPE, P_QUAD, P_CUBE, P_THIRD,
    P_RDISC1, P_RDISC2, P_HEIGHT_DISC, P_BETA_DISC, P_TEMP_DISC, P_TEXP_DISC,
    P_LIN_LIMB_DISC, P_QUAD_LIMB_DISC, P_TEMP_EDGE, P_ABSORB_EDGE,
    P_RADIUS_SPOT, P_LENGTH_SPOT, P_HEIGHT_SPOT, P_EXPON_SPOT, P_EPOW_SPOT, P_ANGLE_SPOT,
    P_YAW_SPOT, P_TEMP_SPOT, P_TILT_SPOT, P_CFRAC_SPOT,
    P_STSP11_LONG, P_STSP11_LAT, P_STSP11_FWHM, P_STSP11_TCEN,
    P_STSP12_LONG, P_STSP12_LAT, P_STSP12_FWHM, P_STSP12_TCEN,
    P_STSP13_LONG, P_STSP13_LAT, P_STSP13_FWHM, P_STSP13_TCEN,
    P_STSP21_LONG, P_STSP21_LAT, P_STSP21_FWHM, P_STSP21_TCEN,
    P_STSP22_LONG, P_STSP22_LAT, P_STSP22_FWHM, P_STSP22_TCEN,
    P_UESP_LONG1, P_UESP_LONG2, P_UESP_LATHW, P_UESP_TAPER, P_UESP_TEMP,
    P_COUNT
};

const char* phys_name(int i);
int phys_index(const char* name);  // -1 if unknown

enum LimbType : int { LIMB_POLY = 0, LIMB_CLARET = 1 };  // types.rs:62-68

struct Model {
    Pparam p[P_COUNT];
    // computational parameters (model.rs:140-181)
    double delta_phase = 0, lfudge = 0, llo = 0, lhi = 0, phase1 = 0, phase2 = 0, wavelength = 0;
    double tperiod = 0, mucrit1 = 0, mucrit2 = 0;
    int32_t nlat1f = 0, nlat2f = 0, nlat1c = 0, nlat2c = 0, nlatfill = 0, nlngfill = 0, nrad = 0, nspot = 0;
    int32_t limb1 = LIMB_POLY, limb2 = LIMB_POLY;
    bool npole = false, roche1 = false, roche2 = false, eclipse1 = false, eclipse2 = false, glens1 = false;
    bool use_radii = false, gdark_bolom1 = false, gdark_bolom2 = false, mirror = false, add_disc = false;
    bool opaque = false, add_spot = false, iscale = false;

    double v(int i) const { return p[i].value; }
};

Model parse_model_text(const std::string& text);   // throws Error(LCB_ERR_PARSE)
Model load_model_file(const std::string& path);    // throws Error(LCB_ERR_IO / LCB_ERR_PARSE)
// Computational parameter access by name with .dat text values.
void set_comp_param(Model& m, const std::string& name, const std::string& value);
std::string get_comp_param(const Model& m, const std::string& name);

std::vector<lcb_datum> read_data_file(const std::string& path);  // types.rs:229-254

// model.rs:445-454
void get_r1r2(const Model& m, double& r1, double& r2);

// Rust-compatible number formatting used by the lroche front end.
std::string fmt_lower_exp(double v, int prec);           // {:.Ne}
std::string fmt_display(double v);                       // {} (shortest round trip, no exponent)
std::string pad_left(const std::string& s, size_t width);

}  // namespace lcb
