// lcb_model.cpp — parameter table, .dat parser, data reader, Rust-style number formatting.
//
// Behaviour follows crates/lcurve/src/model.rs:186-442 (parser), 445-532
// (r1/r2, get/set) and types.rs:229-265 (data files).
#include "lcb_model.h"

#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

namespace lcb {

namespace {

const char* const kPhysNames[P_COUNT] = {
    "q", "iangle", "r1", "r2", "cphi3", "cphi4", "spin1", "spin2", "t1", "t2",
    "ldc1_1", "ldc1_2", "ldc1_3", "ldc1_4", "ldc2_1", "ldc2_2", "ldc2_3", "ldc2_4",
    "velocity_scale", "beam_factor1", "beam_factor2", "t0", "period", "pdot", "deltat",
    "gravity_dark1", "gravity_dark2", "absorb", "slope", "quad", "cube", "third",
    "rdisc1", "rdisc2", "height_disc", "beta_disc", "temp_disc", "texp_disc",
    "lin_limb_disc", "quad_limb_disc", "temp_edge", "absorb_edge",
    "radius_spot", "length_spot", "height_spot", "expon_spot", "epow_spot", "angle_spot",
    "yaw_spot", "temp_spot", "tilt_spot", "cfrac_spot",
    "stsp11_long", "stsp11_lat", "stsp11_fwhm", "stsp11_tcen",
    "stsp12_long", "stsp12_lat", "stsp12_fwhm", "stsp12_tcen",
    "stsp13_long", "stsp13_lat", "stsp13_fwhm", "stsp13_tcen",
    "stsp21_long", "stsp21_lat", "stsp21_fwhm", "stsp21_tcen",
    "stsp22_long", "stsp22_lat", "stsp22_fwhm", "stsp22_tcen",
    "uesp_long1", "uesp_long2", "uesp_lathw", "uesp_taper", "uesp_temp",
};

// Computational parameters: one descriptor drives parsing, set and get.
enum CompType { CT_DOUBLE, CT_INT, CT_BOOL, CT_LIMB };
struct CompDesc {
    const char* name;
    CompType type;
    size_t offset;
};
#define CD(field, t) {#field, t, offsetof(Model, field)}
const CompDesc kComp[] = {
    CD(delta_phase, CT_DOUBLE), CD(nlat1f, CT_INT), CD(nlat2f, CT_INT), CD(nlat1c, CT_INT),
    CD(nlat2c, CT_INT), CD(npole, CT_BOOL), CD(nlatfill, CT_INT), CD(nlngfill, CT_INT),
    CD(lfudge, CT_DOUBLE), CD(llo, CT_DOUBLE), CD(lhi, CT_DOUBLE), CD(phase1, CT_DOUBLE),
    CD(phase2, CT_DOUBLE), CD(wavelength, CT_DOUBLE), CD(roche1, CT_BOOL), CD(roche2, CT_BOOL),
    CD(eclipse1, CT_BOOL), CD(eclipse2, CT_BOOL), CD(glens1, CT_BOOL), CD(use_radii, CT_BOOL),
    CD(tperiod, CT_DOUBLE), CD(gdark_bolom1, CT_BOOL), CD(gdark_bolom2, CT_BOOL),
    CD(mucrit1, CT_DOUBLE), CD(mucrit2, CT_DOUBLE), CD(limb1, CT_LIMB), CD(limb2, CT_LIMB),
    CD(mirror, CT_BOOL), CD(add_disc, CT_BOOL), CD(nrad, CT_INT), CD(opaque, CT_BOOL),
    CD(add_spot, CT_BOOL), CD(nspot, CT_INT), CD(iscale, CT_BOOL),
};
#undef CD
constexpr int kNumComp = sizeof(kComp) / sizeof(kComp[0]);

const CompDesc* find_comp(const std::string& n) {
    for (const auto& c : kComp)
        if (n == c.name) return &c;
    return nullptr;
}

std::string strip(const std::string& s) {
    const char* ws = " \t\r\n\v\f";
    size_t a = s.find_first_not_of(ws);
    if (a == std::string::npos) return std::string();
    size_t b = s.find_last_not_of(ws);
    return s.substr(a, b - a + 1);
}

std::vector<std::string> fields(const std::string& s) {
    std::vector<std::string> out;
    std::istringstream is(s);
    for (std::string t; is >> t;) out.push_back(t);
    return out;
}

Error parse_err(const std::string& m) { return Error(LCB_ERR_PARSE, m); }

// f64::from_str: decimal or exponent notation, "inf"/"infinity"/"nan"; no hex floats.
bool to_f64(const std::string& s, double& out) {
    if (s.empty()) return false;
    size_t sgn = (s[0] == '+' || s[0] == '-') ? 1 : 0;
    std::string body = s.substr(sgn), low;
    for (char c : body) low += (char)std::tolower((unsigned char)c);
    if (low == "inf" || low == "infinity") { out = s[0] == '-' ? -INFINITY : INFINITY; return true; }
    if (low == "nan") { out = NAN; return true; }
    if (body.empty()) return false;
    for (char c : body)
        if (!std::isdigit((unsigned char)c) && c != '.' && c != 'e' && c != 'E' && c != '+' && c != '-') return false;
    char* end = nullptr;
    out = std::strtod(s.c_str(), &end);
    return end != s.c_str() && *end == '\0';
}

bool to_i32(const std::string& s, int32_t& out) {
    if (s.empty()) return false;
    size_t k = (s[0] == '+' || s[0] == '-') ? 1 : 0;
    if (k == s.size()) return false;
    for (size_t i = k; i < s.size(); ++i)
        if (!std::isdigit((unsigned char)s[i])) return false;
    errno = 0;
    long long v = std::strtoll(s.c_str(), nullptr, 10);
    if (errno != 0 || v > INT32_MAX || v < INT32_MIN) return false;
    out = (int32_t)v;
    return true;
}

bool to_bool(const std::string& s, bool& out) {
    if (s == "1" || s == "true" || s == "yes") { out = true; return true; }
    if (s == "0" || s == "false" || s == "no") { out = false; return true; }
    return false;
}

Pparam to_pparam(const std::string& s) {  // model.rs:23-38
    auto f = fields(s);
    if (f.size() < 4) throw parse_err("Pparam: too few fields in '" + s + "'");
    Pparam p;
    if (!to_f64(f[0], p.value)) throw parse_err("bad value: " + f[0]);
    if (!to_f64(f[1], p.range)) throw parse_err("bad range: " + f[1]);
    if (!to_f64(f[2], p.dstep)) throw parse_err("bad dstep: " + f[2]);
    if (!to_bool(f[3], p.vary)) throw parse_err("bad bool: '" + f[3] + "'");
    p.defined = true;
    if (f.size() > 4 && !to_bool(f[4], p.defined)) throw parse_err("bad bool: '" + f[4] + "'");
    return p;
}

void assign_comp(Model& m, const CompDesc& c, const std::string& raw) {
    std::string v = strip(raw);
    char* base = reinterpret_cast<char*>(&m) + c.offset;
    switch (c.type) {
        case CT_DOUBLE: {
            double d;
            if (!to_f64(v, d)) throw parse_err("bad double: '" + v + "'");
            *reinterpret_cast<double*>(base) = d;
            break;
        }
        case CT_INT: {
            int32_t i;
            if (!to_i32(v, i)) throw parse_err("bad int: '" + v + "'");
            *reinterpret_cast<int32_t*>(base) = i;
            break;
        }
        case CT_BOOL: {
            bool b;
            if (!to_bool(v, b)) throw parse_err("bad bool: '" + v + "'");
            *reinterpret_cast<bool*>(base) = b;
            break;
        }
        case CT_LIMB: {
            int32_t t;
            if (v == "Poly") t = LIMB_POLY;
            else if (v == "Claret") t = LIMB_CLARET;
            else throw parse_err(std::string("bad ") + c.name + ": '" + v + "'");
            *reinterpret_cast<int32_t*>(base) = t;
            break;
        }
    }
}

}  // namespace

const char* phys_name(int i) { return (i >= 0 && i < P_COUNT) ? kPhysNames[i] : nullptr; }

int phys_index(const char* name) {
    if (!name) return -1;
    for (int i = 0; i < P_COUNT; ++i)
        if (std::strcmp(kPhysNames[i], name) == 0) return i;
    return -1;
}

Model parse_model_text(const std::string& text) {
    std::map<std::string, std::string> values;  // last assignment wins
    std::istringstream is(text);
    std::string line;
    int lineno = 0;
    while (std::getline(is, line)) {
        ++lineno;
        std::string t = strip(line);
        if (t.empty() || t[0] == '#') continue;
        size_t eq = t.find('=');
        if (eq == std::string::npos) continue;
        std::string key = strip(t.substr(0, eq));
        std::string val = t.substr(eq + 1);
        // '#' starts a comment unless escaped with a backslash (model.rs:299-309)
        for (size_t from = 0;;) {
            size_t h = val.find('#', from);
            if (h == std::string::npos) break;
            if (h > 0 && val[h - 1] == '\\') { from = h + 1; continue; }
            val.erase(h);
            break;
        }
        if (phys_index(key.c_str()) < 0 && !find_comp(key))
            throw parse_err("Parameter '" + key + "' on line " + std::to_string(lineno) + " was not recognised");
        values[key] = strip(val);
    }
    auto has = [&](const std::string& k) { return values.count(k) != 0; };

    // Optional with defaults, spot groups all-or-nothing (model.rs:253-306).
    for (const char* k : {"pdot", "third", "temp_edge", "absorb_edge"})
        if (!has(k)) values[k] = "0 1.e-10 1.e-10 0 0";
    for (int i = 0; i < P_COUNT; ++i) {
        std::string k = kPhysNames[i];
        if (!has(k) && k.compare(0, 4, "stsp") != 0 && k.compare(0, 4, "uesp") != 0)
            throw parse_err("Parameter '" + k + "' was not defined");
    }
    for (const auto& c : kComp)
        if (!has(c.name)) throw parse_err(std::string("Parameter '") + c.name + "' was not defined");
    for (const char* g : {"stsp11", "stsp12", "stsp13", "stsp21", "stsp22"}) {
        int n = 0;
        for (const char* s : {"_long", "_lat", "_fwhm", "_tcen"}) n += has(std::string(g) + s) ? 1 : 0;
        if (n != 0 && n != 4) throw parse_err(std::string("One or more of ") + g + " parameters were not initialised");
    }
    {
        int n = 0;
        for (const char* s : {"uesp_long1", "uesp_long2", "uesp_lathw", "uesp_taper", "uesp_temp"}) n += has(s) ? 1 : 0;
        if (n != 0 && n != 5) throw parse_err("One or more uniform equatorial spot parameters were not initialised");
    }

    Model m;
    // limb types and the glens1/roche1 exclusion are checked before the values (model.rs:309-327)
    assign_comp(m, *find_comp("limb1"), values["limb1"]);
    assign_comp(m, *find_comp("limb2"), values["limb2"]);
    assign_comp(m, *find_comp("roche1"), values["roche1"]);
    assign_comp(m, *find_comp("glens1"), values["glens1"]);
    if (m.glens1 && m.roche1) throw parse_err("glens1=1 and roche1=1 are not simultaneously allowed");
    for (int i = 0; i < P_COUNT; ++i) {
        auto it = values.find(kPhysNames[i]);
        m.p[i] = it == values.end() ? Pparam() : to_pparam(it->second);
    }
    for (const auto& c : kComp) assign_comp(m, c, values[c.name]);
    return m;
}

Model load_model_file(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw Error(LCB_ERR_IO, "cannot open model file '" + path + "'");
    std::stringstream ss;
    ss << f.rdbuf();
    return parse_model_text(ss.str());
}

void set_comp_param(Model& m, const std::string& name, const std::string& value) {
    const CompDesc* c = find_comp(name);
    if (!c) throw Error(LCB_ERR_UNKNOWN_PARAM, "unknown computational parameter '" + name + "'");
    Model tmp = m;
    assign_comp(tmp, *c, value);
    if (tmp.glens1 && tmp.roche1) throw parse_err("glens1=1 and roche1=1 are not simultaneously allowed");
    m = tmp;
}

std::string get_comp_param(const Model& m, const std::string& name) {
    const CompDesc* c = find_comp(name);
    if (!c) throw Error(LCB_ERR_UNKNOWN_PARAM, "unknown computational parameter '" + name + "'");
    const char* base = reinterpret_cast<const char*>(&m) + c->offset;
    switch (c->type) {
        case CT_DOUBLE: return fmt_display(*reinterpret_cast<const double*>(base));
        case CT_INT: return std::to_string(*reinterpret_cast<const int32_t*>(base));
        case CT_BOOL: return *reinterpret_cast<const bool*>(base) ? "1" : "0";
        case CT_LIMB: return *reinterpret_cast<const int32_t*>(base) == LIMB_CLARET ? "Claret" : "Poly";
    }
    return std::string();
}

std::vector<lcb_datum> read_data_file(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw Error(LCB_ERR_IO, "cannot open data file '" + path + "'");
    std::vector<lcb_datum> out;
    std::string line;
    while (std::getline(f, line)) {
        std::string t = strip(line);
        if (t.empty() || t[0] == '#') continue;
        auto p = fields(t);
        if (p.size() < 6) continue;
        lcb_datum d{};
        const char* what[5] = {"time", "expose", "flux", "ferr", "weight"};
        double* dst[5] = {&d.time, &d.expose, &d.flux, &d.ferr, &d.weight};
        for (int i = 0; i < 5; ++i)
            if (!to_f64(p[i], *dst[i])) throw parse_err(std::string("bad ") + what[i] + ": " + p[i]);
        if (!to_i32(p[5], d.ndiv)) throw parse_err("bad ndiv: " + p[5]);
        if (d.ferr < 0.0) { d.ferr = -d.ferr; d.weight = 0.0; }
        out.push_back(d);
    }
    return out;
}

void get_r1r2(const Model& m, double& r1, double& r2) {
    if (m.use_radii) { r1 = m.v(P_R1); r2 = m.v(P_R2); return; }
    const double pi = 3.14159265358979323846;
    double sini = std::sin(m.v(P_IANGLE) * (pi / 180.0));
    double c4 = sini * std::cos(2.0 * pi * m.v(P_CPHI4));
    double c3 = sini * std::cos(2.0 * pi * m.v(P_CPHI3));
    double sum = std::sqrt(1.0 - c4 * c4), diff = std::sqrt(1.0 - c3 * c3);
    r1 = (sum - diff) / 2.0;
    r2 = (sum + diff) / 2.0;
}

// ---- Rust-compatible formatting ------------------------------------------

std::string fmt_lower_exp(double v, int prec) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*e", prec, v);
    std::string s(buf);
    size_t e = s.find('e');
    std::string mant = s.substr(0, e);
    int ex = std::atoi(s.c_str() + e + 1);
    return mant + "e" + std::to_string(ex);
}

std::string fmt_display(double v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
    if (v == 0.0) return std::signbit(v) ? "-0" : "0";
    // the shortest digits that round-trip, the closest to v among them (what Rust's Display
    // prints; a "fewest printf digits that round-trip" search differs at powers of two, where
    // the rounding interval is asymmetric)
    char buf[64];
    const auto r = std::to_chars(buf, buf + sizeof buf - 1, v, std::chars_format::scientific);
    *r.ptr = '\0';
    std::string s(buf);
    bool neg = s[0] == '-';
    if (neg) s = s.substr(1);
    size_t e = s.find('e');
    int ex = std::atoi(s.c_str() + e + 1);
    std::string digits;
    for (size_t i = 0; i < e; ++i)
        if (std::isdigit((unsigned char)s[i])) digits += s[i];
    while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
    std::string out;
    int point = ex + 1;  // digits before the decimal point
    if (point <= 0) {
        out = "0." + std::string((size_t)(-point), '0') + digits;
    } else if ((size_t)point >= digits.size()) {
        out = digits + std::string((size_t)point - digits.size(), '0');
    } else {
        out = digits.substr(0, (size_t)point) + "." + digits.substr((size_t)point);
    }
    return neg ? "-" + out : out;
}

std::string pad_left(const std::string& s, size_t width) {
    return s.size() >= width ? s : std::string(width - s.size(), ' ') + s;
}

}  // namespace lcb
