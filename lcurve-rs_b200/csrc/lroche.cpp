// lroche — command-line light curve, same arguments and output as the
// reference front end (src/main.rs:6-121), computed through liblcurve_b200.so.
//
//   lroche MODEL DATA [--time1 T] [--time2 T] [--ntime N] [--expose E]
//          [--ndivide N] [-o|--output FILE] [--scale] [--device N]
//
// DATA = 'none' generates regularly spaced times (main.rs:57-73).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lcurve_b200.h"
#include "lcb_model.h"

namespace {

void usage() {
    std::fprintf(stderr,
                 "Usage: lroche [OPTIONS] <MODEL> <DATA>\n"
                 "  --time1 <T>    first time when DATA = none [default: -0.2]\n"
                 "  --time2 <T>    last time when DATA = none [default: 0.8]\n"
                 "  --ntime <N>    number of times when DATA = none [default: 500]\n"
                 "  --expose <E>   exposure time when DATA = none [default: 0.001]\n"
                 "  --ndivide <N>  exposure sub-divisions when DATA = none [default: 1]\n"
                 "  -o, --output <FILE>  output file\n"
                 "  --scale        autoscale to minimise chi-squared (only with real data)\n"
                 "  --device <N>   CUDA device [default: 0]\n");
}

int die(const std::string& msg) {
    std::fprintf(stderr, "lroche: %s\n", msg.c_str());
    return 1;
}

std::string line_out(const lcb_datum& d, double calc) {  // main.rs:108-116
    return lcb::pad_left(lcb::fmt_lower_exp(d.time, 15), 20) + " " + lcb::fmt_display(d.expose) + " " +
           lcb::pad_left(lcb::fmt_lower_exp(calc, 10), 17) + " " + lcb::fmt_display(d.ferr) + " " +
           lcb::fmt_display(d.weight) + " " + std::to_string(d.ndiv);
}

}  // namespace

int main(int argc, char** argv) {
    double time1 = -0.2, time2 = 0.8, expose = 0.001;
    long ntime = 500;
    int ndivide = 1, device = 0;
    bool scale = false;
    std::string output;
    std::vector<std::string> pos;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto val = [&](const char* name) -> std::string {
            if (i + 1 >= argc) { usage(); std::exit(2); }
            (void)name;
            return argv[++i];
        };
        if (a == "--time1") time1 = std::atof(val("time1").c_str());
        else if (a == "--time2") time2 = std::atof(val("time2").c_str());
        else if (a == "--ntime") ntime = std::atol(val("ntime").c_str());
        else if (a == "--expose") expose = std::atof(val("expose").c_str());
        else if (a == "--ndivide") ndivide = std::atoi(val("ndivide").c_str());
        else if (a == "-o" || a == "--output") output = val("output");
        else if (a == "--scale") scale = true;
        else if (a == "--device") device = std::atoi(val("device").c_str());
        else if (a == "-h" || a == "--help") { usage(); return 0; }
        else pos.push_back(a);
    }
    if (pos.size() != 2) { usage(); return 2; }

    lcb_model* model = nullptr;
    if (lcb_model_load(pos[0].c_str(), &model) != LCB_OK) return die(lcb_last_error());
    std::string lower = pos[1];
    for (auto& c : lower) c = (char)std::tolower((unsigned char)c);
    const bool no_file = lower == "none";
    std::vector<lcb_datum> data;
    if (no_file) {
        for (long i = 0; i < ntime; ++i) {
            lcb_datum d{};
            d.time = time1 + (time2 - time1) * (double)i / (double)(ntime - 1);
            d.expose = expose; d.flux = 0.0; d.ferr = 0.0; d.weight = 1.0; d.ndiv = ndivide;
            data.push_back(d);
        }
    } else {
        lcb_datum* p = nullptr;
        int64_t n = 0;
        if (lcb_read_data(pos[1].c_str(), &p, &n) != LCB_OK) return die(lcb_last_error());
        data.assign(p, p + n);
        lcb_free_data(p);
    }
    if (data.empty()) return die("No data points");
    const bool do_scale = scale && !no_file, rdata = !no_file;

    lcb_ctx* ctx = nullptr;
    if (lcb_ctx_create(device, &ctx) != LCB_OK) return die(lcb_last_error());
    std::vector<double> calc(data.size());
    lcb_result r{};
    int rc = lcb_light_curve(ctx, model, data.data(), (int64_t)data.size(), do_scale, rdata, calc.data(), &r);
    if (rc != LCB_OK) return die(lcb_last_error());

    std::string iscale;
    char buf[16];
    lcb_model_get_comp(model, "iscale", buf, sizeof buf);
    iscale = buf;
    if (rdata) {  // main.rs:87-96
        std::printf("Weighted chi**2 = %s, wnok = %s\n", lcb::fmt_lower_exp(r.chisq, 12).c_str(),
                    lcb::fmt_lower_exp(r.wnok, 12).c_str());
        if (iscale == "1") {
            std::printf("Scale factors = %s, %s, %s, %s, %s\n", lcb::fmt_lower_exp(r.sfac[0], 12).c_str(),
                        lcb::fmt_lower_exp(r.sfac[1], 12).c_str(), lcb::fmt_lower_exp(r.sfac[2], 12).c_str(),
                        lcb::fmt_lower_exp(r.sfac[3], 12).c_str(), lcb::fmt_lower_exp(r.sfac[4], 12).c_str());
        } else {
            std::printf("Scale factor = %s\n", lcb::fmt_lower_exp(r.sfac[0], 12).c_str());
        }
    }
    std::printf("White dwarf's contribution = %s\n", lcb::fmt_lower_exp(r.wdwarf, 12).c_str());
    std::printf("log10(g1 [cgs]) = %s\n", lcb::fmt_lower_exp(r.logg1, 12).c_str());
    std::printf("log10(g2 [cgs]) = %s\n", lcb::fmt_lower_exp(r.logg2, 12).c_str());
    std::printf("Vol-averaged r1 = %s\n", lcb::fmt_lower_exp(r.rv1, 12).c_str());
    std::printf("Vol-averaged r2 = %s\n", lcb::fmt_lower_exp(r.rv2, 12).c_str());
    if (!output.empty()) {  // main.rs:103-111
        FILE* f = std::fopen(output.c_str(), "w");
        if (!f) return die("cannot write " + output);
        for (size_t i = 0; i < data.size(); ++i) std::fprintf(f, "%s\n", line_out(data[i], calc[i]).c_str());
        std::fclose(f);
        std::printf("Written data to %s\n", output.c_str());
    } else {
        for (size_t i = 0; i < data.size(); ++i) std::printf("%s\n", line_out(data[i], calc[i]).c_str());
    }
    lcb_ctx_destroy(ctx);
    lcb_model_destroy(model);
    return 0;
}
