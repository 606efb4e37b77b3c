// lcb_engine.cu — context, device buffers, batch execution and the C ABI.
//
// A batch runs as one launch sequence on the context's stream:
//   memset(aux, status, counter) -> k_phase -> k_elements -> k_roche (or, for
//   small batches, k_roche_scan -> k_roche_chop2) -> k_aux -> k_flux -> k_epilogue
// For a resident batch (lcb_batch_*) the sequence is captured once in a CUDA
// graph and replayed; between runs only the model table and the tables
// derived from it are uploaded, and the graph is rebuilt only when the
// plan's shapes change.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lcurve_b200.h"
#include "lcb_kernels.cuh"
#include "lcb_model.h"
#include "lcb_plan.h"
#include "lcb_stream.h"

using lcb::Error;

namespace {

thread_local std::string t_last_error;

int fail(int code, const std::string& msg) {
    t_last_error = msg;
    return code;
}

// NVTX range around one host-side stage (planning, uploads, launches, result
// copies): visible in Nsight Systems / ncu's NVTX filters; header-only, inert
// when no tool is attached.
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

#define CUDA_TRY(expr)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (expr);                                                                    \
        if (e_ != cudaSuccess) throw Error(LCB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    void ensure(size_t bytes) {
        if (bytes <= cap && p) return;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(bytes, 256);
        CUDA_TRY(cudaMalloc(&p, want));
        cap = want;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// All device storage of one planned batch.
struct DeviceSet {
    DevBuf models, segs, bands, rings, eblocks, rblocks, ablocks, units, dmodel, dsub0, dsrc, data;
    DevBuf rec, pos, p64, d64, ecl, egrp, aux, status, spe, spphi, sptype, spw, slfac, partial, calc, results, counter,
        datum, ecount, fcomp, svda, firsthit;
    void release() {
        for (DevBuf* b : {&models, &segs, &bands, &rings, &eblocks, &rblocks, &ablocks, &units, &dmodel, &dsub0, &dsrc,
                          &data, &rec, &pos, &p64, &d64, &ecl, &egrp, &aux, &status, &spe, &spphi, &sptype, &spw, &slfac,
                          &partial, &calc, &results, &counter, &datum, &ecount, &fcomp, &svda, &firsthit})
            b->release();
    }
};

}  // namespace

struct lcb_model {
    lcb::Model m;
};

constexpr int kStages = 6;  // phase, elements, roche, aux, flux, epilogue

struct lcb_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::mutex mu;
    std::string last_error;
    DeviceSet scratch;  // buffers of transient (non-resident) calls
    lcb::Plan plan;     // plan of the last transient call (its buffers are reused)
    std::vector<lcb_datum> stage;  // host staging of gathered data
    cudaEvent_t ev[kStages + 1] = {};
    int64_t h2d = 0, d2h = 0;  // bytes moved by the current / last call
    int fblink_cap = lcb::kFblinkEvalCap;  // lcb_ctx_set_search_cap
    DevBuf probe;                          // lcb_wait_probe's status words
};

struct lcb_batch {
    lcb_ctx* ctx = nullptr;
    std::vector<lcb::Model> models;
    std::vector<lcb_datum> data;
    std::vector<int64_t> start, count;
    lcb::Plan plan;
    lcb::Plan spare;  // the plan before the last lcb_batch_set_params: its storage is planned into next
    lcb::PlanTuning tune;  // launch-shape choices (lcb_batch_set_tuning); zeros = heuristics
    DeviceSet dev;
    cudaGraphExec_t graph = nullptr;
    int graph_scale = -1;
    int graph_cap = -1;  // the search cap baked into the captured graph's kernel arguments
    std::vector<int64_t> graph_key;
    bool ran = false;
    bool broken = false;  // a re-plan failed part-way: buffers may not match the plan
    double stage_ms[kStages] = {0, 0, 0, 0, 0, 0};
    std::vector<double> h_results, h_calc;
    std::vector<int> h_status;
    unsigned long long ecount[5] = {0, 0, 0, 0, 0};
};

namespace {

// Upload of the plan's tables (and the data) into a device set.
// Words of the per-group eclipse slot masks (one per kEclGroup elements).
size_t ecl_groups(const lcb::Plan& P) { return (size_t)((P.nelem + lcb::kEclGroup - 1) / lcb::kEclGroup); }

// `prev` (a resident batch's previous plan, its tables already on the device):
// tables equal to prev's are not uploaded again (a re-parameterised batch of
// unchanged shape usually changes only the model table and the grid bands).
void upload_plan(lcb_ctx* C, DeviceSet& D, const lcb::Plan& P, const lcb_datum* data, int64_t ndata_src,
                 bool upload_data, const lcb::Plan* prev = nullptr) {
    cudaStream_t s = C->stream;
    auto put = [&](DevBuf& b, const void* src, size_t bytes) {
        b.ensure(bytes);
        if (bytes) CUDA_TRY(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, s));
        C->h2d += (int64_t)bytes;
    };
    // a table equal to the previous plan's is already on the device
    auto put_new = [&](DevBuf& b, const auto& now, const auto& before) {
        const size_t bytes = now.size() * sizeof(now[0]);
        if (prev && b.p && b.cap >= bytes && before.size() == now.size() &&
            (bytes == 0 || std::memcmp(now.data(), before.data(), bytes) == 0))
            return;
        put(b, now.data(), bytes);
    };
    const int64_t nm = (int64_t)P.models.size();
    put(D.models, P.models.data(), nm * sizeof(lcb::ModelDev));
    const lcb::Plan& Q = prev ? *prev : P;
    put_new(D.segs, P.segs, Q.segs);
    put_new(D.bands, P.bands, Q.bands);
    put_new(D.rings, P.rings, Q.rings);
    put_new(D.eblocks, P.eblocks, Q.eblocks);
    put_new(D.rblocks, P.rblocks, Q.rblocks);
    put_new(D.ablocks, P.ablocks, Q.ablocks);
    put_new(D.units, P.units, Q.units);
    put_new(D.dmodel, P.datum_model, Q.datum_model);
    put_new(D.dsub0, P.datum_sub0, Q.datum_sub0);
    if (upload_data) {
        (void)ndata_src;
        if (P.datum_contiguous && P.ndatum > 0) {
            // ragged data laid out model after model: one copy straight from the caller's buffer
            put(D.datum, data + P.datum_src[0], P.ndatum * sizeof(lcb_datum));
        } else {
            // expanded (model, datum) records; shared data is gathered on the host once
            std::vector<lcb_datum>& ex = C->stage;
            ex.resize(P.ndatum);
            for (int64_t d = 0; d < P.ndatum; ++d) ex[d] = data[P.datum_src[d]];
            put(D.datum, ex.data(), ex.size() * sizeof(lcb_datum));
            // the copy is from pageable memory: it is staged before cudaMemcpyAsync returns
        }
    }
    D.rec.ensure(P.nelem * sizeof(float4));
    D.pos.ensure(P.nelem * sizeof(float4));
    D.p64.ensure(P.nelem * sizeof(double4));
    D.d64.ensure(P.nelem * sizeof(double4));
    D.ecl.ensure(P.nelem * lcb::kMaxEcl * sizeof(double2));
    D.egrp.ensure(ecl_groups(P) * sizeof(unsigned));
    D.aux.ensure(nm * lcb::kNumAux * sizeof(double));
    D.status.ensure(nm * sizeof(int));
    D.spe.ensure(P.nsub * sizeof(float4));
    D.spphi.ensure(P.nsub * sizeof(double));
    D.sptype.ensure(P.nsub * sizeof(int8_t));
    D.spw.ensure(P.nsub * sizeof(double));
    D.slfac.ensure(P.ndatum * sizeof(double));
    D.partial.ensure(P.npartial * sizeof(double));
    D.calc.ensure(P.ndatum * sizeof(double));
    D.results.ensure(nm * 12 * sizeof(double));
    D.counter.ensure(sizeof(int) * 4);
    D.ecount.ensure(sizeof(unsigned long long) * 8);
    const size_t ncomp = P.any_iscale ? (size_t)P.ndatum * 5 : 1;
    D.fcomp.ensure(ncomp * sizeof(double));
    D.svda.ensure(ncomp * sizeof(double));
    D.firsthit.ensure((P.roche_split > 1 ? P.rblocks.size() * lcb::kRocheBlock : 1) * sizeof(int));
}

// Parts of the launch sequence: the element stage (grids, continuum, eclipses:
// k_elements, k_roche) and the rest (k_phase, k_aux, k_flux, k_epilogue).
constexpr int kStageElements = 1, kStageRest = 2, kStagesAll = 3;

// The device launch sequence of one batch evaluation.  nblk / nrblk (>= 0)
// launch only the first nblk element blocks and nrblk Roche blocks of the
// uploaded block lists (an element slab, lcb_model_elements).
void enqueue_run(lcb_ctx* C, DeviceSet& D, const lcb::Plan& P, int scale, int rdata, bool timed,
                 int stages = kStagesAll, int64_t nblk = -1, int64_t nrblk = -1) {
    cudaStream_t s = C->stream;
    const int64_t nm = (int64_t)P.models.size();
    if (nblk < 0) nblk = (int64_t)P.eblocks.size();
    if (nrblk < 0) nrblk = (int64_t)P.rblocks.size();
    CUDA_TRY(cudaMemsetAsync(D.aux.p, 0, nm * lcb::kNumAux * sizeof(double), s));
    CUDA_TRY(cudaMemsetAsync(D.status.p, 0, nm * sizeof(int), s));
    CUDA_TRY(cudaMemsetAsync(D.counter.p, 0, sizeof(int) * 4, s));
    CUDA_TRY(cudaMemsetAsync(D.ecount.p, 0, sizeof(unsigned long long) * 8, s));
    if (timed) CUDA_TRY(cudaEventRecord(C->ev[0], s));
    const bool rest = stages & kStageRest, elem = stages & kStageElements;
    const lcb::Sizes sz{P.nelem, P.nsub, P.npartial, P.ndatum, (int64_t)P.bands.size(), (int64_t)P.rings.size()};
    lcb::PhaseArgs pa{D.models.as<lcb::ModelDev>(), D.datum.as<lcb_datum>(), D.dmodel.as<int32_t>(),
                      D.dsub0.as<int64_t>(), P.ndatum, D.spe.as<float4>(), D.spphi.as<double>(),
                      D.sptype.as<int8_t>(), D.spw.as<double>(), D.slfac.as<double>()};
    if (rest) CUDA_TRY(lcb::launch_phase(pa, s));
    if (timed) CUDA_TRY(cudaEventRecord(C->ev[1], s));
    lcb::ElemArgs ea{D.models.as<lcb::ModelDev>(), D.segs.as<lcb::SegDesc>(), D.eblocks.as<lcb::ElemBlock>(),
                     D.rblocks.as<lcb::ElemBlock>(), D.ablocks.as<lcb::ElemBlock>(), D.bands.as<lcb::Band>(),
                     D.rings.as<lcb::Ring>(), D.rec.as<float4>(), D.pos.as<float4>(), D.p64.as<double4>(),
                     D.d64.as<double4>(), D.ecl.as<double2>(), D.egrp.as<unsigned>(), D.aux.as<double>(),
                     D.status.as<int>(), nblk, nrblk, (int64_t)P.ablocks.size(),
                     D.ecount.as<unsigned long long>(), P.roche_split, D.firsthit.as<int>(), C->fblink_cap, sz};
    if (elem) {
        CUDA_TRY(cudaMemsetAsync(D.egrp.p, 0, ecl_groups(P) * sizeof(unsigned), s));
        if (P.roche_split > 1 && nrblk > 0)
            CUDA_TRY(cudaMemsetAsync(D.firsthit.p, 0x7f, nrblk * lcb::kRocheBlock * sizeof(int), s));
        CUDA_TRY(lcb::launch_elements(ea, s));
    }
    if (timed) CUDA_TRY(cudaEventRecord(C->ev[2], s));
    if (elem) CUDA_TRY(lcb::launch_roche(ea, s));
    if (timed) CUDA_TRY(cudaEventRecord(C->ev[3], s));
    if (!rest) return;
    CUDA_TRY(lcb::launch_aux(ea, s));
    if (timed) CUDA_TRY(cudaEventRecord(C->ev[4], s));
    lcb::FluxArgs fa{D.models.as<lcb::ModelDev>(), D.units.as<lcb::FluxUnit>(), (int64_t)P.units.size(),
                     D.counter.as<int>(), D.rec.as<float4>(), D.pos.as<float4>(), D.ecl.as<double2>(),
                     D.egrp.as<unsigned>(), D.spe.as<float4>(), D.spphi.as<double>(), D.sptype.as<int8_t>(), D.partial.as<double>(),
                     D.status.as<int>(), sz};
    const int bps_max = lcb::flux_blocks_per_sm();
    const int bps = P.flux_blocks_per_sm > 0 ? std::min(P.flux_blocks_per_sm, bps_max) : bps_max;
    int64_t grid = (int64_t)C->num_sms * bps;
    grid = std::min<int64_t>(grid, std::max<int64_t>((int64_t)P.units.size(), 1));
    CUDA_TRY(lcb::launch_flux(fa, (int)grid, s));
    if (timed) CUDA_TRY(cudaEventRecord(C->ev[5], s));
    lcb::EpiArgs pe{D.models.as<lcb::ModelDev>(), D.datum.as<lcb_datum>(), D.dsub0.as<int64_t>(),
                    D.spphi.as<double>(), D.spw.as<double>(), D.slfac.as<double>(), D.partial.as<double>(),
                    D.aux.as<double>(), D.status.as<int>(), scale, rdata, D.calc.as<double>(),
                    D.results.as<double>(), D.fcomp.as<double>(), D.svda.as<double>(), nm, sz, D.status.as<int>()};
    CUDA_TRY(lcb::launch_epilogue(pe, s));
    if (timed) CUDA_TRY(cudaEventRecord(C->ev[6], s));
}

void set_device(lcb_ctx* C) { CUDA_TRY(cudaSetDevice(C->device)); }

void fetch_results(lcb_ctx* C, DeviceSet& D, const lcb::Plan& P, std::vector<double>& res, std::vector<double>* calc,
                   std::vector<int>* status, unsigned long long* ecount = nullptr) {
    const int64_t nm = (int64_t)P.models.size();
    res.resize(nm * 12);
    CUDA_TRY(cudaMemcpyAsync(res.data(), D.results.p, nm * 12 * sizeof(double), cudaMemcpyDeviceToHost, C->stream));
    if (calc) {
        calc->resize(P.ndatum);
        if (P.ndatum)
            CUDA_TRY(cudaMemcpyAsync(calc->data(), D.calc.p, P.ndatum * sizeof(double), cudaMemcpyDeviceToHost, C->stream));
    }
    if (status) {
        status->resize(nm);
        CUDA_TRY(cudaMemcpyAsync(status->data(), D.status.p, nm * sizeof(int), cudaMemcpyDeviceToHost, C->stream));
    }
    if (ecount)  // the eclipse-search counters (5)
        CUDA_TRY(cudaMemcpyAsync(ecount, D.ecount.p, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, C->stream));
    C->d2h += (int64_t)(nm * 12 * sizeof(double)) + (calc ? P.ndatum * (int64_t)sizeof(double) : 0) +
              (status ? nm * (int64_t)sizeof(int) : 0);
    CUDA_TRY(cudaStreamSynchronize(C->stream));
}

// Device checks that fail a whole call (as opposed to one model's NaN): a bounded
// wait that gave up, or (LCURVE_DEBUG_BOUNDS build) an index out of range.
void check_device_status(int st) {
    if (st & lcb::kStatusTmaTimeout) throw Error(LCB_ERR_DEVICE_CHECK, "a bounded device wait timed out");
    if (st & lcb::kStatusBounds) throw Error(LCB_ERR_DEVICE_CHECK, "a device-side bounds check failed");
}

void fill_result(const double* r, lcb_result* out) {
    out->wdwarf = r[0]; out->chisq = r[1]; out->wnok = r[2]; out->logg1 = r[3]; out->logg2 = r[4];
    out->rv1 = r[5]; out->rv2 = r[6];
    for (int k = 0; k < 5; ++k) out->sfac[k] = r[7 + k];
}


// A transient evaluation on the context's scratch buffers.
void run_transient(lcb_ctx* C, const lcb::Model* const* models, int64_t n, const lcb_datum* data,
                   const int64_t* start, const int64_t* count, int scale, int rdata, std::vector<double>& res,
                   std::vector<double>* calc, lcb::Plan& P, std::vector<int>& st) {
    {
        Range r("lcb plan");
        lcb::plan_batch(models, n, data, start, count, C->num_sms, P);
    }
    {
        Range r("lcb upload");
        upload_plan(C, C->scratch, P, data, 0, true);
    }
    {
        Range r("lcb launch");
        enqueue_run(C, C->scratch, P, scale, rdata, false);
    }
    {
        Range r("lcb results");
        fetch_results(C, C->scratch, P, res, calc, &st);
    }
    for (int64_t i = 0; i < n; ++i)
        check_device_status(st[i]);
}

template <class F>
int guarded(lcb_ctx* C, F&& f) {
    try {
        if (C) {
            std::lock_guard<std::mutex> g(C->mu);
            set_device(C);
            (void)cudaGetLastError();  // a stale non-sticky error must not be blamed on this call
            C->h2d = C->d2h = 0;
            f();
        } else {
            f();
        }
        return LCB_OK;
    } catch (const Error& e) {
        if (C) C->last_error = e.what();
        return fail(e.code, e.what());
    } catch (const std::bad_alloc&) {
        if (C) C->last_error = "out of host memory";
        return fail(LCB_ERR_INVALID, "out of host memory");
    } catch (const std::exception& e) {
        if (C) C->last_error = e.what();
        return fail(LCB_ERR_INVALID, e.what());
    }
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* lcb_version(void) { return "lcurve-b200 0.1.0 (sm_100a)"; }
const char* lcb_last_error(void) { return t_last_error.c_str(); }

int lcb_device_count(int* count) {
    if (!count) return fail(LCB_ERR_INVALID, "null pointer");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) { *count = 0; return fail(LCB_ERR_NO_DEVICE, cudaGetErrorString(e)); }
    *count = n;
    return LCB_OK;
}

int lcb_ctx_create(int device, lcb_ctx** out) {
    if (!out) return fail(LCB_ERR_INVALID, "null pointer");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return fail(LCB_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= n) return fail(LCB_ERR_NO_DEVICE, "device id out of range");
    auto C = std::make_unique<lcb_ctx>();
    C->device = device;
    int rc = guarded(nullptr, [&] {
        CUDA_TRY(cudaSetDevice(device));
        cudaDeviceProp prop;
        CUDA_TRY(cudaGetDeviceProperties(&prop, device));
        if (prop.major < 10) throw Error(LCB_ERR_NO_DEVICE, "this library is built for sm_100a (B200)");
        C->num_sms = prop.multiProcessorCount;
        // fails here, not later, if the sm_100a image cannot load on this device
        if (lcb::flux_blocks_per_sm() <= 0) throw Error(LCB_ERR_NO_DEVICE, "kernel image not loadable");
        CUDA_TRY(cudaStreamCreateWithFlags(&C->stream, cudaStreamNonBlocking));
        C->own_stream = true;
        for (auto& e : C->ev) CUDA_TRY(cudaEventCreate(&e));
    });
    if (rc != LCB_OK) return rc;
    *out = C.release();
    return LCB_OK;
}

void lcb_ctx_destroy(lcb_ctx* C) {
    if (!C) return;
    cudaSetDevice(C->device);
    if (C->stream) cudaStreamSynchronize(C->stream);
    C->scratch.release();
    C->probe.release();
    for (auto& e : C->ev)
        if (e) cudaEventDestroy(e);
    if (C->own_stream && C->stream) cudaStreamDestroy(C->stream);
    delete C;
}

int lcb_ctx_set_stream(lcb_ctx* C, void* stream) {
    if (!C) return fail(LCB_ERR_INVALID, "null context");
    return guarded(C, [&] {
        if (C->own_stream && C->stream) {
            CUDA_TRY(cudaStreamSynchronize(C->stream));
            CUDA_TRY(cudaStreamDestroy(C->stream));
        }
        C->own_stream = stream == nullptr;
        if (stream) C->stream = (cudaStream_t)stream;
        else CUDA_TRY(cudaStreamCreateWithFlags(&C->stream, cudaStreamNonBlocking));
    });
}

const char* lcb_ctx_last_error(const lcb_ctx* C) { return C ? C->last_error.c_str() : "null context"; }

// ---- models -----------------------------------------------------------------
int lcb_model_load(const char* path, lcb_model** out) {
    if (!path || !out) return fail(LCB_ERR_INVALID, "null pointer");
    return guarded(nullptr, [&] { *out = new lcb_model{lcb::load_model_file(path)}; });
}
int lcb_model_parse(const char* text, lcb_model** out) {
    if (!text || !out) return fail(LCB_ERR_INVALID, "null pointer");
    return guarded(nullptr, [&] { *out = new lcb_model{lcb::parse_model_text(text)}; });
}
int lcb_model_clone(const lcb_model* m, lcb_model** out) {
    if (!m || !out) return fail(LCB_ERR_INVALID, "null pointer");
    return guarded(nullptr, [&] { *out = new lcb_model{m->m}; });
}
void lcb_model_destroy(lcb_model* m) { delete m; }

int lcb_model_set_param(lcb_model* m, const char* name, double value) {
    if (!m || !name) return fail(LCB_ERR_INVALID, "null pointer");
    int i = lcb::phys_index(name);
    if (i < 0) return fail(LCB_ERR_UNKNOWN_PARAM, std::string("unknown parameter: '") + name + "'");
    m->m.p[i].value = value;
    return LCB_OK;
}
int lcb_model_get_param(const lcb_model* m, const char* name, double* value) {
    if (!m || !name || !value) return fail(LCB_ERR_INVALID, "null pointer");
    int i = lcb::phys_index(name);
    if (i < 0) return fail(LCB_ERR_UNKNOWN_PARAM, std::string("unknown parameter: '") + name + "'");
    *value = m->m.p[i].value;
    return LCB_OK;
}
int lcb_model_get_pparam(const lcb_model* m, const char* name, double* value, double* range, double* dstep,
                         int* vary, int* defined) {
    if (!m || !name) return fail(LCB_ERR_INVALID, "null pointer");
    int i = lcb::phys_index(name);
    if (i < 0) return fail(LCB_ERR_UNKNOWN_PARAM, std::string("unknown parameter: '") + name + "'");
    const lcb::Pparam& p = m->m.p[i];
    if (value) *value = p.value;
    if (range) *range = p.range;
    if (dstep) *dstep = p.dstep;
    if (vary) *vary = p.vary;
    if (defined) *defined = p.defined;
    return LCB_OK;
}
int lcb_model_set_pparam(lcb_model* m, const char* name, const double* value, const double* range,
                         const double* dstep, const int* vary) {
    if (!m || !name) return fail(LCB_ERR_INVALID, "null pointer");
    int i = lcb::phys_index(name);
    if (i < 0) return fail(LCB_ERR_UNKNOWN_PARAM, std::string("unknown parameter: '") + name + "'");
    lcb::Pparam& p = m->m.p[i];
    if (value) p.value = *value;
    if (range) p.range = *range;
    if (dstep) p.dstep = *dstep;
    if (vary) p.vary = *vary != 0;
    return LCB_OK;
}
int lcb_model_set_comp(lcb_model* m, const char* name, const char* value) {
    if (!m || !name || !value) return fail(LCB_ERR_INVALID, "null pointer");
    return guarded(nullptr, [&] { lcb::set_comp_param(m->m, name, value); });
}
int lcb_model_get_comp(const lcb_model* m, const char* name, char* buf, int buflen) {
    if (!m || !name || !buf || buflen <= 0) return fail(LCB_ERR_INVALID, "null pointer");
    return guarded(nullptr, [&] {
        std::string s = lcb::get_comp_param(m->m, name);
        std::snprintf(buf, (size_t)buflen, "%s", s.c_str());
    });
}
const char* lcb_param_name(int i) { return lcb::phys_name(i); }

// ---- data -------------------------------------------------------------------
int lcb_read_data(const char* path, lcb_datum** out, int64_t* n) {
    if (!path || !out || !n) return fail(LCB_ERR_INVALID, "null pointer");
    return guarded(nullptr, [&] {
        std::vector<lcb_datum> d = lcb::read_data_file(path);
        lcb_datum* p = (lcb_datum*)std::malloc(std::max<size_t>(d.size(), 1) * sizeof(lcb_datum));
        if (!p) throw std::bad_alloc();
        if (!d.empty()) std::memcpy(p, d.data(), d.size() * sizeof(lcb_datum));
        *out = p;
        *n = (int64_t)d.size();
    });
}
void lcb_free_data(lcb_datum* d) { std::free(d); }

// ---- evaluation ---------------------------------------------------------------
int lcb_light_curve(lcb_ctx* C, const lcb_model* model, const lcb_datum* data, int64_t n, int scale, int rdata,
                    double* calc_out, lcb_result* res_out) {
    if (!C || !model || (!data && n > 0) || !calc_out) return fail(LCB_ERR_INVALID, "null pointer");
    if (n <= 0) return fail(LCB_ERR_EMPTY, "No data points");
    return guarded(C, [&] {
        const lcb::Model* mp = &model->m;
        int64_t st = 0, cnt = n;
        std::vector<double> res, calc;
        std::vector<int> status;
        lcb::Plan P;
        run_transient(C, &mp, 1, data, &st, &cnt, scale, rdata, res, &calc, P, status);
        if (!P.model_ok[0]) throw Error(LCB_ERR_MODEL, P.model_err[0]);
        if (status[0] & lcb::kStatusIterCap)
            throw Error(LCB_ERR_DEVICE_CHECK, "a device-side iteration cap tripped for this model");
        std::memcpy(calc_out, calc.data(), n * sizeof(double));
        if (res_out) fill_result(res.data(), res_out);
    });
}

int lcb_model_grid(lcb_ctx* C, const lcb_model* model, int which, int64_t* n, double* posn, double* dirn,
                   float* area, float* gravity, float* flux, double* ecl) {
    if (!C || !model || !n || which < 0 || which > 6) return fail(LCB_ERR_INVALID, "bad arguments");
    return guarded(C, [&] {
        const lcb::Model* mp = &model->m;
        lcb_datum d{};
        d.time = 0.0; d.expose = 0.0; d.ferr = 1.0; d.weight = 1.0; d.ndiv = 1;
        int64_t st = 0, cnt = 1;
        lcb::Plan P;
        lcb::plan_batch(&mp, 1, &d, &st, &cnt, C->num_sms, P);
        if (!P.model_ok[0]) throw Error(LCB_ERR_MODEL, P.model_err[0]);
        const lcb::SegDesc* g = nullptr;
        for (const auto& sg : P.segs) {
            bool star = sg.kind == lcb::SEG_STAR1 || sg.kind == lcb::SEG_STAR2;
            int k = sg.kind == lcb::SEG_STAR1 ? 1 : 2;
            if (star && which <= 3) {
                bool fine = which <= 1;
                if ((which % 2 == 0 ? 1 : 2) != k) continue;
                if (sg.role == lcb::ROLE_BOTH || (sg.role == lcb::ROLE_FINE) == fine) { g = &sg; break; }
            } else if ((which == 4 && sg.kind == lcb::SEG_DISC) || (which == 5 && sg.kind == lcb::SEG_EDGE) ||
                       (which == 6 && sg.kind == lcb::SEG_SPOT)) {
                g = &sg;
                break;
            }
        }
        *n = g ? g->count : 0;
        if (!g || !posn) return;
        upload_plan(C, C->scratch, P, &d, 1, true);
        enqueue_run(C, C->scratch, P, 0, 0, false);
        CUDA_TRY(cudaStreamSynchronize(C->stream));
        std::vector<double4> p64(g->count), d64(g->count);
        std::vector<float4> rec(g->count);
        std::vector<double2> e(g->count * lcb::kMaxEcl);
        CUDA_TRY(cudaMemcpy(p64.data(), C->scratch.p64.as<double4>() + g->first, g->count * sizeof(double4),
                            cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(d64.data(), C->scratch.d64.as<double4>() + g->first, g->count * sizeof(double4),
                            cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(rec.data(), C->scratch.rec.as<float4>() + g->first, g->count * sizeof(float4),
                            cudaMemcpyDeviceToHost));
        for (int k = 0; k < lcb::kMaxEcl; ++k)  // slot-major on the device
            CUDA_TRY(cudaMemcpy(e.data() + k * g->count, C->scratch.ecl.as<double2>() + k * P.nelem + g->first,
                                g->count * sizeof(double2), cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < g->count; ++i) {
            posn[3 * i] = p64[i].x; posn[3 * i + 1] = p64[i].y; posn[3 * i + 2] = p64[i].z;
            if (dirn) { dirn[3 * i] = d64[i].x; dirn[3 * i + 1] = d64[i].y; dirn[3 * i + 2] = d64[i].z; }
            if (area) area[i] = (float)p64[i].w;
            if (gravity) gravity[i] = (float)d64[i].w;
            if (flux) flux[i] = rec[i].w;
            if (ecl)
                for (int k = 0; k < lcb::kMaxEcl; ++k) {
                    ecl[8 * i + 2 * k] = e[k * g->count + i].x;
                    ecl[8 * i + 2 * k + 1] = e[k * g->count + i].y;
                }
        }
    });
}

// Element records of one model exchanged across devices (a model split into element slabs):
// five device arrays in the engine's own element order; the eclipse slots element-major
// (kMaxEcl pairs per element), converted from and to the engine's slot-major array.
static const size_t kElemBytes[4] = {sizeof(float4), sizeof(float4), sizeof(double4), sizeof(double4)};

int lcb_model_elements(lcb_ctx* C, const lcb_model* model, int64_t first, int64_t count, void* rec_dev,
                       void* pos_dev, void* p64_dev, void* d64_dev, void* ecl_dev, int64_t* total) {
    if (!C || !model || !total || first < 0 || count < 0) return fail(LCB_ERR_INVALID, "bad arguments");
    return guarded(C, [&] {
        const lcb::Model* mp = &model->m;
        lcb_datum d{};
        d.ferr = 1.0; d.weight = 1.0; d.ndiv = 1;
        int64_t st = 0, cnt = 1;
        lcb::Plan& P = C->plan;
        lcb::plan_batch(&mp, 1, &d, &st, &cnt, C->num_sms, P);
        if (!P.model_ok[0]) throw Error(LCB_ERR_MODEL, P.model_err[0]);
        *total = P.nelem;
        if (!rec_dev) return;
        if (!pos_dev || !p64_dev || !d64_dev || !ecl_dev) throw Error(LCB_ERR_INVALID, "null device array");
        if (first + count > P.nelem) throw Error(LCB_ERR_INVALID, "element range beyond the model's elements");
        if (count == 0) return;
        // the element blocks and Roche blocks that touch [first, first + count): every Roche
        // block lies inside an element block, so the slab's elements are all computed
        const int64_t last = first + count;
        auto touches = [&](const lcb::ElemBlock& b, int64_t width) {
            const int64_t e0 = P.segs[b.seg].first + b.offset;
            return e0 < last && e0 + width > first;
        };
        std::vector<lcb::ElemBlock> eb, rb;
        for (const auto& b : P.eblocks)
            if (touches(b, lcb::kElemThreads)) eb.push_back(b);
        for (const auto& b : P.rblocks)
            if (touches(b, lcb::kRocheBlock)) rb.push_back(b);
        upload_plan(C, C->scratch, P, &d, 1, true);
        DeviceSet& D = C->scratch;
        if (!eb.empty())
            CUDA_TRY(cudaMemcpyAsync(D.eblocks.p, eb.data(), eb.size() * sizeof(lcb::ElemBlock),
                                     cudaMemcpyHostToDevice, C->stream));
        if (!rb.empty())
            CUDA_TRY(cudaMemcpyAsync(D.rblocks.p, rb.data(), rb.size() * sizeof(lcb::ElemBlock),
                                     cudaMemcpyHostToDevice, C->stream));
        enqueue_run(C, D, P, 0, 0, false, kStageElements, (int64_t)eb.size(), (int64_t)rb.size());
        void* dst[4] = {rec_dev, pos_dev, p64_dev, d64_dev};
        const void* src[4] = {D.rec.p, D.pos.p, D.p64.p, D.d64.p};
        for (int k = 0; k < 4; ++k)
            CUDA_TRY(cudaMemcpyAsync(dst[k], (const char*)src[k] + first * kElemBytes[k], count * kElemBytes[k],
                                     cudaMemcpyDeviceToDevice, C->stream));
        CUDA_TRY(lcb::launch_ecl_export(D.ecl.as<double2>(), P.nelem, first, count, (double2*)ecl_dev, C->stream));
        int status = 0;
        CUDA_TRY(cudaMemcpyAsync(&status, D.status.p, sizeof(int), cudaMemcpyDeviceToHost, C->stream));
        CUDA_TRY(cudaStreamSynchronize(C->stream));
        check_device_status(status);
        if (status & lcb::kStatusIterCap)
            throw Error(LCB_ERR_DEVICE_CHECK, "a device-side iteration cap tripped for this model");
    });
}

int lcb_light_curve_elements(lcb_ctx* C, const lcb_model* model, const lcb_datum* data, int64_t n, int scale,
                             int rdata, const void* rec_dev, const void* pos_dev, const void* p64_dev,
                             const void* d64_dev, const void* ecl_dev, double* calc_out, lcb_result* res_out) {
    if (!C || !model || (!data && n > 0) || !calc_out || !rec_dev || !pos_dev || !p64_dev || !d64_dev || !ecl_dev)
        return fail(LCB_ERR_INVALID, "null pointer");
    if (n <= 0) return fail(LCB_ERR_EMPTY, "No data points");
    return guarded(C, [&] {
        const lcb::Model* mp = &model->m;
        int64_t st = 0, cnt = n;
        lcb::Plan& P = C->plan;
        lcb::plan_batch(&mp, 1, data, &st, &cnt, C->num_sms, P);
        if (!P.model_ok[0]) throw Error(LCB_ERR_MODEL, P.model_err[0]);
        upload_plan(C, C->scratch, P, data, 0, true);
        DeviceSet& D = C->scratch;
        const void* src[4] = {rec_dev, pos_dev, p64_dev, d64_dev};
        void* dst[4] = {D.rec.p, D.pos.p, D.p64.p, D.d64.p};
        for (int k = 0; k < 4; ++k)
            if (P.nelem)
                CUDA_TRY(cudaMemcpyAsync(dst[k], src[k], P.nelem * kElemBytes[k], cudaMemcpyDeviceToDevice, C->stream));
        CUDA_TRY(cudaMemsetAsync(D.egrp.p, 0, ecl_groups(P) * sizeof(unsigned), C->stream));
        CUDA_TRY(lcb::launch_ecl_import((const double2*)ecl_dev, P.nelem, D.ecl.as<double2>(), D.egrp.as<unsigned>(),
                                        C->stream));
        enqueue_run(C, D, P, scale, rdata, false, kStageRest);
        std::vector<double> res, calc;
        std::vector<int> status;
        fetch_results(C, D, P, res, &calc, &status);
        check_device_status(status[0]);
        std::memcpy(calc_out, calc.data(), n * sizeof(double));
        if (res_out) fill_result(res.data(), res_out);
    });
}

int lcb_chisq_batch(lcb_ctx* C, const lcb_model* base, const lcb_datum* data, int64_t n, const char* const* names,
                    int ndim, const double* values, int64_t nsets, int scale, double* chisq_out) {
    if (!C || !base || !data || !names || !values || !chisq_out) return fail(LCB_ERR_INVALID, "null pointer");
    if (ndim <= 0 || nsets < 0) return fail(LCB_ERR_INVALID, "ndim must be > 0");
    if (n <= 0) return fail(LCB_ERR_EMPTY, "No data points");
    return guarded(C, [&] {
        std::vector<int> idx(ndim);
        for (int j = 0; j < ndim; ++j) idx[j] = lcb::phys_index(names[j]);  // unknown names are ignored
        std::vector<lcb::Model> ms(nsets, base->m);
        std::vector<const lcb::Model*> mp(nsets);
        for (int64_t i = 0; i < nsets; ++i) {
            for (int j = 0; j < ndim; ++j)
                if (idx[j] >= 0) ms[i].p[idx[j]].value = values[i * ndim + j];
            mp[i] = &ms[i];
        }
        if (nsets == 0) return;
        std::vector<int64_t> st(nsets, 0), cnt(nsets, n);
        std::vector<double> res;
        std::vector<int> status;
        lcb::Plan& P = C->plan;
        run_transient(C, mp.data(), nsets, data, st.data(), cnt.data(), scale, 1, res, nullptr, P, status);
        for (int64_t i = 0; i < nsets; ++i) chisq_out[i] = P.model_ok[i] ? res[i * 12 + 1] : NAN;
    });
}

int lcb_chisq_batch_ragged(lcb_ctx* C, const lcb_model* const* models, int64_t nmodels, const lcb_datum* data,
                           const int64_t* offsets, int scale, double* chisq_out, double* calc_out,
                           lcb_result* res_out) {
    if (!C || !models || !data || !offsets || !chisq_out) return fail(LCB_ERR_INVALID, "null pointer");
    if (nmodels <= 0) return fail(LCB_ERR_INVALID, "nmodels must be > 0");
    return guarded(C, [&] {
        std::vector<const lcb::Model*> mp(nmodels);
        std::vector<int64_t> st(nmodels), cnt(nmodels);
        for (int64_t i = 0; i < nmodels; ++i) {
            if (!models[i]) throw Error(LCB_ERR_INVALID, "null model");
            mp[i] = &models[i]->m;
            st[i] = offsets[i];
            cnt[i] = offsets[i + 1] - offsets[i];
            if (cnt[i] < 0) throw Error(LCB_ERR_INVALID, "offsets must be non-decreasing");
        }
        std::vector<double> res, calc;
        std::vector<int> status;
        lcb::Plan& P = C->plan;
        run_transient(C, mp.data(), nmodels, data, st.data(), cnt.data(), scale, 1, res, calc_out ? &calc : nullptr, P,
                      status);
        for (int64_t i = 0; i < nmodels; ++i) {
            chisq_out[i] = P.model_ok[i] ? res[i * 12 + 1] : NAN;
            if (res_out) {
                if (P.model_ok[i]) fill_result(&res[i * 12], &res_out[i]);
                else {
                    double nanv[12];
                    for (double& v : nanv) v = NAN;
                    fill_result(nanv, &res_out[i]);
                }
            }
        }
        if (calc_out)
            for (int64_t d = 0; d < P.ndatum; ++d) calc_out[offsets[0] + d] = calc[d];
    });
}

// ---- resident batch -------------------------------------------------------------
int lcb_batch_create(lcb_ctx* C, const lcb_model* const* models, int64_t nmodels, const lcb_datum* data,
                     const int64_t* offsets, lcb_batch** out) {
    if (!C || !models || !data || !offsets || !out) return fail(LCB_ERR_INVALID, "null pointer");
    if (nmodels <= 0) return fail(LCB_ERR_INVALID, "nmodels must be > 0");
    *out = nullptr;
    auto B = std::make_unique<lcb_batch>();
    B->ctx = C;
    int rc = guarded(C, [&] {
        int64_t total = offsets[nmodels] - offsets[0];
        if (total < 0) throw Error(LCB_ERR_INVALID, "offsets must be non-decreasing");
        B->data.assign(data + offsets[0], data + offsets[0] + total);
        for (int64_t i = 0; i < nmodels; ++i) {
            if (!models[i]) throw Error(LCB_ERR_INVALID, "null model");
            B->models.push_back(models[i]->m);
            B->start.push_back(offsets[i] - offsets[0]);
            B->count.push_back(offsets[i + 1] - offsets[i]);
            if (B->count.back() < 0) throw Error(LCB_ERR_INVALID, "offsets must be non-decreasing");
        }
        std::vector<const lcb::Model*> mp(nmodels);
        for (int64_t i = 0; i < nmodels; ++i) mp[i] = &B->models[i];
        lcb::plan_batch(mp.data(), nmodels, B->data.data(), B->start.data(), B->count.data(), C->num_sms, B->plan,
                        B->tune);
        upload_plan(C, B->dev, B->plan, B->data.data(), (int64_t)B->data.size(), true);
        CUDA_TRY(cudaStreamSynchronize(C->stream));
    });
    if (rc != LCB_OK) {
        B->dev.release();
        return rc;
    }
    *out = B.release();
    return LCB_OK;
}

void lcb_batch_destroy(lcb_batch* B) {
    if (!B) return;
    std::lock_guard<std::mutex> g(B->ctx->mu);
    cudaSetDevice(B->ctx->device);
    cudaStreamSynchronize(B->ctx->stream);
    if (B->graph) cudaGraphExecDestroy(B->graph);
    B->dev.release();
    delete B;
}

// Re-plans a resident batch after its models or its tuning changed: plans into the spare
// storage, uploads what changed, drops the captured graph when the shapes changed.
// If the uploads fail part-way (a buffer could not grow), the device buffers no longer
// match the plan: the batch is marked broken, its graph dropped and its shape key
// cleared, so no launch runs on it until a later re-plan uploads everything again.
static void replan_batch(lcb_batch* B) {
    lcb_ctx* C = B->ctx;
    const int64_t n = (int64_t)B->models.size();
    std::vector<const lcb::Model*> mp(n);
    for (int64_t i = 0; i < n; ++i) mp[i] = &B->models[i];
    lcb::Plan& P = B->spare;
    Range r("lcb replan");
    lcb::plan_batch(mp.data(), n, B->data.data(), B->start.data(), B->count.data(), C->num_sms, P, B->tune);
    const bool same = !B->broken && P.shape_key == B->plan.shape_key;
    std::swap(B->plan, P);
    try {
        upload_plan(C, B->dev, B->plan, B->data.data(), (int64_t)B->data.size(), !same, same ? &P : nullptr);
        if (!same && B->graph) {
            cudaGraphExecDestroy(B->graph);
            B->graph = nullptr;
        }
        // copies from pageable host memory are staged before cudaMemcpyAsync returns, so the
        // plan's host tables may change at once; a new shape waits for its uploads here
        if (!same) CUDA_TRY(cudaStreamSynchronize(C->stream));
    } catch (...) {
        cudaStreamSynchronize(C->stream);
        if (B->graph) cudaGraphExecDestroy(B->graph);
        B->graph = nullptr;
        B->plan.shape_key.clear();
        B->broken = true;
        throw;
    }
    B->broken = false;
}

static void check_usable(const lcb_batch* B) {
    if (B->broken)
        throw Error(LCB_ERR_INVALID, "the batch's last re-plan failed (device memory); set its parameters or "
                                     "tuning again before running it");
}

int lcb_batch_set_tuning(lcb_batch* B, int flux_chunks, int roche_split, int flux_blocks_per_sm) {
    if (!B) return fail(LCB_ERR_INVALID, "null batch");
    if (flux_chunks < 0 || flux_chunks > 16 || roche_split < 0 || roche_split > 16 || flux_blocks_per_sm < 0)
        return fail(LCB_ERR_INVALID, "tuning out of range (flux_chunks, roche_split 0..16; blocks per SM >= 0)");
    lcb_ctx* C = B->ctx;
    return guarded(C, [&] {
        B->tune.flux_chunks = flux_chunks;
        B->tune.roche_split = roche_split;
        B->tune.flux_blocks_per_sm = flux_blocks_per_sm;
        replan_batch(B);
    });
}

int lcb_batch_get_tuning(const lcb_batch* B, int* out3) {
    if (!B || !out3) return fail(LCB_ERR_INVALID, "null pointer");
    return guarded(B->ctx, [&] {
        const lcb::Plan& P = B->plan;
        const int bps_max = lcb::flux_blocks_per_sm();
        out3[0] = P.flux_chunks;
        out3[1] = P.roche_split;
        out3[2] = P.flux_blocks_per_sm > 0 ? std::min(P.flux_blocks_per_sm, bps_max) : bps_max;
    });
}

int lcb_batch_set_params(lcb_batch* B, const char* const* names, int ndim, const double* values) {
    if (!B || !names || !values || ndim <= 0) return fail(LCB_ERR_INVALID, "bad arguments");
    lcb_ctx* C = B->ctx;
    return guarded(C, [&] {
        const int64_t n = (int64_t)B->models.size();
        for (int j = 0; j < ndim; ++j) {
            int k = lcb::phys_index(names[j]);
            if (k < 0) throw Error(LCB_ERR_UNKNOWN_PARAM, std::string("unknown parameter: '") + names[j] + "'");
            for (int64_t i = 0; i < n; ++i) B->models[i].p[k].value = values[i * ndim + j];
        }
        // planned into the previous call's storage (kept capacity: no allocation or first-touch
        // page faults when a resident batch is re-parameterised step after step); with unchanged
        // shapes only the model table and the tables derived from it are uploaded
        replan_batch(B);
    });
}

int lcb_batch_run(lcb_batch* B, int scale) {
    if (!B) return fail(LCB_ERR_INVALID, "null batch");
    lcb_ctx* C = B->ctx;
    return guarded(C, [&] {
        check_usable(B);
        if (B->graph && (B->graph_scale != scale || B->graph_key != B->plan.shape_key || B->graph_cap != C->fblink_cap)) {
            cudaGraphExecDestroy(B->graph);
            B->graph = nullptr;
        }
        if (!B->graph) {
            // the flux kernel's shared-memory attribute must be set outside capture
            lcb::flux_blocks_per_sm();
            cudaGraph_t g;
            CUDA_TRY(cudaStreamBeginCapture(C->stream, cudaStreamCaptureModeThreadLocal));
            try {
                enqueue_run(C, B->dev, B->plan, scale, 1, false);
            } catch (...) {
                cudaStreamEndCapture(C->stream, &g);
                throw;
            }
            CUDA_TRY(cudaStreamEndCapture(C->stream, &g));
            cudaError_t e = cudaGraphInstantiate(&B->graph, g, 0);
            cudaGraphDestroy(g);
            CUDA_TRY(e);
            B->graph_scale = scale;
            B->graph_key = B->plan.shape_key;
            B->graph_cap = C->fblink_cap;
        }
        Range r("lcb batch run");
        CUDA_TRY(cudaGraphLaunch(B->graph, C->stream));
        fetch_results(C, B->dev, B->plan, B->h_results, nullptr, &B->h_status, B->ecount);
        B->ran = true;
        for (int s : B->h_status)
            check_device_status(s);
    });
}

int lcb_batch_profile(lcb_batch* B, int scale) {
    if (!B) return fail(LCB_ERR_INVALID, "null batch");
    lcb_ctx* C = B->ctx;
    return guarded(C, [&] {
        check_usable(B);
        enqueue_run(C, B->dev, B->plan, scale, 1, true);
        fetch_results(C, B->dev, B->plan, B->h_results, nullptr, &B->h_status);
        CUDA_TRY(cudaMemcpy(B->ecount, B->dev.ecount.p, sizeof(B->ecount), cudaMemcpyDeviceToHost));
        for (int k = 0; k < kStages; ++k) {
            float ms = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&ms, C->ev[k], C->ev[k + 1]));
            B->stage_ms[k] = ms;
        }
        B->ran = true;
        for (int s : B->h_status)
            check_device_status(s);
    });
}

int lcb_batch_results(lcb_batch* B, double* chisq_out, double* calc_out, lcb_result* res_out) {
    if (!B) return fail(LCB_ERR_INVALID, "null batch");
    if (!B->ran) return fail(LCB_ERR_INVALID, "lcb_batch_run has not been called");
    lcb_ctx* C = B->ctx;
    return guarded(C, [&] {
        check_usable(B);
        const lcb::Plan& P = B->plan;
        const int64_t n = (int64_t)P.models.size();
        for (int64_t i = 0; i < n; ++i) {
            if (chisq_out) chisq_out[i] = P.model_ok[i] ? B->h_results[i * 12 + 1] : NAN;
            if (res_out) {
                double nanv[12];
                for (double& v : nanv) v = NAN;
                fill_result(P.model_ok[i] ? &B->h_results[i * 12] : nanv, &res_out[i]);
            }
        }
        if (calc_out && P.ndatum) {
            CUDA_TRY(cudaMemcpy(calc_out, B->dev.calc.p, P.ndatum * sizeof(double), cudaMemcpyDeviceToHost));
        }
    });
}

int lcb_batch_stats(const lcb_batch* B, int64_t* out8) {
    if (!B || !out8) return fail(LCB_ERR_INVALID, "null pointer");
    const lcb::Plan& P = B->plan;
    int64_t v[8] = {(int64_t)P.models.size(), P.nelem, P.nsub, P.evals, (int64_t)P.units.size(), P.roche_elems,
                    (int64_t)B->ecount[0], (int64_t)B->ecount[1]};
    std::memcpy(out8, v, sizeof v);
    return LCB_OK;
}

int lcb_batch_search_counts(const lcb_batch* B, int64_t* out5) {
    if (!B || !out5) return fail(LCB_ERR_INVALID, "null pointer");
    for (int k = 0; k < 5; ++k) out5[k] = (int64_t)B->ecount[k];
    return LCB_OK;
}

int lcb_batch_stage_ms(const lcb_batch* B, double* out6) {
    if (!B || !out6) return fail(LCB_ERR_INVALID, "null pointer");
    for (int k = 0; k < kStages; ++k) out6[k] = B->stage_ms[k];
    return LCB_OK;
}

int lcb_ctx_transfer_bytes(const lcb_ctx* C, int64_t* h2d, int64_t* d2h) {
    if (!C || !h2d || !d2h) return fail(LCB_ERR_INVALID, "null pointer");
    *h2d = C->h2d;
    *d2h = C->d2h;
    return LCB_OK;
}

namespace {

// The planner's GPU path for many bright-spot streams (lcb_plan.h: StreamDeviceFn): one
// k_stream launch on the calling thread's default stream of the current device; false on
// any CUDA error (the planner then integrates on the host).
bool stream_on_device(const double* in, int n, double* out, int* status) {
    if (n <= 0) return true;
    char* buf = nullptr;
    const size_t bin = 3 * sizeof(double) * (size_t)n, bst = sizeof(int) * (size_t)n;
    cudaStream_t s = cudaStreamPerThread;
    bool ok = cudaMalloc(&buf, 2 * bin + bst) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(buf, in, bin, cudaMemcpyHostToDevice, s) == cudaSuccess;
    ok = ok && lcb::launch_stream((const double*)buf, n, (double*)(buf + bin), (int*)(buf + 2 * bin), s) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(out, buf + bin, bin, cudaMemcpyDeviceToHost, s) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(status, buf + 2 * bin, bst, cudaMemcpyDeviceToHost, s) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
    if (buf) cudaFree(buf);
    if (!ok) cudaGetLastError();  // clear a non-sticky error; the host path takes over
    return ok;
}

const bool g_stream_device_registered = (lcb::set_stream_device(&stream_on_device), true);

}  // namespace

int lcb_stream_points(lcb_ctx* C, const double* q, const double* radius, int64_t n, int on_device, double* out) {
    if (!C || (n > 0 && (!q || !radius || !out)) || n < 0 || n > (1 << 24)) return fail(LCB_ERR_INVALID, "bad arguments");
    return guarded(C, [&] {
        (void)g_stream_device_registered;
        std::vector<double> in(3 * n);
        std::vector<int> st(n, lcb::stream::kStreamOk);
        for (int64_t i = 0; i < n; ++i) {
            in[3 * i] = q[i];
            in[3 * i + 1] = lcb::host_xl1(q[i]);
            in[3 * i + 2] = radius[i];
        }
        if (on_device) {
            if (!stream_on_device(in.data(), (int)n, out, st.data()))
                throw Error(LCB_ERR_CUDA, "the gas-stream kernel failed");
        } else {
            for (int64_t i = 0; i < n; ++i)
                st[i] = lcb::stream::stream_to_radius_core(q[i], in[3 * i + 1], radius[i], out + 3 * i);
        }
        bool bad = false;
        for (int64_t i = 0; i < n; ++i)
            if (st[i] != lcb::stream::kStreamOk) {
                out[3 * i] = out[3 * i + 1] = out[3 * i + 2] = NAN;
                bad = true;
            }
        if (bad) throw Error(LCB_ERR_MODEL, "the gas stream did not reach a radius (NaN rows)");
    });
}

int lcb_model_work(const lcb_model* model, const lcb_datum* data, int64_t n, int64_t* out4) {
    if (!model || (!data && n > 0) || !out4 || n < 0) return fail(LCB_ERR_INVALID, "bad arguments");
    return guarded(nullptr, [&] {
        const lcb::Model* mp = &model->m;
        int64_t st = 0, cnt = n;
        lcb::Plan P;
        lcb::plan_batch(&mp, 1, data, &st, &cnt, 148, P);
        const bool ok = !P.model_ok.empty() && P.model_ok[0];
        int64_t v[4] = {ok ? P.nelem : 0, ok ? P.roche_elems : 0, ok ? P.nsub : 0, ok ? P.evals : 0};
        std::memcpy(out4, v, sizeof v);
    });
}

int lcb_ctx_set_search_cap(lcb_ctx* C, int evals) {
    if (!C || evals < 0) return fail(LCB_ERR_INVALID, "bad arguments");
    return guarded(C, [&] { C->fblink_cap = evals > 0 ? evals : lcb::kFblinkEvalCap; });
}

int lcb_wait_probe(lcb_ctx* C, int64_t limit_cycles, int64_t* waited_cycles) {
    if (!C || limit_cycles <= 0 || limit_cycles > 4000000000LL) return fail(LCB_ERR_INVALID, "bad arguments");
    return guarded(C, [&] {
        C->probe.ensure(2 * sizeof(long long));
        int* status = C->probe.as<int>();
        long long* waited = C->probe.as<long long>() + 1;
        CUDA_TRY(cudaMemsetAsync(C->probe.p, 0, 2 * sizeof(long long), C->stream));
        CUDA_TRY(lcb::launch_wait_probe((long long)limit_cycles, status, waited, C->stream));
        long long h[2] = {0, 0};
        CUDA_TRY(cudaMemcpyAsync(h, C->probe.p, sizeof h, cudaMemcpyDeviceToHost, C->stream));
        CUDA_TRY(cudaStreamSynchronize(C->stream));
        if (waited_cycles) *waited_cycles = h[1];
        if ((int)(h[0] & 0xffffffff) & lcb::kStatusTmaTimeout)
            throw Error(LCB_ERR_DEVICE_CHECK, "a bounded device wait timed out");
    });
}

int lcb_measure_fma_peak(lcb_ctx* C, int which, double* tflops) {
    if (!C || !tflops || (which != 0 && which != 1)) return fail(LCB_ERR_INVALID, "bad arguments");
    return guarded(C, [&] { CUDA_TRY(lcb::measure_fma_peak(which, C->num_sms, C->stream, tflops)); });
}

}  // extern "C"

// ===========================================================================
// lcb_light_curve_noalloc: the light curve of one model with no device
// allocation.
//
// Some callers cannot call cudaMalloc: a process whose device memory is
// already claimed by another framework's pool allocator (JAX preallocating
// most of the GPU, a serving runtime with a fixed memory budget), a plugin
// host that forbids allocation inside its callbacks, or a timing-sensitive
// loop that cannot afford the device-wide synchronisation cudaMalloc and
// cudaFree may imply.  For them this entry point runs the same kernels as
// lcb_light_curve, but every device buffer (plan tables, element and
// sub-phase arrays, flux partials, results) is carved out of one statically
// allocated arena of LCB_NOALLOC_ARENA_BYTES.  Host staging uses ordinary
// pageable host memory.
//
// The arena is file-scope device memory: every device on which this
// library's device code is loaded holds it until the process exits.  In host
// code its name is only a host-side shadow; each call looks up the device
// address (cudaGetSymbolAddress, with the context's device current).
//
// Every call on a device shares the arena, which keeps the previous call's
// contents.  The accumulators that must start at zero (per-model sums, status
// words, the work-unit counter and search counters) are cleared by the launch
// sequence itself; every other region is written in full before it is read.
// Two calls whose GPU work overlapped would race on the arena, so calls on one
// device are serialised by a per-device lock, and each call waits for its GPU
// work (also on its error paths) before it returns.
// ===========================================================================
static __device__ __align__(256) unsigned char g_noalloc_arena[LCB_NOALLOC_ARENA_BYTES];

namespace {

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu[kNoallocMaxDevices];   // one per device

// The arena's device address on the current device.  Looked up on every call
// (it is cheap next to the launch sequence), so a device or primary-context
// reset between calls, which reloads the module at a new address, cannot leave
// a stale pointer behind.  Caller holds g_noalloc_mu[device] and has made
// `device` current.
unsigned char* noalloc_arena() {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_arena);
    if (e != cudaSuccess || !p)
        throw Error(LCB_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc arena): ") + cudaGetErrorString(e));
    return static_cast<unsigned char*>(p);
}

// Lays out every buffer of a planned single-model evaluation inside the arena
// (base == nullptr only measures).  Returns the bytes used.
size_t noalloc_carve(const lcb::Plan& P, unsigned char* base, DeviceSet& D) {
    size_t off = 0;
    auto take = [&](DevBuf& b, size_t bytes) {
        b.p = base ? base + off : nullptr;
        b.cap = bytes;
        off += (bytes + 255) & ~size_t(255);
    };
    const size_t nm = P.models.size();
    take(D.models, nm * sizeof(lcb::ModelDev));
    take(D.segs, P.segs.size() * sizeof(lcb::SegDesc));
    take(D.bands, P.bands.size() * sizeof(lcb::Band));
    take(D.rings, P.rings.size() * sizeof(lcb::Ring));
    take(D.eblocks, P.eblocks.size() * sizeof(lcb::ElemBlock));
    take(D.rblocks, P.rblocks.size() * sizeof(lcb::ElemBlock));
    take(D.ablocks, P.ablocks.size() * sizeof(lcb::ElemBlock));
    take(D.units, P.units.size() * sizeof(lcb::FluxUnit));
    take(D.dmodel, P.datum_model.size() * sizeof(int32_t));
    take(D.dsub0, P.datum_sub0.size() * sizeof(int64_t));
    take(D.datum, P.ndatum * sizeof(lcb_datum));
    take(D.rec, P.nelem * sizeof(float4));
    take(D.pos, P.nelem * sizeof(float4));
    take(D.p64, P.nelem * sizeof(double4));
    take(D.d64, P.nelem * sizeof(double4));
    take(D.ecl, P.nelem * lcb::kMaxEcl * sizeof(double2));
    take(D.egrp, ecl_groups(P) * sizeof(unsigned));
    take(D.aux, nm * lcb::kNumAux * sizeof(double));
    take(D.status, nm * sizeof(int));
    take(D.spe, P.nsub * sizeof(float4));
    take(D.spphi, P.nsub * sizeof(double));
    take(D.sptype, P.nsub * sizeof(int8_t));
    take(D.spw, P.nsub * sizeof(double));
    take(D.slfac, P.ndatum * sizeof(double));
    take(D.partial, P.npartial * sizeof(double));
    take(D.calc, P.ndatum * sizeof(double));
    take(D.results, nm * 12 * sizeof(double));
    take(D.counter, sizeof(int) * 4);
    take(D.ecount, sizeof(unsigned long long) * 8);
    const size_t ncomp = P.any_iscale ? (size_t)P.ndatum * 5 : 1;
    take(D.fcomp, ncomp * sizeof(double));
    take(D.svda, ncomp * sizeof(double));
    take(D.firsthit, (P.roche_split > 1 ? P.rblocks.size() * lcb::kRocheBlock : 1) * sizeof(int));
    return off;
}

// Host -> arena copies of the plan's tables and the data (no allocation).
void noalloc_upload(lcb_ctx* C, DeviceSet& D, const lcb::Plan& P, const lcb_datum* data) {
    auto put = [&](DevBuf& b, const void* src, size_t bytes) {
        if (bytes) CUDA_TRY(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, C->stream));
        C->h2d += (int64_t)bytes;
    };
    put(D.models, P.models.data(), P.models.size() * sizeof(lcb::ModelDev));
    put(D.segs, P.segs.data(), P.segs.size() * sizeof(lcb::SegDesc));
    put(D.bands, P.bands.data(), P.bands.size() * sizeof(lcb::Band));
    put(D.rings, P.rings.data(), P.rings.size() * sizeof(lcb::Ring));
    put(D.eblocks, P.eblocks.data(), P.eblocks.size() * sizeof(lcb::ElemBlock));
    put(D.rblocks, P.rblocks.data(), P.rblocks.size() * sizeof(lcb::ElemBlock));
    put(D.ablocks, P.ablocks.data(), P.ablocks.size() * sizeof(lcb::ElemBlock));
    put(D.units, P.units.data(), P.units.size() * sizeof(lcb::FluxUnit));
    put(D.dmodel, P.datum_model.data(), P.datum_model.size() * sizeof(int32_t));
    put(D.dsub0, P.datum_sub0.data(), P.datum_sub0.size() * sizeof(int64_t));
    std::vector<lcb_datum> ex(P.ndatum);
    for (int64_t d = 0; d < P.ndatum; ++d) ex[d] = data[P.datum_src[d]];
    put(D.datum, ex.data(), ex.size() * sizeof(lcb_datum));
}

}  // namespace

extern "C" int lcb_light_curve_noalloc(lcb_ctx* C, const lcb_model* model, const lcb_datum* data, int64_t n,
                                       int scale, int rdata, double* calc_out, lcb_result* res_out) {
    if (!C || !model || (!data && n > 0) || !calc_out) return fail(LCB_ERR_INVALID, "null pointer");
    if (n <= 0) return fail(LCB_ERR_EMPTY, "No data points");
    if (C->device < 0 || C->device >= kNoallocMaxDevices)
        return fail(LCB_ERR_INVALID, "lcb_light_curve_noalloc: device index beyond the supported 64");
    return guarded(C, [&] {
        const lcb::Model* mp = &model->m;
        int64_t st = 0, cnt = n;
        lcb::Plan P;
        lcb::plan_batch(&mp, 1, data, &st, &cnt, C->num_sms, P);
        if (!P.model_ok[0]) throw Error(LCB_ERR_MODEL, P.model_err[0]);
        DeviceSet D;  // views into the arena: never ensure()d or released
        const size_t need = noalloc_carve(P, nullptr, D);
        if (need > (size_t)LCB_NOALLOC_ARENA_BYTES)
            throw Error(LCB_ERR_INVALID, "lcb_light_curve_noalloc: this model and data need " + std::to_string(need) +
                                             " bytes of device scratch, more than the fixed arena's " +
                                             std::to_string((size_t)LCB_NOALLOC_ARENA_BYTES) +
                                             "; use lcb_light_curve (or coarser grids / fewer points)");
        std::lock_guard<std::mutex> lock(g_noalloc_mu[C->device]);
        noalloc_carve(P, noalloc_arena(), D);
        std::vector<double> res, calc;
        std::vector<int> status;
        try {
            noalloc_upload(C, D, P, data);
            enqueue_run(C, D, P, scale, rdata, false);
            fetch_results(C, D, P, res, &calc, &status);  // ends with a stream synchronise
        } catch (...) {
            cudaStreamSynchronize(C->stream);  // no work may touch the arena after the lock is released
            throw;
        }
        check_device_status(status[0]);
        if (status[0] & lcb::kStatusIterCap)
            throw Error(LCB_ERR_DEVICE_CHECK, "a device-side iteration cap tripped for this model");
        std::memcpy(calc_out, calc.data(), n * sizeof(double));
        if (res_out) fill_result(res.data(), res_out);
    });
}
