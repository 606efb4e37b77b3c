// lcb_plan.h — host planning of a batch: per-model constants and work decomposition.
#pragma once

#include <string>
#include <vector>

#include "lcb_internal.h"
#include "lcb_model.h"

namespace lcb {

// Launch-shape choices an autotuner may fix; 0 leaves each to the planner's heuristic.  Every
// value lies in the range the heuristic itself produces, so the kernels handle it as usual.
struct PlanTuning {
    int flux_chunks = 0;         // elements per flux work unit, in chunks of kFluxChunk (1..16)
    int roche_split = 0;         // threads per Roche-eclipsed element in the phase scan (1..16)
    int flux_blocks_per_sm = 0;  // persistent flux blocks per SM (1..occupancy limit)
};

struct Plan {
    std::vector<ModelDev> models;
    std::vector<SegDesc> segs;
    std::vector<Band> bands;
    std::vector<Ring> rings;
    std::vector<ElemBlock> eblocks;    // k_elements
    std::vector<ElemBlock> rblocks;    // k_roche
    std::vector<ElemBlock> ablocks;    // k_aux
    std::vector<FluxUnit> units;
    std::vector<int32_t> datum_model;   // per (model, datum): model index
    std::vector<int64_t> datum_sub0;    // per (model, datum): first global sub-phase
    std::vector<int64_t> datum_src;     // per (model, datum): index into the caller's data array
    std::vector<int32_t> model_ok;      // 1 = planned, 0 = failed (NaN chisq)
    std::vector<std::string> model_err;
    int64_t nelem = 0, nsub = 0, ndatum = 0, npartial = 0;
    int64_t evals = 0, roche_elems = 0;
    // Signature of everything that fixes buffer sizes and launch shapes.
    std::vector<int64_t> shape_key;
    // datum_src[d] == datum_src[0] + d for every d: the data can be copied as one range
    bool datum_contiguous = false;
    bool any_iscale = false;  // some model fits per-component scale factors (needs fcomp scratch)
    int roche_split = 1;      // threads per Roche-eclipsed element in the phase scan
    int flux_chunks = 1;      // elements per flux work unit / kFluxChunk
    int flux_blocks_per_sm = 0;  // persistent flux blocks per SM; 0 = the occupancy limit

    // Empties the plan but keeps every buffer's capacity, so re-planning a
    // batch of the same size touches no fresh memory.
    void reset() {
        models.clear(); segs.clear(); bands.clear(); rings.clear(); eblocks.clear(); rblocks.clear();
        ablocks.clear(); units.clear(); datum_model.clear(); datum_sub0.clear(); datum_src.clear();
        model_ok.clear(); model_err.clear(); shape_key.clear();
        nelem = nsub = ndatum = npartial = evals = roche_elems = 0;
        datum_contiguous = false;
        any_iscale = false;
        roche_split = 1;
        flux_chunks = 1;
        flux_blocks_per_sm = 0;
    }
};

// Plans models[0..n); model i is evaluated on data[start[i] .. start[i]+count[i])
// (ranges may overlap, e.g. one shared data set).  Models that are physically
// invalid are marked failed (model_ok = 0) instead of throwing.
void plan_batch(const Model* const* models, int64_t n, const lcb_datum* data, const int64_t* start,
                const int64_t* count, int num_sms, Plan& out, const PlanTuning& tune = PlanTuning{});

// Host FP64 helpers also used by tests of the planner.
double host_xl1(double q);
double host_xl11(double q, double spin);
double host_xl12(double q, double spin);
void host_stream_spot(double q, double radius, double out[3]);

// Gas-stream end points on a GPU for many (q, radius) pairs at once: in[3 i ..] = (q,
// L1 distance, radius), out[3 i ..] = the position, status[i] = a stream:: code.
// Returns false where no GPU path is available.  The engine registers one; the
// planner calls it for a batch with more new pairs than the host's threads
// integrate quickly (more than four per thread), and memoises the results.
using StreamDeviceFn = bool (*)(const double* in, int n, double* out, int* status);
void set_stream_device(StreamDeviceFn fn);
// The memo's value for (q, radius) if present; stores a result in it.
bool spot_memo_get(double q, double radius, double out[3]);
void spot_memo_put(double q, double radius, const double out[3]);
int64_t host_numface(int nlat);

}  // namespace lcb
