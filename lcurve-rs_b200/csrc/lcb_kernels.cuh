// lcb_kernels.cuh — launch interfaces of the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>

#include "../../include/lcurve_b200.h"
#include "lcb_internal.h"

namespace lcb {

// Sizes of the batch's arrays, for the index checks of the LCURVE_DEBUG_BOUNDS build.
struct Sizes {
    int64_t nelem, nsub, npartial, ndatum, nbands, nrings;
};

struct ElemArgs {
    const ModelDev* models;
    const SegDesc* segs;
    const ElemBlock* blocks;   // k_elements: every element
    const ElemBlock* rblocks;  // k_roche: elements eclipsed by a Roche-distorted star (by = 1 or 2)
    const ElemBlock* ablocks;  // k_aux: star-grid elements
    const Band* bands;
    const Ring* rings;
    float4* el_rec;      // dirn.xyz, flux
    float4* el_pos;      // posn.xyz, 0
    double4* el_p64;     // posn.xyz, area (FP64)
    double4* el_d64;     // dirn.xyz, gravity (FP64)
    double2* el_ecl;     // kMaxEcl (ingress, egress) slots, slot-major: slot k of element e at k * sz.nelem + e
    unsigned* ecl_grp;   // per kEclGroup elements: bit k set if any of them uses slot k (zeroed before k_elements)
    double* aux;         // kNumAux per model
    int* status;         // per model
    int64_t nblocks, nrblocks, nablocks;
    unsigned long long* counters;  // [pot evals, dpot evals, fblink calls, bound nodes, proven misses] or null
    int roche_split;     // threads per Roche-eclipsed element in the phase scan (1: one kernel)
    int* firsthit;       // split scan: first hit per Roche thread (nrblocks x kRocheBlock), starts at 0x7f7f7f7f
    int fblink_cap;      // potential evaluations allowed in one line-of-sight search (kFblinkEvalCap)
    Sizes sz;
};

struct PhaseArgs {
    const ModelDev* models;
    const lcb_datum* data;
    const int32_t* dmodel;
    const int64_t* dsub0;
    int64_t ndatum;
    float4* sp_e;
    double* sp_phi;
    int8_t* sp_type;
    double* sp_w;
    double* d_slfac;
};

struct FluxArgs {
    const ModelDev* models;
    const FluxUnit* units;
    int64_t nunits;
    int* counter;
    const float4* el_rec;
    const float4* el_pos;
    const double2* el_ecl;     // slot-major, as ElemArgs::el_ecl
    const unsigned* ecl_grp;   // slots used per kEclGroup elements
    const float4* sp_e;
    const double* sp_phi;
    const int8_t* sp_type;
    double* partial;
    int* status;         // per model
    Sizes sz;
};

struct EpiArgs {
    const ModelDev* models;
    const lcb_datum* data;
    const int64_t* dsub0;
    const double* sp_phi;
    const double* sp_w;
    const double* d_slfac;
    const double* partial;
    const double* aux;
    const int* status;
    int scale, rdata;
    double* calc;        // per datum
    double* results;     // 12 per model
    double* fcomp;       // iscale: 5 component fluxes per datum
    double* svda;        // iscale: 5 per datum, the weighted design matrix of the scale fit
    int64_t nmodels;
    Sizes sz;
    int* bad;            // LCURVE_DEBUG_BOUNDS: per-model status words the epilogue may set
};

size_t flux_smem_bytes();
cudaError_t launch_phase(const PhaseArgs& a, cudaStream_t s);
cudaError_t launch_elements(const ElemArgs& a, cudaStream_t s);
cudaError_t launch_roche(const ElemArgs& a, cudaStream_t s);
cudaError_t launch_aux(const ElemArgs& a, cudaStream_t s);
int roche_block_size();
cudaError_t launch_flux(const FluxArgs& a, int grid, cudaStream_t s);
cudaError_t launch_epilogue(const EpiArgs& a, cudaStream_t s);
int flux_blocks_per_sm();
cudaError_t measure_fma_peak(int fp64, int num_sms, cudaStream_t s, double* tflops);
// Eclipse slots of elements [first, first + count) between the engine's slot-major
// array (stride nelem) and element-major records of kMaxEcl pairs (the exchange format of
// lcb_model_elements); the import also records the slots used in ecl_grp, which must be
// zeroed first.
cudaError_t launch_ecl_export(const double2* ecl, int64_t nelem, int64_t first, int64_t count, double2* out,
                              cudaStream_t s);
cudaError_t launch_ecl_import(const double2* in, int64_t nelem, double2* ecl, unsigned* ecl_grp, cudaStream_t s);
// Gas-stream end points of n (q, L1 distance, radius) triples, one thread each (k_stream).
cudaError_t launch_stream(const double* in, int n, double* out, int* status, cudaStream_t s);
// One block waiting on an mbarrier that nothing completes, bounded by `limit` cycles.
cudaError_t launch_wait_probe(long long limit, int* status, long long* waited, cudaStream_t s);

}  // namespace lcb
