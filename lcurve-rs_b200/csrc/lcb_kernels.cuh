// lcb_kernels.cuh — launch interfaces of the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>

#include "../../include/lcurve_b200.h"
#include "lcb_internal.h"

namespace lcb {

struct ElemArgs {
    const ModelDev* models;
    const SegDesc* segs;
    const ElemBlock* blocks;
    const Band* bands;
    const Ring* rings;
    float4* el_rec;      // dirn.xyz, flux
    float4* el_pos;      // posn.xyz, 0
    double2* el_ecl;     // 4 (ingress, egress) pairs per element
    double* aux;         // kNumAux per model
    int* status;         // per model
    int64_t nblocks;
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
    const double2* el_ecl;
    const float4* sp_e;
    const double* sp_phi;
    const int8_t* sp_type;
    double* partial;
    int* status;         // per model
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
    int64_t nmodels;
};

size_t flux_smem_bytes();
cudaError_t launch_phase(const PhaseArgs& a, cudaStream_t s);
cudaError_t launch_elements(const ElemArgs& a, cudaStream_t s);
cudaError_t launch_flux(const FluxArgs& a, int grid, cudaStream_t s);
cudaError_t launch_epilogue(const EpiArgs& a, cudaStream_t s);
int flux_blocks_per_sm();

}  // namespace lcb
