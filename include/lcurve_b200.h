/*
 * lcurve_b200.h — C ABI of the B200 light-curve engine (liblcurve_b200.so).
 *
 * Drop-in boundary for the light-curve path of scope-ml/lcurve-rs: the flux
 * sum of every star/disc/edge/bright-spot element over times x exposure
 * sub-divisions, plus the grid generation and Roche eclipse ray-marching that
 * feed it.  Everything behind these entry points runs as sm_100a CUDA
 * kernels; there is no CPU fallback.  A call that cannot get a CUDA device
 * fails with LCB_ERR_NO_DEVICE.
 *
 * Conventions (mirroring the reference's lcuda_* FFI, crates/lcurve-cuda/
 * kernels/flux_kernel.cu:491-627 and crates/lcurve-cuda/src/error.rs:28-37):
 *   - every function returns an int status, 0 = LCB_OK; no exceptions or
 *     aborts cross the ABI;
 *   - all buffers passed in are caller-owned host memory unless the name says
 *     "device"; device memory is owned by the context;
 *   - a context serialises its own calls with an internal mutex, so one
 *     context may be shared by threads (calls then run one at a time), or
 *     each thread may own a context.
 */
#ifndef LCURVE_B200_H
#define LCURVE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define LCB_OK                 0
#define LCB_ERR_INVALID        1  /* bad argument (null pointer, bad size)           */
#define LCB_ERR_PARSE          2  /* model / data file syntax (model.rs:186-442)     */
#define LCB_ERR_IO             3  /* file cannot be read or written                  */
#define LCB_ERR_MODEL          4  /* physically invalid model (LcurveError/RocheError)*/
#define LCB_ERR_CUDA           5  /* CUDA runtime error                              */
#define LCB_ERR_UNKNOWN_PARAM  6  /* name is not a physical parameter (model.rs:459) */
#define LCB_ERR_NO_DEVICE      7  /* no usable CUDA device / kernel image            */
#define LCB_ERR_EMPTY          8  /* no data points                                  */
#define LCB_ERR_DEVICE_CHECK   9  /* a device-side iteration cap or check tripped    */

typedef struct lcb_ctx lcb_ctx;
typedef struct lcb_model lcb_model;
typedef struct lcb_batch lcb_batch;

/* One observation; same fields and meaning as Datum (crates/lcurve/src/
 * types.rs:207-220).  40 bytes of doubles + ndiv + padding = 48 bytes. */
typedef struct lcb_datum {
    double time;    /* mid-exposure time                    */
    double expose;  /* exposure length (time units)         */
    double flux;    /* observed flux                        */
    double ferr;    /* uncertainty                          */
    double weight;  /* weight factor (<= 0: ignored in chi2)*/
    int32_t ndiv;   /* exposure sub-divisions               */
    int32_t _pad;
} lcb_datum;

/* Scalar part of LcResult (crates/lcurve/src/orchestration.rs:9-28). */
typedef struct lcb_result {
    double wdwarf;   /* white dwarf contribution at phase 0.5     */
    double chisq;    /* weighted chi-squared                      */
    double wnok;     /* weighted number of points used            */
    double logg1;    /* flux-weighted log10 g of star 1 (cgs)     */
    double logg2;    /* flux-weighted log10 g of star 2 (cgs)     */
    double rv1;      /* volume-averaged radius of star 1          */
    double rv2;      /* volume-averaged radius of star 2          */
    double sfac[5];  /* scale factors [star1, disc, edge, spot, star2] */
} lcb_result;

/* ---- library / errors ---------------------------------------------------- */
const char* lcb_version(void);
/* Message of the last failing call on this host thread. */
const char* lcb_last_error(void);
/* Number of CUDA devices (reference: lcuda_device_count, flux_kernel.cu:557). */
int lcb_device_count(int* count);

/* ---- context: device, stream, device arena -------------------------------
 * Replaces CudaContext::new (crates/lcurve-cuda/src/context.rs:261) and
 * lcuda_init (flux_kernel.cu:497).  Work is issued on the context's own
 * stream unless lcb_ctx_set_stream gives another one (cudaStream_t). */
int  lcb_ctx_create(int device, lcb_ctx** out);
void lcb_ctx_destroy(lcb_ctx* ctx);
int  lcb_ctx_set_stream(lcb_ctx* ctx, void* cuda_stream);
const char* lcb_ctx_last_error(const lcb_ctx* ctx);

/* ---- models (crates/lcurve/src/model.rs) --------------------------------- */
/* Model::from_file (model.rs:186). */
int  lcb_model_load(const char* path, lcb_model** out);
/* Same parser over an in-memory text. */
int  lcb_model_parse(const char* text, lcb_model** out);
/* Model::clone. */
int  lcb_model_clone(const lcb_model* m, lcb_model** out);
void lcb_model_destroy(lcb_model* m);
/* Model::set_param_value (model.rs:459-493); LCB_ERR_UNKNOWN_PARAM if the
 * name is not a physical parameter. */
int  lcb_model_set_param(lcb_model* m, const char* name, double value);
/* Model::get_param_value (model.rs:495-532). */
int  lcb_model_get_param(const lcb_model* m, const char* name, double* value);
/* Full Pparam record (model.rs:7-13): value, range, dstep, vary, defined. */
int  lcb_model_get_pparam(const lcb_model* m, const char* name, double* value, double* range,
                          double* dstep, int* vary, int* defined);
int  lcb_model_set_pparam(lcb_model* m, const char* name, const double* value, const double* range,
                          const double* dstep, const int* vary);
/* Computational parameter (nlat1f, delta_phase, limb1, ...) by its .dat text. */
int  lcb_model_set_comp(lcb_model* m, const char* name, const char* value);
int  lcb_model_get_comp(const lcb_model* m, const char* name, char* buf, int buflen);
/* Name of the i-th physical parameter (declaration order, model.rs:66-137);
 * NULL when i is out of range. */
const char* lcb_param_name(int i);

/* ---- data files (crates/lcurve/src/types.rs:229-265) --------------------- */
int  lcb_read_data(const char* path, lcb_datum** out, int64_t* n);
void lcb_free_data(lcb_datum* data);

/* ---- light curve ----------------------------------------------------------
 * light_curve_comp(&Model, &Data, scale, rdata) (orchestration.rs:36-318).
 * calc_out receives n fluxes; res_out may be NULL. */
int lcb_light_curve(lcb_ctx* ctx, const lcb_model* model, const lcb_datum* data, int64_t n,
                    int scale, int rdata, double* calc_out, lcb_result* res_out);

/* ---- light curve without device allocation ----------------------------------
 * No counterpart in the reference: an addition for callers that cannot call
 * cudaMalloc (device memory already claimed by another framework's pool
 * allocator, plugin hosts that forbid allocation inside callbacks, loops that
 * cannot afford the synchronisation cudaMalloc/cudaFree may imply).
 * Same arguments, results and errors as lcb_light_curve, but every device
 * buffer lives in one fixed arena of LCB_NOALLOC_ARENA_BYTES, a file-scope
 * device array that each device loading this library holds until the process
 * exits.  Nothing is allocated on the device: a model and data set needing
 * more scratch than the arena is rejected with LCB_ERR_INVALID and a message
 * giving the bytes needed (a grid element takes about 160 B, a datum about
 * 80 B, each exposure sub-division about 40 B plus 8 B per 4,096 elements).
 * Every call looks up the arena's device address on the context's device and
 * waits for its own GPU work, so no call may be made while a CUDA stream
 * capture is in progress on the calling thread.  All calls on a device share
 * the arena: this library serialises them and waits for each call's GPU work
 * before returning, since calls whose GPU work overlapped would race. */
#define LCB_NOALLOC_ARENA_BYTES (64u * 1024u * 1024u)
int lcb_light_curve_noalloc(lcb_ctx* ctx, const lcb_model* model, const lcb_datum* data, int64_t n,
                            int scale, int rdata, double* calc_out, lcb_result* res_out);

/* ---- grid inspection --------------------------------------------------------
 * The elements the GPU builds for one model -- the grids of set_star_grid /
 * set_disc_grid / set_disc_edge / set_bright_spot_grid after continuum and
 * eclipses (grid.rs, brightness.rs; the reference inspects them in
 * crates/lcurve/examples/diag.rs).  which: 0 star1 fine, 1 star2 fine,
 * 2 star1 coarse, 3 star2 coarse, 4 disc, 5 rim, 6 bright spot.  Call with
 * NULL arrays to get *n; then posn/dirn hold 3n doubles, area/gravity/flux n
 * floats and ecl 8n doubles: four (ingress, egress) pairs, unused = (+inf, -inf). */
int lcb_model_grid(lcb_ctx* ctx, const lcb_model* model, int which, int64_t* n, double* posn, double* dirn,
                   float* area, float* gravity, float* flux, double* ecl);

/* ---- one model split into element slabs (no reference counterpart) --------
 * The reference builds a model's grids and eclipses serially per star
 * (crates/lcurve/src/grid.rs:227-320); for a model too large for one device's
 * time budget the element stage splits into slabs over devices:
 * lcb_model_elements computes elements [first, first + count) of the model's
 * element list (grids, continuum and eclipse intervals) into caller-owned
 * DEVICE arrays of count records each -- rec float4 {dirn, flux}, pos float4
 * {posn, 0}, p64 double4 {posn, area}, d64 double4 {dirn, gravity}, ecl 4 x
 * double2 (ingress, egress), unused (+inf, -inf) -- and sets *total to the
 * model's element count (rec_dev NULL: only *total).  After the slabs are
 * gathered into full arrays on a device (the order of lcb_model_elements),
 * lcb_light_curve_elements computes the light curve from them as
 * lcb_light_curve would, without recomputing any element.  A search that
 * reaches the eclipse-search bound fails the slab with LCB_ERR_DEVICE_CHECK. */
int lcb_model_elements(lcb_ctx* ctx, const lcb_model* model, int64_t first, int64_t count, void* rec_dev,
                       void* pos_dev, void* p64_dev, void* d64_dev, void* ecl_dev, int64_t* total);
int lcb_light_curve_elements(lcb_ctx* ctx, const lcb_model* model, const lcb_datum* data, int64_t n,
                             int scale, int rdata, const void* rec_dev, const void* pos_dev, const void* p64_dev,
                             const void* d64_dev, const void* ecl_dev, double* calc_out, lcb_result* res_out);

/* ---- batched chi-squared ---------------------------------------------------
 * chisq_batch(base, data, names, values, scale) (orchestration.rs:329-357)
 * and chisq_batch_gpu (crates/lcurve-cuda/src/batch.rs:73-80): values is an
 * (nsets x ndim) row-major array; each row is applied with set_param_value
 * (unknown names are ignored, as there); a model that fails gives NaN. */
int lcb_chisq_batch(lcb_ctx* ctx, const lcb_model* base, const lcb_datum* data, int64_t n,
                    const char* const* names, int ndim, const double* values, int64_t nsets,
                    int scale, double* chisq_out);

/* Ragged batch (no reference counterpart: the reference shares one Data and
 * one grid size per batch): model i is evaluated on data[offsets[i] ..
 * offsets[i+1]).  calc_out (same length as data) and res_out (nmodels) may be
 * NULL.  Each model is computed with rdata = true. */
int lcb_chisq_batch_ragged(lcb_ctx* ctx, const lcb_model* const* models, int64_t nmodels,
                           const lcb_datum* data, const int64_t* offsets, int scale,
                           double* chisq_out, double* calc_out, lcb_result* res_out);

/* ---- resident batch (repeated evaluation, e.g. MCMC) ----------------------
 * lcb_batch_create plans a ragged batch and uploads its data once;
 * lcb_batch_set_params changes physical parameters (names x values, row-major,
 * one row per model) without re-uploading data; lcb_batch_run evaluates on the
 * device (the launch sequence is captured once in a CUDA graph and replayed);
 * lcb_batch_results copies results back.  Changing a parameter that alters an
 * element count (disc/edge sizes) re-plans the batch transparently. */
int  lcb_batch_create(lcb_ctx* ctx, const lcb_model* const* models, int64_t nmodels,
                      const lcb_datum* data, const int64_t* offsets, lcb_batch** out);
void lcb_batch_destroy(lcb_batch* b);
int  lcb_batch_set_params(lcb_batch* b, const char* const* names, int ndim, const double* values);
int  lcb_batch_run(lcb_batch* b, int scale);
int  lcb_batch_results(lcb_batch* b, double* chisq_out, double* calc_out, lcb_result* res_out);
/* Work counts of the planned batch: [models, elements, sub-phases,
 * element-evals, flux work units, roche-eclipsed elements, Roche potential
 * evaluations and gradient evaluations of the eclipse search in the last run]. */
int  lcb_batch_stats(const lcb_batch* b, int64_t* out8);
/* Eclipse-search counters of the last run: [potential evaluations, gradient
 * evaluations, line-of-sight searches, miss-proof nodes (a potential and a
 * gradient evaluation each), successful miss proofs (one line of sight, or one
 * block of consecutive phase-scan steps proven together)].  The line-of-sight
 * searches are exactly the reference path's (eclipse.rs:123-197 calls). */
int  lcb_batch_search_counts(const lcb_batch* b, int64_t* out5);
/* Launch-shape choices of a resident batch, for an autotuner (no reference
 * counterpart; the reference GPU crate launches one fixed shape, 256-thread
 * blocks, crates/lcurve-cuda/kernels/flux_kernel.cu:81, 543-545): elements
 * per flux work unit in chunks of 256 (1..16), threads per Roche-eclipsed
 * element in the phase scan (1..16; only where the batch has such elements)
 * and persistent flux blocks per SM (>= 1, capped at the occupancy limit);
 * 0 keeps the planner's heuristic for that choice.  Re-plans the batch;
 * results are unchanged up to the FP32 summation order of the flux sum.
 * lcb_batch_get_tuning reports the three values in effect. */
int  lcb_batch_set_tuning(lcb_batch* b, int flux_chunks, int roche_split, int flux_blocks_per_sm);
int  lcb_batch_get_tuning(const lcb_batch* b, int* out3);
/* Same evaluation as lcb_batch_run but issued as direct launches with CUDA
 * events between the stages (events recorded inside a graph carry no timing),
 * for per-kernel device times. */
int  lcb_batch_profile(lcb_batch* b, int scale);
/* Device time (ms) of each stage of the last lcb_batch_profile, measured with
 * CUDA events on the launching stream: [phase, elements (grid + continuum +
 * analytic eclipses), roche (FP64 ray-march), aux (per-model sums), flux,
 * epilogue]. */
int  lcb_batch_stage_ms(const lcb_batch* b, double* out6);

/* ---- work estimate (no reference counterpart) -------------------------------
 * Host-only: plans one model on its data (no device work) and reports
 * [grid elements, elements eclipsed by a Roche-distorted star, exposure
 * sub-divisions, element-evaluations of the flux sum]; zeros for a model that
 * is physically invalid.  Callers that split one batch over several devices
 * (the reference's chisq_batch model loop, orchestration.rs:343-356) weigh
 * models with it. */
int lcb_model_work(const lcb_model* model, const lcb_datum* data, int64_t n, int64_t* out4);
/* Bright-spot positions: the gas stream from L1 integrated to each radius[i] for
 * mass ratio q[i] (replaces crates/roche/src/stream.rs:82-145 stradv as
 * crates/lcurve/src/grid.rs:494 calls it), out[3 i ..] = (x, y, z), on the host
 * (on_device = 0) or one GPU thread per pair on the context's device (1), the
 * same source compiled for both.  Planning uses the GPU path itself for a batch
 * with more new (q, radius) pairs than four per host thread.  Rows whose stream
 * fails are NaN and the call returns LCB_ERR_MODEL. */
int lcb_stream_points(lcb_ctx* ctx, const double* q, const double* radius, int64_t n, int on_device, double* out);

/* ---- failure-path hooks (no reference counterpart) ------------------------
 * The eclipse search bounds one line-of-sight search at 262,144 potential
 * evaluations (the reference's fblink, crates/roche/src/eclipse.rs:123-197,
 * has no bound); a model whose search reaches it fails: NaN in the chisq_batch
 * entry points (as the reference maps a failed model, orchestration.rs:
 * 350-354) and LCB_ERR_DEVICE_CHECK from lcb_light_curve.
 * lcb_ctx_set_search_cap lowers that bound for the context's later calls
 * (0 restores the default), so the failure path can be exercised.
 * lcb_wait_probe runs one block that waits on a barrier nothing completes,
 * with the same bounded wait the flux kernel's copy pipeline uses, limited to
 * limit_cycles SM cycles (<= 4e9); it returns LCB_ERR_DEVICE_CHECK when the
 * wait gives up, as it must, and leaves the context usable. */
int lcb_ctx_set_search_cap(lcb_ctx* ctx, int evals);
int lcb_wait_probe(lcb_ctx* ctx, int64_t limit_cycles, int64_t* waited_cycles);

/* ---- measurement utilities (no reference counterpart) --------------------
 * Bytes the last call on this context copied host->device / device->host. */
int lcb_ctx_transfer_bytes(const lcb_ctx* ctx, int64_t* h2d, int64_t* d2h);
/* FMA throughput of the context's device in TFLOP/s, measured with a CUDA
 * kernel of independent FMA chains: which = 0 FP32, 1 FP64.  These are the
 * roofline denominators of the FP32 flux kernel and the FP64 eclipse kernel. */
int lcb_measure_fma_peak(lcb_ctx* ctx, int which, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* LCURVE_B200_H */
