/*
 * lcurve_b200_surrogate.h — C ABI of the light-curve surrogate (liblcurve_b200.so).
 *
 * A small MLP, n_in -> width x n_hidden (GELU) -> n_out, that maps normalised
 * physical parameters to a light curve on a fixed phase grid, trained and
 * evaluated by hand-written sm_100a BF16 tensor-core kernels (tcgen05 MMA
 * with TMEM accumulators, TMA-staged operands, FP32 accumulation) with FP32
 * master weights and Adam.  It is the cheap first stage of delayed-acceptance
 * MCMC; the light-curve engine (lcurve_b200.h) remains the second stage.
 *
 * The reference has no surrogate: these entry points have no counterpart in
 * it.  The MCMC layer they serve replaces the reference's emcee-based fitter
 * (python/lcurve_rs/fitting.py), whose likelihood calls chisq_batch
 * (crates/lcurve/src/orchestration.rs:329-357).
 *
 * Conventions: status codes as in lcurve_b200.h (0 = LCB_OK); pointers named
 * *_dev are device memory owned by the caller, work is issued on the
 * network's stream (lcb_mlp_set_stream) and is asynchronous unless a
 * function says it synchronises.  Parameters are exchanged in the layout
 * [W0 (width x n_in, row-major), b0, W1 (width x width), b1, ...,
 *  W_last (n_out x width), b_last].
 */
#ifndef LCURVE_B200_SURROGATE_H
#define LCURVE_B200_SURROGATE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lcb_mlp lcb_mlp;

/* Message of the last failing surrogate call on this host thread. */
const char* lcb_mlp_last_error(void);

/* Network with He-uniform initial weights (seeded) and device buffers for
 * batches of up to max_batch rows; width and n_out multiples of 8. */
int  lcb_mlp_create(int device, int n_in, int width, int n_hidden, int n_out, int64_t max_batch, uint64_t seed,
                    lcb_mlp** out);
void lcb_mlp_destroy(lcb_mlp* net);
int  lcb_mlp_set_stream(lcb_mlp* net, void* cuda_stream);
int  lcb_mlp_num_params(const lcb_mlp* net, int64_t* n);
/* FP32 parameters / last gradients to and from host memory (synchronise). */
int  lcb_mlp_get_params(lcb_mlp* net, float* host, int64_t n);
int  lcb_mlp_set_params(lcb_mlp* net, const float* host, int64_t n);
int  lcb_mlp_get_grads(lcb_mlp* net, float* host, int64_t n);
/* Training state for checkpoint / resume: FP32 master parameters and the two
 * Adam moments, each state_size floats in the network's own (padded) device
 * layout, concatenated (3 x state_size), plus the Adam step count.  Valid for
 * a network of the same shape; set_state also refreshes the BF16 weights, so
 * training resumes exactly where get_state left it (synchronise). */
int  lcb_mlp_state_size(const lcb_mlp* net, int64_t* n);
int  lcb_mlp_get_state(lcb_mlp* net, float* host, int64_t n, int64_t* steps);
int  lcb_mlp_set_state(lcb_mlp* net, const float* host, int64_t n, int64_t steps);

/* y_dev[batch x n_out] = net(x_dev[batch x n_in]) (fp32 in and out). */
int  lcb_mlp_forward(lcb_mlp* net, const float* x_dev, int64_t batch, float* y_dev);
/* Gradients of the mean-squared error against target_dev[batch x n_out]
 * (batch a multiple of 8); the loss is added to the network's accumulator. */
int  lcb_mlp_backward(lcb_mlp* net, const float* x_dev, const float* target_dev, int64_t batch);
/* lcb_mlp_backward followed by one Adam step (decoupled weight decay). */
int  lcb_mlp_train_step(lcb_mlp* net, const float* x_dev, const float* target_dev, int64_t batch, float lr,
                        float beta1, float beta2, float eps, float weight_decay);
/* Data-parallel training, one network per GPU: the device buffer of n FP32
 * gradients that lcb_mlp_backward writes (the lcb_mlp_get_params layout), to be
 * reduced in place across ranks (e.g. an NCCL all-reduce averaging it, ordered
 * on the network's stream), then lcb_mlp_adam_step applies it.  backward +
 * adam_step with no reduction in between is exactly lcb_mlp_train_step. */
int  lcb_mlp_grads_device(lcb_mlp* net, float** grads_dev, int64_t* n);
int  lcb_mlp_adam_step(lcb_mlp* net, float lr, float beta1, float beta2, float eps, float weight_decay);
/* Accumulated loss since the last call, then reset (synchronises). */
int  lcb_mlp_take_loss(lcb_mlp* net, double* loss_sum);
/* Waits for the network's stream; LCB_ERR_DEVICE_CHECK if a device wait timed out. */
int  lcb_mlp_sync(lcb_mlp* net);

/* The tensor-core GEMM itself: out[M x N] = A[M x K] . B[N x K]^T with bf16
 * row-major operands (16-byte aligned, N and K multiples of 8) and epilogue
 * mode 0: fp32 out; 1: z = acc + bias, out = bf16(gelu(z)), out2 = fp32 z;
 * 2: fp32 out = acc + bias; 3: out = bf16(acc * gelu'(aux)) with aux fp32
 * M x N.  err_dev (device int) is set to 1 if a bounded wait timed out. */
int  lcb_mlp_gemm(int mode, int64_t M, int64_t N, int64_t K, const void* a_dev, const void* b_dev,
                  const float* bias_dev, const float* aux_dev, void* out_dev, void* out2_dev, int* err_dev,
                  void* cuda_stream);

/* chisq_dev[r] = sum_j ((flux_j - s f_rj) / ferr_j)^2 with
 * f_rj = exp(pred_dev[r][j] * sd_j + mean_j) and s the least-squares scale
 * factor when scale != 0 (re_scale, orchestration.rs:361-401), else 1. */
int  lcb_logflux_chisq(int64_t rows, int n, const float* pred_dev, const float* mean_dev, const float* sd_dev,
                       const double* flux_dev, const double* ferr_dev, int scale, double* chisq_dev, void* cuda_stream);

/* `steps` Metropolis moves of n walkers against m fixed complementary
 * walkers under the surrogate posterior alone, on the network's stream with
 * no host round trip (the sequence is captured once as a CUDA graph and
 * replayed): the first stage of delayed acceptance.  move 0: the stretch move
 * (Goodman & Weare, scale a); move 1: an independence proposal from the
 * Gaussian KDE of the complementary walkers, kernel covariance
 * kde_chol kde_chol^T with inverse kde_prec (host d x d row-major arrays).
 * y_dev (n x d) and ls_dev (n: log probability -chisq/2, finite) are updated
 * in place; rnd_dev holds steps x n x R numbers, R = 3 (stretch) or 3 + d
 * (KDE): a uniform for z (stretch) or the KDE component (KDE), a uniform for
 * the partner (stretch), ln of a uniform for acceptance, then d standard
 * normals (KDE).  Proposals outside [lo, hi] (host arrays of d) are rejected;
 * the network input of dimension k is fadd[k] + fmul[k] * (recip[k] ? 1/x : x);
 * chi-squared as lcb_logflux_chisq against flux_dev / ferr_dev (n_out points). */
int  lcb_surrogate_subchain(lcb_mlp* net, int64_t n, int64_t m, int d, double* y_dev, double* ls_dev,
                            const double* comp_dev, const double* rnd_dev, int steps, double a, const double* lo,
                            const double* hi, const int* recip, const float* fmul, const float* fadd,
                            const float* mean_dev, const float* sd_dev, const double* flux_dev,
                            const double* ferr_dev, int scale, int move, const double* kde_chol,
                            const double* kde_prec);
/* The same sub-chain with y, ls, comp and rnd in host memory (no reference
 * counterpart): the library stages them through one page-locked buffer of the
 * network (one host-to-device copy in, one device-to-host copy of y and ls
 * out, grown on first use outside any capture) and returns with y and ls
 * updated.  Calls on one network must not overlap. */
int  lcb_surrogate_subchain_host(lcb_mlp* net, int64_t n, int64_t m, int d, double* y, double* ls,
                                 const double* comp, const double* rnd, int steps, double a, const double* lo,
                                 const double* hi, const int* recip, const float* fmul, const float* fadd,
                                 const float* mean_dev, const float* sd_dev, const double* flux_dev,
                                 const double* ferr_dev, int scale, int move, const double* kde_chol,
                                 const double* kde_prec);

#ifdef __cplusplus
}
#endif

#endif /* LCURVE_B200_SURROGATE_H */
