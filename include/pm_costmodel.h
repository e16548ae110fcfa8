/* pm_costmodel.h -- C ABI of the tuner's learned cost model
 * (polymage_b200/csrc/mlp.cu, built into libpm_mlp_<hash>.so).
 *
 * The network is a fully connected FP32 MLP  D -> H -> H -> H -> 1  with
 * ReLU, in one flat parameter buffer laid out as
 *   W1[H][D] b1[H] W2[H][H] b2[H] W3[H][H] b3[H] W4[H] b4[1].
 * All pointers are device pointers; every call is asynchronous on `stream`
 * (a cudaStream_t) and returns 0 (ok) or 2 (a CUDA call failed).
 *
 * The reference has no learned cost model (its tuner times every
 * configuration: sandbox/tuner.py:100-384 generates every variant,
 * sandbox/tuner.py:387-600 times each one), so none of these has a
 * counterpart there.
 */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

/* floats in the parameter buffer */
long pm_mlp_param_count(int D, int H);
/* floats of the activation buffer for B rows */
long pm_mlp_act_count(int B, int H);
/* floats of the backward work buffer for B rows */
long pm_mlp_work_count(int B, int H);

/* out[B] <- net(X[B][D]); acts: pm_mlp_act_count(B, H) floats */
int pm_mlp_forward(const float* params, int D, int H, const float* X, int B,
                   float* acts, float* out, void* stream);

/* grads (parameter layout) <- d/dparams of mean((net(X) - y)^2); loss (one
 * float) receives the loss; work: pm_mlp_work_count(B, H) floats */
int pm_mlp_backward(const float* params, int D, int H, const float* X,
                    const float* y, int B, float* acts, float* work,
                    float* grads, float* loss, void* stream);

/* As pm_mlp_forward, with the activations in a fixed array inside the
 * library instead of a caller buffer: allocates nothing.  No counterpart in
 * the reference.  For callers that cannot allocate device memory where they
 * rank configurations (a fixed device budget, or no cudaMalloc between
 * timed kernels).  Limit: B * (6 * H + 1) <= 196864 floats (256 rows at
 * H = 128); larger requests return 1 and launch nothing.  The first call on
 * each device looks up the array's address (make it before any stream
 * capture).  Nothing needs to start at zero.  Calls on one device share the
 * array: two in flight at once race, so issue them on one stream.  The
 * address looked up on a device does not survive a cudaDeviceReset of that
 * device: do not call this entry on a device after resetting it. */
int pm_mlp_forward_static(const float* params, int D, int H, const float* X,
                          int B, float* out, void* stream);

/* one Adam step (t: 1-based step number) */
int pm_mlp_adam(float* params, const float* grads, float* m, float* v, int D,
                int H, int t, float lr, float weight_decay, void* stream);

#ifdef __cplusplus
}
#endif
