// mlp.cu -- training and inference kernels of the tuner's cost model: a
// fully connected FP32 network  in -> H -> H -> H -> 1  with ReLU, trained
// on (pipeline-plan features -> log kernel time) pairs with mean squared
// error and Adam.  The sizes are tiny (H = 128, batches of a few hundred
// configurations), so every kernel is a plain one-thread-per-output loop;
// what matters is that training runs on the GPU with these kernels and
// that their gradients match the FP64 CPU reference (oracle/mlp.py).
//
// Parameter layout (one flat float buffer):
//   W1[H][D] b1[H] W2[H][H] b2[H] W3[H][H] b3[H] W4[H] b4[1]
// Activation buffer (B rows): Z1 A1 Z2 A2 Z3 A3 (each B x H), out[B].
#include <cuda_runtime.h>
#include <math.h>

namespace {

__global__ void linear_fwd(const float* __restrict__ X, int K,
                           const float* __restrict__ W,
                           const float* __restrict__ b, int N, int B,
                           float* __restrict__ Z, float* __restrict__ A) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B * N) return;
  int r = i / N, n = i % N;
  const float* x = X + (size_t)r * K;
  const float* w = W + (size_t)n * K;
  float s = b[n];
  for (int k = 0; k < K; ++k) s = fmaf(x[k], w[k], s);
  if (Z) Z[i] = s;
  if (A) A[i] = s > 0.f ? s : 0.f;
}

// dL/dout for L = mean((out - y)^2); also the loss (atomically summed)
__global__ void mse_grad(const float* __restrict__ out,
                         const float* __restrict__ y, int B,
                         float* __restrict__ dout, float* __restrict__ loss) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B) return;
  float d = out[i] - y[i];
  dout[i] = 2.f * d / (float)B;
  if (loss) atomicAdd(loss, d * d / (float)B);
}

// dW[n][k] = sum_r dZ[r][n] * X[r][k];  db[n] = sum_r dZ[r][n]
__global__ void linear_bwd_w(const float* __restrict__ dZ, int N,
                             const float* __restrict__ X, int K, int B,
                             float* __restrict__ dW, float* __restrict__ db) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * (K + 1)) return;
  int n = i / (K + 1), k = i % (K + 1);
  float s = 0.f;
  if (k < K) {
    for (int r = 0; r < B; ++r) s = fmaf(dZ[(size_t)r * N + n],
                                         X[(size_t)r * K + k], s);
    dW[(size_t)n * K + k] = s;
  } else {
    for (int r = 0; r < B; ++r) s += dZ[(size_t)r * N + n];
    db[n] = s;
  }
}

// dA[r][k] = sum_n dZ[r][n] * W[n][k], then through the ReLU of layer Zp
__global__ void linear_bwd_x(const float* __restrict__ dZ, int N,
                             const float* __restrict__ W, int K, int B,
                             const float* __restrict__ Zprev,
                             float* __restrict__ dZprev) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B * K) return;
  int r = i / K, k = i % K;
  float s = 0.f;
  for (int n = 0; n < N; ++n) s = fmaf(dZ[(size_t)r * N + n],
                                       W[(size_t)n * K + k], s);
  dZprev[i] = Zprev[i] > 0.f ? s : 0.f;
}

__global__ void adam(float* __restrict__ p, const float* __restrict__ g,
                     float* __restrict__ m, float* __restrict__ v, int n,
                     float lr, float b1, float b2, float eps, float c1,
                     float c2, float wd) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = g[i] + wd * p[i];
  float mi = b1 * m[i] + (1.f - b1) * gi;
  float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

inline int nb(long n) { return (int)((n + 255) / 256); }

struct Layout {
  size_t W1, b1, W2, b2, W3, b3, W4, b4, total;
  Layout(int D, int H) {
    W1 = 0; b1 = W1 + (size_t)H * D; W2 = b1 + H; b2 = W2 + (size_t)H * H;
    W3 = b2 + H; b3 = W3 + (size_t)H * H; W4 = b3 + H; b4 = W4 + H;
    total = b4 + 1;
  }
};

void forward(const float* P, int D, int H, const float* X, int B, float* acts,
             cudaStream_t s) {
  Layout L(D, H);
  size_t BH = (size_t)B * H;
  float *Z1 = acts, *A1 = Z1 + BH, *Z2 = A1 + BH, *A2 = Z2 + BH,
        *Z3 = A2 + BH, *A3 = Z3 + BH, *out = A3 + BH;
  linear_fwd<<<nb(BH), 256, 0, s>>>(X, D, P + L.W1, P + L.b1, H, B, Z1, A1);
  linear_fwd<<<nb(BH), 256, 0, s>>>(A1, H, P + L.W2, P + L.b2, H, B, Z2, A2);
  linear_fwd<<<nb(BH), 256, 0, s>>>(A2, H, P + L.W3, P + L.b3, H, B, Z3, A3);
  linear_fwd<<<nb(B), 256, 0, s>>>(A3, H, P + L.W4, P + L.b4, 1, B, out,
                                   nullptr);
}

}  // namespace

extern "C" {

// number of floats in the parameter buffer
long pm_mlp_param_count(int D, int H) { return (long)Layout(D, H).total; }

// floats needed for the activation buffer of B rows (forward) and for the
// gradient work buffer (backward)
long pm_mlp_act_count(int B, int H) { return (long)B * (6L * H + 1); }

// Inference: out[B] <- net(X[B][D]); acts is a work buffer.
int pm_mlp_forward(const float* params, int D, int H, const float* X, int B,
                   float* acts, float* out, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  forward(params, D, H, X, B, acts, s);
  cudaMemcpyAsync(out, acts + (size_t)B * 6 * H, sizeof(float) * B,
                  cudaMemcpyDeviceToDevice, s);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Gradients of the mean squared error over the batch into grads (same
// layout as params); loss (one float, zeroed here) receives the loss.
int pm_mlp_backward(const float* params, int D, int H, const float* X,
                    const float* y, int B, float* acts, float* work,
                    float* grads, float* loss, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  Layout L(D, H);
  forward(params, D, H, X, B, acts, s);
  size_t BH = (size_t)B * H;
  float *Z1 = acts, *A1 = Z1 + BH, *Z2 = A1 + BH, *A2 = Z2 + BH,
        *Z3 = A2 + BH, *A3 = Z3 + BH, *out = A3 + BH;
  float *dout = work, *dZ3 = dout + B, *dZ2 = dZ3 + BH, *dZ1 = dZ2 + BH;
  cudaMemsetAsync(loss, 0, sizeof(float), s);
  mse_grad<<<nb(B), 256, 0, s>>>(out, y, B, dout, loss);
  // output layer
  linear_bwd_w<<<nb(1L * (H + 1)), 256, 0, s>>>(dout, 1, A3, H, B,
                                                 grads + L.W4, grads + L.b4);
  linear_bwd_x<<<nb(BH), 256, 0, s>>>(dout, 1, params + L.W4, H, B, Z3, dZ3);
  // hidden layer 3
  linear_bwd_w<<<nb((long)H * (H + 1)), 256, 0, s>>>(dZ3, H, A2, H, B,
                                                      grads + L.W3,
                                                      grads + L.b3);
  linear_bwd_x<<<nb(BH), 256, 0, s>>>(dZ3, H, params + L.W3, H, B, Z2, dZ2);
  // hidden layer 2
  linear_bwd_w<<<nb((long)H * (H + 1)), 256, 0, s>>>(dZ2, H, A1, H, B,
                                                      grads + L.W2,
                                                      grads + L.b2);
  linear_bwd_x<<<nb(BH), 256, 0, s>>>(dZ2, H, params + L.W2, H, B, Z1, dZ1);
  // input layer
  linear_bwd_w<<<nb((long)H * (D + 1)), 256, 0, s>>>(dZ1, H, X, D, B,
                                                      grads + L.W1,
                                                      grads + L.b1);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

long pm_mlp_work_count(int B, int H) { return (long)B * (3L * H + 1); }

// One Adam step on all parameters (t is the 1-based step number).
int pm_mlp_adam(float* params, const float* grads, float* m, float* v, int D,
                int H, int t, float lr, float weight_decay, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  long n = pm_mlp_param_count(D, H);
  const float b1 = 0.9f, b2 = 0.999f;
  float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
  adam<<<nb(n), 256, 0, s>>>(params, grads, m, v, (int)n, lr, b1, b2, 1e-8f,
                             c1, c2, weight_decay);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Inference that allocates nothing: pm_mlp_forward_static.
//
// pm_mlp_forward takes its activation buffer from the caller.  Some callers
// cannot allocate device memory at the point where they rank configurations:
// a host runtime that hands out a fixed device budget reserved at start-up,
// or a tuning loop that must not add a cudaMalloc (which can synchronize the
// whole device) between the kernels it is timing.  This entry keeps the
// activations in a fixed array of this module instead.  It runs the same
// kernels as pm_mlp_forward, in the same order.
//
// Limit: B * (6 * H + 1) floats of activations, at most
// PM_MLP_STATIC_FLOATS = 196,864 floats (787,456 bytes; 256 rows at H = 128).
// A larger request returns 1 and launches nothing.
// Set-up: the first call on each device looks up the array's device address
// with that device current; make that first call before any stream capture.
// Initial contents: nothing in the array needs to start at zero; every float
// the kernels read was written earlier in the same call.
// Concurrency: all calls on one device share the array, so two calls in
// flight at once (on different streams, or from different host threads
// without ordering) race on it; issue them on one stream.
// Device reset: the address is looked up once per device and kept; a
// cudaDeviceReset unloads this module's device code, after which that
// address is stale, so a process that resets a device must not call this
// entry on that device again.
#include <mutex>

#define PM_MLP_STATIC_FLOATS 196864
#define PM_MLP_STATIC_DEVICES 64

namespace {

__device__ __align__(256) float pm_mlp_static_acts[PM_MLP_STATIC_FLOATS];

float* pm_mlp_static_ptr[PM_MLP_STATIC_DEVICES];
std::mutex pm_mlp_static_mu;

// device address of the array on the current device (looked up once)
float* static_acts(int dev) {
  std::lock_guard<std::mutex> lk(pm_mlp_static_mu);
  if (!pm_mlp_static_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, pm_mlp_static_acts) != cudaSuccess)
      return nullptr;
    pm_mlp_static_ptr[dev] = static_cast<float*>(p);
  }
  return pm_mlp_static_ptr[dev];
}

}  // namespace

extern "C" int pm_mlp_forward_static(const float* params, int D, int H,
                                     const float* X, int B, float* out,
                                     void* stream) {
  if (D <= 0 || H <= 0 || B < 0) return 1;
  if ((long long)B * (6LL * H + 1) > PM_MLP_STATIC_FLOATS) return 1;
  if (B == 0) return 0;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 ||
      dev >= PM_MLP_STATIC_DEVICES)
    return 2;
  float* acts = static_acts(dev);
  if (!acts) return 2;
  cudaStream_t s = (cudaStream_t)stream;
  forward(params, D, H, X, B, acts, s);
  if (cudaMemcpyAsync(out, acts + (size_t)B * 6 * H, sizeof(float) * B,
                      cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return 2;
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
