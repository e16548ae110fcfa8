// Integer-ALU throughput of the GPU, the denominator of the integer
// roofline the camera pipe is held against (its stages are int16/int32
// arithmetic and table gathers, not DRAM traffic).
//
// pm_int_peak_imad: every thread runs `iters` rounds of 8 independent
// 32-bit multiply-add chains (x = x * a + b); pm_int_peak_alu: 8
// independent chains of an add and an xor (x = (x + a) ^ b), the simple
// integer ALU operations index arithmetic consists of.  The chains are
// independent so that issue, not latency, bounds them; the results are
// folded into `out` so that nothing is dead code.  Host side:
// polymage_b200/apps/measure.py (int_peak), which times them with CUDA
// events and counts 8 (IMAD) or 16 (add, xor) integer instructions per
// round and thread.

extern "C" __global__ void __launch_bounds__(256)
pm_int_peak_imad(int* out, int iters, int a, int b) {
  int x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
  int x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
    x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
    x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] =
      x0 ^ x1 ^ x2 ^ x3 ^ x4 ^ x5 ^ x6 ^ x7;
}

extern "C" __global__ void __launch_bounds__(256)
pm_int_peak_alu(int* out, int iters, int a, int b) {
  int x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
  int x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
    x0 = (x0 + a) ^ b; x1 = (x1 + a) ^ b; x2 = (x2 + a) ^ b;
    x3 = (x3 + a) ^ b; x4 = (x4 + a) ^ b; x5 = (x5 + a) ^ b;
    x6 = (x6 + a) ^ b; x7 = (x7 + a) ^ b;
    a += 3; b ^= a;
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] =
      x0 ^ x1 ^ x2 ^ x3 ^ x4 ^ x5 ^ x6 ^ x7;
}

// Host launcher: which = 0 (IMAD chains) or 1 (add/xor chains); `out`
// holds blocks * 256 ints of device memory.  Returns 0, or 2 when the
// launch failed.
extern "C" int pm_int_peak_run(int which, int blocks, int iters, void* out,
                               void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (which == 0)
    pm_int_peak_imad<<<blocks, 256, 0, s>>>((int*)out, iters, 3, 7);
  else
    pm_int_peak_alu<<<blocks, 256, 0, s>>>((int*)out, iters, 3, 7);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
