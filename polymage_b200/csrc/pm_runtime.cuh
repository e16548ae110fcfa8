// pm_runtime.cuh -- device and host support code included by every pipeline
// translation unit that the polymage_b200 code generator emits.
//
// Device side: mbarrier and TMA (cp.async.bulk.tensor, no multicast)
// wrappers for sm_100a, bounded waits that record a timeout in the module's
// error word instead of spinning forever, small integer helpers and atomics
// for reductions.
// Host side: tensor-map encoding through the driver entry point (no link
// against libcuda), a per-device workspace arena reused across calls, and
// status codes shared by all generated entry points.
#pragma once

#include <cuda_runtime.h>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <math.h>
#include <mutex>

#define PM_OK 0
#define PM_ERR_PARAMS 1       // parameter values outside the spec's bounds
#define PM_ERR_CUDA 2         // a CUDA call failed
#define PM_ERR_KERNEL 3       // a kernel reported an error (timeout, overflow)
#define PM_ERR_UNSUPPORTED 4  // request outside what this build supports

// bits of the device error word
#define PM_KERR_TMA_TIMEOUT 1u
#define PM_KERR_REGION 2u
#define PM_KERR_QUEUE 4u
#define PM_KERR_GRID_TIMEOUT 8u

#ifndef PM_WAIT_LIMIT
#define PM_WAIT_LIMIT (1 << 24)
#endif
// polls of a grid barrier (each after a ~128 ns sleep) before it gives up:
// well above the longest kernel that can hold SMs the barrier's CTAs wait for
#ifndef PM_GRID_WAIT_LIMIT
#define PM_GRID_WAIT_LIMIT (1 << 21)
#endif

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int pm_imin(int a, int b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int pm_imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ int pm_clampi(int v, int lo, int hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}
__host__ __device__ __forceinline__ int pm_floordiv(int a, int b) {
  int q = a / b;
  return (q * b != a && ((a < 0) != (b < 0))) ? q - 1 : q;
}

// |v| with the argument's own precision (what C++ std::abs resolves to)
__host__ __device__ __forceinline__ int pm_abs(int v) { return v < 0 ? -v : v; }
__host__ __device__ __forceinline__ long long pm_abs(long long v) { return v < 0 ? -v : v; }
__host__ __device__ __forceinline__ unsigned pm_abs(unsigned v) { return v; }
__host__ __device__ __forceinline__ unsigned long long pm_abs(unsigned long long v) { return v; }
__host__ __device__ __forceinline__ float pm_abs(float v) { return fabsf(v); }
__host__ __device__ __forceinline__ double pm_abs(double v) { return fabs(v); }

__device__ __forceinline__ uint32_t pm_smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void pm_mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(pm_smem_addr(bar)),
               "r"(count)
               : "memory");
}

// make the initialized barrier visible to the async (TMA) proxy
__device__ __forceinline__ void pm_fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// order this thread's generic-proxy shared-memory accesses before later
// async-proxy (TMA) writes to the same bytes
__device__ __forceinline__ void pm_fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// An mbarrier's bytes must be invalidated before they are used for
// anything else (another barrier, staged data of another group).
__device__ __forceinline__ void pm_mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(pm_smem_addr(bar))
               : "memory");
}

// Global loads of a group's kernel body.  A standalone launch reads through
// the read-only (non-coherent) path: nothing it reads is written while it
// runs.  A body inside a chain kernel (several groups, one launch, grid
// barriers between dependent groups) reads data that other CTAs of the same
// launch wrote before the last barrier, so it bypasses L1 (ld.global.cg).
template <bool CH, typename T>
__device__ __forceinline__ T pm_ld(const T* p) {
  if constexpr (CH) return __ldcg(p);
  else return __ldg(p);
}

// Between two phases of a chain kernel: every generic-proxy access of this
// thread (global stores read by later TMA loads, shared memory that a later
// group's TMA overwrites) is ordered before later async-proxy accesses.
__device__ __forceinline__ void pm_fence_proxy_async_all() {
  asm volatile("fence.proxy.async;" ::: "memory");
}

__device__ __forceinline__ unsigned pm_ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p)
               : "memory");
  return v;
}

// Grid-wide barrier of a chain kernel: every CTA arrives on the launch's
// counter (zeroed before the launch) and waits until `target` arrivals
// (gridDim.x times the barrier's ordinal) are counted.  The wait is bounded:
// when it runs out the error word records PM_KERR_GRID_TIMEOUT and every
// thread gets false, so the kernel returns instead of spinning forever.
// The CTAs of a chain launch all fit on the GPU at once (the grid is capped
// by the occupancy calculator), so the wait ends once any concurrently
// running kernel that holds SMs has finished.
__device__ __forceinline__ bool pm_grid_sync(unsigned* ctr, unsigned target,
                                             unsigned* err) {
  pm_fence_proxy_async_all();
  __syncthreads();
  int ok = 1;
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(ctr, 1u);
    int it = 0;
    while (pm_ld_acquire(ctr) < target) {
      if (++it > PM_GRID_WAIT_LIMIT) {
        atomicOr(err, PM_KERR_GRID_TIMEOUT);
        ok = 0;
        break;
      }
      __nanosleep(128);
    }
    __threadfence();
    pm_fence_proxy_async_all();
  }
  return __syncthreads_and(ok) != 0;
}

// Programmatic dependent launch: a kernel launched with programmatic
// stream serialization may start while its predecessor in the stream is
// still running.  pm_grid_dep_wait() returns once every predecessor grid
// has completed and its memory is visible (at once when the launch had no
// such predecessor); pm_grid_dep_launch() lets the next kernel in the
// stream be scheduled once every CTA of this grid has called it.
__device__ __forceinline__ void pm_grid_dep_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void pm_grid_dep_launch() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ void pm_mbar_arrive_expect_tx(uint64_t* bar,
                                                         uint32_t bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          pm_smem_addr(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ bool pm_mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(pm_smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// Wait for a barrier phase with an iteration limit; on timeout set the error
// word and report failure (the caller then skips its compute).
__device__ __forceinline__ bool pm_mbar_wait(uint64_t* bar, uint32_t phase,
                                             unsigned* err) {
  for (int it = 0; it < PM_WAIT_LIMIT; ++it) {
    if (pm_mbar_try_wait(bar, phase)) return true;
  }
  if (err) atomicOr(err, PM_KERR_TMA_TIMEOUT);
  return false;
}

// Tiled TMA loads into this CTA's shared memory; completion is signalled on
// `bar` by transaction bytes.  The innermost coordinate must be 16-byte
// aligned (the callers round it down).
__device__ __forceinline__ void pm_tma_load_1d(void* dst, const CUtensorMap* m,
                                               uint64_t* bar, int c0) {
  asm volatile(
      "cp.async.bulk.tensor.1d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2}], [%3];" ::"r"(pm_smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(c0), "r"(pm_smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void pm_tma_load_2d(void* dst, const CUtensorMap* m,
                                               uint64_t* bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(pm_smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(c0), "r"(c1),
      "r"(pm_smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void pm_tma_load_3d(void* dst, const CUtensorMap* m,
                                               uint64_t* bar, int c0, int c1,
                                               int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(pm_smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(c0), "r"(c1), "r"(c2),
      "r"(pm_smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void pm_tma_load_4d(void* dst, const CUtensorMap* m,
                                               uint64_t* bar, int c0, int c1,
                                               int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(pm_smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
      "r"(pm_smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void pm_tma_load_5d(void* dst, const CUtensorMap* m,
                                               uint64_t* bar, int c0, int c1,
                                               int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(pm_smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
      "r"(c4), "r"(pm_smem_addr(bar))
      : "memory");
}

// ---- atomics used by reductions ------------------------------------------
__device__ __forceinline__ void pm_atomic_add(float* p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void pm_atomic_add(double* p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void pm_atomic_add(int* p, int v) { atomicAdd(p, v); }
__device__ __forceinline__ void pm_atomic_add(unsigned* p, unsigned v) { atomicAdd(p, v); }
__device__ __forceinline__ void pm_atomic_add(long long* p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}
__device__ __forceinline__ void pm_atomic_add(unsigned long long* p,
                                              unsigned long long v) {
  atomicAdd(p, v);
}
__device__ __forceinline__ void pm_atomic_min(int* p, int v) { atomicMin(p, v); }
__device__ __forceinline__ void pm_atomic_max(int* p, int v) { atomicMax(p, v); }
__device__ __forceinline__ void pm_atomic_min(unsigned* p, unsigned v) { atomicMin(p, v); }
__device__ __forceinline__ void pm_atomic_max(unsigned* p, unsigned v) { atomicMax(p, v); }
__device__ __forceinline__ void pm_atomic_min(float* p, float v) {
  int* ip = reinterpret_cast<int*>(p);
  int old = *ip;
  while (__int_as_float(old) > v) {
    int prev = atomicCAS(ip, old, __float_as_int(v));
    if (prev == old) break;
    old = prev;
  }
}
__device__ __forceinline__ void pm_atomic_max(float* p, float v) {
  int* ip = reinterpret_cast<int*>(p);
  int old = *ip;
  while (__int_as_float(old) < v) {
    int prev = atomicCAS(ip, old, __float_as_int(v));
    if (prev == old) break;
    old = prev;
  }
}
__device__ __forceinline__ void pm_atomic_mul(float* p, float v) {
  int* ip = reinterpret_cast<int*>(p);
  int old = *ip;
  while (true) {
    int prev = atomicCAS(ip, old, __float_as_int(__int_as_float(old) * v));
    if (prev == old) break;
    old = prev;
  }
}
__device__ __forceinline__ void pm_atomic_mul(int* p, int v) {
  int old = *p;
  while (true) {
    int prev = atomicCAS(p, old, old * v);
    if (prev == old) break;
    old = prev;
  }
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
typedef CUresult (*pm_encode_tiled_fn)(CUtensorMap*, CUtensorMapDataType,
                                       cuuint32_t, void*, const cuuint64_t*,
                                       const cuuint64_t*, const cuuint32_t*,
                                       const cuuint32_t*, CUtensorMapInterleave,
                                       CUtensorMapSwizzle,
                                       CUtensorMapL2promotion,
                                       CUtensorMapFloatOOBfill);

static pm_encode_tiled_fn pm_get_encode_fn() {
  static pm_encode_tiled_fn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, []() {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault,
                                &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<pm_encode_tiled_fn>(p);
  });
  return fn;
}

static CUtensorMapDataType pm_tma_dtype(int elem_size, int is_float) {
  switch (elem_size) {
    case 1: return CU_TENSOR_MAP_DATA_TYPE_UINT8;
    case 2: return CU_TENSOR_MAP_DATA_TYPE_UINT16;
    case 4: return is_float ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                            : CU_TENSOR_MAP_DATA_TYPE_UINT32;
    default: return is_float ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                             : CU_TENSOR_MAP_DATA_TYPE_INT64;
  }
}

// Device-to-host copy of the box [Bl, Bh] of a dense C-order array whose
// domain is [Dl, Dh] (nd <= 8 dimensions, es-byte elements) into the same
// positions of the host array.  The innermost dimensions the box covers
// whole merge with the first one it does not into one contiguous span per
// point of the dimensions outside it; the spans are the rows of 2-D copies
// (one per point of the dimensions outside the rows' dimension), so an
// interleaved [x][y][3] output written whole is one copy, not one 3-byte
// row per pixel.  Returns 0, or 1 when a copy could not be issued.
static int pm_copy_box_d2h(void* dst, const void* src, int es, int nd,
                           const long long* Dl, const long long* Dh,
                           const long long* Bl, const long long* Bh,
                           cudaStream_t s) {
  if (nd < 1 || nd > 8) return 1;
  long long ext[8], S[8];
  for (int d = 0; d < nd; ++d) {
    if (Bl[d] > Bh[d]) return 0;
    ext[d] = Dh[d] - Dl[d] + 1;
  }
  S[nd - 1] = 1;
  for (int d = nd - 2; d >= 0; --d) S[d] = S[d + 1] * ext[d + 1];
  int j = nd - 1;
  while (j > 0 && Bl[j] == Dl[j] && Bh[j] == Dh[j]) --j;
  const size_t span = (size_t)((Bh[j] - Bl[j] + 1) * S[j]) * es;
  if (j == 0) {
    const size_t o = (size_t)((Bl[0] - Dl[0]) * S[0]) * es;
    return cudaMemcpyAsync((char*)dst + o, (const char*)src + o, span,
                           cudaMemcpyDeviceToHost, s) != cudaSuccess;
  }
  // rows: dimension j - 1; one 2-D copy per point of the dimensions < j - 1
  const int r = j - 1;
  const size_t pitch = (size_t)S[r] * es;
  const size_t rows = (size_t)(Bh[r] - Bl[r] + 1);
  long long idx[8];
  for (int d = 0; d < r; ++d) idx[d] = Bl[d];
  while (true) {
    long long off = (Bl[r] - Dl[r]) * S[r] + (Bl[j] - Dl[j]) * S[j];
    for (int d = 0; d < r; ++d) off += (idx[d] - Dl[d]) * S[d];
    const size_t o = (size_t)off * es;
    if (cudaMemcpy2DAsync((char*)dst + o, pitch, (const char*)src + o, pitch,
                          span, rows, cudaMemcpyDeviceToHost, s) !=
        cudaSuccess)
      return 1;
    int d = r - 1;
    while (d >= 0 && ++idx[d] > Bh[d]) { idx[d] = Bl[d]; --d; }
    if (d < 0) break;
  }
  return 0;
}

// Encode a tiled tensor map over a dense row-major array.  `dims` and `box`
// are given outermost first (C order); returns false when the TMA
// preconditions do not hold (alignment, box limits), in which case the
// kernel falls back to cooperative loads.
// `pitch`: elements between the starts of consecutive innermost rows in
// memory (dims[rank - 1] for a dense array; more for padded rows).
static bool pm_make_tmap(CUtensorMap* m, const void* base, int rank,
                         const long long* dims, const int* box, int elem_size,
                         int is_float, long long pitch) {
  memset(m, 0, sizeof(*m));
  pm_encode_tiled_fn fn = pm_get_encode_fn();
  if (!fn || rank < 1 || rank > 5) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
  cuuint64_t gdim[5], gstride[5];
  cuuint32_t bdim[5], estr[5];
  long long stride = elem_size;
  for (int i = 0; i < rank; ++i) {
    int c = rank - 1 - i;  // reverse to innermost-first
    if (dims[c] <= 0 || box[c] <= 0 || box[c] > 256) return false;
    gdim[i] = (cuuint64_t)dims[c];
    bdim[i] = (cuuint32_t)box[c];
    estr[i] = 1;
    if (i > 0) {
      if (stride % 16 != 0) return false;
      gstride[i - 1] = (cuuint64_t)stride;
    }
    if (i == 0 && pitch < dims[c]) return false;
    stride *= (i == 0) ? pitch : dims[c];
  }
  if ((bdim[0] * elem_size) % 16 != 0) return false;
  CUresult r = fn(m, pm_tma_dtype(elem_size, is_float), (cuuint32_t)rank,
                  const_cast<void*>(base), gdim, gstride, bdim, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Workspace arena: one device allocation per device, grown on demand and
// reused across calls (the device counterpart of the reference's pool
// allocator, sandbox/memory_allocation/simple_pool_allocator.cpp).
struct pm_arena {
  void* ptr[64];
  size_t cap[64];
};

static int pm_arena_get(pm_arena* a, size_t bytes, void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return PM_ERR_CUDA;
  if (bytes == 0) bytes = 256;
  if (a->cap[dev] < bytes) {
    if (a->ptr[dev]) {
      cudaDeviceSynchronize();
      cudaFree(a->ptr[dev]);
    }
    a->ptr[dev] = nullptr;
    a->cap[dev] = 0;
    size_t want = bytes + bytes / 8;
    if (cudaMalloc(&a->ptr[dev], want) != cudaSuccess) {
      cudaGetLastError();
      return PM_ERR_CUDA;
    }
    a->cap[dev] = want;
  }
  *out = a->ptr[dev];
  return PM_OK;
}

static inline size_t pm_align256(size_t x) { return (x + 255) & ~size_t(255); }

// Launch with programmatic stream serialization (the kernel calls
// pm_grid_dep_wait before reading what earlier work in the stream wrote).
template <typename L>
static cudaError_t pm_launch_pdl(void (*k)(L), unsigned grid, unsigned threads,
                                 size_t smem, cudaStream_t s, const L& arg) {
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, arg);
}

// Ordinal of the calling thread's current device, the index of every
// per-device piece of host state (arenas, streams, graphs, kernel
// attributes); a process uses devices 0..63.
static inline int pm_cur_dev() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return 0;
  }
  return dev;
}

// Binary search of a tile index in a batch's tile prefix (descriptors carry
// their first tile); used by batched launches.
template <typename D>
__device__ __forceinline__ int pm_find_image(const D* descs, int n, int tile) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (descs[mid].tile_base <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}
