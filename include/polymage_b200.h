/* polymage_b200.h -- conventions shared by every pipeline library built by
 * polymage_b200 (NVIDIA B200, sm_100a).
 *
 * A pipeline named <name> is compiled into libpm_<name>_<hash>.so, which
 * exports the entry points declared in include/pipeline_<name>.h:
 *
 *   void pipeline_<name>(params..., void* inputs..., void* outputs...);
 *     Replaces the reference's generated `extern "C" void
 *     pipeline_<name>(...)` (sandbox/codegen.py:1002-1007,
 *     sandbox/targetc.py:344-366): same argument order (scalar parameters
 *     sorted by name, then input images sorted by name, then outputs sorted
 *     by name: sandbox/codegen.py:957-999, sandbox/utils.py:87-100), same
 *     meaning (caller-owned dense row-major host buffers shaped by the
 *     functions' domains), blocking.  Points of an output that no Case
 *     covers are left as the caller's buffer had them.
 *
 *   int pipeline_<name>_dev(params..., void* inputs..., void* outputs...,
 *                           void* stream);
 *     Device buffers, asynchronous on a cudaStream_t.
 *
 *   int pipeline_<name>_graph(..., void* stream);
 *     As _dev, replaying a CUDA graph captured on first use.
 *
 *   int pipeline_<name>_batch(int n, const int* iparams,
 *                             const float* fparams, void* const* inputs,
 *                             void* const* outputs, void* stream);
 *     n images, each with its own parameters, one launch per group; a
 *     group with more tiles than fit on the GPU at once runs as a
 *     persistent grid over a device-side tile queue.  A call repeating
 *     the previous call's arguments relaunches the kernels only.
 *
 *   int pipeline_<name>_batch_graph(same arguments as _batch);
 *     The batch as one CUDA graph, captured on first use.
 *
 *   int pipeline_<name>_status(void);   status of the last call
 *   int pipeline_<name>_check(void);    synchronizes, reads the device
 *                                       error word
 *   void pipeline_<name>_clear_error(void);
 *
 * The reference's ABI returns void and has no error reporting
 * (sandbox/codegen.py:1002); the status entry points are additions.
 */
#pragma once

#define PM_OK 0
#define PM_ERR_PARAMS 1       /* parameters outside the spec's bounds */
#define PM_ERR_CUDA 2         /* a CUDA call failed */
#define PM_ERR_KERNEL 3       /* a kernel set the device error word */
#define PM_ERR_UNSUPPORTED 4  /* request outside what the build supports */
