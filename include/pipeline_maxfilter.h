/* pipeline_maxfilter -- C ABI of the PolyMage pipeline 'maxfilter' built for NVIDIA B200 (sm_100a).
 * Generated by polymage_b200; argument order: parameters, then inputs, then
 * outputs, each sorted by name.  pipeline_maxfilter replaces the function of the same
 * name the reference generates (signature built at sandbox/codegen.py:957-1007,
 * sandbox/targetc.py:344-366; called through ctypes as in sandbox/apps/python/
 * img_proc/harris/exec_pipe.py:13-35); the other entry points are additions. */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
/* host buffers, synchronous (reference ABI) */
void pipeline_maxfilter(int C, int R, void* img, void* final);
/* device buffers, asynchronous on `stream` (cudaStream_t); returns a PM status */
int pipeline_maxfilter_dev(int C, int R, void* img, void* final, void* stream);
/* same as _dev through a CUDA graph captured on first use */
int pipeline_maxfilter_graph(int C, int R, void* img, void* final, void* stream);
/* n images; iparams: n x 2 int params, fparams: n x 0 float params, each row in
 * name order; inputs: n x 1 device pointers, outputs: n x 1 device pointers */
int pipeline_maxfilter_batch(int n, const int* iparams, const float* fparams, void* const* inputs, void* const* outputs, void* stream);
/* same as _batch through a CUDA graph captured on first use (re-captured when
 * the arguments change); a repeated _batch call with unchanged arguments
 * relaunches kernels only */
int pipeline_maxfilter_batch_graph(int n, const int* iparams, const float* fparams, void* const* inputs, void* const* outputs, void* stream);
/* status of the last call: 0 ok, 1 bad parameters, 2 CUDA error, 3 kernel error */
int pipeline_maxfilter_status(void);
/* synchronizes and reports the device error word */
int pipeline_maxfilter_check(void);
void pipeline_maxfilter_clear_error(void);
#ifdef __cplusplus
}
#endif
