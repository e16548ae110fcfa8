"""Python side of a compiled pipeline: loads the shared library with ctypes
(as the reference's loader does, sandbox/apps/python/loader.py:4-21) and
calls its entry points on numpy arrays (host buffers, the reference's ABI)
or torch CUDA tensors (device buffers, asynchronous on the current stream).

There is no CPU fallback: the library is the only execution path, and
calls fail loudly when it cannot be loaded or returns an error status.
"""

import ctypes

import numpy as np

from . import constructs as C
from .evaluate import eval_int

STATUS_TEXT = {0: "ok", 1: "parameters outside the pipeline's bounds",
               2: "CUDA error", 3: "kernel reported an error",
               4: "unsupported request"}


class PipelineRuntimeError(RuntimeError):
    pass


def _ctype_of(t):
    return ctypes.c_float if t in (C.Float, C.Double) else ctypes.c_int


class CompiledPipeline(object):
    """A built pipeline.  ``params``/``inputs``/``outputs`` are in C-ABI
    order (each sorted by name)."""

    def __init__(self, pipeline, so_path, module):
        self.pipeline = pipeline
        self.so_path = so_path
        self.module = module
        self.name = module.name
        self.lib = ctypes.CDLL(so_path)
        self.params, self.inputs, self.outputs = pipeline.ordered_params()
        # inputs read only by const tables (the camera pipe's colour
        # matrices): the entry points tabulate them on the host, so they
        # may stay in host memory also for the device entry points, where
        # a device copy would cost a synchronous read-back every call
        from .pipe import body_refs
        readers = dict((id(f), []) for f in self.inputs)
        for comp in pipeline.comps:
            for r in body_refs(comp.func):
                if id(r.objectRef) in readers:
                    readers[id(r.objectRef)].append(comp)
        self.table_only = set(
            id(f) for f in self.inputs if readers[id(f)] and
            all(c.is_const_func for c in readers[id(f)]))
        pt = [_ctype_of(p.typ) for p in self.params]
        vp = [ctypes.c_void_p] * (len(self.inputs) + len(self.outputs))
        n = self.name
        self._host = getattr(self.lib, "pipeline_" + n)
        self._host.argtypes = pt + vp
        self._host.restype = None
        self._dev = getattr(self.lib, "pipeline_%s_dev" % n)
        self._dev.argtypes = pt + vp + [ctypes.c_void_p]
        self._dev.restype = ctypes.c_int
        self._graph = getattr(self.lib, "pipeline_%s_graph" % n)
        self._graph.argtypes = pt + vp + [ctypes.c_void_p]
        self._graph.restype = ctypes.c_int
        self._batch = getattr(self.lib, "pipeline_%s_batch" % n)
        self._batch.argtypes = [ctypes.c_int, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p]
        self._batch.restype = ctypes.c_int
        self._batch_graph = getattr(self.lib, "pipeline_%s_batch_graph" % n)
        self._batch_graph.argtypes = self._batch.argtypes
        self._batch_graph.restype = ctypes.c_int
        self._status = getattr(self.lib, "pipeline_%s_status" % n)
        self._status.restype = ctypes.c_int
        self._check = getattr(self.lib, "pipeline_%s_check" % n)
        self._check.restype = ctypes.c_int
        self._clear = getattr(self.lib, "pipeline_%s_clear_error" % n)
        self._clear.restype = None

    # ---- shapes --------------------------------------------------------------
    def _env(self, params):
        env = {}
        for p in self.params:
            if p.name not in params:
                raise KeyError("missing parameter %s" % p.name)
            v = params[p.name]
            env[p] = int(v) if p.typ not in (C.Float, C.Double) else v
        return env

    def shape_of(self, func, params):
        env = dict((k, v) for k, v in self._env(params).items()
                   if k.typ not in (C.Float, C.Double))
        return tuple(eval_int(d.upperBound - d.lowerBound + 1, env)
                     for d in func.domain)

    def input_shapes(self, params):
        return dict((f.name, self.shape_of(f, params)) for f in self.inputs)

    def output_shapes(self, params):
        return dict((f.name, self.shape_of(f, params)) for f in self.outputs)

    def _param_args(self, params):
        out = []
        for p in self.params:
            v = params[p.name]
            out.append(float(v) if p.typ in (C.Float, C.Double) else int(v))
        return out

    # ---- host buffers ----------------------------------------------------------
    def run_host(self, params, inputs, outputs):
        """Reference ABI: numpy arrays in, numpy arrays (preallocated,
        C-contiguous, domain-shaped) out; synchronous."""
        ptrs = []
        for f in self.inputs:
            a = inputs[f.name]
            self._check_array(f, a, params)
            ptrs.append(a.ctypes.data)
        for f in self.outputs:
            a = outputs[f.name]
            self._check_array(f, a, params)
            ptrs.append(a.ctypes.data)
        self._host(*(self._param_args(params) + ptrs))
        st = self._status()
        if st != 0:
            raise PipelineRuntimeError("pipeline_%s failed: %s" % (
                self.name, STATUS_TEXT.get(st, st)))
        return outputs

    def _check_array(self, f, a, params):
        shape = self.shape_of(f, params)
        if not isinstance(a, np.ndarray) or not a.flags.c_contiguous:
            raise TypeError("%s must be a C-contiguous numpy array" % f.name)
        if a.dtype != f.typ.np_dtype():
            raise TypeError("%s must have dtype %s, got %s" % (
                f.name, f.typ.np_dtype(), a.dtype))
        if a.size != int(np.prod(shape)):
            raise ValueError("%s must have %d elements (shape %s), got %d" % (
                f.name, int(np.prod(shape)), shape, a.size))

    def __call__(self, params, inputs, outputs=None):
        """Convenience: allocate missing outputs (zero-filled) and run."""
        if outputs is None:
            outputs = {}
        first = next(iter(inputs.values())) if inputs else None
        is_torch = first is not None and type(first).__module__.startswith(
            'torch')
        for f in self.outputs:
            if f.name not in outputs:
                shape = self.shape_of(f, params)
                if is_torch:
                    import torch
                    outputs[f.name] = torch.zeros(
                        shape, dtype=_torch_dtype(f.typ), device=first.device)
                else:
                    outputs[f.name] = np.zeros(shape, f.typ.np_dtype())
        if is_torch:
            self.run_dev(params, inputs, outputs)
        else:
            self.run_host(params, inputs, outputs)
        return outputs

    # ---- device buffers ----------------------------------------------------------
    def _dev_ptrs(self, params, inputs, outputs):
        ptrs = []
        for f in self.inputs + self.outputs:
            t = (inputs if any(f is g for g in self.inputs) else outputs)[
                f.name]
            shape = self.shape_of(f, params)
            if not t.is_contiguous() or not t.is_cuda and \
                    id(f) not in self.table_only:
                raise TypeError("%s must be a contiguous CUDA tensor" % f.name)
            if t.numel() != int(np.prod(shape)):
                raise ValueError("%s must have %d elements" % (
                    f.name, int(np.prod(shape))))
            if t.element_size() != f.typ.size():
                raise TypeError("%s must have %d-byte elements" % (
                    f.name, f.typ.size()))
            ptrs.append(t.data_ptr())
        return ptrs

    def run_dev(self, params, inputs, outputs, stream=None, graph=False):
        import torch
        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        ptrs = self._dev_ptrs(params, inputs, outputs)
        fn = self._graph if graph else self._dev
        st = fn(*(self._param_args(params) + ptrs + [stream]))
        if st != 0:
            raise PipelineRuntimeError("pipeline_%s_%s failed: %s" % (
                self.name, "graph" if graph else "dev",
                STATUS_TEXT.get(st, st)))
        return outputs

    def run_batch(self, params_list, inputs_list, outputs_list, stream=None,
                  graph=False):
        """Many images in one launch per group; each entry of the lists is a
        dict as for ``run_dev``.  ``graph=True`` runs the batch as a CUDA
        graph (captured on the first call, re-captured when the arguments
        change)."""
        import torch
        n = len(params_list)
        ip = [p for p in self.params if p.typ not in (C.Float, C.Double)]
        fp = [p for p in self.params if p.typ in (C.Float, C.Double)]
        iarr = np.zeros((n, max(len(ip), 1)), np.int32)
        farr = np.zeros((n, max(len(fp), 1)), np.float32)
        ins = np.zeros((n, max(len(self.inputs), 1)), np.uint64)
        outs = np.zeros((n, max(len(self.outputs), 1)), np.uint64)
        for i in range(n):
            prm = params_list[i]
            for j, p in enumerate(ip):
                iarr[i, j] = int(prm[p.name])
            for j, p in enumerate(fp):
                farr[i, j] = float(prm[p.name])
            ptrs = self._dev_ptrs(prm, inputs_list[i], outputs_list[i])
            for j in range(len(self.inputs)):
                ins[i, j] = ptrs[j]
            for j in range(len(self.outputs)):
                outs[i, j] = ptrs[len(self.inputs) + j]
        iarr = np.ascontiguousarray(iarr[:, :len(ip)]) if ip else iarr
        farr = np.ascontiguousarray(farr[:, :len(fp)]) if fp else farr
        ins = np.ascontiguousarray(ins[:, :len(self.inputs)])
        outs = np.ascontiguousarray(outs[:, :len(self.outputs)])
        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        fn = self._batch_graph if graph else self._batch
        st = fn(n, iarr.ctypes.data, farr.ctypes.data, ins.ctypes.data,
                outs.ctypes.data, stream)
        if st != 0:
            raise PipelineRuntimeError("pipeline_%s_batch%s failed: %s" % (
                self.name, "_graph" if graph else "",
                STATUS_TEXT.get(st, st)))
        return outputs_list

    def check(self):
        """Synchronize and raise if a kernel set the device error word."""
        st = self._check()
        if st != 0:
            self._clear()
            raise PipelineRuntimeError("pipeline_%s: %s" % (
                self.name, STATUS_TEXT.get(st, st)))

    def describe(self):
        return self.pipeline.describe()


def _torch_dtype(t):
    import torch
    return {C.Float: torch.float32, C.Double: torch.float64,
            C.Int: torch.int32, C.UInt: torch.int32, C.Short: torch.int16,
            C.UShort: torch.int16, C.Char: torch.int8, C.UChar: torch.uint8,
            C.Long: torch.int64, C.ULong: torch.int64}[t]
