"""CPU oracle for polymage_b200 -- TEST INFRASTRUCTURE ONLY.

Nothing in the product (the ``polymage_b200`` package and its CUDA
libraries) imports, links or calls anything under ``oracle/``.  Only the
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
use it, as the checker.

Contents:

* numpy FP64 restatements of the reference pipelines' specs, one module per
  app, each function citing the reference file:line it restates
  (``harris``, ``unsharp`` ...);
* ``ref``: ctypes wrappers around the reference's own generated C++
  (``oracle/_ref/*.so``, built from the reference tree by
  ``oracle/Makefile``), used to pin the restatements (tests/golden) and as
  the CPU baseline.

Parity pinning: the Harris and unsharp restatements are checked against the
reference's generated C++ (``refHarris``, ``pipeline_mask``) through the
golden fixtures in tests/golden; see each module for the region where the
reference's output is well defined.
"""
