"""polymage_b200: a B200 (sm_100a) execution backend for PolyMage pipelines.

The language (``constructs``) and the build flow (``compiler.buildPipeline``
-> ``Pipeline`` -> ``generate_code`` / ``build``) follow the reference
PolyMage; the code generator emits CUDA for NVIDIA B200 instead of C++ with
OpenMP, and the compiled pipeline keeps the reference's
``pipeline_<name>(params..., inputs..., outputs...)`` C ABI.
"""

from .constructs import *          # noqa: F401,F403
from .compiler import buildPipeline  # noqa: F401

__version__ = "0.1.0"
