"""bcc -- host-side Python mirror of the batch edge collision checker.

The product path is the CUDA library ``libbcc.so`` (C ABI in include/bcc.h);
this package loads it with ctypes and exposes the reference's operator
semantics (src/batch_cc.hh:4-6): environments + edges + resolution in,
one verdict per (edge, environment) out, True = in collision.
"""
from .envs import EnvSet, KINDS, WIDTH  # noqa: F401
from . import workload  # noqa: F401
