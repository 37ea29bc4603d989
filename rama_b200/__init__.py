"""rama_b200 -- a multicut (correlation clustering) solver for NVIDIA B200.

Drop-in for the RAMA solver's interfaces: ``rama_b200.rama_py`` mirrors the
reference's Python module, include/rama_cuda.h its C++ entry points, and
``rama_b200/bin/rama_text_input`` its command line.  All of them call the
C ABI of librama_b200.so (include/rama_b200.h).
"""
from . import instances  # noqa: F401

__all__ = ["instances", "rama_py", "solver"]
