"""monolis_b200 -- B200-native CG / BiCGSTAB inner loop behind the monolis C API.

The product is the shared library `libmonolis_b200.so` (built from
`monolis_b200/csrc/`); this package holds its ctypes mirror (`api`) and the
seeded synthetic problem generators used by the tests and the benchmark
(`problems`).
"""
from .api import (ITER_BICGSTAB, ITER_CG, PREC_DIAG, PREC_NONE, Monolis, MonolisLib, load_library,  # noqa: F401
                  load_product)

__all__ = ["Monolis", "MonolisLib", "load_product", "load_library", "ITER_CG", "ITER_BICGSTAB", "PREC_NONE",
           "PREC_DIAG"]
