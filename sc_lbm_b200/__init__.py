"""sc_lbm_b200 -- B200-native D2Q9 Shan-Chen lattice-Boltzmann step.

The product is the shared library ``libsclbm_b200.so`` (C ABI in
include/sclbm.h) with sm_100a kernels, plus the C++ drop-in classes under
``host/`` (Geometry / Fluid / LBM, same API as LBMFluids/sc_lbm).  This Python
package is a thin ctypes mirror used by the tests and the benchmark.
"""
from .api import (LBM, Batch, Domain, Fluid, Geometry, io_wait, make_params, read_rows,
                  set_stream, synchronize, tuned_config, version, write_rows)
from .capi import FP16_SHIFTED, FP32_SHIFTED, FP64

__all__ = ["Geometry", "Fluid", "LBM", "Domain", "Batch", "make_params", "synchronize", "tuned_config",
           "io_wait", "write_rows", "read_rows",
           "set_stream", "version", "FP64", "FP32_SHIFTED", "FP16_SHIFTED"]
