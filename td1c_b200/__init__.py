"""td1c_b200 -- B200 (sm_100a) implementation of td1c's orbital-equation RHS.

The hot path (hprod_htot and the RK4 stages around it) runs in the CUDA
library td1c_b200/_lib/libtd1c_b200.so behind a C-ABI (include/td1c_b200.h);
this package holds the host-side set-up (grid, tables, seeded states) and the
ctypes binding.
"""
from . import workloads  # noqa: F401
