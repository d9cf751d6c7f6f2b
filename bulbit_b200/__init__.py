"""bulbit-b200: a B200 (sm_100a) wavefront implementation of Bulbit's
unidirectional path tracer behind a C ABI (include/bbg.h).

The native library (libbulbit_b200.so, built by bulbit_b200.build) is the
product; this package only loads it (bulbit_b200.lib), mirrors its records
(bulbit_b200.abi) and generates workloads (bulbit_b200.scenes).
"""
from . import abi  # noqa: F401
