"""B200-native LPS peridynamics time marcher (Python side of the C ABI).

``files``  reads and writes the preprocessor's input file set and the logs.
``api``    binds liblps_b200.so (include/lps_cuda.h) with ctypes.
``gen``    builds synthetic input sets (lattice discs, pulses, ABC layers).
"""
from .files import InputSet, read_input_set, write_input_set, read_log  # noqa: F401
