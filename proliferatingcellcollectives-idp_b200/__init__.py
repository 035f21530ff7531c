"""B200 (sm_100a) collision hot path of the ProliferatingCellCollectives simulator.

The product is the CUDA library behind include/pcc_gpu.h (csrc/, built into
libpcc_gpu.so next to this file).  Python here is a thin host layer over that
C ABI: `abi` mirrors the header, `device` loads the library and mirrors the
reference's step interface.  The directory name is not a Python identifier;
`load_package()` in the repository root helpers registers it as `pcc_b200`.
"""
from . import abi  # noqa: F401
