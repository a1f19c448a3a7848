"""dcell_b200 -- B200-native (sm_100a) level-set transport for adrielb/DCell.

The product is ``lib/libdcell_ls.so`` behind the C ABI in
``include/dcell_ls.h``; this package binds it (``_lib``), mirrors the
reference's LevelSet entry points over torch device memory (``levelset``)
and generates the synthetic workloads of the benchmark (``fields``).
"""
from ._lib import (BACKTRACE, CUBIC_PLAIN, CUBIC_SEPARABLE, CUBIC_TC, EULER, F32, F64, INTERP, LINEAR, MIDPOINT,
                   DcellError, check, geom, lib)

__all__ = ["DcellError", "lib", "check", "geom", "LINEAR", "CUBIC_PLAIN", "CUBIC_SEPARABLE", "CUBIC_TC", "EULER",
           "MIDPOINT", "F32", "F64", "INTERP", "BACKTRACE"]
