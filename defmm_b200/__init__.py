"""defmm_b200: directional equispaced-interpolation FMM matvec for the
Helmholtz kernel on NVIDIA B200 (sm_100a), a drop-in for IChollet/defmm's
IBFMM_Mat<3> (include/interface.hpp).  See defmm_b200.api."""
from .api import (Batch, CheckFULL, DefmmError, IBFMM_Mat, MultiFreqMat, PRECISION_FP64,  # noqa: F401
                  PRECISION_MIXED, SourceRoot, TargetRoot, gemv)
