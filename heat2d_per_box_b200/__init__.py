"""B200-native box fast Gauss transform: a drop-in for the reference's boxfgt
(bfgt/boxfgt.f) with hand-written sm_100a CUDA kernels behind a C ABI."""
from ._lib import BFGT_PREC_FP64, BFGT_PREC_SPLIT, BfgtError, lib, lib_path  # noqa: F401
from .boxfgt import (Batch, Plan, boxfgt, host_plan_dump, last_call_bytes, plan_cache_clear,  # noqa: F401
                     plan_cache_info, set_default_precision)
from .tree import Tree, build_adaptive, build_uniform, gauss_params  # noqa: F401
