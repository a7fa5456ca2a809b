"""cmfw -- B200-native pFq Conservative Matrix Field walk (host side).

The walk runs in hand-written sm_100a kernels behind the C ABI of
include/cmfw.h (lib/libcmfw.so, built in-tree); this package is the Python
host interface over it. There is no CPU implementation of the walk here.
"""
from ._lib import (BIN_DIR, EXPORTS, F_BATCH_INVARIANT, F_DF64_COMPAT, F_PLAIN_RUNS, F_SEQUENTIAL, F_UNFUSED_COLUMN, IN_DTYPE, LIB_PATH,  # noqa: F401
                   MIXED_ITEM_DTYPE, MixedTuning, OUT_DTYPE, TRAJ_STATUS, CmfwError, Desc, lib)
from .api import (MixedBatch, baseline_tuning, walk_mixed, check_desc, device_banner, exact_residues, launch_walk, make_desc, mt64,  # noqa: F401
                  out_buffer, pipe_peak, records_from_device, reference_inputs, rns_trace, to_device,
                  version, walk, walk_host)
