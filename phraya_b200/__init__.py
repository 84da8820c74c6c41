"""phraya_b200 -- B200-native (sm_100a) seed -> chain -> extend engine for phraya-align.

The compute lives in libphraya_b200.so (CUDA, built by phraya_b200.build); this
package is the host-side mirror of phraya-align's API over its C ABI.
"""
from .api import (AffineCosts, Alignment, AlignmentFailed, Engine, EngineError, EngineUnavailable,  # noqa: F401
                  InvalidInput, SeedAnchor, WfaError, myers_edit_distance, myers_extend, wfa_extend,
                  wfa_extend_affine)
