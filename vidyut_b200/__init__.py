"""vidyut_b200 -- B200-native explicit species / electron-energy update of the
Vidyut plasma fluid solver (hsitaram/vidyut3d), behind a C ABI.

The compute lives in libvidyut_b200.so (hand-written sm_100a kernels); this
package holds the ctypes binding (``_abi``), the runtime mechanism tables
(``mechanism``), seeded workload inputs (``inputs``) and the host-side driver
mirroring the reference's per-box calls (``api``).
"""
from . import _abi  # noqa: F401
from .mechanism import Mechanism, Reaction, argon, synthetic  # noqa: F401

__all__ = ["Mechanism", "Reaction", "argon", "synthetic"]
