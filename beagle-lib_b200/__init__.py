"""beagle-lib_b200: a B200 (sm_100a) resource for BEAGLE's likelihood hot path.

``load()`` opens the native C-ABI library ``lib/libbeagle_b200.so`` (built
in-tree by ``build.py``) through :mod:`.binding`; the seeded workloads and the
lnL + gradient call sequence live in :mod:`.synthetic`; the subtree
checkpointed schedule for trees whose partials do not fit in :mod:`.checkpoint`.  There is no CPU
fallback: without the built library, or without an sm_100 device,
``load()`` / instance creation raise.
"""
import os

from . import binding, checkpoint, shard, synthetic  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libbeagle_b200.so")
PLUGIN_PATH = os.path.join(HERE, "lib", "libhmsbeagle-cuda.so.40.0.0")
_LIB = None


def load():
    """Return the BeagleLib bound to libbeagle_b200.so (prefix ``beagleB200``)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run beagle-lib_b200/build.py")
        _LIB = binding.BeagleLib(LIB_PATH, "beagleB200")
    return _LIB
