"""B200-native batched 2-D MLS-MPM engine for jellyfih.

``jellyfih_b200.Engine`` drives libjellyfih.so (hand-written sm_100a CUDA
behind the C ABI in include/jellyfih.h); ``jellyfih_b200.mpm_sim`` is the
drop-in replacement of the reference's mpm_sim module; ``jellyfih_b200.tank``
builds particle sets from genomes.
"""
from .engine import DT, Engine, InstanceSpec  # noqa: F401
from ._lib import JfError  # noqa: F401

__all__ = ["Engine", "InstanceSpec", "DT", "JfError"]
