"""B200-native implementation of Mjolnir's per-step molecular-dynamics hot path.

The compute lives in ``libmjolnir_b200.so`` (CUDA for sm_100a behind the C ABI
of ``include/mjolnir_b200.h``); :mod:`mjolnir_b200.engine` binds it,
:mod:`mjolnir_b200.systems` describes systems and builds the synthetic
workloads.
"""
from .systems import SystemDesc, PairTerm  # noqa: F401

__all__ = ["SystemDesc", "PairTerm", "Engine"]


def __getattr__(name):
    if name == "Engine":
        from .engine import Engine
        return Engine
    raise AttributeError(name)
