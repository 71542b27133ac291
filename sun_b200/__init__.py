"""sun_b200 -- B200-native SU(N) quenched lattice gauge engine.

The compute path is ``libsun_b200.so`` (hand-written sm_100a CUDA behind the
C ABI of ``include/sun_b200.h``); this package is its Python host binding.
"""
from ._native import SunError, lib  # noqa: F401
from .api import (SOA, SOA8, SOA12, ApplyAPEinSpace, ApplyAPEinTime, ApplyHYPinSpace,  # noqa: F401
                  ApplyHYPinTime, ApplyMultiHit, ApplyMultiHitSpace, ApplyStoutinSpace, ApplyStoutinTime,
                  Batch, Context, EndCULQCD, HeatBath, OnePolyakovLoop, OverRelaxation, ParamHYP,
                  PlaquetteCUB, ReadBin_Gauge, Reunitarize, SaveBin_Gauge, Server, Sweep, SweepMeasure,
                  WilsonLoop, admit_count, gauge, initCULQCD, job_footprint, link_trace_det, make_job,
                  unitarity_violation)

__version__ = "0.1.0"
