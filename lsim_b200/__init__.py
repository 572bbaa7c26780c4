"""B200-native stuck-at fault simulation with LSIM's fsim API and formats.

``Simulator`` mirrors fsim::Simulator; ``Batch`` simulates many circuits in
one launch sequence; ``gen`` writes seeded synthetic .ckt/.flst/.ptn
workloads.  All simulation runs on the GPU through the C ABI
of ``libfsimb200.so`` (include/fsimb.h).
"""
from .simulator import Simulator, FsimbError, RESULT_DTYPE  # noqa: F401
from .batch import Batch  # noqa: F401
from .serve import Server  # noqa: F401
from . import gen  # noqa: F401
