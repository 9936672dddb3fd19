"""B200-native Faceted HyperSARA: Python mirror of the reference interface.

All compute runs in ``libfhs_b200.so`` (hand-written sm_100a CUDA kernels
behind the C ABI of ``include/fhs_b200.h``).
"""
from ._lib import FhsError, lib  # noqa: F401
from .api import *  # noqa: F401,F403
from . import heuristics, io, synth  # noqa: F401
from .io import fitsread, fitswrite, load_checkpoint, save_checkpoint  # noqa: F401
