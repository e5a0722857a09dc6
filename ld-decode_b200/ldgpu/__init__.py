"""ldgpu: B200-native (sm_100a) RF demodulation and time-base correction for
LaserDisc RF captures, a drop-in for the hot path of happycube/ld-decode.

Public API (mirrors lddecode.core):
  RFDecode   -- RFDecode.demodblock on the GPU (lddecode/core.py:253-1046)
  FieldNTSC, FieldPAL -- line locations and Field.downscale (TBC) on the GPU
  synth_capture -- seeded synthetic RF captures for tests and benchmarks
"""

from .params import BLOCKSIZE, SysParams_NTSC, SysParams_PAL  # noqa: F401
from .rfdecode import RFDecode  # noqa: F401
from .synth import synth_capture  # noqa: F401

__version__ = "0.1.0"
