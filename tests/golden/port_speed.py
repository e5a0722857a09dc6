#!/usr/bin/env python3
"""Speed of the CPU oracle port against the unmodified reference, on the
same inputs, one host thread each.

The CPU reference arm of bench.py times the oracle (oracle/, a numpy
restatement of the reference's path) because the reference itself is not
available where the bench runs.  This script, run where a checkout of the
reference is (like make_golden.py), shows how the port's speed compares
with the reference's own code on the same synthetic NTSC blocks and fields:

  demod  RFDecode.demodblock(data=block, mtf_level=1, cut=True)
         (lddecode/core.py:747-879; scipy/numpy FFTs, numba discriminator)
         against oracle.demod.demodblock;
  TBC    lddecode.utils.scale_field (utils.py:127-183, numba) against
         oracle.tbc.scale_field, both on the same pixel coordinates and wow
         factors, plus hz_to_output.

Usage: python tests/golden/port_speed.py --ref <ld-decode checkout>
       (or LDDECODE_REF=<checkout>); prints one JSON line.
"""

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _take_ref(argv):
    if "--ref" in argv:
        i = argv.index("--ref")
        path = argv[i + 1]
        del argv[i:i + 2]
        return path
    return os.environ.get("LDDECODE_REF")


REF = _take_ref(sys.argv)
if not REF or not os.path.isdir(os.path.join(REF, "lddecode")):
    sys.exit("usage: port_speed.py --ref <ld-decode checkout>  (or LDDECODE_REF=<checkout>)")

os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_golden")
os.environ.setdefault("OMP_NUM_THREADS", "1")
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
os.environ.setdefault("MKL_NUM_THREADS", "1")
sys.dont_write_bytecode = True
sys.path.insert(0, os.path.join(REPO, "ld-decode_b200"))
sys.path.insert(0, REPO)
sys.path.insert(0, REF)

import numpy as np  # noqa: E402

from lddecode import core as refcore  # noqa: E402
from lddecode import utils as refutils  # noqa: E402
from ldgpu.linelocs import FieldLogicNTSC  # noqa: E402
from ldgpu.rfdecode import RFParams  # noqa: E402
from ldgpu.synth import synth_capture  # noqa: E402
from oracle import demod as odemod  # noqa: E402
from oracle import tbc as otbc  # noqa: E402

NBLOCKS = 24   # blocks timed through demod
NFIELD_BLOCKS = 64  # blocks demodulated (by the port) to locate a field for the TBC
REPS = 3


def best(fn, reps=REPS):
    fn()  # warm-up (numba compilation, caches)
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    return min(ts)


def main():
    ref = refcore.RFDecode(system="NTSC", decode_analog_audio=44100, decode_digital_audio=True)
    port = RFParams(system="NTSC", decode_analog_audio=44100, decode_digital_audio=True)
    port.delays = {"video_rot": 3}
    N = port.blocklen
    U = N - port.blockcut - port.blockcut_end
    cap = synth_capture("NTSC", (NFIELD_BLOCKS - 1) * U + N, seed=5, start=1004).numpy()
    allblocks = [cap[b * U:b * U + N] for b in range(NFIELD_BLOCKS)]
    blocks = allblocks[:NBLOCKS]

    def ref_demod():
        for x in blocks:
            ref.demodblock(data=x, mtf_level=1, cut=True)

    def port_demod():
        for x in blocks:
            odemod.demodblock(x, port.Filters, system="NTSC", freq_hz=port.freq_hz, blockcut_end=port.blockcut_end,
                              video_rot=port.delays["video_rot"], mtf_level=port.scaled_mtf(1), cut=True, efm=True,
                              audio=port.audio, out_dtype=np.float32)

    t_ref_demod = best(ref_demod)
    t_port_demod = best(port_demod)

    # one field's TBC on the port's demodulation and line locations
    outs = [odemod.demodblock(x, port.Filters, system="NTSC", freq_hz=port.freq_hz, blockcut_end=port.blockcut_end,
                              video_rot=port.delays["video_rot"], mtf_level=port.scaled_mtf(1), cut=True, efm=True,
                              audio=port.audio, out_dtype=np.float32) for x in allblocks]
    keys = ("demod", "demod_05", "demod_burst")
    host = {k: np.concatenate([o["video"][k] for o in outs]) for k in keys}
    from ldgpu.fieldread import field_window
    start, prev, fields = 0.0, None, []
    while len(fields) < 2:
        w = field_window(port, start)
        if w.first_block + w.nblocks > NFIELD_BLOCKS:
            break
        sl = slice(w.startloc, w.startloc + w.length)
        f = FieldLogicNTSC(port, {"video": {k: v[sl] for k, v in host.items()}, "startloc": w.startloc},
                           prevfield=prev, fields_written=len(fields), readloc=w.startloc)
        f.process()
        if not f.valid:
            start += f.nextfieldoffset
            prev = None
            continue
        fields.append((host["demod"][sl], np.asarray(f.linelocs, np.float64), f.lineoffset))
        start += f.nextfieldoffset - (w.readloc - w.startloc)
        prev = f
    buf, ll, lineoffset = fields[-1]
    outw = port.SysParams["outlinelen"]
    outl = port.SysParams["frame_lines"] // 2 + 1
    coords, wow = otbc.pixel_coords(ll, port.linelen, outw, outl, lineoffset)
    lut = np.ascontiguousarray(port.downscale_sinc_lut, dtype=np.float32)
    buf32 = np.ascontiguousarray(buf, dtype=np.float32)
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    wow = np.ascontiguousarray(wow, dtype=np.float64)

    def ref_tbc():
        dsout = np.zeros(outl * outw, dtype=np.float32)
        refutils.scale_field(buf32, dsout, coords, wow, lut, lineoffset, outw)

    def port_tbc():
        otbc.scale_field(buf32, coords, wow, lut, lineoffset, outw, outl * outw)

    t_ref_tbc = best(ref_tbc)
    t_port_tbc = best(port_tbc)
    samples = NBLOCKS * U
    res = {
        "what": "one host thread each, same synthetic NTSC inputs; best of 3 after a warm-up",
        "demod": {"blocks": NBLOCKS, "reference_ms_per_block": 1e3 * t_ref_demod / NBLOCKS,
                  "port_ms_per_block": 1e3 * t_port_demod / NBLOCKS,
                  "reference_msps": samples / t_ref_demod / 1e6, "port_msps": samples / t_port_demod / 1e6,
                  "port_over_reference_speed": t_ref_demod / t_port_demod},
        "tbc": {"pixels": outl * outw, "reference_ms_per_field": 1e3 * t_ref_tbc,
                "port_ms_per_field": 1e3 * t_port_tbc, "port_over_reference_speed": t_ref_tbc / t_port_tbc},
    }
    print(json.dumps(res))


if __name__ == "__main__":
    main()
