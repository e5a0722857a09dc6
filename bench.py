#!/usr/bin/env python3
"""Throughput benchmark: RF demodulation + time-base correction on B200.

Workload (default): an NTSC 10 s capture -- 400 M int16 samples at 40 MSPS
from the seeded synthetic generator (ldgpu.synth), about 12.6 k overlap-save
blocks and 600 fields.  One step = every block of the capture through the
fused demodulator (all outputs: demod, demod_raw, demod_05, demod_burst,
rfhpf, EFM, analog audio stage 1), the line locations of every field (GPU
sync-run scan, native field chain, GPU H-sync / burst / pilot refinement)
and every field through the TBC (uint16 4fsc fields) and the analog audio
downscale (16-bit 44.1 kHz per field; --no-analog-audio leaves it out).
The step runs in
chunks of blocks (--chunks): while the GPU demodulates chunk c+1 (one CTA
per block, so other streams' kernels get SMs between blocks), the host walks
chunk c's fields and higher-priority streams scan, refine and resample them.
The timed steps run back to back on two device buffer sets (the same
capture in each), so one step's last line locations and TBC overlap the
next step's demodulation, as when decoding a stream of captures; each step
alone is reported too (isolated_step_ms).

Prints one JSON line (rank 0).  `--impl reference` times the CPU oracle (a
numpy restatement of the reference's demodblock + scale_field) on the host
cores instead, on a bounded sample of the same workload; its line locations
are computed outside its timed steps.

Multi-GPU (torchrun): each rank decodes its own capture (different seed);
no data-path collective; timing is the max over ranks.
"""

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, os.path.join(ROOT, "ld-decode_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402
from ldgpu.replicas import barrier as replica_barrier  # noqa: E402
from ldgpu.replicas import capture_seed, dist_env, max_over_ranks  # noqa: E402

METRIC = "RF MSPS demod+TBC on 1 B200 (batched FP32 vs plain) + HBM roofline %"
# DRAM bytes (read + write) per block of the demod kernel, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of the NTSC 1 s case divided by
# its 1261 blocks; traffic scales with blocks.  NTSC only (PAL writes a fifth
# float32 output and was not captured).
DRAM_BYTES_PER_BLOCK = {"NTSC": 719_500}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ldgpu", choices=["ldgpu", "reference"])
    ap.add_argument("--system", default="NTSC", choices=["NTSC", "PAL"])
    ap.add_argument("--seconds", type=float, default=10.0)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true",
                    help="skip the CPU-baseline leg (and with it the accuracy check against the oracle)")
    ap.add_argument("--fft-variant", default="auto", choices=["auto", "stockham", "in_place"],
                    help="FFT decomposition of the demodulator; auto: autotune_demod picks it (and blocks per "
                         "CTA) on the capture's first blocks before the warm-up")
    ap.add_argument("--other-system-seconds", type=float, default=2.0,
                    help="also time a capture of this length of the other system (PAL for NTSC) in a "
                         "subprocess and report it under other_system (0: off)")
    ap.add_argument("--dropouts-per-field", type=float, default=4.0,
                    help="seeded disc dropouts (40-1200 samples of lost carrier) per field's worth of capture")
    ap.add_argument("--accuracy-fields", type=int, default=16,
                    help="fields spread over the capture that the CPU-baseline leg runs through the oracle")
    ap.add_argument("--chunks", type=int, default=4,
                    help="pipeline chunks of blocks per step (1: demod, then line locations, then TBC)")
    ap.add_argument("--chunk-taper", type=float, default=0.7,
                    help="chunk c gets a share of the blocks proportional to taper**c")
    ap.add_argument("--e2e-chunks", type=int, default=None,
                    help="end to end: pipeline chunks per step (default: --chunks)")
    ap.add_argument("--e2e-first", type=float, default=0.5,
                    help="end to end: the first chunk's share relative to the taper's (< 1: the first "
                         "demod starts sooner after the capture's copy begins)")
    ap.add_argument("--wow-interp", default="linear", choices=["linear", "quadratic", "cubic"],
                    help="Field.wow_interpolation_method of the TBC (the reference's default is linear)")
    ap.add_argument("--wow-smoothing", type=float, default=0.0,
                    help="Field.wow_level_adjust_smoothing of the TBC (0: off, the reference's default)")
    ap.add_argument("--no-analog-audio", action="store_true",
                    help="leave the 44.1 kHz analog audio of the fields out of the step")
    ap.add_argument("--e2e-efm", default="edges", choices=["edges", "samples"],
                    help="end to end, the EFM output crosses to the host as its zero crossings (what the EFM PLL "
                         "consumes, with each field's slice bounds) or as the int16 samples")
    ap.add_argument("--mixed-sub", type=int, default=8,
                    help="after the default step, a mixed batch of this many captures in a subprocess, reported "
                         "under mixed_batch (0: off)")
    ap.add_argument("--mixed", type=int, default=0,
                    help="mixed-batch workload instead: this many captures, lengths uniform in 0.5-8 s, "
                         "half NTSC / half PAL, own seed and SNR (30-45 dB) each")
    ap.add_argument("--locate-threads", type=int, default=4,
                    help="mixed batch: host threads locating the captures' lines")
    ap.add_argument("--mixed-pipeline", type=int, default=4,
                    help="mixed batch: groups of captures per wave whose line locations and TBC overlap the next "
                         "group's demodulation")
    ap.add_argument("--reserve-sms", type=int, default=40,
                    help="mixed batch, pipelined: SMs the group queues leave to the line-location and TBC kernels")
    ap.add_argument("--mixed-budget-gb", type=float, default=100.0,
                    help="device memory per wave of the mixed batch (inputs + demodulator outputs)")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during timing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if not self.proc:
            return out
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if sm:
            out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                   "samples": len(sm)}
        return out


def run_gpu(args):
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from ldgpu import RFDecode
    from ldgpu import lib as L
    from ldgpu.field import tbc_fields, tbc_status
    from ldgpu.fieldread import blocks_in_capture
    from ldgpu.audio import downscale_audio_located
    from ldgpu.lines import LineLocator, field_levels, tbc_batch
    from ldgpu.efm import EFM_PLL, efm_edges, field_efm_slices
    wow_opts = dict(wow_interpolation_method=args.wow_interp, wow_smoothing=args.wow_smoothing)
    from ldgpu.synth import inject_dropouts, synth_capture

    system = args.system
    rf = RFDecode(system=system, decode_analog_audio=44100, decode_digital_audio=True, device=local)
    N = rf.blocklen
    U = N - rf.blockcut - rf.blockcut_end
    nsamples = int(args.seconds * rf.freq_hz)
    nblocks = blocks_in_capture(rf, nsamples)
    nout = nblocks * U
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream

    cap = synth_capture(system, nsamples, seed=capture_seed(args.seed, rank), device="cuda")
    # seeded disc dropouts (carrier lost for 40-1200 samples), so the dropout
    # detection and the line locations meet them as in a real capture
    ndrop = int(round(args.dropouts_per_field * nsamples * rf.SysParams["FPS"] * 2 / rf.freq_hz))
    drop_spans = inject_dropouts(cap, capture_seed(args.seed, rank) + 7919, ndrop) if ndrop else []
    keys = ["demod", "demod_raw", "demod_05", "demod_burst"] + (["demod_pilot"] if system == "PAL" else [])
    outs = {k: torch.empty(nout, dtype=torch.float32, device="cuda") for k in keys}
    outs["rfhpf"] = torch.empty(nout, dtype=torch.float32, device="cuda")
    outs["efm"] = torch.empty(nout, dtype=torch.int16, device="cuda")
    outs["audio_left"] = torch.empty(nblocks * 991, dtype=torch.float32, device="cuda")
    outs["audio_right"] = torch.empty(nblocks * 991, dtype=torch.float32, device="cuda")
    ptrs = {k: v.data_ptr() for k, v in outs.items()}
    import types

    # FFT decomposition and blocks per CTA: fixed, or timed on the capture's first blocks
    tune = None
    if args.fft_variant == "auto":
        from ldgpu.batch import autotune_demod
        nt = min(nblocks, 16 * torch.cuda.get_device_properties(local).multi_processor_count)
        tune = autotune_demod(rf, cap.data_ptr(), nt, U, ptrs, mtf_level=1, stream=stream)
    else:
        rf.fft_variant = {"stockham": 0, "in_place": 1}[args.fft_variant]

    def demod():
        rf.demod_blocks_device(cap.data_ptr(), nblocks, U, ptrs, mtf_level=1, stream=sh)

    # ---- the step, pipelined in chunks of blocks: the GPU demodulates chunk
    # c+1 (stream A) while the host walks chunk c's fields and stream B
    # (higher priority) scans, refines and resamples them
    fkeys = ["demod", "demod_05", "demod_burst"] + (["demod_pilot"] if system == "PAL" else [])
    farr = {k: outs[k] for k in fkeys}
    loc = LineLocator(rf)
    # one set of device buffers per step in flight: the end-to-end steps
    # alternate two sets, so a step's device->host copies overlap the next
    # step's input copy and demod (a set is reused once its copies are done)
    main = types.SimpleNamespace(cap=cap, outs=outs, ptrs=ptrs, farr=farr, loc=loc, pics=None, aud=None, done=None)

    def make_set():
        o = {k: torch.empty_like(v) for k, v in outs.items()}
        return types.SimpleNamespace(cap=torch.empty_like(cap), outs=o, ptrs={k: v.data_ptr() for k, v in o.items()},
                                     farr={k: o[k] for k in fkeys}, loc=LineLocator(rf), pics=None, aud=None,
                                     done=None)
    levels = field_levels(rf)
    lib = L.load()
    edges_mode = not args.no_e2e and args.e2e_efm == "edges"

    def chunk_plan(n, taper, first=1.0):
        """The step's chunks: chunk c holds a share proportional to taper**c
        of the blocks (the first's scaled by `first`) -- a smaller last chunk
        shortens the tail (its line locations and TBC) after the demod; end to
        end, the EFM output as its zero crossings: room per chunk for one
        crossing per 4 samples (band-limited EFM crosses every ~25)."""
        nonlocal nchunks, bounds, ecap, eoff
        nchunks = max(1, min(n, nblocks // 64))
        w = [taper ** c for c in range(nchunks)]
        w[0] *= first
        cum = np.concatenate([[0.0], np.cumsum(w)]) / sum(w)
        bounds = [int(round(x * nblocks)) for x in cum]
        ecap = np.array([(bounds[c + 1] - bounds[c]) * U // 4 for c in range(nchunks)], np.int64)
        eoff = np.concatenate([[0], np.cumsum(ecap)[:-1]]).astype(np.int64)

    nchunks = bounds = ecap = eoff = None
    chunk_plan(args.chunks, args.chunk_taper)
    streamB = torch.cuda.Stream(priority=-1)   # line locations
    streamC = torch.cuda.Stream(priority=-1)   # TBC of ranges whose line locations are final
    streamS = torch.cuda.Stream(priority=-1)   # sync-run scans
    # analog audio of finished ranges: high priority too, since the range's
    # copies out wait for it and the buffer set's next demod waits for those
    streamA = torch.cuda.Stream(priority=-1)
    # EFM zero crossings of each demodulated chunk (end to end): high priority
    # too -- at the demod's priority each of its three launches waited for a
    # whole demod chunk to be dispatched, and the step's end waits for them
    streamE = torch.cuda.Stream(priority=-1)
    do_audio = not args.no_analog_audio
    elem = {k: v.element_size() for k, v in outs.items()}
    per_block = {k: (991 if k.startswith("audio") else U) for k in outs}

    def demod_range(b0, b1, bs):
        o = {k: v + elem[k] * per_block[k] * b0 for k, v in bs.ptrs.items()}
        rf.demod_blocks_device(bs.cap.data_ptr() + 2 * b0 * U, b1 - b0, U, o, mtf_level=1, stream=sh)

    outlinelen = rf.SysParams["outlinelen"]
    outlines = rf.SysParams["frame_lines"] // 2 + 1
    fsz = outlinelen * outlines
    # analog audio of each field at 44.1 kHz (Field.downscale's dsaudio): one
    # fixed slot of AS int16 per field
    AS = 2 * 1024
    marks = {"audio_ranges": 0}

    streamH = torch.cuda.Stream()              # host -> device input copies (end to end)
    streamD = torch.cuda.Stream()              # device -> host EFM copies, chunk by chunk (end to end)
    streamP = torch.cuda.Stream()              # device -> host picture / audio copies of finished field ranges

    streamJ = torch.cuda.Stream()              # joins a step's streams for its end event (overlapped steps)

    def copy_in(io, bs):
        """Every chunk's host -> device input copy of a step on buffer set
        bs (stream H, once the set's previous demod has read its input);
        returns the per-chunk events."""
        if getattr(bs, "demod_done", None) is not None:
            streamH.wait_event(bs.demod_done)
        hevs = []
        for c in range(nchunks):
            # chunk c's blocks read [b0*U, b1*U + N - U); the previous chunk already copied up to b0*U + N - U
            a0 = bounds[c] * U + (N - U if c else 0)
            a1 = min(bounds[c + 1] * U + (N - U), nsamples)
            with torch.cuda.stream(streamH):
                bs.cap[a0:a1].copy_(io["cap"][a0:a1], non_blocking=True)
                hev = torch.cuda.Event()
                hev.record(streamH)
            hevs.append(hev)
        return hevs

    def step(io=None, bs=None, overlap=False, next_in=None):
        """One pass over the capture with buffer set `bs` (default: the
        main set).  io: pinned host buffers; then each chunk's input is
        copied in before its demod (stream H) and each chunk's EFM/audio
        and each field range's pictures are copied out as soon as they are
        final (streams D, P).  next_in = (io, set) of the next step: its
        input copies are issued as soon as this step's demods are, so the
        next step's first chunk does not wait for the host to reach it."""
        bs = bs or main
        evs = step_start(io, bs)
        if next_in is not None:
            next_in[1].prefetched = copy_in(*next_in)
        return step_finish(io, bs, evs, overlap or io is not None)

    def steps_pipelined(n, ios=None):
        """n steps back to back on the two buffer sets, each step's input copy
        and demods issued before the host works through the step before it
        (its line locations, TBC and copies), so the GPU always has the
        next capture's demod queued."""
        sets_ = (main, alt)
        pend = step_start(ios[0] if ios else None, sets_[0])
        for k in range(n):
            nxt = step_start(ios[(k + 1) % 2] if ios else None, sets_[(k + 1) % 2]) if k + 1 < n else None
            step_finish(ios[k % 2] if ios else None, sets_[k % 2], pend, True)
            pend = nxt

    def step_start(io, bs):
        """A step's input copy (end to end) and demods; returns the chunks'
        demod events."""
        if bs.done is not None:
            # the set's previous step (its line locations, TBC and, end to
            # end, its copies to the host) must be done before its outputs
            # are refilled; its input may be refilled once that step's
            # demodulator has read it
            for e in bs.done:
                stream.wait_event(e)
            bs.done = None
        hevs = None
        if io is not None:
            hevs = bs.prefetched if getattr(bs, "prefetched", None) else copy_in(io, bs)
            bs.prefetched = None
        evs = []
        for c in range(nchunks):
            if hevs is not None:
                stream.wait_event(hevs[c])
            demod_range(bounds[c], bounds[c + 1], bs)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
            evs.append(ev)
            if io is not None and edges_mode:
                # the chunk's EFM zero crossings (stream E, beside the next
                # chunk's demod and off the sync-run scan's stream); the count
                # lands in pinned memory and is read when the copy is issued
                streamE.wait_event(ev)
                base = bounds[c] * U
                L.check(lib.ldg_efm_edges(bs.outs["efm"].data_ptr() + 2 * base, (bounds[c + 1] - bounds[c]) * U,
                                          1 if c else 0, base, bs.edges.data_ptr() + 8 * int(eoff[c]),
                                          int(ecap[c]), io["ecount"].data_ptr() + 8 * c, bs.escratch.data_ptr(),
                                          streamE.cuda_stream))
                eev = torch.cuda.Event()
                eev.record(streamE)
                bs.eevs[c] = eev
            if io is not None and not edges_mode:
                streamD.wait_event(ev)
                o0, o1 = bounds[c] * U, bounds[c + 1] * U
                with torch.cuda.stream(streamD):
                    io["efm"][o0:o1].copy_(bs.outs["efm"][o0:o1], non_blocking=True)
        marks["demod_end"] = evs[-1]
        bs.demod_done = evs[-1]
        if io is not None and edges_mode:
            # stream E holds the next step's crossings by the time this step
            # finishes: the set's reuse waits for its own only
            bs.edges_done = bs.eevs[-1]
        return evs

    def step_finish(io, bs, evs, overlap):
        """The rest of a step started by step_start: line locations chunk by
        chunk, TBC and audio of each finished range, the copies out."""
        loc = bs.loc
        loc.begin(bs.farr)
        pend_e = list(range(nchunks)) if io is not None and edges_mode else []

        def edges_out(block):
            # each chunk's crossings to the host once its count is known (in
            # chunk order; without blocking until the step's end)
            while pend_e:
                c_ = pend_e[0]
                eev = bs.eevs[c_]
                if not block and not eev.query():
                    return
                eev.synchronize()
                k = int(io["ecount"][c_])
                if k > ecap[c_]:
                    raise RuntimeError(f"chunk {c_}: {k} EFM crossings, room for {int(ecap[c_])}")
                io["ecounts"][c_] = k
                streamD.wait_event(eev)
                e0_, e1_ = 8 * int(eoff[c_]), 8 * (int(eoff[c_]) + k)
                with torch.cuda.stream(streamD):
                    io["edges"][e0_:e1_].copy_(bs.edges[e0_:e1_], non_blocking=True)
                pend_e.pop(0)

        for c in range(nchunks):
            streamB.wait_event(evs[c])
            streamS.wait_event(evs[c])
            loc.advance(bounds[c + 1], stream=streamB, scan_stream=streamS)
            edges_out(False)
            # TBC of each range of fields as its line locations become final
            # (stream C: overlaps the NTSC burst chain's next range and the demod)
            while loc.ready and bs.pics is not None:
                lo, hi, ev = loc.ready.pop(0)
                streamC.wait_event(ev)
                tbc_fields(rf, tbc_batch(rf, loc.fields, bs.outs["demod"].data_ptr(), bs.pics.data_ptr(), levels,
                                         first=lo, count=hi - lo, **wow_opts),
                           stream=streamC.cuda_stream, asynchronous=True)
                if do_audio:
                    # the same fields' analog audio, 16-bit 44.1 kHz (one launch)
                    streamA.wait_event(ev)
                    downscale_audio_located(rf, loc.fields, bs.outs["audio_left"], bs.outs["audio_right"], 44100,
                                            stream=streamA.cuda_stream, first=lo, count=hi - lo, out=bs.aud,
                                            stride=AS)
                    marks["audio_ranges"] += 1
                if io is not None:
                    # on their own stream, so that the next chunks' EFM copies do not
                    # queue behind copies that wait for the TBC
                    tev = torch.cuda.Event()
                    tev.record(streamC)
                    streamP.wait_event(tev)
                    if do_audio:
                        aev = torch.cuda.Event()
                        aev.record(streamA)
                        streamP.wait_event(aev)
                    with torch.cuda.stream(streamP):
                        io["pics"][lo * fsz:hi * fsz].copy_(bs.pics[lo * fsz:hi * fsz], non_blocking=True)
                        if do_audio:
                            io["aud"][lo * AS:hi * AS].copy_(bs.aud[lo * AS:hi * AS], non_blocking=True)
                    if edges_mode:
                        # each field's EFM slice for the PLL (its bounds and end samples),
                        # written by the kernel straight into pinned memory; on the TBC's
                        # high-priority stream, not among the copies, where it would wait
                        # for SMs behind the next chunk's demod and hold up the copies
                        field_efm_slices(loc.fields, bs.outs["efm"], lo, hi - lo, bounds=io["ebounds"][lo:hi],
                                         samples=io["esamples"][lo:hi], stream=streamC.cuda_stream)
        edges_out(True)
        end = torch.cuda.Event(enable_timing=True)
        if overlap:
            # the next step (on the other buffer set) starts its demod while
            # this step's line locations, TBC and copies finish
            bs.done = []
            for st_ in ([streamB, streamC, streamS, streamA] + ([streamD, streamP] if io is not None else [])):
                e = torch.cuda.Event()
                e.record(st_)
                bs.done.append(e)
                streamJ.wait_event(e)
            if io is not None and edges_mode:
                bs.done.append(bs.edges_done)
                streamJ.wait_event(bs.edges_done)
            end.record(streamJ)
        else:
            stream.wait_stream(streamB)
            stream.wait_stream(streamC)
            stream.wait_stream(streamS)
            stream.wait_stream(streamA)
            end.record(stream)
        marks["end"] = end
        return loc.fields

    flist = step()
    torch.cuda.synchronize()
    nf = len(flist)
    main.pics = torch.empty(nf * fsz, dtype=torch.uint16, device="cuda")
    main.aud = torch.zeros(nf * AS, dtype=torch.int16, device="cuda")
    pics = main.pics
    # the second buffer set (overlapped and end-to-end steps); its capture is
    # the same, copied once on the device
    alt = make_set()
    alt.cap.copy_(cap)
    alt.pics = torch.empty(nf * fsz, dtype=torch.uint16, device="cuda")
    alt.aud = torch.zeros(nf * AS, dtype=torch.int16, device="cuda")
    def edge_buffers():
        # the sets' crossing buffers for the current chunk plan
        for bs_ in (main, alt):
            bs_.edges = torch.empty(8 * int(ecap.sum()) if edges_mode else 8, dtype=torch.uint8, device="cuda")
            bs_.eevs = [None] * nchunks
            bs_.escratch = torch.empty(max(int(L.load().ldg_efm_edges_scratch_bytes((bounds[c + 1] - bounds[c]) * U))
                                           for c in range(nchunks)), dtype=torch.uint8, device="cuda")

    edge_buffers()

    def barrier():
        replica_barrier(world)

    for _ in range(args.warmup):
        assert len(step()) == nf
    torch.cuda.synchronize()
    # blocks per CTA for the step: the demodulator alone runs a little faster
    # with more blocks per CTA, but the pipelined step needs SMs released
    # between CTAs for the line-location and TBC kernels, so the step itself
    # (back to back on the two buffer sets) is timed under each
    step_tune = None
    if tune is not None:
        step_tune = {}
        for b in (1, 2, 4):
            rf.blocks_per_cta = b
            steps_pipelined(2)
            torch.cuda.synchronize()
            q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            q0.record(stream)
            steps_pipelined(4)
            for st_ in (streamB, streamC, streamS, streamA):
                stream.wait_stream(st_)
            q1.record(stream)
            torch.cuda.synchronize()
            step_tune[b] = q0.elapsed_time(q1) / 4
        rf.blocks_per_cta = min(step_tune, key=step_tune.get)
        steps_pipelined(2)
        torch.cuda.synchronize()
    loc.stats = {k: 0 for k in loc.stats}
    loc.timing = {}

    # ---- timed device-resident steps (line locations inside the step)
    t_start = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    t_demod, t_end = [], []
    clk = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clk.start()
    host_ms = []
    for k in range(args.steps):
        t_start[k].record(stream)
        h0 = time.perf_counter()
        step()
        host_ms.append((time.perf_counter() - h0) * 1e3)
        t_demod.append(marks["demod_end"])
        t_end.append(marks["end"])
    torch.cuda.synchronize()
    # the same steps back to back on the two buffer sets, each step's demod
    # starting while the previous step's line locations and TBC finish: the
    # throughput of a stream of captures (the reported value)
    steps_pipelined(2)
    torch.cuda.synchronize()
    assert len(main.loc.fields) == nf and len(alt.loc.fields) == nf
    barrier()
    o0, o1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    o0.record(stream)
    ar0 = marks["audio_ranges"]
    hw0 = time.perf_counter()
    steps_pipelined(args.steps)
    pipelined_host_ms = (time.perf_counter() - hw0) * 1e3 / args.steps
    audio_ranges = (marks["audio_ranges"] - ar0) / args.steps
    for st_ in (streamB, streamC, streamS, streamA):
        stream.wait_stream(st_)
    o1.record(stream)
    torch.cuda.synchronize()
    barrier()
    overlap_ms = max_over_ranks(o0.elapsed_time(o1), world, "cuda") / args.steps
    clocks = clk.stop()
    rf.demod_status()  # raises if any block was skipped
    tbc_status(rf)     # raises if a TBC tap fell outside its field buffer
    step_ms = [t_start[k].elapsed_time(t_end[k]) for k in range(args.steps)]
    demod_ms = [t_start[k].elapsed_time(t_demod[k]) for k in range(args.steps)]
    tail_ms = [t_demod[k].elapsed_time(t_end[k]) for k in range(args.steps)]
    segs = loc.stats["segments"] / args.steps
    total_ms = max_over_ranks(float(sum(step_ms)), world, "cuda")
    isolated_ms = total_ms / args.steps  # one step at a time (the diagnostics below)
    ms_per_step = overlap_ms             # steps back to back on two buffer sets
    flist = loc.fields
    fields = [(f.window, f.host_linelocs(), f.lineoffset, levels) for f in flist]
    # the threaded field chain against one sequential walk over the same runs (untimed)
    from ldgpu.lines import parallel_chain, run_chain
    runs = [a.copy() for a in loc.sync_runs(farr["demod_05"].data_ptr(), nout, sh)]
    p_plans, _, _ = parallel_chain(rf, runs, nblocks, None, loc.threads, max_plans=8192)
    s_plans, _, _ = run_chain(rf, runs, nblocks, None, max_plans=8192)
    chain_check = bool(p_plans.tobytes() == s_plans.tobytes())

    # ---- end to end: pinned host capture in, fields/efm/audio out
    e2e = None
    if not args.no_e2e:
        host_cap = cap.cpu().pin_memory()
        # end to end the chunks may differ: the first chunk's input copy
        # precedes any demod, so a smaller first chunk starts the pipeline sooner
        dr_plan = (nchunks, bounds, ecap, eoff)
        chunk_plan(args.e2e_chunks or args.chunks, args.chunk_taper, args.e2e_first)
        edge_buffers()

        def make_io():
            io = {"cap": host_cap,
                  "pics": torch.empty(nf * fsz, dtype=torch.uint16).pin_memory(),
                  "aud": torch.zeros(nf * AS, dtype=torch.int16).pin_memory()}
            if edges_mode:
                io.update({"edges": torch.empty(8 * int(ecap.sum()), dtype=torch.uint8).pin_memory(),
                           "ecount": torch.zeros(nchunks, dtype=torch.int64).pin_memory(),
                           "ecounts": [0] * nchunks,
                           "ebounds": torch.zeros((nf, 2), dtype=torch.int64).pin_memory(),
                           "esamples": torch.zeros((nf, 2), dtype=torch.int16).pin_memory()})
            else:
                io["efm"] = torch.empty(nout, dtype=torch.int16).pin_memory()
            return io
        sets, ios = [main, alt], [make_io(), make_io()]
        for k in range(2):  # warm the copy path on both sets
            assert len(step(ios[k], sets[k])) == nf
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record(stream)
        # each step's input copy and demods are issued before the host works
        # through the step before it (the first step's inside the timed region too)
        hw0 = time.perf_counter()
        steps_pipelined(args.steps, ios)
        e2e_host_ms = (time.perf_counter() - hw0) * 1e3 / args.steps
        stream.wait_stream(streamD)
        stream.wait_stream(streamP)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, "cuda")
        h2d = nsamples * 2
        last = ios[(args.steps - 1) % 2]
        efm_d2h = 8 * sum(last["ecounts"]) + nf * (16 + 4) if edges_mode else nout * 2
        d2h = nf * fsz * 2 + efm_d2h + (nf * AS * 2 if do_audio else 0)
        e2e = {"value": world * nout / (e2e_ms * 1e-3) / 1e6, "unit": "MSPS", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
               "path": "pinned host capture -> ldg_demod_blocks -> ldg_sync_runs + ldg_field_chain + "
                       "ldg_lines_refine -> ldg_tbc_fields + ldg_audio_downscale (+ ldg_efm_edges) -> host "
                       "fields, EFM, 44.1 kHz audio; per chunk, the input "
                       "copy and the output copies overlap the other chunks' work; two buffer sets, so a "
                       "step's output copies also overlap the next step"}
        # the end-to-end outputs of the last step equal the device-resident run's
        same = (torch.equal(last["pics"].view(torch.int16), pics.cpu().view(torch.int16)) and
                torch.equal(last["aud"], main.aud.cpu()))
        if edges_mode:
            # the crossings (chunk by chunk) equal those of the whole EFM array,
            # the slices those of the located fields, and the PLL run from them
            # the PLL run from the samples (first 32 fields)
            from ldgpu import lib as Lb
            got = np.concatenate([last["edges"][8 * int(eoff[c]):8 * (int(eoff[c]) + last["ecounts"][c])].numpy()
                                  for c in range(nchunks)]).view(Lb.EFM_EDGE_DTYPE)
            whole = efm_edges(outs["efm"])
            eb, es = field_efm_slices(main.loc.fields, outs["efm"])
            same = same and got.tobytes() == whole.tobytes() and torch.equal(last["ebounds"], eb.cpu()) and \
                torch.equal(last["esamples"], es.cpu())
            xs = outs["efm"].cpu().numpy()
            pa, pb = EFM_PLL(), EFM_PLL()
            pll_same, tvals = True, 0
            for i in range(min(32, nf)):
                lo_, hi_ = (int(v) for v in last["ebounds"][i])
                ta = pa.process(xs[lo_:hi_])
                tb = pb.process_edges(got, lo_, hi_, int(last["esamples"][i, 0]), int(last["esamples"][i, 1]))
                pll_same = pll_same and np.array_equal(ta, tb)
                tvals += len(ta)
            pll_same = pll_same and pa.state() == pb.state()
            e2e["efm"] = {"form": "zero crossings (ldg_efm_edges, 8 bytes each) + per-field slice bounds and end "
                                  "samples; the EFM PLL (ldg_efm_pll_process_edges) turns them into the reference's "
                                  "T-values without the samples",
                          "crossings_per_step": int(sum(last["ecounts"])),
                          "bytes_per_step": int(efm_d2h), "int16_samples_bytes": int(nout * 2),
                          "pll_from_crossings_equals_pll_from_samples": bool(pll_same),
                          "pll_fields_checked": min(32, nf), "t_values_checked": int(tvals)}
        else:
            same = same and torch.equal(last["efm"], outs["efm"].cpu())
        e2e["outputs_match"] = bool(same)
        # the PCIe floor: the step's copies alone, each direction and both at once
        def copies(h2d_on, d2h_on):
            q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            q0.record(stream)
            if h2d_on:
                with torch.cuda.stream(streamH):
                    main.cap.copy_(host_cap, non_blocking=True)
            if d2h_on:
                with torch.cuda.stream(streamD):
                    last["pics"].view(torch.int16).copy_(main.pics.view(torch.int16), non_blocking=True)
                    if edges_mode:
                        nb_ = 8 * sum(last["ecounts"])
                        last["edges"][:nb_].copy_(main.edges[:nb_], non_blocking=True)
                    else:
                        last["efm"].copy_(outs["efm"], non_blocking=True)
            stream.wait_stream(streamH)
            stream.wait_stream(streamD)
            q1.record(stream)
            torch.cuda.synchronize()
            return q0.elapsed_time(q1)
        copies(True, True)
        pcie = {"h2d_ms": copies(True, False), "d2h_ms": copies(False, True), "both_ms": copies(True, True)}
        pcie["h2d_gbs"] = h2d / pcie["h2d_ms"] / 1e6
        pcie["d2h_gbs"] = (nf * fsz * 2 + efm_d2h) / pcie["d2h_ms"] / 1e6
        e2e["pcie_alone"] = pcie
        e2e["host_ms_per_step"] = e2e_host_ms  # the host's own loop (it returns before the GPU finishes)
        e2e["chunks"] = {"n": nchunks, "taper": args.chunk_taper, "first_share": round(bounds[1] / nblocks, 3)}
        nchunks, bounds, ecap, eoff = dr_plan

    # ---- plain form: one demodblock() call per block through the Python API
    plain = None
    if rank == 0:
        hc = cap[: 64 * U + N].cpu().numpy()
        for b in range(3):
            rf.demodblock(data=hc[b * U:b * U + N], mtf_level=1, cut=True)
        t0 = time.perf_counter()
        nplain = 64
        for b in range(nplain):
            rf.demodblock(data=hc[b * U:b * U + N], mtf_level=1, cut=True)
        dt = time.perf_counter() - t0
        plain = {"value": nplain * U / dt / 1e6, "unit": "MSPS",
                 "form": "RFDecode.demodblock per block, host numpy in/out (DemodCache worker style)"}
        # DemodCache's pool (core.py:1165-1200): worker threads, one RFDecode
        # (context, stream) each, blocks handed out in turn
        from concurrent.futures import ThreadPoolExecutor
        nthr = 8
        workers = [RFDecode(system=system, decode_analog_audio=44100, decode_digital_audio=True, device=local)
                   for _ in range(nthr)]
        def run_worker(w):
            for b in range(w, nplain, nthr):
                workers[w].demodblock(data=hc[b * U:b * U + N], mtf_level=1, cut=True)
        with ThreadPoolExecutor(nthr) as ex:
            list(ex.map(run_worker, range(nthr)))  # warm-up
            t0 = time.perf_counter()
            list(ex.map(run_worker, range(nthr)))
            dt = time.perf_counter() - t0
        for w in workers:
            w.close()
        plain["threads"] = {"value": nplain * U / dt / 1e6, "unit": "MSPS", "threads": nthr,
                            "form": "the same calls from a pool of worker threads, one RFDecode each (DemodCache)"}

    # ---- roofline of the dominant kernel (demod)
    # ---- the kernels on their own (whole-capture launches, events on the launching stream)
    def timed(fn, reps=3):
        out = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            out.append(a.elapsed_time(b))
        return statistics.median(out)

    all_descs = tbc_batch(rf, flist, outs["demod"].data_ptr(), pics.data_ptr(), levels, **wow_opts)
    dmed = timed(demod)
    tbc_med = timed(lambda: tbc_fields(rf, all_descs, stream=sh))
    tbc_ms = [tbc_med]

    # dropout detection of every field (Field.dropout_detect; not part of the
    # step, which is demod + TBC): one ldg_dropouts launch
    from ldgpu.dropouts import detect_located
    drop_lists = detect_located(rf, flist, outs, stream=sh)
    drop_total = sum(len(d[0]) for d in drop_lists)
    from ldgpu import dropouts as LD
    a = flist.arrays()
    ddescs = [LD._field(*(outs[k].data_ptr() + 4 * int(a["startloc"][i]) for k in
                          ("demod", "demod_05", "demod_raw", "rfhpf")),
                        a["length"][i], int(a["linelocs_ptr"][i]), a["nlines"][i], a["lineoffset"][i],
                        a["linecount"][i], a["isfirst"][i], a["hsync_len"][i]) for i in range(nf)]
    darr = (L.DropoutField * nf)(*ddescs)
    dprm = LD.dropout_params(rf)
    d_drops = torch.empty(nf * LD.OUT_CAP * 3, dtype=torch.int32, device="cuda")
    d_counts = torch.empty(2 * nf, dtype=torch.int32, device="cuda")
    drop_med = timed(lambda: L.check(rf._ctx._lib.ldg_dropouts(rf._ctx.handle, ctypes.byref(dprm), darr, nf,
                                                               d_drops.data_ptr(), d_counts.data_ptr(), None, sh)))

    peak, peak_kind = peaks()
    # algorithmic bytes: the int16 input once, every output array once (NTSC:
    # 4 float32 video outputs + rfhpf + int16 EFM = 24 B per sample, PAL 28 B,
    # plus the two audio bands' 991 float32 per block)
    demod_bytes = nout * 2 + sum(v.numel() * v.element_size() for v in outs.values())
    achieved = demod_bytes / (dmed * 1e-3) / 1e9
    # TBC: uint16 field written + the demod span of the field read once
    tbc_bytes = nf * fsz * 2 + sum(int(ll[-1] - ll[0]) * 4 for (_, ll, _, _) in fields)
    traffic = DRAM_BYTES_PER_BLOCK[system] * nblocks if system in DRAM_BYTES_PER_BLOCK else None

    cpu = accuracy = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu, accuracy = cpu_baseline(rf, cap, outs, pics, flist, runs, levels, U, fsz, nfields=args.accuracy_fields,
                                     method=args.wow_interp, smoothing=args.wow_smoothing, drop_spans=drop_spans)

    # the other television system, recorded beside the headline: a short
    # PAL capture through the same step (its own process, after this one's
    # timing; no CPU leg and no end-to-end pass)
    other = None
    if rank == 0 and world == 1 and args.other_system_seconds > 0:
        osys = "PAL" if system == "NTSC" else "NTSC"
        cmd = [sys.executable, os.path.abspath(__file__), "--system", osys, "--seconds",
               str(args.other_system_seconds), "--steps", str(args.steps), "--warmup", str(args.warmup),
               "--no-cpu", "--no-e2e", "--other-system-seconds", "0", "--mixed-sub", "0", "--seed", str(args.seed)]
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
            line = [x for x in r.stdout.splitlines() if x.startswith("{")]
            o = json.loads(line[-1]) if r.returncode == 0 and line else None
            other = None if o is None else {
                "system": osys, "value": o["value"], "unit": o["unit"], "ms_per_step": o["ms_per_step"],
                "fields_per_s": o["fields_per_s"], "workload": o["config"]["workload"],
                "kernel_ms": {k: o["kernel_ms"][k] for k in ("demod_alone", "tbc_alone")},
                "roofline_frac": o["roofline"]["frac"], "command": " ".join(cmd[1:])}
            if other is None:
                other = {"system": osys, "error": (r.stderr or r.stdout)[-400:]}
        except Exception as e:  # noqa: BLE001
            other = {"system": osys, "error": str(e)[:400]}

    # the mixed-batch form (many captures of both systems through the device
    # work queue), a few captures in its own process, recorded beside the headline
    mixed = None
    if rank == 0 and world == 1 and args.mixed_sub > 0:
        cmd = [sys.executable, os.path.abspath(__file__), "--mixed", str(args.mixed_sub), "--steps", "2",
               "--warmup", "1", "--seed", str(args.seed)]
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
            line = [x for x in r.stdout.splitlines() if x.startswith("{")]
            o = json.loads(line[-1]) if r.returncode == 0 and line else None
            mixed = {"error": (r.stderr or r.stdout)[-400:]} if o is None else {
                "value": o["value"], "unit": o["unit"], "ms_per_step": o["ms_per_step"],
                "fields_per_s": o.get("fields_per_s"), "workload": o["config"].get("workload"),
                "command": " ".join(cmd[1:])}
        except Exception as e:  # noqa: BLE001
            mixed = {"error": str(e)[:400]}

    res = {
        "metric": METRIC,
        "value": world * nout / (ms_per_step * 1e-3) / 1e6,
        "unit": "MSPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded generator, ldgpu.synth)",
        "config": {
            "workload": f"{system} {args.seconds:g} s capture, {nsamples} int16 samples at 40 MSPS, "
                        f"{nblocks} blocks x 32768 (stride {U}), {nf} fields per GPU",
            "outputs": "demod, demod_raw, demod_05, demod_burst" + (", demod_pilot" if system == "PAL" else "")
                       + ", rfhpf, efm, audio L/R stage 1, uint16 TBC fields, 16-bit 44.1 kHz analog audio "
                         "per field",
            "linelocs": "in the step: GPU sync-run scan, native field chain, GPU H-sync/burst/pilot refinement "
                        f"(FP64); host time per step {statistics.median(host_ms):.1f} ms, overlapped with the GPU",
            "l2": "inputs (800 MB) and outputs (> 8 GB) exceed L2 each step; no flush",
            "parallelism": f"replicas x{world} (one capture per GPU)",
            "mtf_level": 1,
            "wow_interpolation_method": args.wow_interp,
            "wow_level_adjust_smoothing": args.wow_smoothing,
        },
        "fields_per_s": world * nf / (ms_per_step * 1e-3),
        "isolated_step_ms": isolated_ms,
        "host_ms_per_pipelined_step": pipelined_host_ms,
        "kernel_ms": {"demod_alone": dmed, "tbc_alone": tbc_med,
                      "step_demod_chunks_median": statistics.median(demod_ms),
                      "after_last_demod_median": statistics.median(tail_ms),
                      "note": f"{nchunks} chunks: line locations and TBC of chunk c overlap the demod of "
                              "chunk c+1; after_last_demod is the exposed tail of a step run alone "
                              "(isolated_step_ms); ms_per_step runs the steps back to back on two buffer sets, "
                              "each step's demods issued before the host works through the step before it, so a "
                              "step's tail overlaps the next step's demod"},
        "autotune": None if tune is None else {
            "best": {"fft": ("stockham", "in_place")[tune["best"][0]], "blocks_per_cta": tune["best"][1]},
            "step_ms_by_blocks_per_cta": step_tune,
            "step_blocks_per_cta": rf.blocks_per_cta,
            "ms": {f"{('stockham', 'in_place')[k[0]]}_bpc{k[1]}": v for k, v in tune["ms"].items()},
            "blocks": tune["blocks"],
            "swept": "FFT decomposition (Stockham / in-place Cooley-Tukey 16384-point transforms) x blocks per CTA, "
                     "ldg_demod_blocks on the capture's first blocks; one CTA per block (cluster size 1)"},
        "linelocs_host_ms": {k: v / args.steps for k, v in loc.timing.items()},
        "linelocs_chain": {"threads": loc.threads, "equals_sequential_walk": chain_check,
                           "segments": segs, "host_decoded": loc.stats["host"] / args.steps,
                           "prev_resolved": loc.stats["resolved"] / args.steps,
                           "prev_resolved_early": loc.stats["resolved_early"] / args.steps},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": "ldg::demod_ip_kernel" if rf.fft_variant == 1 else "ldg::demod_kernel",
                     "algorithmic_bytes_per_launch": demod_bytes},
        "tbc_roofline": {"achieved": tbc_bytes / (statistics.median(tbc_ms) * 1e-3) / 1e9, "unit": "GB/s"},
        "dropouts": {"ms_all_fields": drop_med, "us_per_field": 1e3 * drop_med / nf, "dropouts_found": drop_total,
                     "note": "ldg_dropouts over every field (Field.dropout_detect); outside the step"},
        "e2e": e2e,
        "plain": plain,
        "cpu_baseline": cpu,
        "accuracy": accuracy,
        "other_system": other,
        "mixed_batch": mixed,
        # per step: demod 1, sync runs 4, refine 3 (NTSC) / 1 (PAL) per segment, TBC 2
        "gpu_launches": int(args.steps * (nchunks * (1 + 2 + 2) + segs * (3 if system == "NTSC" else 1)
                                          + audio_ranges)),
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(res), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    rf.close()


def cpu_demod_sample(rfp, cap, blocks, U, threads, out_dtype=np.float32):
    """Oracle demod of `blocks` (list of block indices) with a thread pool."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import demod as odemod
    N = rfp.blocklen

    def one(b):
        return odemod.demodblock(cap[b * U:b * U + N], rfp.Filters, system=rfp.system, freq_hz=rfp.freq_hz,
                                 blockcut_end=rfp.blockcut_end, video_rot=rfp.delays["video_rot"],
                                 mtf_level=rfp.scaled_mtf(1), cut=True, efm=True, audio=rfp.audio,
                                 out_dtype=out_dtype)
    with ThreadPoolExecutor(threads) as ex:
        return list(ex.map(one, blocks))


def cpu_tbc_field(rfp, buf, ll, lineoffset, levels, method="linear", smoothing=0.0):
    """Oracle TBC of one field (FP64 coordinates): uint16 picture."""
    from oracle import tbc as otbc
    outw = rfp.SysParams["outlinelen"]
    outlines = rfp.SysParams["frame_lines"] // 2 + 1
    coords, wow = otbc.pixel_coords(ll, rfp.linelen, outw, outlines, lineoffset, method=method)
    ds = otbc.scale_field(buf, coords, wow, rfp.downscale_sinc_lut, lineoffset, outw, outlines * outw,
                          smoothing=smoothing)
    return otbc.hz_to_output(ds, levels[0], levels[1], levels[4], levels[2], levels[3])


def cpu_tbc_sample(rfp, outs_by_block, fields, U, first_block, method="linear", smoothing=0.0):
    demod = np.concatenate([o["video"]["demod"] for o in outs_by_block])
    n = 0
    for (w, ll, lineoffset, levels) in fields:
        lo = w.startloc - first_block * U
        if lo < 0 or lo + w.length > len(demod):
            continue
        cpu_tbc_field(rfp, demod[lo:lo + w.length], ll, lineoffset, levels, method, smoothing)
        n += 1
    return n


def _err_stats(got, want, scale=1.0):
    d = (np.asarray(got, dtype=np.float64) - np.asarray(want, dtype=np.float64)) * scale
    return {"rms": float(np.sqrt(np.mean(d * d))), "max": float(np.max(np.abs(d)))}


def cpu_baseline(rf, cap, outs, pics, flist, runs, levels, U, fsz, nfields=16, method="linear", smoothing=0.0,
                 drop_spans=()):
    """The CPU oracle on a bounded sample of the workload (all host threads),
    timed as the CPU baseline: `nfields` fields spread over the capture, each
    with the field before it, through the whole path -- demod of every block
    their reads cover, line locations (the host restatement of the
    reference's Field logic on the oracle's outputs) and TBC.

    The same oracle outputs then check the GPU's outputs of those blocks and
    fields (the accuracy block): per output the error of the float32 GPU
    value against the FP64 oracle, the TBC pictures against the FP64 oracle
    TBC in LSB, and the integer results of line location.  Inside a seeded
    dropout (no carrier: the analytic signal's phase is that of noise near
    zero amplitude, where float32 and FP64 rounding pick different phases)
    the output is noise in both; the error statistics are given both outside
    the dropouts (with a 1024-sample margin, the block filters' reach) and
    over all samples."""
    from ldgpu.linelocs import FieldLogicNTSC, FieldLogicPAL
    threads = os.cpu_count() or 1
    system = rf.system
    nf = len(flist)
    picks = sorted(set(int(x) for x in np.linspace(1, nf - 1, nfields)))
    wins = {i: flist[i].window for j in picks for i in (j - 1, j)}
    blocks = sorted({b for w in wins.values() for b in range(w.first_block, w.first_block + w.nblocks)})
    hi = (blocks[-1] + 1) * U + rf.blocklen
    hc = cap[:hi].cpu().numpy()
    keys = ["demod", "demod_05", "demod_burst"] + (["demod_pilot"] if system == "PAL" else [])
    cls = FieldLogicPAL if system == "PAL" else FieldLogicNTSC

    t0 = time.perf_counter()
    res = dict(zip(blocks, cpu_demod_sample(rf, hc, blocks, U, threads, out_dtype=np.float64)))
    t1 = time.perf_counter()
    located = {}
    for j in picks:
        prev = None
        for i in (j - 1, j):
            w = wins[i]
            bl = range(w.first_block, w.first_block + w.nblocks)
            video = {k: np.concatenate([res[b]["video"][k] for b in bl]).astype(np.float32) for k in keys}
            f = cls(rf, {"video": video, "startloc": w.startloc}, prevfield=prev, fields_written=i,
                    readloc=w.startloc)
            f.process()
            located[(j, i)] = (f, video["demod"])
            prev = f
    t2 = time.perf_counter()
    cpu_pics = {}
    for j in picks:
        f, demod = located[(j, j)]
        if f.valid:
            lv = (levels[0], levels[1], levels[2], f.out_scale, levels[4])
            cpu_pics[j] = cpu_tbc_field(rf, demod, np.asarray(f.linelocs, dtype=np.float64), f.lineoffset, lv,
                                        method, smoothing)
    t3 = time.perf_counter()
    cpu = {"value": len(blocks) * U / (t3 - t0) / 1e6, "unit": "MSPS", "cores": threads, "kind": "port",
           "sample": f"{len(picks)} fields spread over the capture, each with the field before it: demod of the "
                     f"{len(blocks)} blocks their reads cover ({len(blocks) * U} samples, counted once), their "
                     f"line locations (host restatement of the reference's Field logic) and TBC; demod "
                     f"{t1 - t0:.1f} s, line locations {t2 - t1:.1f} s, TBC {t3 - t2:.1f} s",
           "impl": "oracle/ numpy FP64 restatement of demodblock + scale_field; host Field logic"}

    # ---- accuracy of the GPU outputs against the FP64 oracle (untimed)
    ok = {k: outs[k] for k in keys + ["demod_raw", "rfhpf", "efm", "audio_left", "audio_right"]}
    sel = torch_index(blocks, U)
    # raw sample of each compared output sample, and whether it is clear of the dropouts
    raw = sel.cpu().numpy() + rf.blockcut
    clear = np.ones(len(raw), dtype=bool)
    margin = 1024
    if len(drop_spans):
        ds = np.array(drop_spans, dtype=np.int64)
        lo, hi = ds[:, 0] - margin, np.maximum.accumulate(ds[:, 0] + ds[:, 1] + margin)
        k = np.searchsorted(lo, raw, side="right") - 1
        clear = ~((k >= 0) & (raw < hi[np.maximum(k, 0)]))
    dem, dem_all = {}, {}
    for k in keys + ["demod_raw", "rfhpf"]:
        g = ok[k][sel].cpu().numpy()
        src = (lambda b: res[b]["rfhpf"]) if k == "rfhpf" else (lambda b, k=k: res[b]["video"][k])
        w = np.concatenate([src(b) for b in blocks])
        dem[k] = _err_stats(g[clear], w[clear])
        dem_all[k] = _err_stats(g, w)
    pb = len(res[blocks[0]]["audio"]["audio_left"])
    asel = torch_index(blocks, pb)
    aud = {ch: _err_stats(ok["audio_" + ch][asel].cpu().numpy(),
                          np.concatenate([res[b]["audio"]["audio_" + ch] for b in blocks]))
           for ch in ("left", "right")}
    ge = ok["efm"][sel].cpu().numpy().astype(np.int64)[clear]
    we = np.concatenate([res[b]["efm"] for b in blocks]).astype(np.int64)[clear]
    lsb, lsb_clear = [], []
    for j, pic in cpu_pics.items():
        g = pics[j * fsz:(j + 1) * fsz].cpu().numpy().astype(np.int64)
        d = np.abs(g - pic.astype(np.int64))
        lsb.append(d)
        # output pixels whose input window is clear of the dropouts
        f, _ = located[(j, j)]
        w = flist[j].window
        from oracle import tbc as otbc
        outw = rf.SysParams["outlinelen"]
        outlines = rf.SysParams["frame_lines"] // 2 + 1
        coords, _ = otbc.pixel_coords(np.asarray(f.linelocs, dtype=np.float64), rf.linelen, outw, outlines,
                                      f.lineoffset, method="linear")
        c = coords[outw * (f.lineoffset + 1):outw * (f.lineoffset + 1) + fsz].astype(np.int64)
        praw = w.startloc + rf.blockcut + c
        pc = np.ones(len(praw), dtype=bool)
        if len(drop_spans):
            k = np.searchsorted(lo, praw, side="right") - 1
            pc = ~((k >= 0) & (praw < hi[np.maximum(k, 0)]))
        lsb_clear.append(d[pc])
    lsb = np.concatenate(lsb) if lsb else np.zeros(0, np.int64)
    lsb_clear = np.concatenate(lsb_clear) if lsb_clear else np.zeros(0, np.int64)

    def lsb_stats(x):
        if not len(x):
            return None
        return {"max": int(x.max()), "p99_99": float(np.percentile(x, 99.99)),
                "frac_within_1": float(np.mean(x <= 1)), "frac_exact": float(np.mean(x == 0)), "samples": len(x)}
    # integers: GPU line location against the host restatement on the oracle's outputs
    rs, rl = runs[0], runs[1]
    ints = {"linecount": True, "field_order": True, "lineoffset": True, "phase_id": True, "sync_pulses": True}
    for (j, i), (f, _) in located.items():
        gf = flist[i]
        if not f.valid:
            ints["linecount"] = False
            continue
        ints["linecount"] &= f.linecount == gf.linecount
        ints["field_order"] &= bool(f.isFirstField) == bool(gf.isFirstField)
        ints["lineoffset"] &= f.lineoffset == gf.lineoffset
        if i == j:
            ints["phase_id"] &= int(f.fieldPhaseID) == int(gf.fieldPhaseID)
        w = gf.window
        hp = [(p.start, p.len) for p in f.rawpulses if p.start > 0 and p.start + p.len < w.length - 1]
        m = (rs > w.startloc) & (rs + rl < w.startloc + w.length - 1)
        gp = list(zip((rs[m] - w.startloc).tolist(), rl[m].tolist()))
        ints["sync_pulses"] &= hp == gp
    acc = {
        "oracle": "FP64 numpy restatement of demodblock (core.py:755-879, complex128 FFTs) and of scale_field "
                  "without the float32 coordinate cast (utils.py:127-183); line locations by the host "
                  "restatement of the reference's Field logic on the oracle's outputs",
        "sample": f"{len(blocks)} blocks ({len(blocks) * U} samples) under {len(picks)} fields spread over the "
                  f"capture; TBC of {len(cpu_pics)} fields ({len(lsb)} samples)",
        "dropouts": f"{len(drop_spans)} seeded in the capture; 'demod_hz', 'efm' and 'tbc_lsb' exclude samples "
                    f"within {margin} samples of one ({int((~clear).sum())} of {len(clear)} compared demod "
                    "samples), the '_all' keys include them",
        "demod_hz": dem,
        "demod_hz_all": dem_all,
        "audio_stage1_hz": aud,
        "efm": {"max_abs": int(np.max(np.abs(ge - we))), "frac_exact": float(np.mean(ge == we))},
        "tbc_lsb": lsb_stats(lsb_clear),
        "tbc_lsb_all": lsb_stats(lsb),
        "integers_equal": dict(ints, all=all(ints.values()), fields=len(located)),
        "targets": "demod <= 1 kHz RMS; TBC within 1 LSB on >= 99.99 % of samples; integers bit-exact",
    }
    return cpu, acc


def torch_index(blocks, per):
    """Device index of the capture-wide samples of `blocks` (per samples each)."""
    import torch
    b = torch.as_tensor(blocks, dtype=torch.int64, device="cuda")
    return (b[:, None] * per + torch.arange(per, device="cuda")[None, :]).reshape(-1)


def run_reference(args):
    """CPU reference arm, rank 0 only: the oracle port of the reference's
    path on the host cores, each step one bounded sample of the workload
    through the same stages as the GPU step -- demod of every block of the
    sample (a thread pool, one worker per host thread, as DemodCache's
    workers), line locations of every field whose read lies in the sample
    (the host restatement of the reference's Field logic, field after field
    as LDdecode.readfield does) and TBC of each of them.  MSPS counts the
    input samples those fields cover (up to where the next field would
    start).  A single-thread step is reported beside it."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    from ldgpu.linelocs import FieldLogicNTSC, FieldLogicPAL
    from ldgpu.rfdecode import RFParams
    from ldgpu.synth import synth_capture

    rf = RFParams(system=args.system, decode_analog_audio=44100, decode_digital_audio=True)
    rf.delays = {"video_rot": 3}
    N = rf.blocklen
    U = N - rf.blockcut - rf.blockcut_end
    nblk = 100  # blocks per step (~3.2 M samples, 4 NTSC / 3 PAL fields whose reads fit)
    nsamples = (nblk - 1) * U + N
    cap = synth_capture(args.system, nsamples, seed=args.seed).numpy()
    cls = FieldLogicPAL if args.system == "PAL" else FieldLogicNTSC
    keys = ["demod", "demod_05", "demod_burst"] + (["demod_pilot"] if args.system == "PAL" else [])

    def one_step(threads):
        o = cpu_demod_sample(rf, cap, list(range(nblk)), U, threads)
        host = {k: np.concatenate([x["video"][k] for x in o]) for k in keys}
        fields, covered = _fields_cpu(rf, host, nblk, cls)
        for (w, ll, lineoffset, lv) in fields:
            cpu_tbc_field(rf, host["demod"][w.startloc:w.startloc + w.length], ll, lineoffset, lv,
                          args.wow_interp, args.wow_smoothing)
        return len(fields), covered

    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        one_step(threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        nft, covered = one_step(threads)
    dt = (time.perf_counter() - t0) / args.steps
    v = covered / dt / 1e6
    t0 = time.perf_counter()
    one_step(1)
    dt1 = time.perf_counter() - t0
    sample = (f"{nblk} blocks demod, line locations and TBC of the {nft} fields whose reads lie in them "
              f"({covered} input samples covered) per step")
    res = {"metric": METRIC, "value": v, "unit": "MSPS", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, ldgpu.synth)",
           "impl": "reference",
           "config": {"workload": f"{args.system} capture sample: {nblk} blocks x 32768 (stride {U}), "
                                  f"{nft} fields per step (bounded sample of the {args.seconds:g} s workload)",
                      "parallelism": f"{threads} host threads", "wow_interpolation_method": args.wow_interp,
                      "wow_level_adjust_smoothing": args.wow_smoothing},
           "cpu_baseline": {"value": v, "unit": "MSPS", "cores": threads, "kind": "port", "sample": sample},
           "single_thread": {"value": covered / dt1 / 1e6, "unit": "MSPS", "cores": 1, "ms_per_step": dt1 * 1e3},
           "e2e": {"value": v, "unit": "MSPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(res), flush=True)


def _fields_cpu(rf, host, nblocks, cls):
    """Every field whose read lies in the first `nblocks` blocks, located one
    after the other (LDdecode.readfield's walk); returns the fields and the
    input samples they cover (where the next field would start)."""
    from ldgpu.fieldread import field_window
    fields = []
    start = 0.0
    prev = None
    while True:
        w = field_window(rf, start)
        if w.first_block + w.nblocks > nblocks:
            break
        sl = slice(w.startloc, w.startloc + w.length)
        f = cls(rf, {"video": {k: v[sl] for k, v in host.items()}, "startloc": w.startloc},
                prevfield=prev, fields_written=len(fields), readloc=w.startloc)
        f.process()
        if not f.valid:
            start += f.nextfieldoffset
            prev = None
            continue
        lv = (rf.DecoderParams["ire0"], rf.DecoderParams["hz_ire"], rf.DecoderParams["vsync_ire"],
              f.out_scale, rf.SysParams["outputZero"])
        fields.append((w, np.asarray(f.linelocs, dtype=np.float64), f.lineoffset, lv))
        start += f.nextfieldoffset - (w.readloc - w.startloc)
        prev = f
    return fields, int(start)


def mixed_plan(seed, n):
    """(system, samples, seed, snr_db) per capture of the mixed batch."""
    rng = np.random.default_rng(seed)
    secs = rng.uniform(0.5, 8.0, n)
    systems = ["NTSC"] * (n // 2) + ["PAL"] * (n - n // 2)
    rng.shuffle(systems)
    snr = rng.uniform(30.0, 45.0, n)
    seeds = rng.integers(1, 2**31 - 1, n)
    return [(systems[i], int(secs[i] * 40e6), int(seeds[i]), float(snr[i])) for i in range(n)]


def run_mixed(args):
    """Mixed batch: every block of every capture of a wave in one persistent
    demodulator launch from the device work queue (CUDA graph), line
    locations per capture, one TBC launch per wave.  One step = one pass over
    every wave; the captures are regenerated per wave (untimed), so a step's
    time is the sum of its waves' timed passes."""
    import torch
    import torch.distributed as dist
    from ldgpu import RFDecode
    from ldgpu.batch import DemodQueue, MixedBatch, autotune, output_bytes_per_sample, waves
    from ldgpu.field import tbc_status
    from ldgpu.synth import synth_capture

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    plan = mixed_plan(capture_seed(args.seed, rank), args.mixed)
    groups = waves([p[1] for p in plan], [p[0] for p in plan], args.mixed_budget_gb * 1e9)
    rfs = {s: RFDecode(system=s, decode_analog_audio=44100, decode_digital_audio=True, device=local)
           for s in ("NTSC", "PAL")}
    queue = DemodQueue(local)
    loc_rfs = []  # per locate thread {system: RFDecode}, kept across waves
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    tune = None
    wave_ms, demod_ms, samples, fields, launches = [], [], 0, 0, 0
    clk = Clocks(local)
    gen_s = 0.0
    for gi, g in enumerate(groups):
        t0 = time.perf_counter()
        caps = [(plan[i][0], synth_capture(plan[i][0], plan[i][1], seed=plan[i][2], snr_db=plan[i][3],
                                           start=plan[i][2] % 1000003, device="cuda")) for i in g]
        torch.cuda.synchronize()
        gen_s += time.perf_counter() - t0
        mb = MixedBatch(caps, device=local, rfs=rfs, queue=queue, locate_threads=args.locate_threads,
                        locate_rfs=loc_rfs, pipeline=args.mixed_pipeline, reserve_sms=args.reserve_sms)
        st = mb.stream
        if tune is None:
            tune = autotune(queue, st, grabs=(1, 2, 4, 8), ctas=(0, 2 * sms), reps=2, variants=(0, 1))
        for _ in range(args.warmup):
            mb.run()
        torch.cuda.synchronize()
        # the queue launch alone (graph replay), then the whole path
        d = []
        for _ in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            mb.demod()
            b.record(st)
            b.synchronize()
            d.append(a.elapsed_time(b))
        demod_ms.append(statistics.median(d))
        replica_barrier(world)
        torch.cuda.synchronize()
        if gi == 0:
            clk.start()
        for loc in mb.locators:
            loc.stats = {k: 0 for k in loc.stats}
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        for _ in range(args.steps):
            nf = mb.run()
        b.record(st)
        torch.cuda.synchronize()
        replica_barrier(world)
        tbc_status(mb.rfs[mb.captures[0][0]])
        wave_ms.append(a.elapsed_time(b) / args.steps)
        samples += mb.samples
        fields += nf
        # per pass: the queue kernel, 4 sync-run kernels per capture, the TBC's 2;
        # refinement: 3 (NTSC) / 1 (PAL) per batched segment
        launches += args.steps * (1 + 4 * len(caps) + 2)
        for loc, (system, _) in zip(mb.locators, mb.captures):
            launches += loc.stats["segments"] * (3 if system == "NTSC" else 1)
        del mb, caps
        torch.cuda.empty_cache()
    clocks = clk.stop()
    step_ms = max_over_ranks(float(sum(wave_ms)), world, "cuda")
    dsum = sum(demod_ms)
    peak, peak_kind = peaks()
    nsys = {s: sum(1 for p in plan if p[0] == s) for s in ("NTSC", "PAL")}
    alg = sum(p[1] * output_bytes_per_sample(p[0]) for p in plan) + 2 * sum(p[1] for p in plan)
    res = {
        "metric": METRIC,
        "value": world * samples / (step_ms * 1e-3) / 1e6,
        "unit": "MSPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": step_ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded generator, ldgpu.synth)",
        "config": {
            "workload": f"mixed batch of {args.mixed} captures ({nsys['NTSC']} NTSC, {nsys['PAL']} PAL), lengths "
                        f"uniform in 0.5-8 s ({sum(p[1] for p in plan) / 40e6:.1f} s in all), SNR 30-45 dB, "
                        "own seed each",
            "waves": len(groups),
            "per_wave": f"{args.mixed_pipeline} groups of captures, one ldg_queue launch (CUDA graph) per group "
                        f"on {148 - args.reserve_sms} of the SMs; each group's line locations (on "
                        f"{args.locate_threads} host threads) and one TBC launch overlap the next group's demod",
            "l2": "inputs and outputs exceed L2 each pass; no flush",
            "parallelism": f"replicas x{world}",
            "mtf_level": 1,
        },
        "fields_per_s": world * fields / (step_ms * 1e-3),
        "fields": fields,
        "kernel_ms": {"queue_demod_alone_sum": dsum},
        "queue_demod_msps": samples / (dsum * 1e-3) / 1e6,
        "roofline": {"bound": "hbm", "achieved": alg / (dsum * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (dsum * 1e-3) / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                     "kernel": "ldg::demod_queue_kernel"},
        "autotune": {"best": {"grab": tune["best"][0], "ctas": tune["best"][1] or sms,
                              "fft": ("stockham", "in_place")[tune["best"][2]]},
                     "ms": {f"{('stockham', 'in_place')[k[2]]}_grab{k[0]}_ctas{k[1] or sms}": v
                            for k, v in tune["ms"].items()},
                     "swept": "FFT decomposition (Stockham / in-place Cooley-Tukey 16384-point transforms), blocks "
                              "per queue pop and persistent CTAs; one CTA per block (cluster size 1)"},
        "synth_s": gen_s,
        "gpu_launches": int(launches),
        "clocks": clocks,
        "e2e": None,
    }
    if rank == 0:
        print(json.dumps(res), flush=True)
    queue.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.mixed:
        run_mixed(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
