"""Analog audio to 16-bit 44.1 kHz (or line-locked) output, per field.

Restates lddecode/core.py:1423-1580 (`_downscale_audio_compute_locs_and_swow`,
`_downscale_audio_to_output`, `downscale_audio`) and utils.py:1328-1332
(`dsa_rescale_and_clip`).  The work per field is ~1500 output samples, each
the mean of a ~28-sample run of the field's 1.25 MHz audio; it runs on the
host in FP64 numpy (vectorised; only the reference's 1.5 % wow clamp, which
depends on the previous clamped value, is a scalar scan, and only where a
jump exists).

Same call signature and results as the reference: int16 interleaved L/R,
negated (`-dsa_rescale_and_clip`), samples whose run falls outside the audio
muted to 0 with a warning, and the time offset for the next field.

`downscale_audio_located` does the same for every field of a batched
decode in one GPU launch (ldg_audio_downscale): each field's output clock
and A/V offset are scalars the host computes as the reference does (the
offset comes from the previous written field's position, not from the
previous field's audio, so the fields are independent).
"""

import ctypes
import logging

import numpy as np

logger = logging.getLogger("lddecode")


def compute_locs_and_swow(lineinfo, line_period, linelen, linecount, timeoffset, freq, scale):
    """core.py:1423-1490: (locs, swow, arange, frametime)."""
    if freq < 0:
        timeoffset = 0
        freq = (1000000 / line_period) * -freq
    frametime = linecount / (1000000 / line_period)
    soundgap = 1 / freq
    # the reference's compiled np.arange: ceil((stop - start) / step) ticks at
    # start + i * step (numpy's own arange steps by (start + step) - start)
    stop = frametime + (soundgap / 2)
    nticks = max(int(np.ceil((stop - timeoffset) / soundgap)), 0)
    arange = timeoffset + np.arange(nticks, dtype=np.float64) * soundgap

    li = np.asarray(lineinfo, dtype=np.float64)
    linenum = ((arange * 1000000) / line_period) + 1
    intlinenum = linenum.astype(np.int64)  # int() truncates toward zero
    cur = np.empty_like(linenum)
    nxt = np.empty_like(linenum)
    neg = linenum < 0
    inside = ~neg & (len(li) > linenum + 2)
    past = ~neg & ~inside
    if neg.any():
        c = (li[0] + (linelen * linenum[neg])).astype(np.int64).astype(np.float64)
        cur[neg] = c
        nxt[neg] = c + linelen
    if inside.any():
        k = intlinenum[inside]
        cur[inside] = li[k]
        nxt[inside] = li[k + 1]
    if past.any():
        cur[past] = li[-2]
        nxt[past] = li[-2] + linelen
    sampleloc = cur + (nxt - cur) * (linenum - np.floor(linenum))
    swow = (nxt - cur) / linelen
    swow = (swow - 1) + 1
    # no disc turns more than 1.5 % off speed: a jump larger than that keeps
    # the previous (already clamped) factor
    jumps = np.nonzero(np.abs(np.diff(swow)) > 0.015)[0]
    if len(jumps):
        for i in range(int(jumps[0]) + 1, len(swow)):
            if np.abs(swow[i] - swow[i - 1]) > 0.015:
                swow[i] = swow[i - 1]
    locs = sampleloc / scale
    return locs, swow, arange, frametime


def rescale_and_clip(x):
    """utils.py:1328-1332 over an array: round half to even, clip to +-32766."""
    v = np.round(np.asarray(x, dtype=np.float64) * 32767.0 / 371081.0)
    return np.clip(v, -32766, 32766).astype(np.int64)


def to_output(arange, locs, swow, audio_left, audio_right, audio_lfreq, audio_rfreq):
    """core.py:1493-1533: interleaved int16 L/R and whether any sample was
    muted.  Sample i is the mean of audio[int(locs[i]):int(locs[i+1])]."""
    n = len(arange) - 1
    out = np.zeros(2 * n, dtype=np.int16)
    if n <= 0:
        return out, False
    al = np.asarray(audio_left)
    ar = np.asarray(audio_right)
    start = locs[:-1].astype(np.int64)
    end = locs[1:].astype(np.int64)
    na = len(al)
    ok = (end > start) & (end < na)
    # the bounds of the slice audio[start:end] as numpy and numba take it: a
    # negative bound counts from the end, then clamps at 0
    s0 = np.where(start < 0, np.maximum(start + na, 0), start)
    e0 = np.where(end < 0, np.maximum(end + na, 0), end)
    # an empty slice (a run from before the buffer's start to after it) makes
    # the reference's compiled np.mean divide by zero, which raises; such a
    # sample is muted here like the other failed runs
    ok &= e0 > s0
    failed = not bool(ok.all())
    idx = np.nonzero(ok)[0]
    if len(idx):
        s, e = s0[idx], e0[idx]
        acc = al.dtype if al.dtype.kind == "f" else np.dtype(np.float64)
        ml = _run_means(al, s, e, acc)
        mr = _run_means(ar, s, e, acc)
        left = (ml * swow[idx]) - audio_lfreq
        right = (mr * swow[idx]) - audio_rfreq
        out[2 * idx] = -rescale_and_clip(left)
        out[2 * idx + 1] = -rescale_and_clip(right)
    return out, failed


def _run_means(a, s, e, acc):
    """Mean of a[s_i:e_i] for every run, each sum accumulated in order in the
    array's own precision (float32 audio sums in float32, as the reference's
    compiled np.mean does), vectorised across runs; the sum is divided by the
    run length in float64."""
    lens = e - s
    total = np.zeros(len(s), dtype=acc)
    for k in range(int(lens.max())):
        m = lens > k
        total[m] += a[s[m] + k].astype(acc, copy=False)
    return total.astype(np.float64) / lens


def downscale_audio(audio, lineinfo, rf, linecount, timeoffset=0, freq=44100, rv=None):
    """core.py:1538-1580: (int16 interleaved L/R, next field's time offset)."""
    locs, swow, arange, frametime = compute_locs_and_swow(
        lineinfo, rf.SysParams["line_period"], rf.linelen, linecount, timeoffset, freq,
        rf.Filters["audio_fdiv"])
    output16, failed = to_output(arange, locs, swow, audio["audio_left"], audio["audio_right"],
                                 rf.SysParams["audio_lfreq"], rf.SysParams["audio_rfreq"])
    if failed:
        logger.warning("Analog audio processing error, muting samples")
    if rv is not None:
        rv["dsaudio"] = output16
        rv["audio_next_offset"] = arange[-1] - frametime
    return output16, arange[-1] - frametime


def downscale_audio_gpu(audio, lineinfo, rf, linecount, timeoffset=0, freq=44100, rv=None):
    """downscale_audio (core.py:1538-1580) of one field on the GPU
    (ldg_audio_downscale, one CTA): the same int16 samples, mute warning and
    next-field offset as the host form."""
    import torch

    from . import lib as L
    sp = rf.SysParams
    off, soundgap, nticks, nxt = field_clock(sp["line_period"], linecount, timeoffset, freq)
    n_out = 2 * max(nticks - 1, 0)
    out16 = np.zeros(n_out, dtype=np.int16)
    if n_out:
        dev = torch.device("cuda", rf.device)
        al = torch.from_numpy(np.ascontiguousarray(audio["audio_left"], dtype=np.float32)).to(dev)
        ar = torch.from_numpy(np.ascontiguousarray(audio["audio_right"], dtype=np.float32)).to(dev)
        ll = torch.from_numpy(np.ascontiguousarray(lineinfo, dtype=np.float64)).to(dev)
        out = torch.empty(n_out, dtype=torch.int16, device=dev)
        muted = torch.zeros(1, dtype=torch.int32, device=dev)
        d = np.zeros(1, _AUDIO_DTYPE)
        d["audio_left"], d["audio_right"], d["audio_len"] = al.data_ptr(), ar.data_ptr(), len(al)
        d["linelocs"], d["nlines"], d["nticks"] = ll.data_ptr(), len(ll), nticks
        d["timeoffset"], d["soundgap"], d["out"] = off, soundgap, out.data_ptr()
        p = L.AudioParams(float(sp["line_period"]), float(rf.linelen), float(rf.Filters["audio_fdiv"]),
                          float(sp["audio_lfreq"]), float(sp["audio_rfreq"]))
        torch.cuda.current_stream(dev).synchronize()
        descs = (L.AudioField * 1).from_buffer_copy(d.tobytes())
        L.check(rf._ctx._lib.ldg_audio_downscale(rf._ctx.handle, descs, 1, ctypes.byref(p), muted.data_ptr(), 1))
        torch.cuda.synchronize(dev)
        out16 = out.cpu().numpy()
        if int(muted.item()):
            logger.warning("Analog audio processing error, muting samples")
    if rv is not None:
        rv["dsaudio"] = out16
        rv["audio_next_offset"] = nxt
    return out16, nxt


def av_offset(rf, readloc, is_first, audio, lastfieldwritten):
    """Field.downscale's A/V alignment offset of a field's first audio
    sample (core.py:2644-2670): from the last written field's number and
    read position; 0 without one or below 16 kHz."""
    if lastfieldwritten and audio >= 16000:
        sp = rf.SysParams
        rf_samples_per_field = rf.freq_hz / sp["FPS"] / 2
        read_gap = (readloc - lastfieldwritten[1]) / rf_samples_per_field
        field_number = int(np.round(lastfieldwritten[0] + read_gap))
        linecount = sum(sp["field_lines"]) * (field_number // 2)
        if not is_first:
            linecount += sp["field_lines"][0]
        samples_per_line = (sp["line_period"] / 1000000) / (1 / audio)
        cnt = linecount * samples_per_line
        frac = cnt - np.floor(cnt)
        return (1 - frac) * (1 / audio) if frac > .5 else -frac * (1 / audio)
    return 0


def field_clock(line_period, linecount, timeoffset, freq):
    """(timeoffset, soundgap, nticks, next field's offset) of a field's
    output clock, as compute_locs_and_swow sets it up (core.py:1445-1455)."""
    if freq < 0:
        timeoffset = 0
        freq = (1000000 / line_period) * -freq
    frametime = linecount / (1000000 / line_period)
    soundgap = 1 / freq
    stop = frametime + (soundgap / 2)
    nticks = max(int(np.ceil((stop - timeoffset) / soundgap)), 0)
    last = timeoffset + np.float64(nticks - 1) * soundgap
    return timeoffset, soundgap, nticks, last - frametime


def field_clocks(rf, startloc, isfirst, linecount, first, count, freq):
    """av_offset and field_clock for fields [first, first + count) of a
    decode whose field i follows lastfieldwritten = (i, startloc[i - 1]),
    as numpy arrays (the same double operations, element by element):
    (timeoffset, soundgap, nticks, next_offset)."""
    sp = rf.SysParams
    i = np.arange(first, first + count, dtype=np.int64)
    startloc = np.asarray(startloc, dtype=np.int64)
    isfirst = np.asarray(isfirst, dtype=bool)[first:first + count]
    linecount = np.asarray(linecount, dtype=np.int64)[first:first + count]
    off = np.zeros(count, dtype=np.float64)
    if freq >= 16000 and count:
        rf_samples_per_field = rf.freq_hz / sp["FPS"] / 2
        prev = startloc[np.maximum(i - 1, 0)]
        read_gap = (startloc[i] - prev) / rf_samples_per_field
        field_number = np.round(i + read_gap).astype(np.int64)
        lc = sum(sp["field_lines"]) * (field_number // 2) + np.where(isfirst, 0, sp["field_lines"][0])
        samples_per_line = (sp["line_period"] / 1000000) / (1 / freq)
        cnt = lc * samples_per_line
        frac = cnt - np.floor(cnt)
        off = np.where(frac > .5, (1 - frac) * (1 / freq), -frac * (1 / freq))
        off[i == 0] = 0
    if freq < 0:
        off = np.zeros(count, dtype=np.float64)
        freq = (1000000 / sp["line_period"]) * -freq
    frametime = linecount / (1000000 / sp["line_period"])
    soundgap = 1 / freq
    stop = frametime + (soundgap / 2)
    nticks = np.maximum(np.ceil((stop - off) / soundgap).astype(np.int64), 0)
    last = off + (nticks - 1).astype(np.float64) * soundgap
    return off, soundgap, nticks, last - frametime


def downscale_audio_located(rf, fields, audio_left, audio_right, freq=44100, stream=None, first=0, count=None,
                            out=None, stride=None, muted=None):
    """The analog audio of located fields on the GPU, one launch.

    `fields`: ldgpu.lines.LocatedFields (in decode order, all written);
    `audio_left` / `audio_right`: the capture-wide stage-1 audio (device
    float32 tensors, audio_fdiv-th of the demod rate per block, as
    demod_blocks_device writes it).  Field i is given lastfieldwritten =
    (i, startloc of field i - 1), as LDdecode.readfield passes it.  Fields
    [first, first + count) are done (default: all).

    Without `out`: returns (out, offsets, muted, next_offsets), `out` one
    device int16 tensor with field first + j's interleaved L/R samples (the
    reference's dsaudio) at out[offsets[j]:offsets[j+1]], `muted` a device
    int32 flag per field (a sample fell outside the audio and was muted),
    `next_offsets` the fields' audio_next_offset (host).  With `out` (device
    int16) and `stride`: field i's samples start at out[i * stride]; the
    offsets returned are those starts and ends; `muted` may be given (one
    int32 per field, indexed from `first`) or None."""
    import torch

    from . import lib as L
    a = fields.arrays()
    n_all = len(a["startloc"])
    count = n_all - first if count is None else count
    sp = rf.SysParams
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    scale = float(rf.Filters["audio_fdiv"])
    per_block = int(round(U / scale))
    off, soundgap, nticks, nxt = field_clocks(rf, a["startloc"], a["isfirst"], a["linecount"], first, count, freq)
    nsamp = 2 * np.maximum(nticks - 1, 0)
    if out is None:
        starts = np.concatenate([[0], np.cumsum(nsamp)[:-1]]).astype(np.int64) if count else np.zeros(0, np.int64)
        out = torch.empty(max(int(nsamp.sum()), 1), dtype=torch.int16, device=audio_left.device)
        ret_muted = muted = torch.zeros(max(count, 1), dtype=torch.int32, device=audio_left.device)
    else:
        if stride is None or (count and int(nsamp.max()) > stride):
            raise ValueError("stride must hold 2 * (nticks - 1) samples of every field")
        starts = np.arange(first, first + count, dtype=np.int64) * stride
        ret_muted = muted
    sel = slice(first, first + count)
    d = np.zeros(count, _AUDIO_DTYPE)
    fb = (np.asarray(a["startloc"][sel], dtype=np.int64) // U).astype(np.uint64)
    d["audio_left"] = np.uint64(audio_left.data_ptr()) + np.uint64(4 * per_block) * fb
    d["audio_right"] = np.uint64(audio_right.data_ptr()) + np.uint64(4 * per_block) * fb
    d["audio_len"] = (np.asarray(a["length"][sel], dtype=np.int64) // U) * per_block
    d["linelocs"] = np.asarray(a["linelocs_ptr"][sel], dtype=np.uint64)
    d["nlines"] = a["nlines"][sel]
    d["nticks"] = nticks
    d["timeoffset"] = off
    d["soundgap"] = soundgap
    d["out"] = np.uint64(out.data_ptr()) + np.uint64(2) * starts.astype(np.uint64)
    p = L.AudioParams(float(sp["line_period"]), float(rf.linelen), scale, float(sp["audio_lfreq"]),
                      float(sp["audio_rfreq"]))
    if count:
        descs = (L.AudioField * count).from_buffer_copy(d.tobytes())
        L.check(rf._ctx._lib.ldg_audio_downscale(rf._ctx.handle, descs, count, ctypes.byref(p),
                                                 muted.data_ptr() if muted is not None else None,
                                                 stream if stream else 1))
    return out, np.concatenate([starts, [starts[-1] + nsamp[-1]] if count else [0]]), ret_muted, nxt


def _audio_dtype():
    from . import lib as L
    fmt = {"audio_left": "u8", "audio_right": "u8", "audio_len": "i8", "linelocs": "u8", "nlines": "i4",
           "nticks": "i4", "timeoffset": "f8", "soundgap": "f8", "out": "u8"}
    names = [n for n, _ in L.AudioField._fields_]
    return np.dtype({"names": names, "formats": [fmt[k] for k in names],
                     "offsets": [getattr(L.AudioField, k).offset for k in names],
                     "itemsize": ctypes.sizeof(L.AudioField)})


_AUDIO_DTYPE = _audio_dtype()
