"""Host restatement of the reference's field sync / line-location logic.

Field.process() and its helpers (lddecode/core.py:1636-2589, 2754-2827,
2998-3047, 3053-3239, 3349-3495): sync-pulse detection on demod_05, the
vertical blanking state machine, line 0 and field parity, per-line H-sync
zero crossings, colour-burst (NTSC) / pilot (PAL) phase refinement and
bad-line repair.  It runs on the host in FP64 over the GPU-demodulated
field arrays.  The steps, thresholds and tie-breaking rules are the
reference's (they decide integer results: pulse positions, line count,
field order, phase ID), so the control flow follows it closely; numba
helpers of the reference are replaced by numpy with the same numeric
semantics (float64 means/medians of float32 data).
"""

from collections import namedtuple

import numpy as np

from .hostmath import calczc

Pulse = namedtuple("Pulse", "start len")

# vertical-blanking state machine states (core.py:1584)
HSYNC, EQPL1, VSYNC, EQPL2 = range(4)


def inrange(a, lo, hi):
    return (a >= lo) & (a <= hi)


def nround(x):
    return int(np.round(x))


def fmean(a):
    """Mean in float64 (numba's np.mean of float32 data accumulates in float64)."""
    return float(np.mean(np.asarray(a), dtype=np.float64))


def fmedian(a):
    return float(np.median(np.asarray(a)))


def frms(a):
    a = np.asarray(a, dtype=np.float64)
    return float(np.sqrt(np.mean(np.square(a - np.mean(a)))))


def find_pulses(sync_ref, high, min_len=0, max_len=5000):
    """Runs of samples <= high that end inside the array, as (start, len)
    pulses; a run starting at index 0 is dropped, as is a trailing run
    (utils.py:1101-1157)."""
    x = np.asarray(sync_ref)
    below = x.astype(np.float64) <= float(high)  # float32 samples vs a float64 level
    if len(x) < 2:
        return []
    b = below.astype(np.int8)
    d = np.diff(b)
    starts = np.nonzero(d == 1)[0] + 1
    ends = np.nonzero(d == -1)[0] + 1
    if below[0]:
        starts = np.concatenate([[0], starts])
    # pair each end with the run start before it
    n = min(len(starts), len(ends))
    starts, ends = starts[:n], ends[:n]
    lens = ends - starts
    keep = (starts != 0) & (lens >= min_len) & (lens <= max_len)
    return [Pulse(int(s), int(ln)) for s, ln in zip(starts[keep], lens[keep])]


def find_bursts(burstarea, threshold, bstart, s_rem, zcburstdiv, phase_adjust):
    """Zero crossings of a colour burst and the phase update they imply
    (utils.py:1339-1368, clb_findbursts).  Works on fixed 16-slot arrays
    like the reference, including the unused slots in the median and the
    rising count."""
    isrising = np.zeros(16, dtype=np.bool_)
    zcs = np.zeros(16, dtype=np.float32)
    zc_count = 0
    j = 0
    end = len(burstarea) - 1
    while j < end and zc_count < 16:
        if abs(float(burstarea[j])) > threshold:
            zc = calczc(burstarea, j, 0)
            if zc is None:
                break
            isrising[zc_count] = burstarea[j] < 0
            zcs[zc_count] = zc
            zc_count += 1
            j = int(zc) + 1
        else:
            j += 1
    rising_count = 0
    if zc_count:
        zc_cycles = ((bstart + zcs.astype(np.float64) - s_rem) / zcburstdiv) + phase_adjust
        zc_rounds = (zc_cycles + .5).astype(np.int32)
        phase_adjust += fmedian(zc_rounds - zc_cycles)
        rising_count = int(np.sum(np.bitwise_xor(isrising, (zc_rounds % 2) != 0)))
    return zc_count, phase_adjust, rising_count


def _angle_mean_phase(x, cycle_len=1.0):
    """Mean phase (0..1) of values taken modulo 1 (utils.py:1288-1301 and
    core.py:3085-3088)."""
    x = np.asarray(x, dtype=np.float64)
    x2 = x - x.astype(np.int32)
    angles = np.exp(1j * x2 * np.pi * 2 / cycle_len)
    am = np.angle(np.mean(angles)) / (np.pi * 2)
    return 1 + am if am < 0 else am


def phase_distance(x, c=0.75):
    """Shortest signed distance between phases x and c (utils.py:1305-1314)."""
    d = (x - np.floor(x)) - c
    if d < -0.5:
        d += 1
    elif d > 0.5:
        d -= 1
    return d


class FieldLogic:
    """Constructor and shared line-location logic (core.py:1587-2996)."""

    def __init__(self, rf, decode, prevfield=None, initphase=False, fields_written=0, readloc=0,
                 use_threads=True, wow_level_adjust_smoothing=0, wow_interpolation_method="linear"):
        self.rawdata = decode.get("input")
        self.data = decode
        self.initphase = initphase
        self.readloc = readloc
        self.prevfield = prevfield
        self.fields_written = fields_written
        self.rf = rf
        self.freq = rf.freq
        self.inlinelen = rf.linelen
        self.outlinelen = rf.SysParams["outlinelen"]
        self.lineoffset = 0
        self.needrerun = False
        self.valid = False
        self.sync_confidence = 100
        self.dspicture = None
        self.dsaudio = None
        self.interpolated_pixel_locs = None
        self.wowfactors = None
        self.outlinecount = (rf.SysParams["frame_lines"] // 2) + 1
        self.linecount = None
        self.use_threads = use_threads
        self.wow_level_adjust_smoothing = wow_level_adjust_smoothing
        self.wow_interpolation_method = wow_interpolation_method

    # ---- process

    def process(self):
        """core.py:1636-1653."""
        self.linelocs1, self.linebad, self.nextfieldoffset = self.compute_linelocs()
        if self.linelocs1 is None:
            if self.nextfieldoffset is None:
                self.nextfieldoffset = self.rf.linelen * 200
            return
        self.linebad = self.compute_deriv_error(self.linelocs1, self.linebad)
        self.linelocs2 = self.refine_linelocs_hsync()
        self.linebad = self.compute_deriv_error(self.linelocs2, self.linebad)
        self.linelocs = self.linelocs2
        self.valid = True

    # ---- unit conversions (core.py:1655-1712)

    def get_linelen(self, line=None, linelocs=None):
        if linelocs is None and hasattr(self, "linelocs"):
            linelocs = self.linelocs
        if line is None or linelocs is None:
            return self.rf.linelen
        if line >= self.linecount + self.lineoffset:
            length = (linelocs[line + 0] - linelocs[line - 1]) / 1
        elif line > 0:
            length = (linelocs[line + 1] - linelocs[line - 1]) / 2
        elif line == 0:
            length = (linelocs[line + 1] - linelocs[line - 0]) / 1
        if length <= 0:
            return self.rf.linelen
        return length

    def get_linefreq(self, line=None, linelocs=None):
        return self.rf.samplesperline * self.get_linelen(line, linelocs)

    def usectoinpx(self, x, line=None):
        return x * self.get_linefreq(line)

    def inpxtousec(self, x, line=None):
        return x / self.get_linefreq(line)

    def lineslice(self, l, begin=None, length=None, linelocs=None, begin_offset=0):
        l_adj = l + self.lineoffset
        _begin = linelocs[l_adj] if linelocs is not None else self.linelocs[l_adj]
        _begin += self.usectoinpx(begin, l_adj) if begin is not None else 0
        _length = length if length else self.rf.SysParams["line_period"]
        _length = self.usectoinpx(_length)
        return slice(int(_begin + begin_offset), int(_begin + _length + begin_offset + 1))

    def usectooutpx(self, x):
        return x * self.rf.SysParams["outfreq"]

    def outpxtousec(self, x):
        return x / self.rf.SysParams["outfreq"]

    def output_to_ire(self, output):
        return ((output - self.rf.SysParams["outputZero"]) / self.out_scale) + self.rf.DecoderParams["vsync_ire"]

    def lineslice_tbc(self, l, begin=None, length=None, linelocs=None, keepphase=False):
        _begin = self.rf.SysParams["outlinelen"] * (l - 1)
        begin_offset = self.usectooutpx(begin) if begin is not None else 0
        if keepphase:
            begin_offset = (begin_offset // 4) * 4
        _begin += begin_offset
        _length = self.usectooutpx(length) if length is not None else self.rf.SysParams["outlinelen"]
        return slice(nround(_begin), nround(_begin + _length))

    # ---- sync pulses (core.py:1760-2322)

    def get_timings(self):
        SP = self.rf.SysParams
        pulses = self.rawpulses
        hsync_typical = self.usectoinpx(SP["hsyncPulseUS"])
        lo = self.usectoinpx(SP["hsyncPulseUS"] - 1.75)
        hi = self.usectoinpx(SP["hsyncPulseUS"] + 2)
        hlens = [p.len for p in pulses if inrange(p.len, lo, hi)]
        LT = {}
        LT["hsync_median"] = np.median(hlens) if len(hlens) > 0 else SP["hsyncPulseUS"]
        LT["hsync"] = (LT["hsync_median"] + self.usectoinpx(-0.5), LT["hsync_median"] + self.usectoinpx(0.5))
        LT["hsync_offset"] = LT["hsync_median"] - hsync_typical
        LT["eq"] = (self.usectoinpx(SP["eqPulseUS"] - 0.5) + LT["hsync_offset"],
                    self.usectoinpx(SP["eqPulseUS"] + 0.5) + LT["hsync_offset"])
        LT["vsync"] = (self.usectoinpx(SP["vsyncPulseUS"] * 0.5) + LT["hsync_offset"],
                       self.usectoinpx(SP["vsyncPulseUS"] + 1) + LT["hsync_offset"])
        return LT

    def pulse_qualitycheck(self, prevpulse, pulse):
        if prevpulse[0] > 0 and pulse[0] > 0:
            exprange = (0.4, 0.6)
        elif prevpulse[0] == 0 and pulse[0] == 0:
            exprange = (0.9, 1.1)
        else:
            exprange = (0.4, 1.1)
        linelen = (pulse[1].start - prevpulse[1].start) / self.inlinelen
        return inrange(linelen, *exprange)

    def run_vblank_state_machine(self, pulses, LT):
        """Classify a run of pulses through EQ / VSYNC / EQ back to HSYNC
        (core.py:1825-1911).  Returns (done, [(state, pulse, good), ...])."""
        done = False
        vsyncs = []
        valid = []
        vsync_start = None
        state_end = 0
        state_length = None
        half = self.rf.SysParams["numPulses"] / 2
        for p in pulses:
            spulse = None
            state = valid[-1][0] if valid else -1
            is_h = inrange(p.len, *LT["hsync"])
            is_eq = inrange(p.len, *LT["eq"])
            is_v = inrange(p.len, *LT["vsync"])
            if state == -1:
                if is_h:
                    spulse = (HSYNC, p)
            elif state == HSYNC:
                if is_h:
                    spulse = (HSYNC, p)
                elif is_eq:
                    spulse = (EQPL1, p)
                    state_length = half
                elif is_v:
                    vsync_start = len(valid) - 1
                    spulse = (VSYNC, p)
            elif state == EQPL1:
                if is_eq:
                    spulse = (EQPL1, p)
                elif is_v:
                    vsync_start = len(valid) - 1
                    spulse = (VSYNC, p)
                    state_length = half
                elif is_h:
                    spulse = (HSYNC, p)
            elif state == VSYNC:
                if is_eq:
                    vsyncs.append((vsync_start, len(valid) - 1))
                    spulse = (EQPL2, p)
                    state_length = half
                elif is_v:
                    spulse = (VSYNC, p)
                elif p.start > state_end and is_h:
                    spulse = (HSYNC, p)
            elif state == EQPL2:
                if is_eq:
                    spulse = (EQPL2, p)
                elif is_h:
                    spulse = (HSYNC, p)
                    done = True
            if spulse is not None and spulse[0] != state:
                if spulse[1].start < state_end:
                    spulse = None
                elif state_length:
                    state_end = spulse[1].start + ((state_length - 0.1) * self.inlinelen)
                    state_length = None
            if spulse is not None:
                good = self.pulse_qualitycheck(valid[-1], spulse) if valid else False
                valid.append((spulse[0], spulse[1], good))
            if done:
                return done, valid
        return done, valid

    def refinepulses(self):
        """core.py:1913-1949."""
        self.LT = self.get_timings()
        i = 0
        valid = []
        raw = self.rawpulses
        while i < len(raw):
            cur = raw[i]
            if inrange(cur.len, *self.LT["hsync"]):
                good = self.pulse_qualitycheck(valid[-1], (0, cur)) if valid else False
                valid.append((HSYNC, cur, good))
                i += 1
            elif i > 2 and inrange(cur.len, *self.LT["eq"]) and (valid and valid[-1][0] == HSYNC):
                done, vblank = self.run_vblank_state_machine(raw[i - 2:i + 24], self.LT)
                if done:
                    valid.extend(vblank[2:])
                    i += len(vblank) - 2
                else:
                    i += 1
            else:
                i += 1
        return valid

    def getBlankRange(self, validpulses, start=0):
        """core.py:1951-1978."""
        vp_type = np.array([p[0] for p in validpulses])
        vs = np.where(vp_type[start:] == VSYNC)[0]
        firstvsync = vs[0] + start if len(vs) else None
        if firstvsync is None or firstvsync < 10:
            return None, None
        for newstart in range(firstvsync - 10, firstvsync - 4):
            blank = np.where(vp_type[newstart:] > 0)[0]
            if len(blank) == 0:
                continue
            firstblank = blank[0] + newstart
            hs = np.where(vp_type[firstblank:] == 0)[0]
            if len(hs) == 0:
                continue
            lastblank = hs[0] + firstblank - 1
            if (lastblank - firstblank) > 12:
                return firstblank, lastblank
        return None, None

    def getVBlankLength(self, isFirstField):
        core = self.rf.SysParams["numPulses"] * 3 * 0.5
        if self.rf.system == "NTSC":
            return core + 1
        return core + 0.5 + (0 if isFirstField else 1)

    def processVBlank(self, validpulses, start, limit=None):
        """Line 0 and field parity from one vertical blanking interval
        (core.py:1988-2088)."""
        firstblank, lastblank = self.getBlankRange(validpulses, start)
        lastvalid = len(validpulses) if limit is None else start + limit
        if firstblank is None or firstblank > lastvalid:
            return None, None, None, None
        SP = self.rf.SysParams
        loc_presync = validpulses[firstblank - 1][1].start
        pt = np.array([v[0] for v in validpulses[firstblank:]])
        pstart = np.array([v[1].start for v in validpulses[firstblank:]])
        plen = np.array([v[1].len for v in validpulses[firstblank:]])
        numPulses = SP["numPulses"]
        for i in (VSYNC, EQPL1, EQPL2):
            ptmatch = pt == i
            grouploc = None
            for j in range(0, lastblank - firstblank):
                if ptmatch[j:j + numPulses].all():
                    if ptmatch[j:j + numPulses + 4].sum() != numPulses:
                        break
                    gaps = np.diff(np.diff(pstart[j:j + numPulses]))
                    lengths = np.diff(plen[j:j + numPulses])
                    if np.max(gaps) < (self.rf.freq * 0.2) and np.max(lengths) < (self.rf.freq * 0.2):
                        grouploc = j
                        break
            if grouploc is None:
                continue
            firstloc = validpulses[firstblank + grouploc][1].start
            distfroml1 = ((i - 1) * numPulses) * 0.5
            dist = (firstloc - loc_presync) / self.inlinelen
            hdist = nround(dist * 2)
            isfirstfield = (hdist % 2) == (SP["firstFieldH"][1] != 1)
            if (distfroml1 * 2) % 2:
                isfirstfield = not isfirstfield
            eqgap = SP["firstFieldH"][isfirstfield]
            line0 = firstloc - ((eqgap + distfroml1) * self.inlinelen)
            return int(line0), isfirstfield, firstblank, 100

        if (validpulses[firstblank - 1][2] and validpulses[firstblank][2]
                and validpulses[lastblank][2] and validpulses[lastblank + 1][2]):
            gap1 = validpulses[firstblank][1].start - validpulses[firstblank - 1][1].start
            gap2 = validpulses[lastblank + 1][1].start - validpulses[lastblank][1].start
            if self.rf.system == "PAL" and inrange(np.abs(gap2 - gap1), 0, self.rf.freq * 1):
                isfirstfield = inrange((gap1 / self.inlinelen), 0.45, 0.55)
            elif self.rf.system == "NTSC" and inrange(np.abs(gap2 + gap1), self.inlinelen * 1.4,
                                                      self.inlinelen * 1.6):
                isfirstfield = inrange((gap1 / self.inlinelen), 0.95, 1.05)
            else:
                self.sync_confidence = 0
                return None, None, None, 0
            return validpulses[firstblank - 1][1].start, isfirstfield, firstblank, 50
        return None, None, None, 0

    def computeLineLen(self, validpulses):
        """Mean H-sync spacing over the longest run of HSYNC pulses
        (core.py:2090-2119)."""
        longrun = [-1, -1]
        currun = None
        for i, v in enumerate(p[0] for p in validpulses):
            if v != 0:
                if currun is not None and currun[1] > longrun[1]:
                    longrun = currun
                currun = None
            elif currun is None:
                currun = [i, 0]
            else:
                currun[1] += 1
        if currun is not None and currun[1] > longrun[1]:
            longrun = currun
        linelens = []
        for i in range(longrun[0] + 1, longrun[0] + longrun[1]):
            ll = validpulses[i][1].start - validpulses[i - 1][1].start
            if inrange(ll / self.inlinelen, 0.95, 1.05):
                linelens.append(ll)
        return np.mean(linelens) if linelens else self.inlinelen

    def skip_check(self):
        """Probability that a VSYNC follows this field (core.py:2122-2151)."""
        score = 0
        vsync_lines = 0
        vsync_ire = self.rf.DecoderParams["vsync_ire"]
        for l in range(self.outlinecount, self.outlinecount + 8):
            sl = self.lineslice(l, 0, self.rf.SysParams["line_period"])
            line_ire = self.rf.hztoire(fmedian(self.data["video"]["demod"][sl]))
            if inrange(line_ire, vsync_ire - 10, vsync_ire / 2):
                vsync_lines += 1
            elif inrange(line_ire, -5, 5):
                score += 1
            else:
                score -= 1
        if vsync_lines >= 2:
            return 100
        if vsync_lines == 1 and score > 0:
            return 50
        if score > 0:
            return 25
        return 0

    def getLine0(self, validpulses, meanlinelen):
        """Line 0 from this field's vblank, the next one and the previous
        field, voting by median when all three agree (core.py:2156-2239)."""
        self.sync_confidence = 100
        limit = 100 if (self.prevfield is not None and self.prevfield.skip_check() >= 50) else None
        l0_local, first_local, fb_local, conf_local = self.processVBlank(validpulses, 0, limit)
        l0_next, first_next, conf_next = None, None, None
        if l0_local is not None:
            self.vblank_next, notfirst_next, fb_next, conf_next = self.processVBlank(validpulses, fb_local + 40)
            if self.vblank_next is not None:
                first_next = not notfirst_next
                fieldlen = meanlinelen * self.rf.SysParams["field_lines"][0 if first_next else 1]
                l0_next = nround(self.vblank_next - fieldlen)
                if l0_next < 0:
                    self.sync_confidence = 10
        else:
            self.vblank_next = None
        l0_prev, first_prev = None, None
        if self.prevfield is not None and self.prevfield.valid:
            frameoffset = self.data["startloc"] - self.prevfield.data["startloc"]
            l0_prev = self.prevfield.linelocs[self.prevfield.linecount] - frameoffset
            first_prev = not self.prevfield.isFirstField
            conf_prev = self.prevfield.sync_confidence
        if l0_local is not None and l0_next is not None and l0_prev is not None:
            first_all = (first_local + first_prev + first_next) >= 2
            return np.median([l0_local, l0_next, l0_prev]), self.vblank_next, first_all
        if l0_local is not None and conf_local > 50:
            self.sync_confidence = min(self.sync_confidence, 90)
            return l0_local, self.vblank_next, first_local
        if l0_prev is not None:
            newconf = max(np.max(conf_prev - 10, 0), 10)
            self.sync_confidence = min(self.sync_confidence, newconf)
            return l0_prev, self.vblank_next, first_prev
        if l0_next is not None:
            self.sync_confidence = conf_next
            return l0_next, self.vblank_next, first_next
        return None, None, None

    def getpulses(self, do_retry=True):
        """Sync pulses of demod_05, re-levelled from the VSYNC and EQ pulse
        levels when the standard levels are off (core.py:2242-2322)."""
        rf = self.rf
        d05 = self.data["video"]["demod_05"]
        pulse_hz_max = rf.iretohz(-20)
        pulses = find_pulses(d05, pulse_hz_max)
        if len(pulses) == 0:
            if do_retry and not self.fields_written:
                rf.DecoderParams["ire0"] = np.percentile(d05, 15)
                return self.getpulses(do_retry=False)
            return pulses
        vsync_locs = []
        vsync_means = []
        minlength = self.usectoinpx(10)
        for i, p in enumerate(pulses):
            if p.len > minlength:
                vsync_locs.append(i)
                vsync_means.append(np.mean(d05[int(p.start + rf.freq):int(p.start + p.len - rf.freq)]))
        if len(vsync_means) == 0:
            return None
        synclevel = np.median(vsync_means)
        if np.abs(rf.hztoire(synclevel) - rf.DecoderParams["vsync_ire"]) < 5:
            return pulses
        black_means = []
        for i in list(range(vsync_locs[0] - 5, vsync_locs[0])) + list(range(vsync_locs[-1] + 1, vsync_locs[-1] + 6)):
            if i < 0 or i >= len(pulses):
                continue
            p = pulses[i]
            if inrange(p.len, rf.freq * 0.75, rf.freq * 2.5):
                black_means.append(np.mean(d05[int(p.start + (rf.freq * 5)):int(p.start + (rf.freq * 20))]))
        blacklevel = np.median(black_means)
        pulse_hz_max = (blacklevel + synclevel) / 2
        return find_pulses(d05, pulse_hz_max)

    # ---- line locations (core.py:2324-2589)

    def compute_linelocs(self):
        self.rawpulses = self.getpulses()
        if self.rawpulses is None or len(self.rawpulses) == 0:
            if self.fields_written:
                return None, None, None
            return None, None, int(self.rf.freq_hz)

        self.validpulses = validpulses = self.refinepulses()
        meanlinelen = self.computeLineLen(validpulses)
        line0loc, lastlineloc, self.isFirstField = self.getLine0(validpulses, meanlinelen)
        self.linecount = 263 if self.isFirstField else 262

        proclines = self.outlinecount + self.lineoffset + 10
        if self.rf.system == "PAL":
            proclines += 3

        if lastlineloc is not None:
            numlines = (lastlineloc - line0loc) / self.inlinelen
            self.skipdetected = numlines < (self.linecount - 5)
        else:
            self.skipdetected = False

        if line0loc is None:
            return None, None, self.inlinelen * 200

        lastline = (self.rawpulses[-1].start - line0loc) / meanlinelen
        if lastline < proclines:
            return None, None, line0loc - (meanlinelen * 20)

        ll_dict = {}
        ll_dist = {}
        for p in validpulses:
            lineloc = (p[1].start - line0loc) / meanlinelen
            rlineloc = nround(lineloc)
            dist = np.abs(lineloc - rlineloc)
            if self.skipdetected:
                lineloc_end = self.linecount - ((lastlineloc - p[1].start) / meanlinelen)
                rlineloc_end = nround(lineloc_end)
                dist_end = np.abs(lineloc_end - rlineloc_end)
                if p[0] == 0 and rlineloc > 23 and dist_end < dist:
                    lineloc = lineloc_end
                    rlineloc = rlineloc_end
                    dist = dist_end
            if dist > self.rf.hsync_tolerance or (rlineloc in ll_dict and dist > ll_dist[rlineloc]):
                continue
            if rlineloc > 0 and not p[2]:
                if p[0] > 0 or (p[0] == 0 and rlineloc < 10):
                    continue
            ll_dict[rlineloc] = p[1].start
            ll_dist[rlineloc] = dist

        rv_err = np.full(proclines, False)
        linelocs = [ll_dict[l] if l in ll_dict else -1 for l in range(0, proclines)]
        filled = linelocs.copy()
        self.linelocs0 = linelocs.copy()

        if filled[0] < 0:
            next_valid = None
            for i in range(0, self.outlinecount + 1):
                if linelocs[i] > 0:
                    next_valid = i
                    break
            if next_valid is None:
                return None, None, line0loc + (self.inlinelen * self.outlinecount - 7)
            filled[0] = filled[next_valid] - (next_valid * meanlinelen)
            if filled[0] < self.inlinelen:
                return None, None, line0loc + (self.inlinelen * self.outlinecount - 7)

        for l in range(1, proclines):
            if filled[l] < 0:
                rv_err[l] = True
                prev_valid = None
                next_valid = None
                for i in range(l, -1, -1):
                    if linelocs[i] > 0:
                        prev_valid = i
                        break
                for i in range(l, self.outlinecount + 1):
                    if linelocs[i] > 0:
                        next_valid = i
                        break
                if prev_valid is None:
                    filled[l] = linelocs[next_valid] - (self.inlinelen * (next_valid - l))
                elif next_valid is not None:
                    avglen = (linelocs[next_valid] - linelocs[prev_valid]) / (next_valid - prev_valid)
                    filled[l] = linelocs[prev_valid] + (avglen * (l - prev_valid))
                else:
                    filled[l] = linelocs[prev_valid] + (self.inlinelen * (l - prev_valid))

        rv_ll = [filled[l] for l in range(0, proclines)]
        if self.vblank_next is None:
            nextfield = filled[self.outlinecount - 7]
        else:
            nextfield = self.vblank_next - (self.inlinelen * 8)
        return rv_ll, rv_err, nextfield

    def refine_linelocs_hsync(self):
        """Sub-sample H-sync leading edges at the sync/porch mid level
        (core.py:2483-2551)."""
        rf = self.rf
        d05 = self.data["video"]["demod_05"]
        ll2 = self.linelocs1.copy()
        half_sync = rf.iretohz(rf.DecoderParams["vsync_ire"] / 2)
        lo_ok, hi_ok = rf.iretohz(-55), rf.iretohz(30)
        for i in range(len(self.linelocs1)):
            if inrange(i, 3, 6) or (rf.system == "PAL" and inrange(i, 1, 2)):
                self.linebad[i] = True
                continue
            ll1 = self.linelocs1[i] - rf.freq
            zc = calczc(d05, ll1, half_sync, reverse=False, count=rf.freq * 2)
            if zc is not None and not self.linebad[i]:
                ll2[i] = zc
                area = d05[int(zc - (rf.freq * 0.75)):int(zc + (rf.freq * 8))]
                if float(np.min(area)) < lo_ok or float(np.max(area)) > hi_ok:
                    self.linebad[i] = True
                    ll2[i] = self.linelocs1[i]
                else:
                    porch = fmedian(d05[int(zc + (rf.freq * 8)):int(zc + (rf.freq * 9))])
                    sync = fmedian(d05[int(zc + (rf.freq * 1)):int(zc + (rf.freq * 2.5))])
                    zc2 = calczc(d05, ll1, (porch + sync) / 2, reverse=False, count=400)
                    if zc2 is not None and np.abs(zc2 - zc) < (rf.freq / 2):
                        ll2[i] = zc2
                    else:
                        self.linebad[i] = True
            else:
                self.linebad[i] = True
            if self.linebad[i]:
                ll2[i] = self.linelocs1[i]
        return ll2

    def compute_deriv_error(self, linelocs, baserr):
        """Lines whose second difference exceeds 4 samples (core.py:2553-2564)."""
        d2 = np.abs(np.diff(np.diff(linelocs))) > 4
        e1 = np.full(len(linelocs), False)
        e1[1:-1] = d2
        e2 = np.full(len(linelocs), False)
        e2[2:] = d2
        return baserr | e1 | e2

    def fix_badlines(self, linelocs_in, linelocs_backup_in=None):
        """Interpolate bad lines from their good neighbours (core.py:2566-2589)."""
        self.linebad = self.compute_deriv_error(linelocs_in, self.linebad)
        linelocs = np.array(linelocs_in.copy())
        if linelocs_backup_in is not None:
            backup = np.array(linelocs_backup_in.copy())
            bad = np.isnan(linelocs)
            linelocs[bad] = backup[bad]
        firstcheck = 0 if self.rf.system == "PAL" else 1
        for l in np.where(self.linebad)[0]:
            prevgood = l - 1
            while prevgood >= 0 and self.linebad[prevgood]:
                prevgood -= 1
            nextgood = l + 1
            while nextgood < len(linelocs) and self.linebad[nextgood]:
                nextgood += 1
            if prevgood >= firstcheck and nextgood < (len(linelocs) + self.lineoffset):
                gap = (linelocs[nextgood] - linelocs[prevgood]) / (nextgood - prevgood)
                linelocs[l] = (gap * (l - prevgood)) + linelocs[prevgood]
        return linelocs

    # ---- field metadata used by process() (core.py:2754-2827)

    def decodephillipscode(self, linenum):
        """24-bit Philips VBI code of one line, or None (core.py:2754-2789)."""
        linestart = self.linelocs[linenum]
        data = self.data["video"]["demod"]
        level = self.rf.iretohz(50)
        curzc = calczc(data, int(linestart + self.usectoinpx(2)), level, count=int(self.usectoinpx(12)))
        zc = []
        while curzc is not None:
            zc.append((curzc, data[int(curzc - self.usectoinpx(0.5))] < level))
            curzc = calczc(data, curzc + self.usectoinpx(1.9), level, count=int(self.usectoinpx(0.2)))
        usecgap = self.inpxtousec(np.diff([z[0] for z in zc]))
        if len(zc) == 24 and np.min(usecgap) > 1.85 and np.max(usecgap) < 2.15:
            bits = [z[1] for z in zc]
            code = np.int64(0)
            for b in range(0, 24, 4):
                code *= 0x10
                code += (np.packbits(bits[b:b + 4]) >> 4)[0]
            return code
        return None

    def compute_syncconf(self):
        """core.py:2791-2806."""
        newconf = 100
        lld = np.diff(self.linelocs[self.lineoffset:self.lineoffset + self.linecount])
        lld2max = np.max(np.diff(lld))
        if lld2max > 4:
            newconf = int(50 - (5 * np.sum(lld2max > 4)))
        newconf = max(newconf, 0)
        self.sync_confidence = min(self.sync_confidence, newconf)
        return int(self.sync_confidence)

    def get_vsync_area(self):
        vsync_begin = int(self.linelocs[0])
        vsync_end_line = int(self.getVBlankLength(self.isFirstField) + 0.6)
        vsync_end = int(self.linelocs[vsync_end_line]) + 1
        return vsync_begin, vsync_end_line, vsync_end

    def get_vsync_lines(self):
        rv = list(range(1, 10 if self.isFirstField else 9))
        if self.rf.system == "PAL":
            rv.extend(range(311 if self.isFirstField else 310, 318))
        return rv

    def compute_line_bursts(self, linelocs, _line, prev_phaseadjust=0):
        """Colour-burst zero crossings of one line: (rising, phase adjust)
        (core.py:2998-3047)."""
        line = _line + self.lineoffset
        s = int(linelocs[line])
        s_rem = linelocs[line] - s
        lfreq = self.get_linefreq(line)
        fsc_inv = 1 / self.rf.SysParams["fsc_mhz"]
        bstart = int(21 * fsc_inv * lfreq)
        bend = int(28 * fsc_inv * lfreq)
        burstarea = self.data["video"]["demod_burst"][s + bstart:s + bend]
        if len(burstarea) == 0:
            return None, None
        burstarea = burstarea - fmean(burstarea)
        threshold = frms(burstarea)
        bd = self.data["video"]["demod"][s + bstart:s + bend]
        bd = bd - fmean(bd)
        if float(np.max(np.abs(bd))) > (30 * self.rf.DecoderParams["hz_ire"]):
            return None, None
        zcburstdiv = (lfreq * fsc_inv) / 2
        phase_adjust = -prev_phaseadjust
        for _ in range(2):
            zc_count, phase_adjust, rising_count = find_bursts(burstarea, threshold, bstart, s_rem,
                                                               zcburstdiv, phase_adjust)
        rising = rising_count > (zc_count / 2)
        return rising, -phase_adjust


class FieldLogicNTSC(FieldLogic):
    """NTSC colour-burst line refinement (core.py:3349-3495)."""

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.phase_adjust_median = 0
        self.out_scale = np.double(0xC800 - 0x0400) / (100 - self.rf.DecoderParams["vsync_ire"])

    def get_burstlevel(self, l, linelocs=None):
        area = self.data["video"]["demod"][self.lineslice(l, 5.5, 2.4, linelocs)]
        if len(area) == 0:
            return 0
        return frms(area) * np.sqrt(2)

    def compute_burst_offsets(self, linelocs):
        rising_sum = 0
        adjs = {}
        for l in range(0, 266):
            prev = self.phase_adjust_median
            if prev == 0 and self.prevfield:
                prev = self.prevfield.phase_adjust_median
            rising, pa = self.compute_line_bursts(linelocs, l, prev)
            if rising is None:
                continue
            adjs[l] = pa / 2
            if (not (l % 2)) and rising:
                rising_sum += 1
        field14 = rising_sum > (len(adjs.keys()) // 4)
        self.phase_adjust_median = np.median([adjs[a] for a in adjs]) * 2
        return field14, adjs

    def refine_linelocs_burst(self, linelocs=None):
        if linelocs is None:
            linelocs = self.linelocs2
        adj_ll = linelocs.copy()
        field14, adjs_new = self.compute_burst_offsets(adj_ll)
        adjs = {}
        for l in range(1, 266):
            if l not in adjs_new:
                self.linebad[l] = True
        for l in range(0, 266):
            if not (np.isnan(adj_ll[l]) or self.linebad[l]):
                lfreq = self.get_linefreq(l, linelocs)
                if l in adjs_new:
                    adjs[l] = adjs_new[l] * lfreq * (1 / self.rf.SysParams["fsc_mhz"])
        if len(adjs.keys()):
            med = np.median([adjs[a] for a in adjs])
            lastvalid = med
            for l in range(0, 266):
                if l in adjs and inrange(adjs[l] - med, -2, 2):
                    adj_ll[l] += adjs[l]
                    lastvalid = adjs[l]
                else:
                    adj_ll[l] += lastvalid
            map4 = {(True, True): 1, (False, False): 2, (True, False): 3, (False, True): 4}
            self.fieldPhaseID = map4[(self.isFirstField, field14)]
        else:
            self.fieldPhaseID = 1
        return adj_ll

    def calc_burstmedian(self):
        return np.median([self.get_burstlevel(l) for l in range(11, 264)]) / self.rf.DecoderParams["hz_ire"]

    def apply_offsets(self, linelocs, phaseoffset, picoffset=0):
        return np.array(linelocs) + picoffset + (phaseoffset * (self.rf.freq / (4 * 315 / 88)))

    def process(self):
        FieldLogic.process(self)
        self.out_scale = np.double(0xC800 - 0x0400) / (100 - self.rf.DecoderParams["vsync_ire"])
        if not self.valid:
            return
        self.linecode = [self.decodephillipscode(l + self.lineoffset) for l in (16, 17, 18)]
        self.linelocs3 = self.refine_linelocs_burst(self.linelocs2)
        self.linelocs4 = self.fix_badlines(self.linelocs3, self.linelocs2)
        self.burstmedian = self.calc_burstmedian()
        # subcarrier phase offset calibrated for ~147 degree output burst phase
        fsc_phase_deg = 117.25
        shift = (fsc_phase_deg / 360) / self.rf.SysParams["fsc_mhz"] * self.rf.freq
        self.linelocs = np.array(self.linelocs4) - shift


class FieldLogicPAL(FieldLogic):
    """PAL pilot line refinement and 8-field sequence (core.py:3053-3239)."""

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.out_scale = np.double(0xD300 - 0x0100) / (100 - self.rf.DecoderParams["vsync_ire"])

    def refine_linelocs_pilot(self, linelocs=None):
        linelocs = (self.linelocs2 if linelocs is None else linelocs).copy()
        plen = {}
        zcs = []
        pilot = self.data["video"]["demod_pilot"]
        for l in range(0, 323):
            adjfreq = self.rf.freq
            if l > 1:
                adjfreq /= (linelocs[l] - linelocs[l - 1]) / self.rf.linelen
            plen[l] = (adjfreq / self.rf.SysParams["pilot_mhz"]) / 2
            ls = self.lineslice(l, 0, 6, linelocs)
            lsoffset = linelocs[l] - ls.start
            pilots = pilot[ls]
            peakloc = np.argmax(np.abs(pilots))
            zc_base = calczc(pilots, peakloc, 0)
            if zc_base is not None:
                zc = (zc_base - lsoffset) / plen[l]
            else:
                zc = zcs[-1] if len(zcs) else 0
            zcs.append(zc)
        am = _angle_mean_phase(np.array(zcs))
        for l in range(0, 323):
            linelocs[l] += (phase_distance(zcs[l], am) * plen[l]) * 1
        return np.array(linelocs)

    def get_burstlevel(self, l, linelocs=None):
        area = self.data["video"]["demod"][self.lineslice(l, 5.5, 2.4, linelocs)].astype(np.float32).copy()
        area -= np.float32(fmean(area))
        if max(area) > (30 * self.rf.DecoderParams["hz_ire"]):
            return None
        return frms(area) * np.sqrt(2)

    def calc_burstmedian(self):
        levels = [b for b in (self.get_burstlevel(l) for l in range(11, 313)) if b is not None]
        if levels == []:
            return 0.0
        return np.median(levels) / self.rf.DecoderParams["hz_ire"]

    def get_following_field_number(self):
        if self.prevfield is not None:
            newphase = self.prevfield.fieldPhaseID + 1
            return 1 if newphase == 9 else newphase
        return 1

    def determine_field_number(self):
        """PAL 8-field sequence from line-6 burst presence and the burst phase
        of lines 7, 11, 15, 19 (core.py:3128-3203)."""
        map4 = {(True, False): 1, (False, True): 2, (True, True): 3, (False, False): 4}
        b6 = self.get_burstlevel(6)
        if b6 is None:
            return self.get_following_field_number()
        b6 /= self.rf.DecoderParams["hz_ire"]
        if inrange(b6, self.burstmedian * 0.8, self.burstmedian * 1.2):
            hasburst = True
        elif b6 < self.burstmedian * 0.2:
            hasburst = False
        else:
            return self.get_following_field_number()
        m4 = map4[(self.isFirstField, hasburst)]
        rcount = 0
        count = 0
        self.phase_adjust = {}
        for l in range(7, 22, 4):
            prev = 0
            try:
                if self.prevfield.phase_adjust[l] is not None:
                    prev = self.prevfield.phase_adjust[l]
            except AttributeError:
                pass
            rising, self.phase_adjust[l] = self.compute_line_bursts(self.linelocs, l, prev)
            if rising is not None:
                rcount += (rising is True)
                count += 1
        if count == 0 or (rcount * 2) == count:
            return self.get_following_field_number()
        is_firstfour = (rcount * 2) > count
        if m4 == 2:
            is_firstfour = not is_firstfour
        return m4 + (0 if is_firstfour else 4)

    def process(self):
        FieldLogic.process(self)
        self.out_scale = np.double(0xD300 - 0x0100) / (100 - self.rf.DecoderParams["vsync_ire"])
        if not self.valid:
            return
        self.linelocs3 = self.refine_linelocs_pilot(self.linelocs2)
        self.linelocs3a = self.refine_linelocs_pilot(self.linelocs3)
        self.linelocs = self.fix_badlines(self.linelocs3a)
        self.burstmedian = self.calc_burstmedian()
        self.linecount = 312 if self.isFirstField else 313
        self.lineoffset = 2 if self.isFirstField else 3
        self.linecode = [self.decodephillipscode(l + self.lineoffset) for l in (16, 17, 18)]
        self.fieldPhaseID = self.determine_field_number()
