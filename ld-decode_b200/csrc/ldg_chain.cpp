// Field read chain and pulse-level line locations, on the host in FP64.
//
// Restates the part of Field.process() that works on sync pulses
// (lddecode/core.py:1760-2481): pulse timing classes (get_timings), the
// vertical-blanking state machine (run_vblank_state_machine, refinepulses),
// line 0 and field parity (getBlankRange, processVBlank, getLine0), mean
// line length (computeLineLen) and the integer-rounded line slots with gap
// filling (compute_linelocs), plus LDdecode.readfield's next-field offset
// (core.py:4090-4097) that walks field after field through a capture.
//
// The pulses themselves come from the GPU: runs of demod_05 at or below the
// sync threshold over the whole capture-wide output array, and the mean
// level inside every long run (ldg_sync_runs).  A field read window
// [startloc, startloc + length) sees the runs that start after its first
// sample and end before its last one, exactly the pulses findpulses
// (utils.py:1101-1157) finds in the window.
//
// Decisions that depend on the previous field's GPU-refined line locations
// (the line-0 vote of getLine0 when it can change the result, the
// skip_check limit of processVBlank) are detected instead of guessed: the
// field is retried with the range the previous field's pulse-level line
// locations put its refined line at, and only if that range leaves the
// result open does the chain stop before the field (LDG_CHAIN_STOP_PREV)
// for the caller to decode it with full information.  The same holds for the
// reference's level-recalibration branches of getpulses
// (LDG_CHAIN_STOP_LEVELS).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ldg_chain.h"

namespace {

enum { HSYNC = 0, EQPL1 = 1, VSYNC = 2, EQPL2 = 3 };

struct Pulse {
    long long start;
    long long len;
};

struct VPulse {
    int type;
    Pulse p;
    bool good;
};

inline bool inrange(double a, double lo, double hi) { return a >= lo && a <= hi; }

// numpy round-half-to-even of a double, as int
inline long long nround(double x) { return (long long)std::nearbyint(x); }

// np.median: the middle value, or the mean of the two middle values
double median_of(std::vector<double> v) {
    const size_t n = v.size();
    std::nth_element(v.begin(), v.begin() + n / 2, v.end());
    const double hi = v[n / 2];
    if (n % 2) return hi;
    const double lo = *std::max_element(v.begin(), v.begin() + n / 2);
    return (lo + hi) / 2.0;
}

struct Timings {
    double hsync_lo, hsync_hi, eq_lo, eq_hi, vsync_lo, vsync_hi;
    // the same ranges for integer pulse lengths: len >= lo <=> len >= ceil(lo)
    long long ih_lo, ih_hi, ieq_lo, ieq_hi, iv_lo, iv_hi;
    void integerise() {
        ih_lo = (long long)std::ceil(hsync_lo);
        ih_hi = (long long)std::floor(hsync_hi);
        ieq_lo = (long long)std::ceil(eq_lo);
        ieq_hi = (long long)std::floor(eq_hi);
        iv_lo = (long long)std::ceil(vsync_lo);
        iv_hi = (long long)std::floor(vsync_hi);
    }
    bool is_h(long long len) const { return len >= ih_lo && len <= ih_hi; }
    bool is_eq(long long len) const { return len >= ieq_lo && len <= ieq_hi; }
    bool is_v(long long len) const { return len >= iv_lo && len <= iv_hi; }
};

struct VBlank {
    bool ok = false;       // line0 found
    long long line0 = 0;
    bool isfirst = false;
    int firstblank = 0;
    int conf = 0;
    bool zeroed_conf = false;  // the branch that sets sync_confidence = 0
    bool operator==(const VBlank& o) const {
        return ok == o.ok && line0 == o.line0 && isfirst == o.isfirst && firstblank == o.firstblank &&
               conf == o.conf && zeroed_conf == o.zeroed_conf;
    }
};

// Integer spacing bounds equivalent to inrange(d / inlinelen, lo, hi) for
// integer d: d / L is monotonic in d, so the smallest d whose quotient
// reaches lo and the largest whose quotient stays <= hi decide it exactly.
struct SpacingBounds {
    long long lo, hi;
};

SpacingBounds spacing_bounds(double L, double lo, double hi) {
    long long a = (long long)std::floor(lo * L) - 2;
    while ((double)a / L < lo) ++a;
    while ((double)(a - 1) / L >= lo) --a;
    long long b = (long long)std::ceil(hi * L) + 2;
    while ((double)b / L > hi) --b;
    while ((double)(b + 1) / L <= hi) ++b;
    return {a, b};
}

class FieldPulses {
public:
    FieldPulses(const LdgChainParams& P, std::vector<Pulse> raw) : P(P), raw(std::move(raw)) {
        q_eq = spacing_bounds(P.inlinelen, 0.4, 0.6);
        q_h = spacing_bounds(P.inlinelen, 0.9, 1.1);
        q_mix = spacing_bounds(P.inlinelen, 0.4, 1.1);
    }

    double usectoinpx(double x) const { return x * P.linefreq0; }

    Timings get_timings() const {
        const double lo = usectoinpx(P.hsync_pulse_us - 1.75), hi = usectoinpx(P.hsync_pulse_us + 2);
        // integer lengths within [lo, hi]: len >= ceil(lo), len <= floor(hi)
        const long long ilo = (long long)std::ceil(lo), ihi = (long long)std::floor(hi);
        std::vector<long long> hl;
        hl.reserve(raw.size());
        for (const Pulse& p : raw)
            if (p.len >= ilo && p.len <= ihi) hl.push_back(p.len);
        double med = P.hsync_pulse_us;
        if (!hl.empty()) {
            const size_t n = hl.size();
            std::nth_element(hl.begin(), hl.begin() + n / 2, hl.end());
            const double h = (double)hl[n / 2];
            med = (n % 2) ? h : ((double)*std::max_element(hl.begin(), hl.begin() + n / 2) + h) / 2.0;
        }
        const double off = med - usectoinpx(P.hsync_pulse_us);
        Timings t;
        t.hsync_lo = med + usectoinpx(-0.5);
        t.hsync_hi = med + usectoinpx(0.5);
        t.eq_lo = usectoinpx(P.eq_pulse_us - 0.5) + off;
        t.eq_hi = usectoinpx(P.eq_pulse_us + 0.5) + off;
        t.vsync_lo = usectoinpx(P.vsync_pulse_us * 0.5) + off;
        t.vsync_hi = usectoinpx(P.vsync_pulse_us + 1) + off;
        t.integerise();
        return t;
    }

    // pulse_qualitycheck (core.py:1803-1823): the spacing to the previous
    // valid pulse, in lines, within 0.4-0.6 (both blanking pulses), 0.9-1.1
    // (both H-sync) or 0.4-1.1
    bool qualitycheck(const VPulse& prev, int type, const Pulse& p) const {
        const SpacingBounds& q = (prev.type > 0 && type > 0) ? q_eq : (prev.type == 0 && type == 0) ? q_h : q_mix;
        const long long d = p.start - prev.p.start;
        return d >= q.lo && d <= q.hi;
    }

    SpacingBounds q_eq, q_h, q_mix;

    // core.py:1825-1911
    bool vblank_state_machine(size_t from, size_t to, const Timings& LT, std::vector<VPulse>& valid) const {
        bool done = false;
        double state_end = 0;
        double state_length = 0;  // 0: None
        const double half = P.num_pulses / 2.0;
        for (size_t k = from; k < to; ++k) {
            const Pulse& p = raw[k];
            int stype = -1;
            const int state = valid.empty() ? -1 : valid.back().type;
            const bool is_h = LT.is_h(p.len);
            const bool is_eq = LT.is_eq(p.len);
            const bool is_v = LT.is_v(p.len);
            if (state == -1) {
                if (is_h) stype = HSYNC;
            } else if (state == HSYNC) {
                if (is_h) stype = HSYNC;
                else if (is_eq) {
                    stype = EQPL1;
                    state_length = half;
                } else if (is_v) stype = VSYNC;
            } else if (state == EQPL1) {
                if (is_eq) stype = EQPL1;
                else if (is_v) {
                    stype = VSYNC;
                    state_length = half;
                } else if (is_h) stype = HSYNC;
            } else if (state == VSYNC) {
                if (is_eq) {
                    stype = EQPL2;
                    state_length = half;
                } else if (is_v) stype = VSYNC;
                else if ((double)p.start > state_end && is_h) stype = HSYNC;
            } else if (state == EQPL2) {
                if (is_eq) stype = EQPL2;
                else if (is_h) {
                    stype = HSYNC;
                    done = true;
                }
            }
            if (stype >= 0 && stype != state) {
                if ((double)p.start < state_end) stype = -1;
                else if (state_length != 0) {
                    state_end = (double)p.start + (state_length - 0.1) * P.inlinelen;
                    state_length = 0;
                }
            }
            if (stype >= 0) {
                const bool good = valid.empty() ? false : qualitycheck(valid.back(), stype, p);
                valid.push_back({stype, p, good});
            }
            if (done) return true;
        }
        return done;
    }

    // core.py:1913-1949
    std::vector<VPulse> refinepulses(const Timings& LT) const {
        std::vector<VPulse> valid;
        valid.reserve(raw.size());
        size_t i = 0;
        while (i < raw.size()) {
            const Pulse& cur = raw[i];
            if (LT.is_h(cur.len)) {
                const bool good = valid.empty() ? false : qualitycheck(valid.back(), HSYNC, cur);
                valid.push_back({HSYNC, cur, good});
                i += 1;
            } else if (i > 2 && LT.is_eq(cur.len) && !valid.empty() &&
                       valid.back().type == HSYNC) {
                std::vector<VPulse> vb;
                vb.reserve(32);
                const bool done = vblank_state_machine(i - 2, std::min(raw.size(), i + 24), LT, vb);
                if (done) {
                    for (size_t k = 2; k < vb.size(); ++k) valid.push_back(vb[k]);
                    i += vb.size() - 2;
                } else {
                    i += 1;
                }
            } else {
                i += 1;
            }
        }
        return valid;
    }

    // core.py:1951-1978; returns false when no blanking range is found
    static bool blank_range(const std::vector<VPulse>& vp, int start, int& firstblank, int& lastblank) {
        const int n = (int)vp.size();
        int firstvsync = -1;
        for (int k = std::max(start, 0); k < n; ++k)
            if (vp[k].type == VSYNC) {
                firstvsync = k;
                break;
            }
        if (firstvsync < 0 || firstvsync < 10) return false;
        for (int newstart = firstvsync - 10; newstart < firstvsync - 4; ++newstart) {
            int fb = -1;
            for (int k = newstart; k < n; ++k)
                if (vp[k].type > 0) {
                    fb = k;
                    break;
                }
            if (fb < 0) continue;
            int hs = -1;
            for (int k = fb; k < n; ++k)
                if (vp[k].type == 0) {
                    hs = k;
                    break;
                }
            if (hs < 0) continue;
            const int lb = hs - 1;
            if (lb - fb > 12) {
                firstblank = fb;
                lastblank = lb;
                return true;
            }
        }
        return false;
    }

    // Python's negative-index wrap for validpulses[idx]
    static const VPulse& at(const std::vector<VPulse>& vp, int idx) {
        return vp[idx < 0 ? idx + (int)vp.size() : idx];
    }

    // core.py:1988-2088; limit < 0 means None
    VBlank process_vblank(const std::vector<VPulse>& vp, int start, int limit) const {
        VBlank r;
        int firstblank, lastblank;
        if (!blank_range(vp, start, firstblank, lastblank)) return r;
        const int lastvalid = limit < 0 ? (int)vp.size() : start + limit;
        if (firstblank > lastvalid) return r;
        const long long loc_presync = at(vp, firstblank - 1).p.start;
        const int n = (int)vp.size() - firstblank;
        const int np_ = P.num_pulses;
        const int order[3] = {VSYNC, EQPL1, EQPL2};
        for (int oi = 0; oi < 3; ++oi) {
            const int ty = order[oi];
            int grouploc = -1;
            for (int j = 0; j < lastblank - firstblank; ++j) {
                // ptmatch[j:j+numPulses].all(), slices truncated at the end
                bool all = true;
                for (int k = j; k < std::min(j + np_, n); ++k)
                    if (vp[firstblank + k].type != ty) {
                        all = false;
                        break;
                    }
                if (!all) continue;
                int cnt = 0;
                for (int k = j; k < std::min(j + np_ + 4, n); ++k) cnt += vp[firstblank + k].type == ty;
                if (cnt != np_) break;
                // gaps = diff(diff(starts)), lengths = diff(lens) over the group
                double gmax = -1e300, lmax = -1e300;
                for (int k = j; k + 2 < j + np_; ++k) {
                    const long long a = vp[firstblank + k].p.start, b = vp[firstblank + k + 1].p.start,
                                    c = vp[firstblank + k + 2].p.start;
                    gmax = std::max(gmax, (double)((c - b) - (b - a)));
                }
                for (int k = j; k + 1 < j + np_; ++k)
                    lmax = std::max(lmax, (double)(vp[firstblank + k + 1].p.len - vp[firstblank + k].p.len));
                if (gmax < P.freq * 0.2 && lmax < P.freq * 0.2) {
                    grouploc = j;
                    break;
                }
            }
            if (grouploc < 0) continue;
            const long long firstloc = vp[firstblank + grouploc].p.start;
            const double distfroml1 = ((ty - 1) * np_) * 0.5;
            const double dist = (double)(firstloc - loc_presync) / P.inlinelen;
            const long long hdist = nround(dist * 2);
            const long long hmod = ((hdist % 2) + 2) % 2;
            bool isfirst = hmod == (long long)(P.first_field_h[1] != 1.0);
            if (std::fmod(distfroml1 * 2, 2.0) != 0.0) isfirst = !isfirst;
            const double eqgap = P.first_field_h[isfirst ? 1 : 0];
            const double line0 = (double)firstloc - ((eqgap + distfroml1) * P.inlinelen);
            r.ok = true;
            r.line0 = (long long)line0;  // int() truncates toward zero
            r.isfirst = isfirst;
            r.firstblank = firstblank;
            r.conf = 100;
            return r;
        }
        if (at(vp, firstblank - 1).good && vp[firstblank].good && vp[lastblank].good && vp[lastblank + 1].good) {
            const double gap1 = (double)(vp[firstblank].p.start - at(vp, firstblank - 1).p.start);
            const double gap2 = (double)(vp[lastblank + 1].p.start - vp[lastblank].p.start);
            bool isfirst;
            if (P.system == 1 && inrange(std::fabs(gap2 - gap1), 0, P.freq * 1)) {
                isfirst = inrange(gap1 / P.inlinelen, 0.45, 0.55);
            } else if (P.system == 0 && inrange(std::fabs(gap2 + gap1), P.inlinelen * 1.4, P.inlinelen * 1.6)) {
                isfirst = inrange(gap1 / P.inlinelen, 0.95, 1.05);
            } else {
                r.zeroed_conf = true;
                return r;
            }
            r.ok = true;
            r.line0 = at(vp, firstblank - 1).p.start;
            r.isfirst = isfirst;
            r.firstblank = firstblank;
            r.conf = 50;
            return r;
        }
        return r;
    }

    // core.py:2090-2119
    double compute_line_len(const std::vector<VPulse>& vp) const {
        int lr0 = -1, lr1 = -1;
        int c0 = -1, c1 = 0;
        bool have = false;
        for (int i = 0; i < (int)vp.size(); ++i) {
            if (vp[i].type != 0) {
                if (have && c1 > lr1) {
                    lr0 = c0;
                    lr1 = c1;
                }
                have = false;
            } else if (!have) {
                have = true;
                c0 = i;
                c1 = 0;
            } else {
                c1 += 1;
            }
        }
        if (have && c1 > lr1) {
            lr0 = c0;
            lr1 = c1;
        }
        const SpacingBounds q = spacing_bounds(P.inlinelen, 0.95, 1.05);
        long long sum = 0, cnt = 0;
        for (int i = lr0 + 1; i < lr0 + lr1; ++i) {
            const long long ll = vp[i].p.start - vp[i - 1].p.start;
            if (ll >= q.lo && ll <= q.hi) {
                sum += ll;
                cnt += 1;
            }
        }
        return cnt ? (double)sum / (double)cnt : P.inlinelen;
    }

    const LdgChainParams& P;
    std::vector<Pulse> raw;
};

// Line slots from pulses for a given line 0 (core.py:2394-2481).
struct Slots {
    bool ok = false;
    bool error = false;     // no valid line anywhere to fill from (the reference raises)
    bool skipdetected = false;
    double nextfield = 0;
    std::vector<double> filled;
    std::vector<unsigned char> err;
};

Slots line_slots(const LdgChainParams& P, const std::vector<VPulse>& vp, const std::vector<Pulse>& raw,
                 double line0loc, double meanlinelen, double lastlineloc, bool have_lastline, int linecount,
                 bool have_vblank_next, double vblank_next, int proclines) {
    Slots s;
    bool skipdetected = false;
    if (have_lastline) skipdetected = (lastlineloc - line0loc) / P.inlinelen < (double)(linecount - 5);
    s.skipdetected = skipdetected;
    const double lastline = ((double)raw.back().start - line0loc) / meanlinelen;
    if (lastline < proclines) {
        s.nextfield = line0loc - (meanlinelen * 20);
        return s;
    }
    // ll_dict / ll_dist over the line slots that reach the output; slots
    // outside [0, proclines) never influence it and are not kept
    std::vector<double> linelocs(proclines, -1.0);
    std::vector<double> ll_dist(proclines, 0.0);
    std::vector<unsigned char> have(proclines, 0);
    // only pulses within two lines of the slots can land in one (the skip rule
    // only moves a pulse to a later slot); the valid pulses are in time order
    const double s_lo = line0loc - 2.0 * meanlinelen, s_hi = line0loc + (proclines + 2.0) * meanlinelen;
    const auto first = std::lower_bound(vp.begin(), vp.end(), s_lo,
                                        [](const VPulse& a, double v) { return (double)a.p.start < v; });
    for (auto it = first; it != vp.end() && (double)it->p.start <= s_hi; ++it) {
        const VPulse& p = *it;
        double lineloc = ((double)p.p.start - line0loc) / meanlinelen;
        long long rlineloc = nround(lineloc);
        double dist = std::fabs(lineloc - (double)rlineloc);
        if (skipdetected) {
            const double lineloc_end = linecount - ((lastlineloc - (double)p.p.start) / meanlinelen);
            const long long rend = nround(lineloc_end);
            const double dist_end = std::fabs(lineloc_end - (double)rend);
            if (p.type == 0 && rlineloc > 23 && dist_end < dist) {
                lineloc = lineloc_end;
                rlineloc = rend;
                dist = dist_end;
            }
        }
        if (rlineloc < 0 || rlineloc >= proclines) continue;
        if (dist > P.hsync_tolerance || (have[rlineloc] && dist > ll_dist[rlineloc])) continue;
        if (rlineloc > 0 && !p.good) {
            if (p.type > 0 || (p.type == 0 && rlineloc < 10)) continue;
        }
        linelocs[rlineloc] = (double)p.p.start;
        ll_dist[rlineloc] = dist;
        have[rlineloc] = 1;
    }
    std::vector<double> filled = linelocs;
    std::vector<unsigned char> err(proclines, 0);
    const int olc = P.outlinecount;
    if (filled[0] < 0) {
        int next_valid = -1;
        for (int i = 0; i < std::min(olc + 1, proclines); ++i)
            if (linelocs[i] > 0) {
                next_valid = i;
                break;
            }
        if (next_valid < 0) {
            s.nextfield = line0loc + (P.inlinelen * olc - 7);
            return s;
        }
        filled[0] = filled[next_valid] - (next_valid * meanlinelen);
        if (filled[0] < P.inlinelen) {
            s.nextfield = line0loc + (P.inlinelen * olc - 7);
            return s;
        }
    }
    for (int l = 1; l < proclines; ++l) {
        if (filled[l] < 0) {
            err[l] = 1;
            int pv = -1, nv = -1;
            for (int i = l; i >= 0; --i)
                if (linelocs[i] > 0) {
                    pv = i;
                    break;
                }
            for (int i = l; i < std::min(olc + 1, proclines); ++i)
                if (linelocs[i] > 0) {
                    nv = i;
                    break;
                }
            if (pv < 0) {
                if (nv < 0) {
                    s.error = true;  // the reference raises here
                    return s;
                }
                filled[l] = linelocs[nv] - (P.inlinelen * (nv - l));
            } else if (nv >= 0) {
                const double avglen = (linelocs[nv] - linelocs[pv]) / (double)(nv - pv);
                filled[l] = linelocs[pv] + (avglen * (l - pv));
            } else {
                filled[l] = linelocs[pv] + (P.inlinelen * (l - pv));
            }
        }
    }
    s.ok = true;
    s.filled = filled;
    s.err = err;
    s.nextfield = have_vblank_next ? vblank_next - (P.inlinelen * 8) : filled[olc - 7];
    return s;
}

bool same_slots(const Slots& a, const Slots& b) {
    return a.ok == b.ok && a.nextfield == b.nextfield && a.filled == b.filled && a.err == b.err;
}

// compute_deriv_error (core.py:2553-2564): second differences above 4 samples
void deriv_error(const std::vector<double>& ll, std::vector<unsigned char>& bad) {
    const int n = (int)ll.size();
    for (int j = 0; j + 2 < n; ++j) {
        const double d2 = std::fabs((ll[j + 2] - ll[j + 1]) - (ll[j + 1] - ll[j]));
        if (d2 > 4) {
            bad[j + 1] = 1;
            bad[j + 2] = 1;
        }
    }
}

struct Window {
    long long readloc, first_block, nblocks, startloc, length;
};

// LDdecode.decodefield's read of blocks (core.py:4030-4042, 1358-1409)
Window field_window(const LdgChainParams& P, double start) {
    Window w;
    w.readloc = std::max((long long)(start - P.blockcut), 0LL);
    const long long bs = P.blocklen;
    const long long U = P.blocklen - P.blockcut - P.blockcut_end;
    const long long begin = (w.readloc / bs) * bs;
    const long long length = ((P.readlen / bs) + 2) * bs;
    const long long end = begin + length;
    w.first_block = begin / U;
    const long long last = end / U;
    w.nblocks = last - w.first_block + 1;
    w.startloc = w.first_block * U;
    w.length = w.nblocks * U;
    return w;
}

thread_local std::string g_chain_err;

// The chain state after plan p (read at state s): the next read position,
// the previous-field flags and the estimate of the field's line at
// linecount; the caller's refined-line inputs are cleared.
LdgChainState advance_state(const LdgChainParams& P, const LdgChainState& s, const LdgFieldPlan& p) {
    LdgChainState n = s;
    n.prev_known = 0;
    if (p.valid) {
        n.start += p.nextfieldoffset - (double)(p.readloc - p.startloc);
        n.prev_valid = 1;
        n.prev_isfirst = p.isfirst;
        n.prev_startloc = p.startloc;
        n.fields_written += 1;
        const int lc = P.system == 1 ? (p.isfirst ? 312 : 313) : p.linecount;
        n.prev_est_valid = lc >= 0 && lc < p.proclines;
        n.prev_est = n.prev_est_valid ? (double)p.startloc + p.linelocs1[lc] : 0.0;
        n.prev_est_conf = p.sync_confidence;
    } else {
        n.start += p.nextfieldoffset;
        n.prev_valid = 0;
        n.prev_est_valid = 0;
    }
    return n;
}

}  // namespace

extern "C" {

const char* ldg_chain_last_error(void) { return g_chain_err.c_str(); }

int ldg_field_chain(const LdgChainParams* P, const int64_t* run_start, const int64_t* run_len, const double* run_mean,
                    int64_t nruns, const LdgChainState* state_in, LdgChainState* state_out, LdgFieldPlan* plans,
                    int32_t max_plans, int32_t* nplans, int32_t* stop) {
    if (!P || (!run_start && nruns) || (!run_len && nruns) || (!run_mean && nruns) || !state_in || !state_out ||
        !plans || !nplans || !stop) {
        g_chain_err = "ldg_field_chain: NULL argument";
        return -1;
    }
    if (P->proclines > LDG_CHAIN_MAX_LINES || P->proclines < P->outlinecount + 1) {
        g_chain_err = "ldg_field_chain: proclines out of range";
        return -1;
    }
    LdgChainState st = *state_in;
    int np_out = 0;
    *stop = LDG_CHAIN_STOP_END;
    const double minlength = 10.0 * P->linefreq0;  // usectoinpx(10)
    // the field at st.start is being retried with the previous field's estimate
    bool est_tried = false;
    // a field that needs the previous field's refined line locations: retry
    // it once with the range the previous field's pulse-level estimate gives
    auto retry_with_estimate = [&](const Window& w) {
        if (est_tried || st.prev_known || !st.prev_est_valid || !st.prev_valid) return false;
        const double e = st.prev_est - (double)w.startloc;
        st.prev_known = 1;
        st.prev_line0 = e - LDG_CHAIN_PREV_MARGIN;
        st.prev_line0_hi = e + LDG_CHAIN_PREV_MARGIN;
        st.prev_skip = -1;
        st.prev_conf = st.prev_est_conf;
        est_tried = true;
        return true;
    };
    auto give_up = [&]() {
        if (est_tried) st.prev_known = 0;  // the caller's inputs were not given
        est_tried = false;
        *stop = LDG_CHAIN_STOP_PREV;
    };
    while (np_out < max_plans) {
        const Window w = field_window(*P, st.start);
        if (w.first_block + w.nblocks > P->nblocks) {
            *stop = LDG_CHAIN_STOP_END;
            break;
        }
        // window pulses: runs starting after the first sample and ending before the last
        const long long lo = w.startloc, hi = w.startloc + w.length;
        const int64_t* b = std::upper_bound(run_start, run_start + nruns, (int64_t)lo);
        std::vector<Pulse> raw;
        raw.reserve(1024);
        std::vector<double> vmeans;
        bool any_long = false;
        for (const int64_t* q = b; q < run_start + nruns && *q < hi; ++q) {
            const size_t k = q - run_start;
            if (*q + run_len[k] > hi - 1) break;  // runs are sorted; an unterminated one ends the window
            if (run_len[k] > P->max_pulse_len) continue;
            raw.push_back({*q - lo, run_len[k]});
            if ((double)run_len[k] > minlength) {
                vmeans.push_back(run_mean[k]);
                any_long = true;
            }
        }
        LdgFieldPlan& pl = plans[np_out];
        std::memset(&pl, 0, sizeof(pl));
        pl.start = st.start;
        pl.readloc = w.readloc;
        pl.first_block = w.first_block;
        pl.nblocks = w.nblocks;
        pl.startloc = w.startloc;
        pl.length = w.length;
        pl.has_prev = st.prev_valid;
        pl.proclines = P->proclines;

        // getpulses (core.py:2242-2322)
        if (raw.empty() && st.fields_written == 0) {
            *stop = LDG_CHAIN_STOP_LEVELS;  // the reference re-levels ire0 from this field's data
            break;
        }
        bool invalid = false;
        double nextfieldoffset = 0;
        bool have_next = false;
        if (raw.empty()) {
            invalid = true;  // compute_linelocs returns (None, None, None)
        } else if (!any_long) {
            invalid = true;  // getpulses returns None: no VSYNC-length pulse
            if (st.fields_written == 0) {
                nextfieldoffset = P->freq_hz;
                have_next = true;
            }
        } else {
            const double synclevel = median_of(vmeans);
            const double sync_ire = (synclevel - P->ire0) / P->hz_ire;
            if (!(std::fabs(sync_ire - P->vsync_ire) < 5)) {
                *stop = LDG_CHAIN_STOP_LEVELS;  // black-level re-threshold of the pulses
                break;
            }
        }
        FieldPulses fp(*P, raw);
        Slots slots;
        bool isfirst = false;
        int dep = 0;
        if (!invalid) {
            const Timings LT = fp.get_timings();
            pl.hsync_len = (int)LT.hsync_hi;
            const std::vector<VPulse> vp = fp.refinepulses(LT);
            const double meanlinelen = fp.compute_line_len(vp);
            // getLine0 (core.py:2156-2239)
            const VBlank loc_none = fp.process_vblank(vp, 0, -1);
            VBlank loc = loc_none;
            if (st.prev_valid) {
                const VBlank loc_100 = fp.process_vblank(vp, 0, 100);
                if (!(loc_100 == loc_none)) {
                    if (st.prev_skip >= 0 && st.prev_known) {
                        if (st.prev_skip) loc = loc_100;  // limit 100 when prevfield.skip_check() >= 50
                    } else {
                        dep |= 1;  // needs the previous field's skip_check
                    }
                }
            }
            int sync_conf = 100;
            if (loc.zeroed_conf) sync_conf = 0;
            bool have_l0next = false, first_next = false, have_vbn = false;
            long long l0_next = 0;
            double vbn = 0;
            int conf_next = 0;
            if (loc.ok) {
                const VBlank nx = fp.process_vblank(vp, loc.firstblank + 40, -1);
                if (nx.zeroed_conf) sync_conf = 0;
                if (nx.ok) {
                    have_vbn = true;
                    vbn = (double)nx.line0;
                    first_next = !nx.isfirst;
                    conf_next = nx.conf;
                    const double fieldlen = meanlinelen * P->field_lines[first_next ? 0 : 1];
                    l0_next = nround(vbn - fieldlen);
                    have_l0next = true;
                    if (l0_next < 0) sync_conf = 10;
                }
            }
            const bool have_prev_l0 = st.prev_valid != 0;
            double l0 = 0;
            bool have_l0 = false;
            bool range = false;
            double l0_lo = 0, l0_hi = 0;
            if (loc.ok && have_l0next && have_prev_l0) {
                const int votes = (int)loc.isfirst + (int)(!st.prev_isfirst) + (int)first_next;
                isfirst = votes >= 2;
                have_l0 = true;
                if (st.prev_known) {
                    // np.median of (l0_local, l0_next, l0_prev), monotonic in
                    // l0_prev: the range its known bounds allow
                    auto med3 = [](double a, double b, double c) {
                        double v[3] = {a, b, c};
                        std::sort(v, v + 3);
                        return v[1];
                    };
                    l0_lo = med3((double)loc.line0, (double)l0_next, st.prev_line0);
                    l0_hi = med3((double)loc.line0, (double)l0_next, st.prev_line0_hi);
                    range = l0_hi != l0_lo;
                    l0 = l0_lo;
                } else {
                    // somewhere between the first two
                    l0_lo = (double)std::min(loc.line0, l0_next);
                    l0_hi = (double)std::max(loc.line0, l0_next);
                    range = true;
                    l0 = l0_lo;
                }
            } else if (loc.ok && loc.conf > 50) {
                sync_conf = std::min(sync_conf, 90);
                l0 = (double)loc.line0;
                isfirst = loc.isfirst;
                have_l0 = true;
            } else if (have_prev_l0) {
                if (st.prev_known) {
                    // line 0 from the previous field's end (or the range it is known in)
                    l0 = l0_lo = st.prev_line0;
                    l0_hi = st.prev_line0_hi;
                    range = l0_hi != l0_lo;
                    isfirst = !st.prev_isfirst;
                    sync_conf = std::min(sync_conf, std::max(st.prev_conf - 10, 10));
                    have_l0 = true;
                } else {
                    dep |= 2;  // line 0 is the previous field's refined line location
                }
            } else if (have_l0next) {
                sync_conf = conf_next;
                l0 = (double)l0_next;
                isfirst = first_next;
                have_l0 = true;
            }
            pl.sync_confidence = sync_conf;
            if (dep) {
                if (retry_with_estimate(w)) continue;
                give_up();
                break;
            }
            const int linecount = isfirst ? 263 : 262;
            if (!have_l0) {
                invalid = true;
                nextfieldoffset = P->inlinelen * 200;
                have_next = true;
            } else {
                slots = line_slots(*P, vp, raw, l0, meanlinelen, vbn, have_vbn, linecount, have_vbn, vbn,
                                   P->proclines);
                if (range && l0_hi != l0_lo) {
                    const Slots s2 = line_slots(*P, vp, raw, l0_hi, meanlinelen, vbn, have_vbn, linecount,
                                                have_vbn, vbn, P->proclines);
                    // the slot assignment is piecewise constant in line 0; equal results at
                    // both ends of the vote's range hold inside it unless the skip rule,
                    // which compares against a line-0-independent estimate, is active
                    if (!same_slots(slots, s2) || slots.skipdetected || s2.skipdetected) {
                        if (retry_with_estimate(w)) continue;
                        give_up();
                        break;
                    }
                }
                if (slots.error) {
                    *stop = LDG_CHAIN_STOP_ERROR;
                    break;
                }
                if (!slots.ok) {
                    invalid = true;
                    nextfieldoffset = slots.nextfield;
                    have_next = true;
                }
            }
            pl.linecount = linecount;
        }
        pl.prev_range = est_tried ? 1 : 0;
        est_tried = false;
        if (invalid) {
            if (!have_next) nextfieldoffset = P->linelen * 200;
            pl.valid = 0;
            pl.nextfieldoffset = nextfieldoffset;
            st = advance_state(*P, st, pl);
            np_out += 1;
            continue;
        }
        // process(): compute_deriv_error on the pulse-level line locations
        std::vector<unsigned char> bad = slots.err;
        deriv_error(slots.filled, bad);
        pl.valid = 1;
        pl.isfirst = isfirst;
        pl.nextfieldoffset = slots.nextfield;
        for (int l = 0; l < P->proclines; ++l) {
            pl.linelocs1[l] = slots.filled[l];
            pl.linebad[l] = bad[l];
        }
        st = advance_state(*P, st, pl);
        np_out += 1;
    }
    if (est_tried) st.prev_known = 0;  // stopped while retrying: the estimate is not the caller's
    if (np_out >= max_plans && *stop == LDG_CHAIN_STOP_END) *stop = LDG_CHAIN_STOP_FULL;
    *nplans = np_out;
    *state_out = st;
    return 0;
}

}  // extern "C"

extern "C" int64_t ldg_abi_sizeof(const char* name) {
    if (!name) return -1;
    const std::string n(name);
    if (n == "ldg_chain_params") return sizeof(ldg_chain_params);
    if (n == "ldg_chain_state") return sizeof(ldg_chain_state);
    if (n == "ldg_field_plan") return sizeof(ldg_field_plan);
    if (n == "ldg_lines_consts") return sizeof(ldg_lines_consts);
    if (n == "ldg_lines_args") return sizeof(ldg_lines_args);
    if (n == "ldg_tbc_field") return sizeof(ldg_tbc_field);
    if (n == "ldg_demod_args") return sizeof(ldg_demod_args);
    if (n == "ldg_slice") return sizeof(ldg_slice);
    if (n == "ldg_work_item") return sizeof(ldg_work_item);
    if (n == "ldg_dropout_field") return sizeof(ldg_dropout_field);
    if (n == "ldg_dropout_params") return sizeof(ldg_dropout_params);
    if (n == "ldg_rftbc_field") return sizeof(ldg_rftbc_field);
    if (n == "ldg_audio2_segment") return sizeof(ldg_audio2_segment);
    if (n == "ldg_audio_field") return sizeof(ldg_audio_field);
    if (n == "ldg_audio_params") return sizeof(ldg_audio_params);
    if (n == "ldg_efm_edge") return sizeof(ldg_efm_edge);
    return -1;
}

// ---- the chain in pieces on host threads

#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>

namespace {

struct Key {
    long long readloc;
    int prev_valid, prev_isfirst;
    bool written;
    bool operator==(const Key& o) const {
        return readloc == o.readloc && prev_valid == o.prev_valid && prev_isfirst == o.prev_isfirst &&
               written == o.written;
    }
};

long long readloc_of(const LdgChainParams& P, double start) { return std::max((long long)(start - P.blockcut), 0LL); }

Key key_of(const LdgChainParams& P, const LdgChainState& s) {
    return {readloc_of(P, s.start), s.prev_valid, s.prev_valid ? s.prev_isfirst : 0, s.fields_written > 0};
}


struct Piece {
    std::vector<LdgFieldPlan> plans;
    LdgChainState in{}, out{};
    int32_t stop = 0;
    int rc = 0;
};

// Host threads kept for the chain's pieces: a call hands its pieces to the
// pool instead of starting and joining threads of its own (tens of
// microseconds each, several calls per capture chunk).  Any number of
// callers may share it; each waits for its own pieces only.  The pool is
// never torn down (its idle threads block on a condition variable).
class PiecePool {
  public:
    static PiecePool& get() {
        static PiecePool* pool = new PiecePool();
        return *pool;
    }
    // run fn(1) .. fn(n-1) on pool threads and fn(0) on the caller; returns
    // when all n have finished
    void run(int n, const std::function<void(int)>& fn) {
        struct Latch {
            std::mutex m;
            std::condition_variable cv;
            int left;
        } latch;
        latch.left = n - 1;
        ensure(n - 1);
        {
            std::lock_guard<std::mutex> lk(m_);
            for (int t = 1; t < n; ++t)
                q_.push_back([&fn, &latch, t] {
                    fn(t);
                    std::lock_guard<std::mutex> l2(latch.m);
                    if (--latch.left == 0) latch.cv.notify_all();
                });
        }
        cv_.notify_all();
        fn(0);
        std::unique_lock<std::mutex> lk(latch.m);
        latch.cv.wait(lk, [&] { return latch.left == 0; });
    }

  private:
    void ensure(int k) {
        std::lock_guard<std::mutex> lk(m_);
        while ((int)nthreads_ < k) {
            std::thread([this] { loop(); }).detach();
            ++nthreads_;
        }
    }
    void loop() {
        for (;;) {
            std::function<void()> task;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return !q_.empty(); });
                task = std::move(q_.front());
                q_.erase(q_.begin());
            }
            task();
        }
    }
    std::mutex m_;
    std::condition_variable cv_;
    std::vector<std::function<void()>> q_;
    size_t nthreads_ = 0;
};

void run_piece(const LdgChainParams& P, int64_t limit, const int64_t* rs, const int64_t* rl, const double* rm,
               int64_t nruns, int32_t cap, Piece& pc) {
    LdgChainParams q = P;
    q.nblocks = limit;
    pc.plans.resize(cap);
    int32_t n = 0;
    pc.rc = ldg_field_chain(&q, rs, rl, rm, nruns, &pc.in, &pc.out, pc.plans.data(), cap, &n, &pc.stop);
    pc.plans.resize(pc.rc == 0 ? n : 0);
}

}  // namespace

extern "C" int ldg_field_chain_mt(const LdgChainParams* P, const int64_t* run_start, const int64_t* run_len,
                                  const double* run_mean, int64_t nruns, const LdgChainState* state_in,
                                  LdgChainState* state_out, LdgFieldPlan* plans, int32_t max_plans,
                                  int32_t* nplans, int32_t* stop, int32_t nthreads, int64_t margin_blocks,
                                  int64_t min_seg_blocks) {
    if (!P || !state_in || !state_out || !plans || !nplans || !stop) {
        g_chain_err = "ldg_field_chain_mt: NULL argument";
        return -1;
    }
    const long long U = P->blocklen - P->blockcut - P->blockcut_end;
    const long long b0 = std::max((long long)state_in->start / U, 0LL);
    const long long seg = nthreads > 0 ? (P->nblocks - b0) / nthreads : 0;
    if (nthreads <= 1 || seg < min_seg_blocks || U <= 0)
        return ldg_field_chain(P, run_start, run_len, run_mean, nruns, state_in, state_out, plans, max_plans, nplans,
                               stop);
    std::vector<Piece> pcs(nthreads);
    std::vector<int64_t> limit(nthreads);
    for (int t = 0; t < nthreads; ++t) {
        if (t == 0) {
            pcs[t].in = *state_in;
        } else {
            pcs[t].in.start = (double)((b0 + t * seg) * U);
            pcs[t].in.fields_written = state_in->fields_written + 1;
        }
        limit[t] = t == nthreads - 1 ? P->nblocks : std::min<long long>(P->nblocks, b0 + (t + 1) * seg + margin_blocks);
    }
    {
        // a field read advances at least ~10 blocks; a piece that fills its
        // buffer stops (LDG_CHAIN_STOP_FULL) and the caller resumes
        auto cap = [&](int t) {
            const long long first = t == 0 ? b0 : b0 + t * seg;
            return (int32_t)std::min<long long>(max_plans, (limit[t] - first) / 8 + 16);
        };
        PiecePool::get().run(nthreads, [&](int t) {
            run_piece(*P, limit[t], run_start, run_len, run_mean, nruns, cap(t), pcs[t]);
        });
    }
    for (const Piece& pc : pcs)
        if (pc.rc != 0) return pc.rc;
    // join the pieces: merged plans with the state before each of them
    std::vector<LdgFieldPlan> merged = std::move(pcs[0].plans);
    std::vector<LdgChainState> before;
    {
        LdgChainState s = pcs[0].in;
        for (const LdgFieldPlan& p : merged) {
            before.push_back(s);
            s = advance_state(*P, s, p);
        }
    }
    int32_t stp = pcs[0].stop;
    LdgChainState st_end = pcs[0].out;
    bool serial_rest = false;
    for (int t = 1; t < nthreads && stp == LDG_CHAIN_STOP_END; ++t) {
        Piece& pc = pcs[t];
        if (pc.plans.empty()) {
            serial_rest = true;
            break;
        }
        std::vector<Key> tk;
        std::vector<LdgChainState> ts;  // the piece's state before each of its plans
        {
            LdgChainState s = pc.in;
            for (const LdgFieldPlan& p : pc.plans) {
                tk.push_back(key_of(*P, s));
                ts.push_back(s);
                s = advance_state(*P, s, p);
            }
        }
        const long long lo = pc.plans[0].readloc;
        int ji = -1, jj = -1;
        for (size_t i = 0; i < before.size() && ji < 0; ++i) {
            const Key k = key_of(*P, before[i]);
            if (k.readloc < lo) continue;
            for (size_t j = 0; j < tk.size(); ++j)
                if (tk[j] == k) {
                    ji = (int)i;
                    jj = (int)j;
                    break;
                }
        }
        if (ji < 0) {
            serial_rest = true;
            break;
        }
        // re-walk the piece's plans from the true state; the fraction of a
        // sample in `start` differs, the read windows must not
        merged.resize(ji);
        before.resize(ji);
        LdgChainState s = ji ? advance_state(*P, before.back(), merged.back()) : pcs[0].in;
        bool moved = false;
        for (size_t j = jj; j < pc.plans.size(); ++j) {
            LdgFieldPlan p = pc.plans[j];
            if (readloc_of(*P, s.start) != p.readloc) {
                moved = true;
                break;
            }
            // a plan decided from the previous field's estimate holds for the
            // true chain when its estimate is the same to within a sample
            if (p.prev_range && (!s.prev_est_valid || std::fabs(s.prev_est - ts[j].prev_est) > 1.0)) {
                moved = true;
                break;
            }
            p.start = s.start;
            merged.push_back(p);
            before.push_back(s);
            s = advance_state(*P, s, p);
        }
        st_end = s;
        stp = pc.stop;
        if (moved) {
            serial_rest = true;
            break;
        }
    }
    if (serial_rest) {
        std::vector<LdgFieldPlan> rest(std::max<int64_t>(max_plans - (int64_t)merged.size(), 1));
        int32_t n = 0, sp = 0;
        LdgChainState so{};
        const int rc = ldg_field_chain(P, run_start, run_len, run_mean, nruns, &st_end, &so, rest.data(),
                                       (int32_t)rest.size(), &n, &sp);
        if (rc != 0) return rc;
        merged.insert(merged.end(), rest.begin(), rest.begin() + n);
        st_end = so;
        stp = sp;
    }
    if ((int64_t)merged.size() > max_plans) {
        // the caller's buffer is full: stop where it ends
        LdgChainState s = pcs[0].in;
        for (int32_t k = 0; k < max_plans; ++k) s = advance_state(*P, s, merged[k]);
        merged.resize(max_plans);
        st_end = s;
        stp = LDG_CHAIN_STOP_FULL;
    }
    std::copy(merged.begin(), merged.end(), plans);
    *nplans = (int32_t)merged.size();
    *state_out = st_end;
    *stop = stp;
    return 0;
}
