// EFM phase-locked loop: T-values (run lengths in EFM bit periods) from the
// EFM-filtered RF that the demodulator writes (its int16 `efm` output).
//
// Restates EFM_PLL (lddecode/efm_pll.py:80-244): an interpolated
// zero-crossing detector (process, efm_pll.py:124-167) feeding each edge's
// sub-sample distance from the previous one to a software PLL (pushEdge,
// efm_pll.py:169-240) whose reference clock counts bit periods between
// edges, nudges its phase by 0.5 % of each edge's error and its period by
// at most 0.01 % per edge after two errors of the same sign.  Every value
// is the reference's: FP64 state, int8 T counter, int32 hysteresis counter,
// and the same operation order, so the T-values are identical.
//
// The work is serial and edge-driven (the loop state carries from edge to
// edge and from field to field), so it runs on the host, one PLL per
// decoded stream; callers decode several streams on several threads.  The
// zero-crossing scan does one sign test per sample; the reference's
// per-sample `delta += 1.0` between crossings is reproduced with one
// addition per binade the running delta crosses (see add_ones), which
// rounds exactly as the per-sample additions do.
#include <cmath>
#include <cstdint>
#include <new>
#include <string>

#include "ldgpu.h"

namespace ldg {
int api_fail(int code, const std::string& msg);
}

struct ldg_efm_pll {
    // zero-crossing detector
    int16_t zc_prev = 0;
    double delta = 0.0;
    // loop constants (efm_pll.py:108-114)
    double base_period = 40000000.0 / 4321800.0;
    double minimum_period = base_period * 0.90;
    double maximum_period = base_period * 1.10;
    double period_adjust_base = base_period * 0.0001;
    // loop state (efm_pll.py:116-121)
    double current_period = base_period;
    double phase_adjust = 0.0;
    double ref_clock_time = 0.0;
    int32_t frequency_hysteresis = 0;
    int8_t t_counter = 1;
};

namespace {

// `d` after k successive additions of 1.0, each rounded to double as the
// reference's per-sample loop rounds it.  Inside a binade [2^(e-1), 2^e)
// whose ulp is at most 1 an addition of 1.0 that stays in the binade is
// exact, so a whole stretch of them is one exact addition; only the
// addition that enters the next binade (where the ulp doubles) and those
// below 1.0 can round, and they are done one at a time.
double add_ones(double d, int64_t k) {
    while (k > 0) {
        if (!(d >= 1.0) || d >= 9007199254740992.0) {  // below 1, or ulp above 1 (never in practice)
            d += 1.0;
            --k;
            continue;
        }
        int e = 0;
        std::frexp(d, &e);                       // d in [2^(e-1), 2^e)
        const double next = std::ldexp(1.0, e);  // 2^e
        const double room = next - d;            // exact (Sterbenz)
        int64_t m = (int64_t)std::ceil(room) - 1;  // d + m < next
        if (m > k) m = k;
        if (m > 0) {
            d += (double)m;  // exact: stays in the binade, a multiple of its ulp
            k -= m;
        }
        if (k > 0) {
            d += 1.0;  // into the next binade: rounds as the reference's addition does
            --k;
        }
    }
    return d;
}

// pushEdge (efm_pll.py:169-240).  Returns false if `out` is full.
bool push_edge(ldg_efm_pll& s, double sample_delta, int8_t* out, int64_t cap, int64_t& count) {
    while (sample_delta >= s.ref_clock_time) {
        const double next_time = s.ref_clock_time + s.current_period + s.phase_adjust;
        s.ref_clock_time = next_time;
        // runs of 1 or 2 periods are not valid EFM (the edge is pushed), and
        // runs beyond 11 are pulled
        if ((sample_delta > next_time || s.t_counter < 3) && s.t_counter < 11) {
            s.phase_adjust = 0.0;
            s.t_counter = (int8_t)(s.t_counter + 1);
        } else {
            const double edge_delta = sample_delta - (next_time - s.current_period / 2.0);
            s.phase_adjust = edge_delta * 0.005;
            // the reference's counter is int32 and wraps
            if (edge_delta < 0) {
                s.frequency_hysteresis = s.frequency_hysteresis < 0
                                             ? (int32_t)((uint32_t)s.frequency_hysteresis - 1u)
                                             : -1;
            } else if (edge_delta > 0) {
                s.frequency_hysteresis = s.frequency_hysteresis > 0
                                             ? (int32_t)((uint32_t)s.frequency_hysteresis + 1u)
                                             : 1;
            } else {
                s.frequency_hysteresis = 0;
            }
            if ((double)s.frequency_hysteresis < -1.0 || (double)s.frequency_hysteresis > 1.0) {
                double aper = s.period_adjust_base * edge_delta / s.current_period;
                // a long gap (a dropout) makes edge_delta large: limit the step
                if (aper < -s.period_adjust_base) {
                    aper = -s.period_adjust_base;
                } else if (aper > s.period_adjust_base) {
                    aper = s.period_adjust_base;
                }
                s.current_period += aper;
                if (s.current_period < s.minimum_period) {
                    s.current_period = s.minimum_period;
                } else if (s.current_period > s.maximum_period) {
                    s.current_period = s.maximum_period;
                }
            }
            if (count >= cap) return false;
            out[count++] = s.t_counter;
            s.t_counter = 1;
        }
    }
    // keep the error for the next delta
    s.ref_clock_time -= sample_delta;
    return true;
}

}  // namespace

extern "C" {

int ldg_efm_pll_create(ldg_efm_pll** out) {
    if (!out) return ldg::api_fail(LDG_ERR_ARG, "ldg_efm_pll_create: out is NULL");
    *out = new (std::nothrow) ldg_efm_pll();
    if (!*out) return ldg::api_fail(LDG_ERR_ARG, "ldg_efm_pll_create: out of host memory");
    return LDG_OK;
}

int ldg_efm_pll_destroy(ldg_efm_pll* pll) {
    delete pll;
    return LDG_OK;
}

int ldg_efm_pll_process(ldg_efm_pll* pll, const int16_t* in, int64_t n, int8_t* out, int64_t out_cap,
                        int64_t* out_count) {
    if (!pll || !out_count || (n > 0 && (!in || !out)))
        return ldg::api_fail(LDG_ERR_ARG, "ldg_efm_pll_process: NULL argument");
    if (n < 0 || out_cap < n)
        return ldg::api_fail(LDG_ERR_ARG, "ldg_efm_pll_process: out must hold n values (the reference's buffer)");
    ldg_efm_pll& s = *pll;
    int64_t count = 0;
    int16_t prev = s.zc_prev;
    double delta = s.delta;
    int64_t run_start = 0;  // first sample not yet counted into delta
    for (int64_t i = 0; i < n; ++i) {
        const int16_t cur = in[i];
        // (prev < 0) != (cur < 0): the sign bits differ
        if (((int)prev ^ (int)cur) < 0) {
            delta = add_ones(delta, i - run_start);
            const double fraction = (double)(-(int64_t)prev) / (double)((int64_t)cur - (int64_t)prev);
            if (!push_edge(s, delta + fraction, out, out_cap, count)) {
                *out_count = count;
                return ldg::api_fail(LDG_ERR_RANGE, "ldg_efm_pll_process: more T-values than input samples");
            }
            delta = 1.0 - fraction;
            run_start = i + 1;
        }
        prev = cur;
    }
    s.delta = add_ones(delta, n - run_start);
    s.zc_prev = prev;
    *out_count = count;
    return LDG_OK;
}

int ldg_efm_pll_process_edges(ldg_efm_pll* pll, const ldg_efm_edge* edges, int64_t nedges, int64_t lo, int64_t hi,
                              int16_t first, int16_t last, int8_t* out, int64_t out_cap, int64_t* out_count) {
    if (!pll || !out_count || (nedges > 0 && !edges) || (hi > lo && !out))
        return ldg::api_fail(LDG_ERR_ARG, "ldg_efm_pll_process_edges: NULL argument");
    if (nedges < 0 || hi < lo || lo < 0 || out_cap < hi - lo)
        return ldg::api_fail(LDG_ERR_ARG, "ldg_efm_pll_process_edges: bad range or out smaller than the slice");
    ldg_efm_pll& s = *pll;
    int64_t count = 0;
    *out_count = 0;
    if (hi == lo) return LDG_OK;
    double delta = s.delta;
    int64_t run_start = lo;
    auto edge = [&](int64_t i, int16_t prev, int16_t cur) {
        delta = add_ones(delta, i - run_start);
        const double fraction = (double)(-(int64_t)prev) / (double)((int64_t)cur - (int64_t)prev);
        if (!push_edge(s, delta + fraction, out, out_cap, count)) return false;
        delta = 1.0 - fraction;
        run_start = i + 1;
        return true;
    };
    // the sample at lo against the PLL's previous sample
    if ((((int)s.zc_prev) ^ (int)first) < 0 && !edge(lo, s.zc_prev, first)) {
        *out_count = count;
        return ldg::api_fail(LDG_ERR_RANGE, "ldg_efm_pll_process_edges: more T-values than input samples");
    }
    // crossings strictly inside the slice: their previous sample is in it too
    int64_t a = 0, b = nedges;
    while (a < b) {  // first edge with pos > lo
        const int64_t m = (a + b) / 2;
        if ((int64_t)edges[m].pos <= lo) a = m + 1;
        else b = m;
    }
    for (int64_t k = a; k < nedges && (int64_t)edges[k].pos < hi; ++k) {
        if (!edge(edges[k].pos, edges[k].prev, edges[k].cur)) {
            *out_count = count;
            return ldg::api_fail(LDG_ERR_RANGE, "ldg_efm_pll_process_edges: more T-values than input samples");
        }
    }
    s.delta = add_ones(delta, hi - run_start);
    s.zc_prev = last;
    *out_count = count;
    return LDG_OK;
}

int ldg_efm_pll_state(const ldg_efm_pll* pll, double* dstate, int32_t* istate) {
    if (!pll || !dstate || !istate) return ldg::api_fail(LDG_ERR_ARG, "ldg_efm_pll_state: NULL argument");
    dstate[0] = pll->delta;
    dstate[1] = pll->current_period;
    dstate[2] = pll->phase_adjust;
    dstate[3] = pll->ref_clock_time;
    istate[0] = pll->zc_prev;
    istate[1] = pll->frequency_hysteresis;
    istate[2] = pll->t_counter;
    return LDG_OK;
}

}  // extern "C"
