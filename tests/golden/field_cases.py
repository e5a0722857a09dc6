"""Seeded captures for the multi-field line-location fixtures
(fields_<case>.npz), shared by make_golden.py and the tests (no reference
import).  Each case decodes `nfields` consecutive fields."""

import numpy as np

FIELD_CASES = [
    # name, system, fields, seed, snr_db, dropouts per field, wow (amplitude, period) in samples,
    # fields whose vertical sync gets a dropout, PAL 8-field sequence
    ("ntsc_clean", "NTSC", 10, 61, 40.0, 0, None, (), False),
    ("ntsc_30db", "NTSC", 10, 62, 30.0, 0, None, (), False),
    ("ntsc_dropouts", "NTSC", 10, 63, 38.0, 6, None, (), False),
    ("ntsc_wow", "NTSC", 10, 64, 40.0, 0, (0.8, 1334667.0), (), False),
    ("ntsc_vsync_dropouts", "NTSC", 10, 65, 38.0, 0, None, (2, 5, 7), False),
    ("pal_8phase", "PAL", 12, 66, 40.0, 0, None, (), True),
    ("pal_30db_dropouts_wow", "PAL", 10, 67, 30.0, 5, (0.8, 1600000.0), (4,), True),
]


def field_case(name):
    for c in FIELD_CASES:
        if c[0] == name:
            return c
    raise KeyError(name)


def field_case_capture(case, blocklen, readlen):
    """(int16 numpy capture, metadata dict) of a case: the synthetic capture
    with its wow, seeded dropouts and dropouts laid over the vertical sync
    pulses of the listed fields."""
    from ldgpu import params
    from ldgpu.synth import inject_dropouts, synth_capture
    name, system, nfields, seed, snr, dpf, wow, vfields, pal8 = case
    sp = params.sysparams(system)
    fieldlen = int(40e6 / (sp["FPS"] * 2))
    ncap = (nfields + 3) * fieldlen + readlen + 8 * blocklen
    start = 123457 + 1009 * seed
    cap = synth_capture(system, ncap, seed=seed, start=start, snr_db=snr, wow=wow, pal8=pal8).numpy()
    spans = inject_dropouts(cap, seed + 5000, dpf * (nfields + 3)) if dpf else []
    # the raster's field k starts its vertical interval at absolute half-line
    # k * frame_lines; its broad (vertical sync) pulses follow numPulses
    # half-lines of equalising pulses
    hl = sp["line_period"] / 2 * 40.0  # samples per half-line
    fper = sp["frame_lines"] * hl
    k0 = int(np.ceil(start / fper))
    vspans = []
    rng = np.random.default_rng(seed + 7000)
    for f in vfields:
        i0 = int((k0 + f) * fper - start + (sp["numPulses"] + 1.3) * hl)
        ln = 600
        cap[i0:i0 + ln] = rng.integers(-30, 31, ln).astype(np.int16)
        vspans.append((i0, ln))
    meta = {"seed": seed, "start": start, "snr_db": snr, "dropouts_per_field": dpf,
            "wow": np.array(wow if wow else (0.0, 0.0)), "drop_spans": np.array(spans, np.int64).reshape(-1, 2),
            "vsync_spans": np.array(vspans, np.int64).reshape(-1, 2), "pal8": pal8}
    return cap, meta
