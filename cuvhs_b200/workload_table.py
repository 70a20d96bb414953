"""Parameters of the named synthetic workloads (seeded synthetic NTSC and PAL
VHS RF captures), as cuvhs_synth_params fields (include/cuvhs_synth.h).

This module imports nothing from the package, so a process can read the table
(by path) and synthesize a capture with the stand-alone cuvhs-synth tool
without loading libcuvhs.
"""

WORKLOADS = {
    # 6 fields at 28 MHz, clean (small parity case)
    "small28": dict(sample_rate_hz=28e6, n_fields=6, seed=7, snr_db=40, jitter_bound=0.5),
    # 8 fields at 28 MHz with 1% dropout lines, head switch, 36 dB
    "dropouts28": dict(sample_rate_hz=28e6, n_fields=8, seed=11, snr_db=36, jitter_bound=1.0,
                       dropout_line_rate=0.01, headswitch_min=3, headswitch_max=8),
    # plain decode: 40 fields at 28 MHz, 40 dB, +/-0.5 sample jitter, no dropouts
    "plain40_28": dict(sample_rate_hz=28e6, n_fields=40, seed=1001, snr_db=40, jitter_bound=0.5),
    # harder signal: 600 fields at 40 MHz, 32 dB, +/-2 jitter, 0.1% dropouts, head switch 3-8
    "hard600_40": dict(sample_rate_hz=40e6, n_fields=600, seed=2001, snr_db=32, jitter_bound=2.0,
                       dropout_line_rate=0.001, headswitch_min=3, headswitch_max=8),
    # 35.8 MHz rate coverage
    "small358": dict(sample_rate_hz=35.8e6, n_fields=6, seed=31, snr_db=38, jitter_bound=1.0),
    # PAL (--system PAL): 6 clean fields at 28 MHz; 8 fields at 28 MHz with dropouts and head switch
    "small28pal": dict(sample_rate_hz=28e6, n_fields=6, seed=41, snr_db=40, jitter_bound=0.5, system=1),
    "dropouts28pal": dict(sample_rate_hz=28e6, n_fields=8, seed=43, snr_db=36, jitter_bound=1.0,
                          dropout_line_rate=0.01, headswitch_min=3, headswitch_max=8, system=1),
    # PAL at 40 MHz, 20 fields
    "pal20_40": dict(sample_rate_hz=40e6, n_fields=20, seed=47, snr_db=38, jitter_bound=1.0, system=1),
    # long-stream sample: 300 fields at 40 MHz with +/-0.2% tape-speed drift, 0.2% dropout lines, head switch
    "drift300_40": dict(sample_rate_hz=40e6, n_fields=300, seed=5003, snr_db=36, jitter_bound=1.0,
                        dropout_line_rate=0.002, headswitch_min=3, headswitch_max=8, speed_drift=0.002),
    # adversarial: the FM carrier raised by 20 IRE + 1 Hz, so the sync tip sits 1 Hz above the pulse
    # threshold and noise puts thousands of sync samples within a few Hz of it
    "tipthr28": dict(sample_rate_hz=28e6, n_fields=6, seed=53, snr_db=40, jitter_bound=0.5,
                     carrier_offset_hz=20 * 1e6 / 140 + 1.0),
}


BATCH_RATES = (28.0, 35.8, 40.0)


def batch_specs(count=64, min_fields=2, max_fields=240, seed=3000):
    """Per-capture synthesis parameters of a mixed batch: lengths uniform in
    [min_fields, max_fields], rates from 28 / 35.8 / 40 MHz, SNR 30-45 dB,
    jitter bound 0.5-2 samples, dropout-line rate 0-0.5%; capture i is seeded
    seed + i."""
    import numpy as np
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        mhz = float(BATCH_RATES[int(rng.integers(0, len(BATCH_RATES)))])
        specs.append(dict(sample_rate_hz=mhz * 1e6, n_fields=int(rng.integers(min_fields, max_fields + 1)),
                          seed=seed + i, snr_db=float(rng.uniform(30, 45)),
                          jitter_bound=float(rng.uniform(0.5, 2.0)),
                          dropout_line_rate=float(rng.uniform(0.0, 0.005))))
    return specs
