"""Named synthetic workloads (seeded synthetic NTSC and PAL VHS RF captures).

They stand in for real tape captures: the reference was developed on private
captures, so every measurement and parity case here runs on seeded synthetic
signals with the stated sizes and impairments.
"""
from ._lib import synth_capture

from .workload_table import BATCH_RATES, WORKLOADS, batch_specs  # noqa: F401


def system_of(name):
    """The video system ("NTSC" or "PAL") of a named workload."""
    return "PAL" if WORKLOADS[name].get("system", 0) == 1 else "NTSC"


def make_workload(name, **overrides):
    kw = dict(WORKLOADS[name])
    kw.update(overrides)
    return synth_capture(**kw)


def make_batch_workload(count=64, min_fields=2, max_fields=240, seed=3000):
    """[(capture u8, sample_rate_mhz), ...] for batch_specs(...)."""
    return [(synth_capture(**kw), kw["sample_rate_hz"] / 1e6)
            for kw in batch_specs(count, min_fields, max_fields, seed)]
