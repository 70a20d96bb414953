import functools
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


# A case name is a workload name, or one with this suffix: the same workload
# decoded with the single-pass line locator (the reference's CUVHS_K2B_DISABLE).
SINGLE = "_singlepass"


def base_name(name):
    return name[:-len(SINGLE)] if name.endswith(SINGLE) else name


def single_pass(name):
    return name.endswith(SINGLE)


def system(name):
    import cuvhs_b200 as cv
    return cv.system_of(base_name(name))


def rate_mhz(name):
    import cuvhs_b200 as cv
    return cv.WORKLOADS[base_name(name)]["sample_rate_hz"] / 1e6


@functools.lru_cache(maxsize=None)
def workload(name):
    import cuvhs_b200 as cv
    return cv.make_workload(base_name(name))


@functools.lru_cache(maxsize=None)
def oracle_decode(name):
    """FP64 oracle decode of a named case (cached per session)."""
    from oracle.oracle import Oracle
    x = workload(name)
    o = Oracle(rate_mhz(name), system=system(name), single_pass_lines=single_pass(name))
    o.decode(x)
    return o


def golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        g = {k: z[k] for k in z.files}
    with open(os.path.join(GOLDEN, name + ".tbc.json")) as f:
        g["json_text"] = f.read()
    return g


def tile_stride(mhz, system="NTSC"):
    pal = system == "PAL"
    spl = int(round(mhz * 1e6 / (15625.0 if pal else 15734.264)))
    return spl * (313 if pal else 263) + 20 * spl


def inside_fields(file_locs, n_input, mhz, system="NTSC"):
    """Fields whose analysis window (one tile stride from the field start) lies
    inside the capture.  Past the end the reference decodes zero-filled samples,
    whose FM phase is FP64 round-off noise, so no implementation can match
    those fields sample for sample."""
    spp = tile_stride(mhz, system)
    return [i for i, f in enumerate(file_locs) if int(f) + spp <= n_input]


def json_fields(text):
    return json.loads(text)["fields"]
