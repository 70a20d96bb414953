"""Tape parameter calibration through the adjoint decode model (cuvhs_adjoint_*).

The model redoes the parameter-dependent part of the decode -- de-emphasis and
video low-pass, FM carrier offset and deviation, per-line start offsets,
per-line chroma phase -- on the demod, pre-band-pass, line locations and
tracks of a normal decode, and scores luma/chroma against target planes.
`Adjoint.grad` returns the gradient from the library's adjoint kernels;
`calibrate` runs Adam (a gradient-descent method) on it.
"""
import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import AdjointParams, Config, CuvhsError, FIELD_H, FIELD_W, _vp, lib

ROWS = FIELD_H + 1  # line offsets per field (rows 0..263)
NAMES = ("deemph", "carrier_hz", "deviation", "line_offset", "chroma_phase")


@dataclass
class Params:
    deemph: np.ndarray                 # n1, n2, m1, m2
    carrier_hz: float
    deviation: float
    line_offset: np.ndarray            # [fields, 264] samples
    chroma_phase: np.ndarray           # [fields, 263] radians

    def copy(self):
        return Params(np.array(self.deemph, np.float64), float(self.carrier_hz), float(self.deviation),
                      np.array(self.line_offset, np.float64), np.array(self.chroma_phase, np.float64))

    def _c(self):
        self.deemph = np.asarray(self.deemph, np.float64)
        self.line_offset = np.ascontiguousarray(self.line_offset, np.float64)
        self.chroma_phase = np.ascontiguousarray(self.chroma_phase, np.float64)
        p = AdjointParams()
        p.deemph = (ctypes.c_double * 4)(*self.deemph)
        p.carrier_hz = float(self.carrier_hz)
        p.deviation = float(self.deviation)
        p.line_offset = self.line_offset.ctypes.data
        p.chroma_phase = self.chroma_phase.ctypes.data
        return p


def deemph_response(deemph, w):
    """H(e^{iw}) of the de-emphasis parameters (n1, n2, m1, m2), unit DC gain."""
    n1, n2, m1, m2 = deemph
    n0 = 1.0 + m1 + m2 - n1 - n2
    z1 = np.exp(-1j * np.asarray(w))
    return (n0 + n1 * z1 + n2 * z1 * z1) / (1.0 + m1 * z1 + m2 * z1 * z1)


SHELF_NOMINAL = (273755.82, 13.9794, 0.462088186)  # corner (Hz), gain (dB), Q of the pre-emphasis shelf


def shelf_deemph(fs_hz, scale=(1.0, 1.0, 1.0)):
    """De-emphasis parameters (n1, n2, m1, m2) inverting the pre-emphasis high
    shelf whose corner, gain and Q are SHELF_NOMINAL times `scale` (the RBJ
    shelf the decoder inverts; its DC gain is 1)."""
    f0, g, q = (v * k for v, k in zip(SHELF_NOMINAL, scale))
    A = 10.0 ** (g / 40.0)
    w0 = 2.0 * np.pi * f0 / fs_hz
    alpha = np.sin(w0) / (2.0 * q)
    c, sa = np.cos(w0), np.sqrt(A)
    b0 = A * ((A + 1) + (A - 1) * c + 2 * sa * alpha)
    b1 = -2 * A * ((A - 1) + (A + 1) * c)
    b2 = A * ((A + 1) + (A - 1) * c - 2 * sa * alpha)
    a1 = 2 * ((A - 1) - (A + 1) * c)
    a2 = (A + 1) - (A - 1) * c - 2 * sa * alpha
    return np.array([a1 / b0, a2 / b0, b1 / b0, b2 / b0])


class Adjoint:
    """The calibration model of one capture's first `fields` fields."""

    def __init__(self, samples, sample_rate_mhz=28.0, fields=8, device=0):
        samples = np.ascontiguousarray(samples, np.uint8)
        cfg = Config()
        lib.cuvhs_default_config(ctypes.byref(cfg))
        cfg.sample_rate_mhz = float(sample_rate_mhz)
        cfg.device = int(device)
        h = _vp()
        st = lib.cuvhs_adjoint_create(ctypes.byref(cfg), samples.ctypes.data, samples.size, int(fields),
                                      ctypes.byref(h))
        if st != 0:
            raise CuvhsError(st, "cuvhs_adjoint_create failed")
        self._h = h
        self.fields = lib.cuvhs_adjoint_fields(h)
        self.sample_rate_mhz = float(sample_rate_mhz)

    def close(self):
        if getattr(self, "_h", None):
            lib.cuvhs_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @staticmethod
    def _check(st, what):
        if st != 0:
            raise CuvhsError(st, what)

    def zeros(self) -> Params:
        return Params(np.zeros(4), 0.0, 0.0, np.zeros((self.fields, ROWS)), np.zeros((self.fields, FIELD_H)))

    def default_params(self) -> Params:
        p = self.zeros()
        c = p._c()
        self._check(lib.cuvhs_adjoint_default_params(self._h, ctypes.byref(c)), "default params")
        p.deemph = np.array(c.deemph[:], np.float64)
        p.carrier_hz, p.deviation = c.carrier_hz, c.deviation
        return p

    def set_target(self, luma, chroma):
        y = np.ascontiguousarray(luma, np.float32).reshape(self.fields, FIELD_H, FIELD_W)
        c = np.ascontiguousarray(chroma, np.float32).reshape(self.fields, FIELD_H, FIELD_W)
        self._check(lib.cuvhs_adjoint_set_target(self._h, y.ctypes.data, c.ctypes.data), "set target")

    def planes(self, p: Params):
        """The model's luma and chroma planes (float, TBC units) at p."""
        y = np.empty((self.fields, FIELD_H, FIELD_W), np.float32)
        c = np.empty_like(y)
        cp = p._c()
        self._check(lib.cuvhs_adjoint_fwd(self._h, ctypes.byref(cp), None, y.ctypes.data, c.ctypes.data), "forward")
        return y, c

    def loss(self, p: Params) -> float:
        out = ctypes.c_double(0.0)
        cp = p._c()
        self._check(lib.cuvhs_adjoint_fwd(self._h, ctypes.byref(cp), ctypes.byref(out), None, None), "forward")
        return out.value

    def grad(self, p: Params):
        """(loss, Params holding dL/dparameter)."""
        g = self.zeros()
        gc = g._c()
        cp = p._c()
        out = ctypes.c_double(0.0)
        self._check(lib.cuvhs_adjoint_bwd(self._h, ctypes.byref(cp), ctypes.byref(out), ctypes.byref(gc)),
                    "backward")
        g.deemph = np.array(gc.deemph[:], np.float64)
        g.carrier_hz, g.deviation = gc.carrier_hz, gc.deviation
        return out.value, g

    def array(self, name):
        dt = {"linelocs": np.float64, "gains": np.float32, "tracks": np.int32, "demod": np.float32,
              "pre": np.float32}[name]
        n = lib.cuvhs_adjoint_array(self._h, name.encode(), None, 0)
        a = np.empty(n, dt)
        lib.cuvhs_adjoint_array(self._h, name.encode(), a.ctypes.data, n)
        return a


# Adam step sizes per parameter group, in their own units.  The de-emphasis is
# stepped in the relative corner / gain / Q of the shelf it inverts: its
# coefficients sit next to a DC pole-zero pair, where equal coefficient steps
# have wildly unequal effects.
DEFAULT_LR = {"shelf": 1.6e-2, "carrier_hz": 4000.0, "deviation": 1.6e-2, "line_offset": 0.32, "chroma_phase": 0.16}


def calibrate(adj: Adjoint, start: Params, steps=200, lr=None, betas=(0.9, 0.999), eps=1e-30, callback=None,
              final_lr=0.05):
    """Adam on the adjoint gradient, the step sizes decaying on a cosine from
    lr to final_lr * lr.  The de-emphasis coefficients follow the shelf scales
    s (start 1, 1, 1) through shelf_deemph; their gradient is the adjoint's
    coefficient gradient times the FP64 Jacobian d(coefficients)/ds.
    Returns (params, shelf scales, loss per step + final)."""
    lr = dict(DEFAULT_LR, **(lr or {}))
    fs = adj.sample_rate_mhz * 1e6
    p = start.copy()
    shelf = np.ones(3)
    p.deemph = shelf_deemph(fs, shelf)
    names = ("carrier_hz", "deviation", "line_offset", "chroma_phase")
    m = {k: np.zeros_like(np.asarray(getattr(p, k), np.float64)) for k in names}
    v = {k: np.zeros_like(m[k]) for k in names}
    m["shelf"], v["shelf"] = np.zeros(3), np.zeros(3)
    hist = []

    def adam(k, x, gk, it):
        m[k] = betas[0] * m[k] + (1 - betas[0]) * gk
        v[k] = betas[1] * v[k] + (1 - betas[1]) * gk * gk
        mh = m[k] / (1 - betas[0] ** it)
        vh = v[k] / (1 - betas[1] ** it)
        decay = final_lr + (1 - final_lr) * 0.5 * (1 + np.cos(np.pi * (it - 1) / max(1, steps - 1)))
        return x - decay * lr[k] * mh / (np.sqrt(vh) + eps)

    for it in range(1, steps + 1):
        loss, g = adj.grad(p)
        hist.append(loss)
        J = np.empty((4, 3))
        for j in range(3):
            e = np.zeros(3)
            e[j] = 1e-6
            J[:, j] = (shelf_deemph(fs, shelf + e) - shelf_deemph(fs, shelf - e)) / 2e-6
        shelf = adam("shelf", shelf, J.T @ g.deemph, it)
        p.deemph = shelf_deemph(fs, shelf)
        for k in names:
            val = adam(k, np.asarray(getattr(p, k), np.float64), np.asarray(getattr(g, k), np.float64), it)
            setattr(p, k, float(val) if np.ndim(val) == 0 else val)
        if callback:
            callback(it, loss, p)
    hist.append(adj.loss(p))
    return p, shelf, np.array(hist)
