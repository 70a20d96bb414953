"""FP64 restatement of the calibration decode model (test infrastructure).

The checker for the library's adjoint kernels (cuvhs_adjoint_*): the same
model -- de-emphasis and video low-pass (here as a linear convolution with the
filter's taps within the decoder's +/-b_pos support), Catmull-Rom luma, heterodyned and band-passed chroma with
the burst-driven ACC gain, mean squared error over lines 10..261, columns
80..893 -- evaluated in FP64 with numpy on the fixed inputs the GPU model
holds (demod, pre-band-pass, line locations, tracks), so that FP64 central
differences of it give a reference gradient."""
import math

import numpy as np
from scipy.signal import fftconvolve

W, H, LPF, NFFT, BURST_LEN = 910, 263, 525, 1024, 36
ROW0, ROW1, COL0, COL1 = 10, 262, 80, 894
FSC = 3579545.0
OUT_RATE = 4.0 * FSC
CHROMA_UNDER = (525.0 * (30.0 / 1.001)) * 40.0
HZ_IRE = 1e6 / 140.0
OUTPUT_SCALE = (51200.0 - 1024.0) / 140.0
KNB = 8192


def super_gauss(f, corner, order):
    scale = (math.log(2.0) / 2.0) ** (1.0 / (2.0 * order))
    x = 2.0 * f * scale / corner
    return np.exp(-2.0 * x ** (2.0 * order))


class RefModel:
    def __init__(self, adj, tgt_y, tgt_c):
        self.fs = adj.sample_rate_mhz * 1e6
        self.P = adj.fields
        self.pre = adj.array("pre").astype(np.float64)
        self.total = self.pre.size
        self.dem = adj.array("demod").astype(np.float64)[: self.total]
        self.ll = adj.array("linelocs").reshape(self.P, LPF)
        self.track = adj.array("tracks")
        self.tgt_y = np.asarray(tgt_y, np.float64).reshape(self.P, H, W)
        self.tgt_c = np.asarray(tgt_c, np.float64).reshape(self.P, H, W)
        self.b_pos = min(64 * math.ceil(self.fs * 1e-6 * 25.6 / 64), 2048)
        self.het_scale = (FSC + CHROMA_UNDER) / OUT_RATE
        self.fsc_bin = int(FSC / OUT_RATE * NFFT + 0.5)
        self.bw_bins = max(10, int(500000.0 / OUT_RATE * NFFT + 0.5))
        self.burst_start = int(5.3e-6 * OUT_RATE + 0.5)
        self.luma_gain = OUTPUT_SCALE / HZ_IRE
        self.luma_offset = 40.0 * OUTPUT_SCALE + 1024.0
        k = np.arange(NFFT)
        kk = np.minimum(k, NFFT - k)
        lo, hi = self.fsc_bin - self.bw_bins, self.fsc_bin + self.bw_bins
        self.mask = ((kk >= lo) & (kk <= hi)).astype(np.float64)
        self.npix = self.P * (ROW1 - ROW0) * (COL1 - COL0)
        self.col_frac = np.arange(W) / float(W)

    def video(self, deemph):
        n1, n2, m1, m2 = deemph
        n0 = 1.0 + m1 + m2 - n1 - n2
        k = np.arange(KNB)
        kk = np.where(k <= KNB // 2, k, k - KNB)
        z = np.exp(-1j * 2.0 * np.pi * kk / KNB)
        R = (n0 + n1 * z + n2 * z * z) / (1.0 + m1 * z + m2 * z * z) * super_gauss(np.abs(kk) * self.fs / KNB, 3.0e6, 9)
        h = np.fft.ifft(R).real
        taps = h[np.arange(-self.b_pos, self.b_pos + 1) % KNB]
        return fftconvolve(self.dem, taps, mode="full")[self.b_pos:self.b_pos + self.total]

    def _coords(self, off):
        r = np.arange(H)
        a0 = self.ll[:, r] + off[:, r]
        a1 = self.ll[:, r + 1] + off[:, r + 1]
        return a0[:, :, None] + self.col_frac[None, None, :] * (a1 - a0)[:, :, None]

    def _cr(self, s, x):
        ci = np.floor(x).astype(np.int64)
        ok = (ci >= 1) & (ci + 2 < self.total)
        c = np.clip(ci, 1, self.total - 3)
        fr = x - c
        p0, p1, p2, p3 = s[c - 1], s[c], s[c + 1], s[c + 2]
        c1 = p2 - p0
        c2 = 2 * p0 - 5 * p1 + 4 * p2 - p3
        c3 = 3 * (p1 - p2) + p3 - p0
        return np.where(ok, p1 + 0.5 * fr * (c1 + fr * (c2 + fr * c3)), 0.0), ok

    def planes(self, p):
        off = np.asarray(p.line_offset, np.float64)
        x = self._coords(off)
        v, ok = self._cr(self.video(p.deemph), x)
        Y = np.where(ok, (v - p.carrier_hz) / p.deviation * self.luma_gain + self.luma_offset, 1024.0)
        s, okc = self._cr(self.pre, x)
        r = np.arange(H)
        rot = np.where(self.track != 0, 1, 3)
        lp = (r[None, :] * rot[:, None]) & 3
        u = self.het_scale * (r[:, None] * W + np.arange(W)[None, :])
        fr = u - np.floor(u)
        arg = 2.0 * fr[None] + 0.5 * lp[:, :, None] + np.asarray(p.chroma_phase)[:, :, None] / np.pi
        sig = np.where(okc, s * -np.cos(np.pi * arg), 0.0)
        buf = np.zeros((self.P, H, NFFT))
        buf[:, :, :W] = sig
        bp = np.fft.ifft(np.fft.fft(buf, axis=2) * self.mask, axis=2).real
        rms = np.sqrt(np.mean(bp[:, :, self.burst_start:self.burst_start + BURST_LEN] ** 2, axis=2))
        g = np.where(rms > 1.0, 4416.0 / np.maximum(rms, 1e-300), 0.0)
        C = g[:, :, None] * bp[:, :, :W] + 32768.0
        return Y, C, ok

    def loss(self, p):
        Y, C, ok = self.planes(p)
        sl = (slice(None), slice(ROW0, ROW1), slice(COL0, COL1))
        ey = np.where(ok[sl], Y[sl] - self.tgt_y[sl], 0.0)
        ec = C[sl] - self.tgt_c[sl]
        return float(np.sum(ey * ey) / self.npix + np.sum(ec * ec) / self.npix)
