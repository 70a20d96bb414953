"""Adjoint calibration model (cuvhs_adjoint_*, cuvhs_b200.calibrate).

A synthetic tape is recorded twice from the same seeded test pattern: once
nominally, once with a perturbed pre-emphasis shelf, an FM carrier offset, a
deviation change, per-line picture delays and per-line colour-under phase
offsets.  The nominal tape decoded by the model at the nominal parameters is
the target.  The gradients of the perturbed tape's loss must agree with
central finite differences of the model and with FP64 central differences of
an FP64 restatement of the model, and 200 gradient-descent steps must bring
the parameters back towards the perturbation."""
import numpy as np
import pytest

import cuvhs_b200 as cv
from cuvhs_b200.calibrate import Adjoint, calibrate, deemph_response, shelf_deemph

BASE = dict(sample_rate_hz=28e6, n_fields=10, seed=404, snr_db=40, jitter_bound=0.5)
PERT = dict(BASE, carrier_offset_hz=30e3, deviation_scale=1.03, preemph_perturb=(0.1, -0.1, 0.1),
            line_offset_bound=1.5, chroma_phase_bound=np.deg2rad(20))
GRAD_RTOL = 1e-3


def test_shelf_deemph_inverts_the_synthesized_preemphasis():
    w = np.linspace(0.01, 3.0, 50)
    z = np.exp(-1j * w)
    for pp in ((0.0, 0.0, 0.0), (0.1, -0.1, 0.1), (-0.08, 0.1, -0.1)):
        b, a = cv.synth_preemphasis(sample_rate_hz=28e6, preemph_perturb=pp)
        d = shelf_deemph(28e6, [1 + v for v in pp])
        assert np.allclose(d, np.array([a[1], a[2], b[1], b[2]]) / b[0], rtol=1e-12, atol=1e-14)
        h_pre = (b[0] + b[1] * z + b[2] * z * z) / (a[0] + a[1] * z + a[2] * z * z)
        assert np.allclose(deemph_response(d, w) * h_pre, 1.0, rtol=1e-9)
        assert np.all(np.abs(np.roots(a)) < 1) and np.all(np.abs(np.roots(b)) < 1)  # stays a stable shelf


def test_calibration_perturbations_are_seeded_and_leave_the_nominal_tape_alone():
    small = dict(BASE, n_fields=2)
    x0 = cv.synth_capture(**small)
    assert np.array_equal(x0, cv.synth_capture(**small, preemph_perturb=(0, 0, 0), line_offset_bound=0.0,
                                               chroma_phase_bound=0.0))
    pert = dict(PERT, n_fields=2)
    assert np.array_equal(cv.synth_capture(**pert), cv.synth_capture(**pert))
    assert not np.array_equal(cv.synth_capture(**pert), x0)
    st, off, ph = cv.synth_lines(**pert)
    assert np.all(np.diff(st) > 0)
    assert np.abs(off).max() <= 1.5 and off.std() > 0.7  # uniform in +/-1.5: std 0.87
    assert np.abs(ph).max() <= np.deg2rad(20) and ph.std() > np.deg2rad(9)  # uniform: std 11.5 degrees


@pytest.fixture(scope="module")
def tapes():
    """(model of the perturbed tape with the nominal tape's target, nominal
    parameters, the perturbation's parameters)."""
    clean = Adjoint(cv.synth_capture(**BASE), 28.0, fields=8)
    p0 = clean.default_params()
    yt, ct = clean.planes(p0)
    pert = Adjoint(cv.synth_capture(**PERT), 28.0, fields=8)
    pert.set_target(yt, ct)
    F = clean.fields
    llc = clean.array("linelocs").reshape(F, 525)
    llp = pert.array("linelocs").reshape(F, 525)
    st, off, ph = cv.synth_lines(**PERT)
    k = np.array([[int(np.argmin(np.abs(st - llp[f, r]))) for r in range(264)] for f in range(F)])
    truth = p0.copy()
    truth.deemph = shelf_deemph(28e6, [1 + v for v in PERT["preemph_perturb"]])
    truth.carrier_hz = PERT["carrier_offset_hz"]
    truth.deviation = PERT["deviation_scale"]
    truth.line_offset = off[k] + (llc[:, :264] - llp[:, :264])  # picture delay + line-location difference
    truth.chroma_phase = ph[k[:, :263]]
    yield pert, p0, truth
    pert.close()
    clean.close()


def _largest(g, rows, n):
    """Indices (field, row) of the n largest |g| over the given rows."""
    sub = np.abs(g[:, rows])
    flat = np.argsort(sub.ravel())[::-1][:n]
    return [(int(i // sub.shape[1]), int(i % sub.shape[1]) + rows.start) for i in flat]


@pytest.mark.gpu
def test_adjoint_gradient_matches_central_differences(tapes):
    """Central differences of the model's own forward with h = 1e-3 of each
    parameter's scale (samples, radians, relative deviation, kHz of carrier);
    the de-emphasis denominator, which sits next to a DC pole-zero pair,
    takes h = 1e-6."""
    adj, p0, _ = tapes
    loss, g = adj.grad(p0)
    assert loss > 0 and np.isfinite(loss)

    def fd(setter, h):
        a = p0.copy()
        setter(a, h)
        b = p0.copy()
        setter(b, -h)
        return (adj.loss(a) - adj.loss(b)) / (2 * h)

    checks = []
    for j, h in enumerate((1e-3, 1e-3, 1e-6, 1e-6)):
        def s(p, d, j=j):
            p.deemph[j] += d
        checks.append((f"deemph[{j}]", g.deemph[j], fd(s, h)))
    checks.append(("carrier", g.carrier_hz, fd(lambda p, d: setattr(p, "carrier_hz", p.carrier_hz + d), 1.0)))
    checks.append(("deviation", g.deviation, fd(lambda p, d: setattr(p, "deviation", p.deviation + d), 1e-3)))
    for f, r in _largest(g.line_offset, slice(22, 258), 4):
        def s(p, d, f=f, r=r):
            p.line_offset[f, r] += d
        checks.append((f"line_offset[{f},{r}]", g.line_offset[f, r], fd(s, 1e-3)))
    for f, r in _largest(g.chroma_phase, slice(22, 169), 4):
        def s(p, d, f=f, r=r):
            p.chroma_phase[f, r] += d
        checks.append((f"chroma_phase[{f},{r}]", g.chroma_phase[f, r], fd(s, 1e-3)))
    bad = [(n, a, b) for n, a, b in checks if abs(a - b) > GRAD_RTOL * abs(b)]
    assert not bad, bad


@pytest.mark.gpu
def test_adjoint_gradient_matches_fp64_reference():
    """The FP64 restatement (tests/adjoint_ref.py) of the same model on the same
    decoded inputs: its loss agrees with the GPU forward and its FP64 central
    differences with the GPU adjoint within 1e-3 relative, at a parameter point
    with non-zero offsets and phases (two fields, to keep the FP64 model quick)."""
    from adjoint_ref import RefModel
    clean = Adjoint(cv.synth_capture(**BASE), 28.0, fields=2)
    p0 = clean.default_params()
    yt, ct = clean.planes(p0)
    adj = Adjoint(cv.synth_capture(**PERT), 28.0, fields=2)
    adj.set_target(yt, ct)
    rng = np.random.default_rng(9)
    p = p0.copy()
    p.deemph = shelf_deemph(28e6, (1.03, 0.97, 1.02))
    p.carrier_hz, p.deviation = 10e3, 1.01
    p.line_offset = rng.uniform(-0.5, 0.5, p.line_offset.shape)
    p.chroma_phase = rng.uniform(-0.1, 0.1, p.chroma_phase.shape)
    ref = RefModel(adj, yt, ct)
    l_gpu, g = adj.grad(p)
    l_ref = ref.loss(p)
    assert abs(l_gpu - l_ref) <= 1e-4 * l_ref, (l_gpu, l_ref)

    def fd(setter, h):
        a = p.copy()
        setter(a, h)
        b = p.copy()
        setter(b, -h)
        return (ref.loss(a) - ref.loss(b)) / (2 * h)

    checks = []
    for j, h in enumerate((1e-6, 1e-6, 1e-8, 1e-8)):
        def s(q, d, j=j):
            q.deemph[j] += d
        checks.append((f"deemph[{j}]", g.deemph[j], fd(s, h)))
    checks.append(("carrier", g.carrier_hz, fd(lambda q, d: setattr(q, "carrier_hz", q.carrier_hz + d), 1e-2)))
    checks.append(("deviation", g.deviation, fd(lambda q, d: setattr(q, "deviation", q.deviation + d), 1e-6)))
    for f, r in _largest(g.line_offset, slice(22, 258), 3):
        def s(q, d, f=f, r=r):
            q.line_offset[f, r] += d
        checks.append((f"line_offset[{f},{r}]", g.line_offset[f, r], fd(s, 1e-5)))
    for f, r in _largest(g.chroma_phase, slice(22, 169), 3):
        def s(q, d, f=f, r=r):
            q.chroma_phase[f, r] += d
        checks.append((f"chroma_phase[{f},{r}]", g.chroma_phase[f, r], fd(s, 1e-5)))
    bad = [(n, a, b) for n, a, b in checks if abs(a - b) > GRAD_RTOL * abs(b)]
    assert not bad, bad
    adj.close()
    clean.close()


@pytest.mark.gpu
def test_calibration_recovers_tape_parameters(tapes):
    """200 Adam steps from the nominal parameters reach the loss of the true
    perturbation and recover the global parameters; the per-line parameters
    come back as far as the data determines them (the FM band limit and the
    luma-into-chroma crosstalk of a re-recorded tape leave a residual that the
    true parameters share)."""
    adj, p0, truth = tapes
    l_truth = adj.loss(truth)
    pc, shelf, hist = calibrate(adj, p0, steps=200)
    assert hist[0] > 50 * hist[-1], (hist[0], hist[-1])
    assert hist[-1] < 1.05 * l_truth, (hist[-1], l_truth)
    assert abs(pc.carrier_hz - truth.carrier_hz) < 1000.0, pc.carrier_hz
    assert abs(pc.deviation - truth.deviation) < 0.003, pc.deviation
    w = np.linspace(0.02, 2 * np.pi * 3e6 / 28e6, 100)
    h_true = deemph_response(truth.deemph, w)
    err0 = np.max(np.abs(deemph_response(p0.deemph, w) / h_true - 1))
    err1 = np.max(np.abs(deemph_response(pc.deemph, w) / h_true - 1))
    assert err1 < 0.5 * err0, (err0, err1, shelf)
    rows = slice(22, 258)
    off_err = np.sqrt(np.mean((pc.line_offset - truth.line_offset)[:, rows] ** 2))
    off_rms = np.sqrt(np.mean(truth.line_offset[:, rows] ** 2))
    assert off_err < 0.6 * off_rms, (off_err, off_rms)
    crows = slice(22, 169)  # lines that carry chroma
    ph_err = np.sqrt(np.mean(np.angle(np.exp(1j * (pc.chroma_phase - truth.chroma_phase)))[:, crows] ** 2))
    ph_rms = np.sqrt(np.mean(truth.chroma_phase[:, crows] ** 2))
    assert ph_err < 0.25 * ph_rms, (np.rad2deg(ph_err), np.rad2deg(ph_rms))
