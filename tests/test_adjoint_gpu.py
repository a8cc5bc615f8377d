"""Adjoint of linear absorption against finite differences and gradcheck.

nise_absorption_model is the differentiable FP64 Trotter absorption with
per-site shifts, a coupling scale and the lifetime as parameters;
nise_backward_absorption back-propagates dL/dspectrum to them by
reverse-time propagation from checkpoints.  The loss is the L2 distance to
a target spectrum made by the same model with shifts ~ N(0, 5 cm^-1) and a
coupling scale of 1.1.
"""
import numpy as np
import pytest

import helpers
import nise_2017_b200 as nise
from nise_2017_b200 import synth

pytestmark = pytest.mark.gpu

ADJ_VS_FD = 1e-6   # per component, relative (central differences, one Richardson step)
# Absolute floor of the per-component comparison, as a fraction of the largest
# component: below it a component is compared absolutely, at ADJ_VS_FD times
# the floor (the finite differences' own rounding, eps * |L| / h, sits there).
FLOOR = 1e-4


def per_component(adj, fd):
    """max_i |adj_i - fd_i| / max(|fd_i|, FLOOR * max|fd|)."""
    adj, fd = np.asarray(adj, float), np.asarray(fd, float)
    den = np.maximum(np.abs(fd), FLOOR * np.abs(fd).max())
    return float((np.abs(adj - fd) / den).max())


def make_case(tmp_path, n=8, frames=400, tmax=40, ts=5):
    s = synth.spec(n_sites=n, frames=frames, dt_fs=2.0, geometry=synth.CHAIN, seed=51)
    files = synth.write(s, str(tmp_path))
    kw = synth.c0_keywords(Singles=n, Length=frames, RunTimes="%d 0 0" % tmax, Samplerate=25, FFT=256,
                           Lifetime=600, Trotter=ts)
    return kw, files


def central(f, x, h):
    """Central difference with one Richardson step: error O(h^4)."""
    d1 = (f(x + h) - f(x - h)) / (2 * h)
    d2 = (f(x + h / 2) - f(x - h / 2)) / h
    return (4 * d2 - d1) / 3


def loss_and_grad(c, target, shift, scale, lifetime):
    w, sr, si = c.absorption_model(shift, scale, lifetime)
    tr, ti = target
    L = float(((sr - tr) ** 2).sum() + ((si - ti) ** 2).sum())
    return L, 2 * (sr - tr), 2 * (si - ti)


def test_model_equals_fp64_absorption(tmp_path):
    """At zero shifts and unit scale the model is the engine's FP64 absorption."""
    kw, files = make_case(tmp_path)
    p = nise.params_from_keywords(kw, files, precision=nise.FP64)
    with nise.Context(p) as c:
        c.load_files()
        re, im, n = c.absorption()
        w0, sr0, si0 = c.absorption_fft(re, im, n)
        w, sr, si = c.absorption_model(np.zeros(p.singles), 1.0, p.lifetime)
    assert np.allclose(w, w0, rtol=0, atol=1e-9)
    assert helpers.rel(sr + 1j * si, sr0 + 1j * si0) < 1e-11


def test_adjoint_matches_central_differences(tmp_path):
    kw, files = make_case(tmp_path)
    p = nise.params_from_keywords(kw, files, precision=nise.FP64)
    rng = np.random.default_rng(3)
    n = p.singles
    with nise.Context(p) as c:
        c.load_files()
        _, tr, ti = c.absorption_model(rng.normal(0, 5, n), 1.1, 500.0)
        target = (tr, ti)
        shift, scale, lt = np.zeros(n), 1.0, 600.0
        L, dre, dim = loss_and_grad(c, target, shift, scale, lt)
        g, gs, gl = c.backward_absorption(shift, scale, lt, dre, dim)
        h = 1e-3  # cm^-1 for shifts, fs for the lifetime, 1e-3 relative for the scale
        fd = np.zeros(n + 2)
        for a in range(n):
            e = np.zeros(n)
            e[a] = 1.0
            fd[a] = central(lambda x: loss_and_grad(c, target, shift + x * e, scale, lt)[0], 0.0, h)
        fd[n] = central(lambda x: loss_and_grad(c, target, shift, x, lt)[0], scale, h)
        fd[n + 1] = central(lambda x: loss_and_grad(c, target, shift, scale, x)[0], lt, h)
    adj = np.concatenate([g, [gs, gl]])
    assert L > 0 and np.abs(adj).max() > 0
    err = per_component(adj, fd)
    print("adjoint vs central differences, N=8: per-component %.2e" % err)
    assert err < ADJ_VS_FD, (adj, fd)


def test_checkpoint_reconstruction_long_run(tmp_path):
    """Many checkpoint segments (tmax 200, K = 32): the reverse-time
    reconstruction stays exact enough for 1e-6 gradients."""
    kw, files = make_case(tmp_path, n=6, frames=700, tmax=200, ts=2)
    p = nise.params_from_keywords(kw, files, precision=nise.FP64)
    n = p.singles
    with nise.Context(p) as c:
        c.load_files()
        _, tr, ti = c.absorption_model(np.linspace(-4, 4, n), 1.05, 600.0)
        shift = np.zeros(n)
        L, dre, dim = loss_and_grad(c, (tr, ti), shift, 1.0, 600.0)
        g, gs, gl = c.backward_absorption(shift, 1.0, 600.0, dre, dim)
        h = 1e-3
        a = 2
        e = np.zeros(n)
        e[a] = 1.0
        fa = central(lambda x: loss_and_grad(c, (tr, ti), shift + x * e, 1.0, 600.0)[0], 0.0, h)
        fs = central(lambda x: loss_and_grad(c, (tr, ti), shift, x, 600.0)[0], 1.0, h)
    err = per_component([g[a], gs], [fa, fs])
    print("adjoint vs central differences, 200 steps: per-component %.2e" % err)
    assert err < ADJ_VS_FD


def test_gradcheck_autograd_function(tmp_path):
    """A test-only torch.autograd.Function around the C ABI passes gradcheck."""
    import torch
    kw, files = make_case(tmp_path, n=5, frames=300, tmax=24)
    p = nise.params_from_keywords(kw, files, precision=nise.FP64)
    c = nise.Context(p)
    c.load_files()

    class Spectrum(torch.autograd.Function):
        @staticmethod
        def forward(ctx, shift, scale, lifetime):
            ctx.save_for_backward(shift, scale, lifetime)
            _, sr, si = c.absorption_model(shift.detach().numpy(), float(scale), float(lifetime))
            return torch.from_numpy(np.stack([sr, si], 1))

        @staticmethod
        def backward(ctx, grad):
            shift, scale, lifetime = ctx.saved_tensors
            g = grad.detach().numpy()
            gsh, gs, gl = c.backward_absorption(shift.detach().numpy(), float(scale), float(lifetime),
                                                np.ascontiguousarray(g[:, 0]), np.ascontiguousarray(g[:, 1]))
            return (torch.from_numpy(gsh), torch.tensor(gs, dtype=torch.float64),
                    torch.tensor(gl, dtype=torch.float64))

    try:
        shift = torch.zeros(p.singles, dtype=torch.float64, requires_grad=True)
        scale = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
        lifetime = torch.tensor(600.0, dtype=torch.float64, requires_grad=True)
        assert torch.autograd.gradcheck(Spectrum.apply, (shift, scale, lifetime), eps=1e-4, atol=1e-9, rtol=1e-5)
    finally:
        c.close()


def test_adjoint_rejects_other_schemes(tmp_path):
    """Coupling, RK4 and the exact propagator have adjoints (tests/test_adjoint_rk4_gpu.py,
    tests/test_adjoint_exact_gpu.py); the truncated propagator (Sparse with a
    Threshold in (0, 1], propagate_vec_DIA_S) is not differentiable and is refused."""
    kw, files = make_case(tmp_path)
    kw = dict(kw, Propagation="Sparse", Threshold=0.001)
    p = nise.params_from_keywords(kw, files, precision=nise.FP64)
    with nise.Context(p) as c:
        c.load_files()
        with pytest.raises(nise.NiseError) as e:
            c.absorption_model(np.zeros(p.singles), 1.0, 600.0)
        assert e.value.code == -6


def test_adjoint_c3_configuration(tmp_path):
    """The full adjoint workload: a 256-site chain over 20000 frames (994 start
    points, 128 steps, checkpoints every 32).  Adjoint gradients of the L2
    spectrum loss against central differences (h = 1e-3) for sites at both ends
    and the middle, the coupling scale and the lifetime."""
    s = synth.c3_spec(seed=53)
    files = synth.write(s, str(tmp_path))
    p = nise.params_from_keywords(synth.c3_keywords(), files, precision=nise.FP64)
    n, lt = p.singles, float(p.lifetime)
    rng = np.random.default_rng(20173)
    with nise.Context(p) as c:
        c.load_files()
        _, tr, ti = c.absorption_model(rng.normal(0, 5, n), 1.1, lt)
        target = (tr, ti)
        shift = np.zeros(n)
        L, dre, dim = loss_and_grad(c, target, shift, 1.0, lt)
        g, gs, gl = c.backward_absorption(shift, 1.0, lt, dre, dim)
        h = 1e-3
        checks = []
        for a in (0, 128, 255):
            e = np.zeros(n)
            e[a] = 1.0
            checks.append((g[a], central(lambda x: loss_and_grad(c, target, shift + x * e, 1.0, lt)[0], 0.0, h)))
        checks.append((gs, central(lambda x: loss_and_grad(c, target, shift, x, lt)[0], 1.0, h)))
        checks.append((gl, central(lambda x: loss_and_grad(c, target, shift, 1.0, x)[0], lt, h)))
    assert L > 0 and max(np.abs(g).max(), abs(gs), abs(gl)) > 0
    err = per_component([a for a, _ in checks], [f for _, f in checks])
    print("adjoint vs central differences, adjoint workload: per-component %.2e" % err)
    assert err < ADJ_VS_FD, checks
