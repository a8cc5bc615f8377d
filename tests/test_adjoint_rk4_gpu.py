"""Adjoint of linear absorption with Propagation RK4 (propagate_vec_RK4,
propagate.c:261-373): the FP64 model at zero shifts and unit coupling scale
is the engine's FP64 RK4 absorption, and nise_backward_absorption's
gradient (the sub-steps' polynomial and renormalisation differentiated,
states recomputed from checkpoints) matches central differences of the
model per component."""
import numpy as np
import pytest

import helpers
import nise_2017_b200 as nise
from nise_2017_b200 import synth
from test_adjoint_gpu import ADJ_VS_FD, central, loss_and_grad, per_component

pytestmark = pytest.mark.gpu


def make_case(tmp_path, n=8, frames=400, tmax=40, ts=3):
    s = synth.spec(n_sites=n, frames=frames, dt_fs=2.0, geometry=synth.CHAIN, seed=61)
    files = synth.write(s, str(tmp_path))
    kw = synth.c0_keywords(Singles=n, Length=frames, RunTimes="%d 0 0" % tmax, Samplerate=25, FFT=256,
                           Lifetime=600, Trotter=ts, Propagation="RK4")
    return kw, files


def test_rk4_model_equals_fp64_absorption(tmp_path):
    kw, files = make_case(tmp_path)
    p = nise.params_from_keywords(kw, files, precision=nise.FP64)
    with nise.Context(p) as c:
        c.load_files()
        re, im, n = c.absorption()
        w0, sr0, si0 = c.absorption_fft(re, im, n)
        w, sr, si = c.absorption_model(np.zeros(p.singles), 1.0, p.lifetime)
    assert np.allclose(w, w0, rtol=0, atol=1e-9)
    assert helpers.rel(sr + 1j * si, sr0 + 1j * si0) < 1e-11


@pytest.mark.parametrize("tmax, frames", [(40, 400), (100, 500)])
def test_rk4_adjoint_matches_central_differences(tmax, frames, tmp_path):
    """tmax 40: one checkpoint block; tmax 100: four (K = 32)."""
    kw, files = make_case(tmp_path, frames=frames, tmax=tmax)
    p = nise.params_from_keywords(kw, files, precision=nise.FP64)
    rng = np.random.default_rng(7)
    n = p.singles
    with nise.Context(p) as c:
        c.load_files()
        _, tr, ti = c.absorption_model(rng.normal(0, 5, n), 1.1, 500.0)
        target = (tr, ti)
        shift, scale, lt = np.zeros(n), 1.0, 600.0
        L, dre, dim = loss_and_grad(c, target, shift, scale, lt)
        g, gs, gl = c.backward_absorption(shift, scale, lt, dre, dim)
        h = 1e-3
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
    print("RK4 adjoint vs central differences, tmax %d: per-component %.2e" % (tmax, err))
    assert err < ADJ_VS_FD, (adj, fd)
