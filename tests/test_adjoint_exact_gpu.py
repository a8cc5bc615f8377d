"""Adjoint of linear absorption with the exact propagator exp(-i H f)
(propagate_vec_DIA, propagate.c:60-125: Propagation Sparse with Threshold 0,
or Diagonal).  The FP64 model (a degree-18 Taylor polynomial of A/m with
||A/m|| <= 1, remainder below 2e-17) at zero shifts and unit coupling scale is
the engine's FP64 exact-propagator absorption, and nise_backward_absorption's
gradient matches central differences of the model per component, with one
and with several sub-steps per frame."""
import numpy as np
import pytest

import helpers
import nise_2017_b200 as nise
from nise_2017_b200 import synth
from test_adjoint_gpu import ADJ_VS_FD, central, loss_and_grad, per_component

pytestmark = pytest.mark.gpu

F_PER_FS = float(np.float32(2.99792458e-5)) * float(np.float32(2 * 3.14159265359))


def make_case(tmp_path, n=8, frames=400, tmax=40, dt=2.0, ham="Coupling", prop="Sparse", seed=71, sigma=10.0):
    """Chain around 1650 cm^-1; a wide disorder (sigma) gets a window of +-650 cm^-1."""
    ht = synth.COUPLING if ham == "Coupling" else synth.FULL
    s = synth.spec(n_sites=n, frames=frames, dt_fs=dt, geometry=synth.CHAIN, ham_type=ht, seed=seed, sigma=sigma)
    files = synth.write(s, str(tmp_path))
    lo, hi = (1550, 1750) if sigma < 50 else (1000, 2300)
    kw = synth.c0_keywords(Singles=n, Length=frames, RunTimes="%d 0 0" % tmax, Samplerate=25, FFT=256,
                           Lifetime=600, Timestep=dt, Propagation=prop, HamiltonianType=ham,
                           MinFrequencies="%d %d %d" % (lo, lo, lo), MaxFrequencies="%d %d %d" % (hi, hi, hi))
    if prop == "Sparse":
        kw["Threshold"] = 0
    return kw, files


def norm_bound(kw, files, n):
    """max over frames of (max |h_a - shift| + ||J||_F) f: the sub-step count is its ceiling."""
    lo = float(kw["MinFrequencies"].split()[0])
    hi = float(kw["MaxFrequencies"].split()[0])
    shift = float(np.float32((np.float32(lo) + np.float32(hi)) / np.float32(2)))
    nn2 = n * (n + 1) // 2
    E = np.fromfile(files["energy"], dtype=np.float32)
    if kw["HamiltonianType"] == "Coupling":
        d = E.reshape(-1, 1 + n)[:, 1:].astype(float) - shift
        rec = np.fromfile(files["coupling"], dtype=np.float32)[1:1 + nn2]
        J = [rec[b + a * (2 * n - a - 1) // 2] for a in range(n) for b in range(a + 1, n)]
        jf = np.sqrt(2 * np.sum(np.square(J)))
        return float((np.abs(d).max(axis=1) + jf).max() * float(kw["Timestep"]) * F_PER_FS)
    raise NotImplementedError


@pytest.mark.parametrize("ham, prop", [("Coupling", "Sparse"), ("Coupling", "Diagonal"), ("Full", "Sparse")])
def test_exact_model_equals_fp64_absorption(ham, prop, tmp_path):
    kw, files = make_case(tmp_path, ham=ham, prop=prop)
    p = nise.params_from_keywords(kw, files, precision=nise.FP64)
    with nise.Context(p) as c:
        c.load_files()
        re, im, n = c.absorption()
        w0, sr0, si0 = c.absorption_fft(re, im, n)
        w, sr, si = c.absorption_model(np.zeros(p.singles), 1.0, p.lifetime)
    err = helpers.rel(sr + 1j * si, sr0 + 1j * si0)
    print("exact model vs FP64 absorption (%s, %s): %.2e" % (ham, prop, err))
    assert np.allclose(w, w0, rtol=0, atol=1e-9)
    assert err < 1e-11


@pytest.mark.parametrize("tmax, frames, dt, sigma", [(40, 400, 2.0, 10.0), (100, 500, 2.0, 10.0),
                                                     (40, 400, 12.0, 250.0)])
def test_exact_adjoint_matches_central_differences(tmax, frames, dt, sigma, tmp_path):
    """tmax 40: one checkpoint block; tmax 100: four (K = 32); a 12 fs step
    over a 250 cm^-1 disorder: ||H|| f above 1, so every frame takes several
    sub-steps."""
    kw, files = make_case(tmp_path, frames=frames, tmax=tmax, dt=dt, sigma=sigma)
    bound = norm_bound(kw, files, 8)
    assert (bound > 1.0) == (dt > 10)
    p = nise.params_from_keywords(kw, files, precision=nise.FP64)
    rng = np.random.default_rng(11)
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
    print("exact adjoint vs central differences, tmax %d, dt %g (|H| f %.2f): per-component %.2e"
          % (tmax, dt, bound, err))
    assert err < ADJ_VS_FD, (adj, fd)
