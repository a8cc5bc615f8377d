"""The eigen route above the shared-memory Jacobi's 120 sites.

Per-frame couplings (HamiltonianType Full), truncating thresholds and
kernel_config 2 need each frame's exact propagator U = V exp(-i e f) V^T
(propagate_vec_DIA / propagate_vec_DIA_S, propagate.c:60-258): frames above
120 sites are diagonalised by Householder tridiagonalisation and implicit QR
(eigen_large.cu).  Checked against the FP64 exact restatement
(oracle.absorption_exact: numpy eigendecompositions, one per frame), the
static-coupling Taylor route, and the reference program's output at 256
sites (tests/golden/make_golden_large.py).
"""
import json
import os

import numpy as np
import pytest

import helpers
import nise_2017_b200 as nise
import oracle
from nise_2017_b200 import synth

pytestmark = pytest.mark.gpu

SPARSE_FP32 = 3e-6
# the tensor-core apply against the per-start-point FP32 kernel: the tensor
# core's product alignment rounds toward zero (measured 1.2e-6 over 48 steps)
TC_VS_SCALAR = 2e-6


def absorb(kw, files, **engine):
    p = nise.params_from_keywords(kw, files, **engine)
    with nise.Context(p) as c:
        c.load_files()
        re, im, n = c.absorption()
    return re + 1j * im, n


@pytest.mark.parametrize("n_sites, geometry", [(256, synth.CHAIN), (512, synth.LATTICE)])
def test_full_type_exact_propagator(n_sites, geometry, tmp_path):
    """Propagation Sparse, Threshold 0, per-frame couplings, FP32 and FP64."""
    extra = dict(spacing=8.0, eps0=15000.0, sigma=300.0, tau_fs=50.0, jcut=2.0, dt_fs=1.0) \
        if geometry == synth.LATTICE else dict(dt_fs=2.0)
    s = synth.spec(n_sites=n_sites, frames=70, geometry=geometry, seed=400 + n_sites, **extra)
    files = synth.write(s, str(tmp_path))
    if geometry == synth.LATTICE:
        kw = synth.c1_keywords(Singles=n_sites, Length=70, RunTimes="10 0 0", Samplerate=20, HamiltonianType="Full")
    else:
        kw = synth.c0_keywords(Singles=n_sites, Length=70, RunTimes="10 0 0", Samplerate=20, Propagation="Sparse",
                               Threshold=0)
    ex_re, ex_im, en = oracle.absorption_exact(kw, files)
    ex = ex_re + 1j * ex_im
    r32, n32 = absorb(kw, files)
    r64, n64 = absorb(kw, files, precision=nise.FP64)
    assert n32 == n64 == en == 3
    assert helpers.rel(r64, ex) < 1e-9
    assert helpers.rel(r32, ex) < SPARSE_FP32
    # Diagonal is the same exact propagator
    rd, _ = absorb(dict(kw, Propagation="Diagonal"), files, precision=nise.FP64)
    assert helpers.rel(rd, ex) < 1e-9


def test_truncated_sparse_above_120_sites(tmp_path):
    """Threshold > 0 (propagate_vec_DIA_S): elements of U with |U|^2 below the
    scaled threshold are dropped before the step."""
    s = synth.spec(n_sites=200, frames=70, dt_fs=2.0, geometry=synth.CHAIN, j_nn=-12.0, seed=410)
    files = synth.write(s, str(tmp_path))
    kw = synth.c0_keywords(Singles=200, Length=70, RunTimes="10 0 0", Samplerate=20, Propagation="Sparse",
                           Threshold=100000)
    ex_re, ex_im, en = oracle.absorption_exact(kw, files)
    ex = ex_re + 1j * ex_im
    full_re, full_im, _ = oracle.absorption_exact(dict(kw, Threshold=0), files)
    assert helpers.rel(full_re + 1j * full_im, ex) > 1e-4  # the truncation matters
    r64, _ = absorb(kw, files, precision=nise.FP64)
    r32, _ = absorb(kw, files)
    assert helpers.rel(r64, ex) < 1e-9
    assert helpers.rel(r32, ex) < SPARSE_FP32


def test_forced_eigen_route_matches_taylor_route_on_a_lattice(tmp_path):
    """kernel_config 2 diagonalises every frame of a static-coupling lattice
    (300 sites); the default for static couplings is the sparse Taylor series,
    the same exact propagator."""
    s = synth.c1_spec(n_sites=300, frames=60, seed=420)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Singles=300, Length=60, RunTimes="12 0 0", Samplerate=12, Propagation="Diagonal")
    re_e, ne = absorb(kw, files, precision=nise.FP64, kernel_config=2)
    re_t, nt = absorb(kw, files, precision=nise.FP64)
    assert ne == nt
    assert helpers.rel(re_e, re_t) < 1e-9


@pytest.mark.parametrize("case", ["full_256", "trunc_256"])
def test_eigen_route_matches_reference_at_256_sites(case, tmp_path):
    """Against the reference program (absorption.c with propagate_vec_DIA[_S]
    at 256 sites): the engine's FP32 error against the FP64 exact responses is
    no larger than the reference's, and the two agree to 1e-5."""
    d = np.load(os.path.join(helpers.GOLDEN, "large_eig.npz"))
    spec = json.loads(str(d["meta"]))[case]
    files = synth.write(synth.spec(**spec["spec"]), str(tmp_path))
    r32, n = absorb(spec["keywords"], files)
    ex = (d[case + "_exact"][0] + 1j * d[case + "_exact"][1]) / int(d[case + "_samples"])
    td = d[case + "_td"][:, 1] + 1j * d[case + "_td"][:, 2]
    err_ref = helpers.rel(td, ex)
    err32 = helpers.rel(r32 / n, ex)
    print("eigen route %s: engine FP32 %.2e, reference %.2e of the FP64 exact responses; engine vs reference %.2e"
          % (case, err32, err_ref, helpers.rel(r32 / n, td)))
    assert err32 <= max(err_ref, 2e-7)
    assert helpers.rel(r32 / n, td) < 1e-5


def test_linear_technique_above_120_sites(tmp_path):
    """LD with Propagation Sparse on per-frame couplings (the per-frame
    propagator tables of the linear techniques), 200 sites, FP64 against the
    FP64 restatement."""
    s = synth.spec(n_sites=200, frames=40, dt_fs=2.0, geometry=synth.CHAIN, seed=430)
    files = synth.write(s, str(tmp_path))
    kw = synth.c0_keywords(Singles=200, Length=40, RunTimes="6 0 0", Samplerate=30, Propagation="Sparse",
                           Threshold=0, Technique="LD", EndPoint=1)
    p = nise.params_from_keywords(kw, files, precision=nise.FP64)
    with nise.Context(p) as c:
        c.load_files()
        re, im, n = c.linear()
    ore, oim, on = oracle.linear(oracle.params(kw, files), "f64")
    assert n == on
    assert helpers.rel(np.asarray(re) + 1j * np.asarray(im), ore + 1j * oim) < 1e-9


@pytest.mark.parametrize("name", ["abs_sparse_full", "abs_sparse_trunc"])
def test_tensor_core_apply_matches_scalar_apply(name, tmp_path):
    """kernel_config 17 applies the propagators on the tensor cores (3xTF32,
    time-major) even below 120 sites; 16 keeps the per-start-point kernel with
    the reference's float accumulation.  Both against each other and against
    the FP64 restatement."""
    case = helpers.cases()[name]
    files = helpers.materialise(case, str(tmp_path))
    tc, n1 = absorb(case["keywords"], files, kernel_config=17)
    sc, n2 = absorb(case["keywords"], files, kernel_config=16)
    ore, oim, on = oracle.absorption(oracle.params(case["keywords"], files), "f64")
    assert n1 == n2 == on
    print("%s: tensor cores vs per-start-point kernel %.2e; vs FP64 %.2e (per-start-point %.2e)"
          % (name, helpers.rel(tc, sc), helpers.rel(tc, ore + 1j * oim), helpers.rel(sc, ore + 1j * oim)))
    assert helpers.rel(tc, sc) < TC_VS_SCALAR
    assert helpers.rel(tc, ore + 1j * oim) < SPARSE_FP32


def test_tensor_core_apply_wide_state(tmp_path):
    """64 state columns (20 start points in flight, 3 polarisations), 160
    sites (a partial 128-row tile and 32-site chunk), against the FP64
    restatement."""
    s = synth.spec(n_sites=160, frames=120, dt_fs=2.0, geometry=synth.CHAIN, seed=440)
    files = synth.write(s, str(tmp_path))
    kw = synth.c0_keywords(Singles=160, Length=120, RunTimes="40 0 0", Samplerate=2, Propagation="Sparse",
                           Threshold=0)
    ex_re, ex_im, en = oracle.absorption_exact(kw, files)
    r32, n = absorb(kw, files)
    sc, _ = absorb(kw, files, kernel_config=16)
    assert n == en == 40
    print("wide state: tensor cores vs FP64 %.2e, per-start-point kernel vs FP64 %.2e"
          % (helpers.rel(r32, ex_re + 1j * ex_im), helpers.rel(sc, ex_re + 1j * ex_im)))
    assert helpers.rel(r32, ex_re + 1j * ex_im) < SPARSE_FP32
    assert helpers.rel(r32, sc) < TC_VS_SCALAR


def test_streamed_propagators_above_1024_sites(tmp_path):
    """A batched FP32 eigen-route job builds and applies the propagators in
    chunks of frames (only a chunk of U is held), which takes it past 1024
    sites: 1100 sites, per-frame couplings, against the FP64 exact
    restatement."""
    s = synth.spec(n_sites=1100, frames=24, geometry=synth.LATTICE, spacing=8.0, eps0=15000.0, sigma=300.0,
                   tau_fs=50.0, jcut=2.0, dt_fs=1.0, seed=450)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Singles=1100, Length=24, RunTimes="4 0 0", Samplerate=10, HamiltonianType="Full")
    ex_re, ex_im, en = oracle.absorption_exact(kw, files)
    r32, n = absorb(kw, files)
    assert n == en > 0
    print("1100 sites, streamed propagators: FP32 vs FP64 exact %.2e" % helpers.rel(r32, ex_re + 1j * ex_im))
    assert helpers.rel(r32, ex_re + 1j * ex_im) < SPARSE_FP32
    # FP64 has no tensor-core apply, so it keeps every frame's U: 1024 sites at most
    p = nise.params_from_keywords(kw, files, precision=nise.FP64)
    with nise.Context(p) as c:
        c.load_files()
        with pytest.raises(nise.NiseError):
            c.absorption()
