"""Linear absorption on the GPU, through the C ABI, against the oracle.

FP32 contexts reproduce the reference's single-precision operations, so for
the Trotter (Coupling) and RK4 schemes every propagated vector is
bit-identical to the oracle's FP32 restatement and the FP64 response sums
differ only in summation order.  The Sparse scheme (exact exp(-iHdt)) is
compared with the FP64 oracle, whose eigen-propagator is exact to rounding.
"""
import os
import subprocess

import numpy as np
import pytest

import helpers
import nise_2017_b200 as nise
import oracle

pytestmark = pytest.mark.gpu

CASES = helpers.cases()
ABS = [k for k, c in CASES.items() if c["keywords"]["Technique"] == "Absorption"]
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# Tolerances (max |difference| / max |reference|):
SUM_ORDER = 1e-11      # same arithmetic, different FP64 summation order
PRINT = 2e-6           # reference output printed with 7 significant digits
SPARSE_FP32 = 3e-6     # FP32 Taylor series vs exact propagator
REF_EIGEN = 1.5e-5     # reference's own ssyev_ rounding (Sparse cases)


def run_engine(case, files, **engine):
    p = nise.params_from_keywords(case["keywords"], files, **engine)
    with nise.Context(p) as c:
        c.load_files()
        re, im, n = c.absorption()
        spec = c.absorption_fft(re, im, n)
        ms, main_ms, launches = c.timing()
        flops, hbm = c.work()
    assert launches >= 2 and 0 < main_ms <= ms and flops > 0 and hbm > 0
    return p, re, im, n, spec


@pytest.mark.parametrize("name", ABS)
def test_fp32_matches_oracle_and_reference(name, tmp_path):
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    p, re, im, n, (w, sr, si) = run_engine(case, files)
    po = oracle.params(case["keywords"], files)
    g = helpers.golden(name)
    if helpers.uses_eigen(case):
        ore, oim, on = oracle.absorption(po, "f64")
        assert n == on
        assert helpers.rel(re + 1j * im, ore + 1j * oim) < SPARSE_FP32
        assert helpers.rel(np.stack([re / n, im / n], 1), g["td"][:, 1:]) < REF_EIGEN
    else:
        ore, oim, on = oracle.absorption(po, "f32a64")
        assert n == on
        assert helpers.rel(re + 1j * im, ore + 1j * oim) < SUM_ORDER
        assert helpers.rel(np.stack([re / n, im / n], 1), g["td"][:, 1:]) < PRINT
    # 1D spectrum on the device vs the reference's Absorption.dat
    spec = g["spec"]
    assert len(w) == len(spec)
    assert np.abs(w - spec[:, 0]).max() < 1e-3
    tol = REF_EIGEN if helpers.uses_eigen(case) else PRINT
    assert helpers.rel(np.stack([sr, si], 1), spec[:, 1:]) < tol


@pytest.mark.parametrize("name", ABS)
def test_fp64_matches_fp64_oracle(name, tmp_path):
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    p, re, im, n, (w, sr, si) = run_engine(case, files, precision=nise.FP64)
    po = oracle.params(case["keywords"], files)
    ore, oim, on = oracle.absorption(po, "f64")
    assert n == on
    tol = 1e-9 if helpers.uses_eigen(case) else 1e-10
    assert helpers.rel(re + 1j * im, ore + 1j * oim) < tol
    ow, osr, osi = oracle.spectrum(po, ore, oim, on, "f64")
    assert np.allclose(w, ow, rtol=0, atol=1e-9)
    assert helpers.rel(sr + 1j * si, osr + 1j * osi) < 1e-9


@pytest.mark.parametrize("name", ["abs_coupling_full", "abs_rk4_full", "abs_sparse_static"])
def test_plain_equals_batched(name, tmp_path):
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    _, re_b, im_b, n_b, _ = run_engine(case, files)
    _, re_p, im_p, n_p, _ = run_engine(case, files, launch_mode=nise.PLAIN)
    assert n_b == n_p
    if case["keywords"]["Propagation"] == "Sparse":
        assert helpers.rel(re_p + 1j * im_p, re_b + 1j * im_b) < 1e-6
    else:
        assert np.array_equal(re_b, re_p) and np.array_equal(im_b, im_p)


@pytest.mark.parametrize("name", ["abs_sparse_full", "abs_sparse_trunc"])
def test_eigen_route_plain_equals_batched(name, tmp_path):
    """The eigen route runs the same per-start-point kernel batched or one start point per launch."""
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    _, re_b, im_b, n_b, _ = run_engine(case, files)
    _, re_p, im_p, n_p, _ = run_engine(case, files, launch_mode=nise.PLAIN)
    assert n_b == n_p
    assert np.array_equal(re_b, re_p) and np.array_equal(im_b, im_p)


def test_diagonal_scheme_matches_reference_sparse(tmp_path):
    """Propagation Diagonal (rejected by the reference) is checked against the
    reference's Sparse + Threshold 0 output on the same trajectory."""
    case = CASES["abs_sparse_full"]
    files = helpers.materialise(case, str(tmp_path))
    kw = dict(case["keywords"], Propagation="Diagonal")
    p, re, im, n, (w, sr, si) = run_engine(dict(case, keywords=kw), files)
    g = helpers.golden("abs_sparse_full")
    assert helpers.rel(np.stack([re / n, im / n], 1), g["td"][:, 1:]) < REF_EIGEN
    assert helpers.rel(np.stack([sr, si], 1), g["spec"][:, 1:]) < REF_EIGEN
    ore, oim, on = oracle.absorption(oracle.params(case["keywords"], files), "f64")
    assert helpers.rel(re + 1j * im, ore + 1j * oim) < SPARSE_FP32


@pytest.mark.parametrize("prop", ["Sparse", "Diagonal"])
def test_eigen_route_matches_taylor_route(prop, tmp_path):
    """Two exact propagators of static couplings: the eigen route (forced by
    kernel_config 2) and the sparse Taylor series (the default for static
    couplings), both in FP64."""
    case = CASES["abs_sparse_static"]
    files = helpers.materialise(case, str(tmp_path))
    kw = dict(case["keywords"], Propagation=prop)
    _, re_t, im_t, _, _ = run_engine(dict(case, keywords=kw), files, precision=nise.FP64)
    _, re_e, im_e, _, _ = run_engine(dict(case, keywords=kw), files, precision=nise.FP64, kernel_config=2)
    assert helpers.rel(re_e + 1j * im_e, re_t + 1j * im_t) < 1e-9


@pytest.mark.parametrize("cfg", [3, 8, 9, 10, 12])
def test_exact_propagator_kernels_agree(cfg, tmp_path):
    """Every kernel of the static-coupling exact propagator (Taylor series with
    4 or 8 vectors per CTA, sliced-ELL Taylor, sliced-ELL Chebyshev) against
    the FP64 oracle's eigen-propagator."""
    case = CASES["abs_sparse_static"]
    files = helpers.materialise(case, str(tmp_path))
    _, re, im, n, _ = run_engine(case, files, kernel_config=cfg)
    ore, oim, on = oracle.absorption(oracle.params(case["keywords"], files), "f64")
    assert n == on
    assert helpers.rel(re + 1j * im, ore + 1j * oim) < SPARSE_FP32


@pytest.mark.parametrize("n", [1300, 2048])
def test_taylor_route_large_lattice(n, tmp_path):
    """Static lattice couplings beyond what the shared-memory ELL kernel holds
    (the launcher falls back to smaller tiles): FP32 against FP64, and plain
    against batched."""
    from nise_2017_b200 import synth
    s = synth.c1_spec(n_sites=n, frames=48, seed=70 + n)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Singles=n, Length=48, RunTimes="8 0 0", Samplerate=12)
    case = dict(keywords=kw)
    _, re32, im32, n32, _ = run_engine(case, files)
    _, re64, im64, n64, _ = run_engine(case, files, precision=nise.FP64)
    _, rep, imp, np_, _ = run_engine(case, files, launch_mode=nise.PLAIN)
    assert n32 == n64 == np_
    assert helpers.rel(re32 + 1j * im32, re64 + 1j * im64) < SPARSE_FP32
    assert helpers.rel(rep + 1j * imp, re32 + 1j * im32) < 1e-6


def test_taylor3_full_waves_and_tail(tmp_path):
    """More vectors than one wave of 8-vector CTAs: whole waves run on the
    8-vector layout and the rest on 1-vector CTAs; every start point must
    match the FP64 oracle, wherever its vectors landed."""
    from nise_2017_b200 import synth
    s = synth.c1_spec(n_sites=27, frames=900, seed=78)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Singles=27, Length=900, RunTimes="16 0 0", Samplerate=2)
    case = dict(keywords=kw)
    p = nise.params_from_keywords(kw, files, kernel_config=8)
    with nise.Context(p) as c:
        c.load_files()
        re, im, n = c.absorption()
        _, _, launches = c.timing()
    assert n == 442 and launches >= 3  # 1326 vectors: 148 CTAs of 8, then 142 vectors on 1-vector CTAs
    ore, oim, on = oracle.absorption(oracle.params(kw, files), "f64")
    assert n == on
    assert helpers.rel(re + 1j * im, ore + 1j * oim) < SPARSE_FP32


def test_taylor3_wide_ctas_on_1024_sites(tmp_path):
    """The benchmark lattice with more than a wave of vectors: 8-vector CTAs
    of 768 threads (the FP32 layout for 513..1056 sites) plus 1-vector CTAs,
    against the FP64 run and against the 4-vector Taylor kernel."""
    from nise_2017_b200 import synth
    s = synth.c1_spec(frames=816, seed=79)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Length=816, RunTimes="16 0 0", Samplerate=2)
    case = dict(keywords=kw)
    _, re32, im32, n32, _ = run_engine(case, files, kernel_config=8)
    _, re64, im64, n64, _ = run_engine(case, files, precision=nise.FP64)
    _, ret2, imt2, nt2, _ = run_engine(case, files, kernel_config=3)
    assert n32 == n64 == nt2 == 400  # 1200 vectors: 148 CTAs of 8, then 16 on 1-vector CTAs
    assert helpers.rel(re32 + 1j * im32, re64 + 1j * im64) < SPARSE_FP32
    assert helpers.rel(re32 + 1j * im32, ret2 + 1j * imt2) < SPARSE_FP32


def test_c1_lattice_full_coherence_time(tmp_path):
    """The benchmark lattice (N = 1024, static couplings, Propagation Sparse)
    over its full 256-step coherence time: the FP32 series, truncated below
    the FP32 unit roundoff per step, stays within 1e-5 of the FP64 run."""
    from nise_2017_b200 import synth
    s = synth.c1_spec(frames=560, seed=77)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Length=560, Samplerate=150)
    case = dict(keywords=kw)
    _, re32, im32, n32, _ = run_engine(case, files)
    _, re64, im64, n64, _ = run_engine(case, files, precision=nise.FP64)
    assert n32 == n64 == 3
    assert helpers.rel(re32 + 1j * im32, re64 + 1j * im64) < 1e-5


def random_hamiltonians(rng, nvec, n, cut):
    nn2 = n * (n + 1) // 2
    H = np.zeros((nvec, nn2), np.float32)
    for v in range(nvec):
        full = rng.normal(0, 30, size=(n, n))
        full = (full + full.T) / 2
        for a in range(n):
            for b in range(a, n):
                x = full[a, b] if a == b else full[a, b] / 4
                if a != b and abs(x) < cut:
                    x = 0.0
                H[v, b + a * (2 * n - a - 1) // 2] = x
    return H


@pytest.mark.parametrize("prop", ["Coupling", "RK4", "Sparse"])
@pytest.mark.parametrize("sign", [1, -1])
def test_single_steps_match_oracle(prop, sign):
    rng = np.random.default_rng(7)
    n, nvec = 9, 40
    kw = dict(Propagation=prop, Singles=n, Length=100, Samplerate=10, Timestep=2, RunTimes="10 0 0", Trotter=3,
              Couplingcut=1.0, Threshold=0, Technique="Absorption", MinFrequencies="-100 0 0",
              MaxFrequencies="100 0 0")
    H = random_hamiltonians(rng, nvec, n, 1.0)
    re = rng.normal(size=(nvec, n)).astype(np.float32)
    im = rng.normal(size=(nvec, n)).astype(np.float32)
    po = oracle.params(kw, {})
    for prec, dt in ((nise.FP32, np.float32), (nise.FP64, np.float64)):
        p = nise.params_from_keywords(kw, precision=prec)
        with nise.Context(p) as c:
            gr, gi = c.propagate(H, re.astype(dt), im.astype(dt), sign)
        olib = "f32" if prec == nise.FP32 else "f64"
        orr, oii = re.astype(dt).copy(), im.astype(dt).copy()
        for v in range(nvec):
            a, b = orr[v].copy(), oii[v].copy()
            oracle.lib(olib).oracle_propagate_vector(oracle.ctypes.byref(po), H[v].ctypes.data_as(oracle.ctypes.POINTER(
                oracle.ctypes.c_float)), a.ctypes.data, b.ctypes.data, sign)
            orr[v], oii[v] = a, b
        if prop == "Sparse":
            tol = 2e-6 if prec == nise.FP32 else 1e-11
            assert helpers.rel(gr + 1j * gi, orr + 1j * oii) < tol
        elif prec == nise.FP32:
            assert np.array_equal(gr, orr) and np.array_equal(gi, oii)
        else:
            assert helpers.rel(gr + 1j * gi, orr + 1j * oii) < 1e-13


@pytest.mark.parametrize("prop", ["Coupling", "Sparse"])
def test_unitarity_at_large_size(prop):
    """Trotter rotations and the exact propagator conserve the norm (N = 384)."""
    rng = np.random.default_rng(11)
    n, nvec = 384, 8
    kw = dict(Propagation=prop, Singles=n, Length=100, Samplerate=10, Timestep=1, RunTimes="10 0 0",
              Couplingcut=0.0, Technique="Absorption", MinFrequencies="-500 0 0", MaxFrequencies="500 0 0")
    nn2 = n * (n + 1) // 2
    H = np.zeros((nvec, nn2), np.float32)
    for v in range(nvec):
        for a in range(n):
            H[v, a * n + a - a * (a + 1) // 2] = rng.normal(0, 300)
            for b in (a + 1, a + 2):
                if b < n:
                    H[v, b + a * (2 * n - a - 1) // 2] = rng.normal(-8, 3)
    re = rng.normal(size=(nvec, n))
    im = rng.normal(size=(nvec, n))
    p = nise.params_from_keywords(kw, precision=nise.FP64)
    with nise.Context(p) as c:
        gr, gi = c.propagate(H, re, im, 1)
        br, bi = c.propagate(H, gr, gi, -1)
    n0 = (re ** 2 + im ** 2).sum(1)
    n1 = (gr ** 2 + gi ** 2).sum(1)
    assert np.allclose(n0, n1, rtol=1e-10)
    if prop == "Sparse":  # exact propagator: forward then backward is the identity
        assert helpers.rel(br + 1j * bi, re + 1j * im) < 1e-10


def test_driver_end_to_end(tmp_path):
    name = "abs_coupling_full"
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    from nise_2017_b200 import synth
    inp = synth.write_input(str(tmp_path / "input1D"), case["keywords"], files)
    exe = os.path.join(ROOT, "nise_2017_b200", "nise")
    r = subprocess.run([exe, inp], cwd=str(tmp_path), stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    g = helpers.golden(name)
    td = np.loadtxt(str(tmp_path / "TD_Absorption.dat"), ndmin=2)
    sp = np.loadtxt(str(tmp_path / "Absorption.dat"), ndmin=2)
    assert td.shape == g["td"].shape and sp.shape == g["spec"].shape
    assert helpers.rel(td[:, 1:], g["td"][:, 1:]) < PRINT
    assert helpers.rel(sp[:, 1:], g["spec"][:, 1:]) < PRINT
    assert np.abs(sp[:, 0] - g["spec"][:, 0]).max() < 1e-3


def test_error_paths(tmp_path):
    case = CASES["abs_coupling_full"]
    files = helpers.materialise(case, str(tmp_path))
    kw = dict(case["keywords"], Length=5000)  # longer than the 600-frame trajectory
    p = nise.params_from_keywords(kw, files)
    with nise.Context(p) as c:
        with pytest.raises(nise.NiseError) as e:
            c.absorption()
        assert e.value.code == -8  # no trajectory loaded
        c.load_files()
        with pytest.raises(nise.NiseError) as e:
            c.absorption()
        assert e.value.code == -2  # trajectory too short
