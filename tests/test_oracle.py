"""The oracle is pinned before it is trusted: the C restatement (FP32 build,
reference arithmetic) must reproduce the reference program's outputs stored in
tests/golden (generated from the reference compiled from its own sources), and
the FP64 build must stay within the reference's own single-precision error."""
import numpy as np
import pytest

import helpers
import oracle

CASES = helpers.cases()
ABS = [k for k, c in CASES.items() if c["keywords"]["Technique"] == "Absorption"]
LIN = [k for k, c in CASES.items() if c["keywords"]["Technique"] in oracle.LINEAR_FILES]
TWO_D = [k for k in CASES if k not in ABS and k not in LIN]
# print precision of the reference's %e output, plus float summation order
PRINT_TOL = 2e-6


@pytest.mark.parametrize("name", ABS)
def test_absorption_restatement_matches_reference(name, tmp_path):
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    g = helpers.golden(name)
    p = oracle.params(case["keywords"], files)
    re, im, n = oracle.absorption(p, "f32")
    td = g["td"]
    tol = 1e-5 if helpers.uses_eigen(case) else PRINT_TOL  # ssyev_ vs Jacobi eigenvectors
    assert helpers.rel(np.stack([re / n, im / n], 1), td[:, 1:]) < tol
    assert np.allclose(td[:, 0], np.arange(p.tmax1) * p.deltat)
    w, sr, si = oracle.spectrum(p, re, im, n, "f32")
    assert len(w) == len(g["spec"])
    assert np.abs(w - g["spec"][:, 0]).max() <= 1.5e-6 * np.abs(w).max() + 1e-6
    assert helpers.rel(np.stack([sr, si], 1), g["spec"][:, 1:]) < max(tol, PRINT_TOL)


@pytest.mark.parametrize("name", ABS)
def test_absorption_fp64_within_reference_rounding(name, tmp_path):
    """The FP32 reference itself is only accurate to ~1e-5 of the response."""
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    g = helpers.golden(name)
    p = oracle.params(case["keywords"], files)
    re, im, n = oracle.absorption(p, "f64")
    err = helpers.rel(np.stack([re / n, im / n], 1), g["td"][:, 1:])
    assert err < 1e-4


@pytest.mark.parametrize("name", LIN)
def test_linear_restatement_matches_reference(name, tmp_path):
    """LD, Raman, SFG, DOS, CD, Luminescence: every TD_*.dat and spectrum file."""
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    g = helpers.golden(name)
    p = oracle.params(case["keywords"], files)
    re, im, n = oracle.linear(p, "f32")
    tdk = helpers.td_channels(case["keywords"]["Technique"], oracle.LINEAR_FILES)
    assert len(re) == len(oracle.LINEAR_FILES[case["keywords"]["Technique"]]) and len(tdk) == len(g["td"])
    tol = 1e-5 if helpers.uses_eigen(case) else PRINT_TOL
    for j, k in enumerate(tdk):
        assert helpers.rel(np.stack([re[k] / n, im[k] / n], 1), g["td"][j][:, 1:]) < tol
    for k in range(len(re)):
        w, sr, si = oracle.spectrum(p, re[k], im[k], n, "f32")
        assert len(w) == len(g["spec"][k])
        assert helpers.rel(np.stack([sr, si], 1), g["spec"][k][:, 1:]) < max(tol, PRINT_TOL)


@pytest.mark.parametrize("name", LIN)
def test_linear_fp64_within_reference_rounding(name, tmp_path):
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    g = helpers.golden(name)
    p = oracle.params(case["keywords"], files)
    re, im, n = oracle.linear(p, "f64")
    # CD and SSP responses are small differences of large terms: the reference's
    # single-precision propagation error reaches 3e-4 of them (static CD)
    for j, k in enumerate(helpers.td_channels(case["keywords"]["Technique"], oracle.LINEAR_FILES)):
        assert helpers.rel(np.stack([re[k] / n, im[k] / n], 1), g["td"][j][:, 1:]) < 5e-4


@pytest.mark.parametrize("name", TWO_D)
def test_2d_restatement_matches_reference(name, tmp_path):
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    g = helpers.golden(name)["R"]
    p = oracle.params(case["keywords"], files)
    R, n = oracle.twodir(p, "f32")
    Rn = helpers.R12_to_files(oracle.normalize_2d(p, R, n, "f32"))
    # Eigen paths (t2 > 0 or Sparse) differ from ssyev_ by eigenvector
    # rounding, which GB+SE+EA cancellation amplifies.
    tol = 5e-4 if helpers.uses_eigen(case) else PRINT_TOL
    assert helpers.rel2d(Rn, g) < tol


@pytest.mark.parametrize("name", TWO_D)
def test_2d_fp64_within_reference_rounding(name, tmp_path):
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    g = helpers.golden(name)["R"]
    p = oracle.params(case["keywords"], files)
    R, n = oracle.twodir(p, "f64")
    Rn = helpers.R12_to_files(oracle.normalize_2d(p, R, n, "f64"))
    assert helpers.rel2d(Rn, g) < 2e-3


def test_diagonal_hamiltonian_is_exact(tmp_path):
    """With no couplings NISE is exact: S(t) = sum_i mu_i^2 exp(-i sum_k w_i f)."""
    from nise_2017_b200 import synth
    s = synth.spec(n_sites=6, frames=200, dt_fs=2.0, j_nn=0.0, j_sigma=0.0, mu_jitter=0.0, ham_type=synth.FULL,
                   seed=5)
    files = synth.write(s, str(tmp_path))
    kw = synth.c0_keywords(Singles=6, Length=200, RunTimes="32 0 0", Samplerate=50)
    p = oracle.params(kw, files)
    re, im, n = oracle.absorption(p, "f64")
    E = np.fromfile(files["energy"], dtype=np.float32).reshape(200, 1 + 21)[:, 1:]
    mu = np.fromfile(files["dipole"], dtype=np.float32).reshape(-1, 1 + 18)[:, 1:]
    diag_idx = [i * 6 + i - i * (i + 1) // 2 for i in range(6)]
    shift = (1550 + 1750) / 2
    f = np.float64(np.float32(np.float32(2.0 * np.float32(2.99792458e-5)) * np.float32(2 * 3.14159265359)))
    S = np.zeros(32, complex)
    for smp in range(n):
        ti = smp * 50
        for x in range(3):
            m0 = mu[ti, x * 6:(x + 1) * 6].astype(np.float64)
            ph = np.zeros(6)
            for t1 in range(32):
                mt = mu[ti + t1, x * 6:(x + 1) * 6].astype(np.float64)
                S[t1] += np.sum(mt * m0 * np.exp(-1j * ph))
                ph += (E[ti + t1, diag_idx].astype(np.float32) - np.float32(shift)).astype(np.float64) * f
    assert helpers.rel(re + 1j * im, S) < 1e-8  # 10 rounded half-phase products per step


def test_fft_restatement_matches_numpy():
    """Direct DFT of the restatement equals numpy's FFT of the same input."""
    p = oracle.OracleParams()
    p.tmax1, p.fft, p.deltat, p.min1, p.max1 = 64, 256, 2.0, -1e9, 1e9
    rng = np.random.default_rng(0)
    re, im = rng.normal(size=64), rng.normal(size=64)
    w, sr, si = oracle.spectrum(p, re, im, 1, "f64")
    x = np.zeros(256, complex)
    x[:64] = im + 1j * re
    x[0] *= 0.5
    X = np.fft.fft(x) * 2 * np.float64(np.float32(2.0)) * np.float64(np.float32(2.99792458e-5))
    order = list(range(128, 256)) + list(range(0, 128))
    assert np.allclose(sr, X.imag[order], rtol=0, atol=1e-12 * np.abs(X).max())
    assert np.allclose(si, X.real[order], rtol=0, atol=1e-12 * np.abs(X).max())


@pytest.mark.parametrize("case", ["t2_0", "t2_4"])
def test_restatement_reproduces_reference_at_2dir_benchmark_size(case, tmp_path):
    """The FP32 restatement (float response sums, the reference's arithmetic)
    against the reference program's R*.dat files on the 64-site cluster of
    the 2DIR benchmark (tests/golden/make_golden_large.py): print precision
    for t2 = 0; with t2 > 0 the t2 step's eigenvectors (ssyev_ vs Jacobi)
    differ by rounding that the GB + SE + EA cancellation amplifies."""
    import json
    import os
    from nise_2017_b200 import synth
    d = np.load(os.path.join(helpers.GOLDEN, "large_c2_2dir.npz"))
    spec = json.loads(str(d["meta"]))[case]
    files = synth.write(synth.c2_spec(**spec["spec"]), str(tmp_path))
    po = oracle.params(spec["keywords"], files)
    R, n = oracle.twodir(po, "f32")
    Rn = helpers.R12_to_files(oracle.normalize_2d(po, R, n, "f64"))
    t2 = int(str(spec["keywords"]["RunTimes"]).split()[1])
    assert helpers.rel2d(Rn, d[case]) < (5e-4 if t2 > 0 else 2e-6)


@pytest.mark.parametrize("name", ["abs_sparse_static", "abs_sparse_full", "abs_sparse_trunc", "abs_sparse_trunc_static"])
def test_exact_restatement_matches_c_restatement(name, tmp_path):
    """oracle.absorption_exact (numpy FP64: one eigendecomposition per frame,
    shared by every vector crossing it; truncation as propagate_vec_DIA_S)
    against the C restatement's FP64 build and the reference's output: the
    checker of the large-site tests."""
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    re, im, n = oracle.absorption_exact(case["keywords"], files)
    ore, oim, on = oracle.absorption(oracle.params(case["keywords"], files), "f64")
    assert n == on
    assert helpers.rel(re + 1j * im, ore + 1j * oim) < 1e-12
    assert helpers.rel(np.stack([re / n, im / n], 1), helpers.golden(name)["td"][:, 1:]) < 1e-5
