"""2DIR family on the GPU, through the C ABI, against the oracle.

The engine reorganises the reference's work items (per-component singles
vectors, conjugated SE snapshots as EA right vectors, 9+9*tmax1 doubles
vectors per start point) but keeps every propagated vector's single-precision
operations, so FP32 results match the FP32-propagation/FP64-sum oracle to
summation-order rounding wherever no eigendecomposition is involved.
"""
import os
import subprocess

import numpy as np
import pytest

import helpers
import nise_2017_b200 as nise
import oracle
from nise_2017_b200 import synth

pytestmark = pytest.mark.gpu

CASES = helpers.cases()
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SUPPORTED = ["2d_coupling", "2d_coupling_t2", "2d_rk4", "2d_sparse", "2d_sparse_trunc", "2d_full_anhfile", "2d_gbir",
             "2d_seir", "2d_eair", "2d_tdc", "2d_uvvis", "2d_uvvis_rk4", "2d_uvvis_sparse", "2d_eauvvis_full",
             "2d_noeauvvis"]

SUM_ORDER = 1e-10   # same single-precision operations, FP64 sums in another order
T2_EIGEN = 1e-5     # t2 eigenvectors from a different Jacobi ordering (rounded to float)
REF_FP32_SUMS = 1e-5  # the reference sums the 2D response in float; GB+SE+EA cancellation amplifies it
REF_EIGEN = 5e-4    # the reference's ssyev_ rounding, amplified by GB+SE+EA cancellation


def run(kw, files, **engine):
    p = nise.params_from_keywords(kw, files, **engine)
    with nise.Context(p) as c:
        c.load_files()
        R, n = c.twodir()
        tot, main, launches = c.timing()
    assert launches >= 4 and main > 0
    return p, R, n


@pytest.mark.parametrize("name", SUPPORTED)
def test_fp32_matches_oracle_and_reference(name, tmp_path):
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    p, R, n = run(case["keywords"], files)
    po = oracle.params(case["keywords"], files)
    oR, on = oracle.twodir(po, "f32a64")
    assert n == on
    eig = helpers.uses_eigen(case)
    if case["keywords"].get("Propagation") in ("Sparse", "Diagonal"):
        # Exact propagators from FP64 eigenvectors: the engine's FP32 run must be
        # at least as close to the FP64 result as the FP32 restatement is.
        oR64, _ = oracle.twodir(po, "f64")
        assert helpers.rel2d(R, oR64) <= max(helpers.rel2d(oR, oR64), T2_EIGEN)
    else:
        assert helpers.rel2d(R, oR) < (T2_EIGEN if eig else SUM_ORDER)
    Rn = helpers.R12_to_files(oracle.normalize_2d(po, R, n, "f64"))
    assert helpers.rel2d(Rn, helpers.golden(name)["R"]) < (REF_EIGEN if eig else REF_FP32_SUMS)


@pytest.mark.parametrize("name", ["2d_coupling", "2d_coupling_t2", "2d_eair", "2d_sparse", "2d_uvvis",
                                  "2d_uvvis_sparse", "2d_uvvis_rk4"])
def test_fp64_matches_fp64_oracle(name, tmp_path):
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    p, R, n = run(case["keywords"], files, precision=nise.FP64)
    oR, on = oracle.twodir(oracle.params(case["keywords"], files), "f64")
    assert n == on
    assert helpers.rel2d(R, oR) < (1e-9 if helpers.uses_eigen(case) else 1e-11)


@pytest.mark.parametrize("tech", ["GBIR", "SEIR", "noEAIR", "EAIR", "2DIR"])
def test_rk4_techniques(tech, tmp_path):
    s = synth.c2_spec(n_sites=6, frames=300, seed=31)
    files = synth.write(s, str(tmp_path))
    kw = synth.c2_keywords(Singles=6, Length=300, RunTimes="8 2 8", Samplerate=40, Propagation="RK4", Technique=tech)
    p, R, n = run(kw, files)
    oR, on = oracle.twodir(oracle.params(kw, files), "f32a64")
    assert n == on and helpers.rel2d(R, oR) < T2_EIGEN


@pytest.mark.parametrize("tech", ["GBUVvis", "SEUVvis", "noEAUVvis", "EAUVvis", "2DUVvis"])
def test_rk4_uvvis_techniques(tech, tmp_path):
    """The two-level (calc_2DES) doubles with RK4 and t2 > 0; no anharmonicity
    or overtone file is read."""
    s = synth.c2_spec(n_sites=6, frames=300, seed=32)
    files = synth.write(s, str(tmp_path))
    kw = synth.c2_keywords(Singles=6, Length=300, RunTimes="8 2 8", Samplerate=40, Propagation="RK4", Technique=tech,
                           Anharmonicity=0)
    p, R, n = run(kw, files)
    oR, on = oracle.twodir(oracle.params(kw, files), "f32a64")
    assert n == on and helpers.rel2d(R, oR) < T2_EIGEN


def test_uvvis_cluster_n40(tmp_path):
    """2DUVvis at N = 40 (two columns per lane in the doubles kernel)."""
    s = synth.c2_spec(n_sites=40, frames=200, seed=44)
    files = synth.write(s, str(tmp_path))
    kw = synth.c2_keywords(Singles=40, Length=200, RunTimes="6 0 6", Samplerate=80, Technique="2DUVvis",
                           Anharmonicity=0)
    p, R, n = run(kw, files)
    oR, on = oracle.twodir(oracle.params(kw, files), "f32a64")
    assert n == on
    assert helpers.rel2d(R, oR) < SUM_ORDER


def test_larger_cluster_and_chunks(tmp_path):
    """N = 24 oscillators, 7 start points, t2 > 0."""
    s = synth.c2_spec(n_sites=24, frames=400, seed=41)
    files = synth.write(s, str(tmp_path))
    kw = synth.c2_keywords(Singles=24, Length=400, RunTimes="12 4 12", Samplerate=60)
    p, R, n = run(kw, files)
    oR, on = oracle.twodir(oracle.params(kw, files), "f32a64")
    assert n == on == 7
    assert helpers.rel2d(R, oR) < T2_EIGEN


def test_cluster_n40(tmp_path):
    """N = 40 (two columns per lane in the doubles kernel), tmax 6, no t2."""
    s = synth.c2_spec(n_sites=40, frames=200, seed=43)
    files = synth.write(s, str(tmp_path))
    kw = synth.c2_keywords(Singles=40, Length=200, RunTimes="6 0 6", Samplerate=80)
    p, R, n = run(kw, files)
    oR, on = oracle.twodir(oracle.params(kw, files), "f32a64")
    assert n == on
    assert helpers.rel2d(R, oR) < SUM_ORDER


@pytest.mark.parametrize("name", ["2d_coupling", "2d_coupling_t2", "2d_uvvis"])
def test_plain_matches_batched(name, tmp_path):
    """One start point per launch of every kernel gives the batched result
    (the start points' responses are summed in another grouping)."""
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    _, Rb, nb = run(case["keywords"], files)
    _, Rp, np_ = run(case["keywords"], files, launch_mode=nise.PLAIN)
    assert nb == np_
    assert helpers.rel2d(Rp, Rb) < 1e-12


def test_diagonal_scheme_matches_reference_sparse(tmp_path):
    """Propagation Diagonal (rejected by the reference) against the reference's
    Sparse + Threshold 0 response files on the same trajectory."""
    case = CASES["2d_sparse"]
    files = helpers.materialise(case, str(tmp_path))
    kw = dict(case["keywords"], Propagation="Diagonal")
    p, R, n = run(kw, files)
    po = oracle.params(case["keywords"], files)
    Rn = helpers.R12_to_files(oracle.normalize_2d(po, R, n, "f64"))
    assert helpers.rel2d(Rn, helpers.golden("2d_sparse")["R"]) < REF_EIGEN


def test_eigen_schemes_size_limit(tmp_path):
    """Sparse/Diagonal 2DIR needs the per-frame eigensolver (at most 120 sites)."""
    s = synth.c2_spec(n_sites=121, frames=40, seed=5)
    files = synth.write(s, str(tmp_path))
    kw = synth.c2_keywords(Singles=121, Length=40, RunTimes="2 0 2", Samplerate=10, Propagation="Sparse",
                           Threshold=0)
    p = nise.params_from_keywords(kw, files)
    with nise.Context(p) as c:
        c.load_files()
        with pytest.raises(nise.NiseError) as e:
            c.twodir()
        assert e.value.code == -6


def test_driver_writes_reference_files(tmp_path):
    name = "2d_coupling"
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    inp = synth.write_input(str(tmp_path / "input2D"), case["keywords"], files)
    exe = os.path.join(ROOT, "nise_2017_b200", "nise")
    r = subprocess.run([exe, inp], cwd=str(tmp_path), stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    g = helpers.golden(name)["R"]
    T1 = 8
    got = np.zeros_like(g)
    for k, fn in enumerate(oracle.R2D_FILES):
        got[k, 0], got[k, 1] = oracle.read_2d(str(tmp_path / fn), T1, T1)
    assert helpers.rel2d(got, g) < REF_FP32_SUMS


@pytest.mark.parametrize("n_sites, tech, prec", [(40, "2DIR", "fp32"), (64, "2DIR", "fp32"), (64, "2DIR", "fp64"),
                                                 (48, "2DUVvis", "fp32")])
def test_two_warp_doubles_kernel_is_bitwise_the_one_warp_kernel(n_sites, tech, prec, tmp_path):
    """For 32 < N <= 64 the doubles vectors run on two warps each (one
    column per thread, named barriers where the rotations cross warps);
    kernel_config 1 keeps one warp per vector.  Same float operations in the
    same order: in FP32, whose operations are all separately rounded, the
    responses are bitwise equal; FP64 lets the compiler fuse multiply-adds,
    differently in the two kernels."""
    s = synth.c2_spec(n_sites=n_sites, frames=240, seed=60 + n_sites)
    files = synth.write(s, str(tmp_path))
    extra = dict(Anharmonicity=0) if tech == "2DUVvis" else {}
    kw = synth.c2_keywords(Singles=n_sites, Length=240, RunTimes="6 0 6", Samplerate=70, Technique=tech, **extra)
    precision = nise.FP64 if prec == "fp64" else nise.FP32
    _, R2w, n2 = run(kw, files, precision=precision)
    _, R1w, n1 = run(kw, files, precision=precision, kernel_config=1)
    assert n1 == n2 > 0
    if prec == "fp32":
        assert np.array_equal(R2w, R1w)
    else:
        assert helpers.rel2d(R2w, R1w) < 1e-12
    assert np.abs(R2w).max() > 0
