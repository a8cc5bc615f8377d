"""LD, Raman, SFG, DOS and CD on the GPU, through the C ABI, against the oracle.

The vectors are propagated with the reference's single-precision operations
(FP32 contexts), so the Trotter and RK4 cases match the FP32-propagation /
FP64-sum oracle to summation order; the Sparse cases use the exact
propagator from FP64 eigenvectors and are held to the FP64 oracle at least as
closely as the FP32 restatement is.  Every case is also compared with the
reference program's own output files (tests/golden).
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
LIN = [k for k, c in CASES.items() if c["keywords"]["Technique"] in oracle.LINEAR_FILES]
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SUM_ORDER = 1e-10   # same single-precision operations, FP64 sums in another order
PRINT = 2e-6        # reference output printed with 7 significant digits
EIGEN_FLOOR = 1e-5  # FP32 vectors through propagators built from FP64 eigenvectors
REF_FP32 = 1e-5     # the reference sums the response in float


def run(kw, files, **engine):
    p = nise.params_from_keywords(kw, files, **engine)
    with nise.Context(p) as c:
        c.load_files()
        re, im, n = c.linear()
        specs = [c.absorption_fft(re[k], im[k], n) for k in range(len(re))]
        ms, main_ms, launches = c.timing()
    assert launches >= 2 and 0 < main_ms <= ms
    return p, re, im, n, specs


def cplx(re, im):
    return np.asarray(re) + 1j * np.asarray(im)


@pytest.mark.parametrize("name", LIN)
def test_fp32_matches_oracle_and_reference(name, tmp_path):
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    p, re, im, n, specs = run(case["keywords"], files)
    po = oracle.params(case["keywords"], files)
    ore, oim, on = oracle.linear(po, "f32a64")
    assert n == on and len(re) == len(ore) == len(oracle.LINEAR_FILES[case["keywords"]["Technique"]])
    g = helpers.golden(name)
    eig = helpers.uses_eigen(case)
    if eig:
        o64r, o64i, _ = oracle.linear(po, "f64")
        # within 10 % of the float restatement's own error (the engine's initial
        # vectors can come from FP64 weights, as the luminescence ones do)
        assert helpers.rel(cplx(re, im), cplx(o64r, o64i)) <= 1.1 * max(
            helpers.rel(cplx(ore, oim), cplx(o64r, o64i)), EIGEN_FLOOR)
    else:
        assert helpers.rel(cplx(re, im), cplx(ore, oim)) < SUM_ORDER
    fr, fi, _ = oracle.linear(po, "f32")  # float sums, as the reference's (matches its files to print precision)
    tdk = helpers.td_channels(case["keywords"]["Technique"], oracle.LINEAR_FILES)
    for k in range(len(re)):
        # the reference's float sums differ from FP64 sums; CD and SSP cancellations amplify that
        tol = max(REF_FP32, 2 * helpers.rel(np.stack([fr[k], fi[k]], 1) / n, np.stack([ore[k], oim[k]], 1) / n))
        if eig:
            tol = max(tol, 5e-4)
        if k in tdk:
            td = g["td"][tdk.index(k)]
            assert helpers.rel(np.stack([re[k] / n, im[k] / n], 1), td[:, 1:]) < tol
        w, sr, si = specs[k]
        assert len(w) == len(g["spec"][k])
        assert np.abs(w - g["spec"][k][:, 0]).max() < 1e-3
        assert helpers.rel(np.stack([sr, si], 1), g["spec"][k][:, 1:]) < tol


@pytest.mark.parametrize("name", LIN)
def test_fp64_matches_fp64_oracle(name, tmp_path):
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    p, re, im, n, _ = run(case["keywords"], files, precision=nise.FP64)
    ore, oim, on = oracle.linear(oracle.params(case["keywords"], files), "f64")
    assert n == on
    tol = 1e-9 if helpers.uses_eigen(case) else 1e-11
    assert helpers.rel(cplx(re, im), cplx(ore, oim)) < tol


@pytest.mark.parametrize("name", ["lin_cd", "lin_raman_rk4"])
def test_plain_matches_batched(name, tmp_path):
    """One start point per launch gives the batched sums (another grouping)."""
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    _, rb, ib, nb, _ = run(case["keywords"], files)
    _, rp, ip, np_, _ = run(case["keywords"], files, launch_mode=nise.PLAIN)
    assert nb == np_
    assert helpers.rel(cplx(rp, ip), cplx(rb, ib)) < 1e-12


@pytest.mark.parametrize("tech", ["LD", "DOS", "CD"])
def test_rk4_and_begin_end(tech, tmp_path):
    """RK4 propagation with BeginPoint/EndPoint on a Full trajectory."""
    s = synth.c0_spec(n_sites=7, frames=260, seed=71)
    files = synth.write(s, str(tmp_path))
    if tech == "CD":
        files.update(synth.write_positions(str(tmp_path), 7, 260, seed=72))
    kw = synth.c0_keywords(Singles=7, Length=260, RunTimes="24 0 0", Samplerate=20, Technique=tech,
                           Propagation="RK4", Trotter=2, BeginPoint=2, EndPoint=9)
    p, re, im, n, _ = run(kw, files)
    ore, oim, on = oracle.linear(oracle.params(kw, files), "f32a64")
    assert n == on == 9
    assert helpers.rel(cplx(re, im), cplx(ore, oim)) < SUM_ORDER


@pytest.mark.parametrize("name", ["lin_raman_rk4", "lin_dos"])
def test_driver_writes_reference_files(name, tmp_path):
    """The nise driver writes every TD_*.dat and spectrum file of the
    technique in the reference's format (TD_DOS.dat without trailing blanks)."""
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    inp = synth.write_input(str(tmp_path / "input"), case["keywords"], files)
    exe = os.path.join(ROOT, "nise_2017_b200", "nise")
    r = subprocess.run([exe, inp], cwd=str(tmp_path), stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    g = helpers.golden(name)
    for k, (tdf, spf) in enumerate(oracle.LINEAR_FILES[case["keywords"]["Technique"]]):
        text = open(str(tmp_path / tdf)).read().splitlines()
        assert all(line.endswith(" ") != (tdf == "TD_DOS.dat") for line in text)
        td = np.loadtxt(str(tmp_path / tdf), ndmin=2)
        sp = np.loadtxt(str(tmp_path / spf), ndmin=2)
        assert td.shape == g["td"][k].shape and sp.shape == g["spec"][k].shape
        assert helpers.rel(td[:, 1:], g["td"][k][:, 1:]) < REF_FP32
        assert helpers.rel(sp[:, 1:], g["spec"][k][:, 1:]) < REF_FP32


def test_missing_operator_files_fail_cleanly(tmp_path):
    case = CASES["lin_sfg_shift"]
    files = helpers.materialise(case, str(tmp_path))
    files["alpha"] = str(tmp_path / "absent.bin")
    p = nise.params_from_keywords(case["keywords"], files)
    with nise.Context(p) as c:
        with pytest.raises(nise.NiseError) as e:
            c.load_files()
        assert e.value.code == -2  # NISE_ERR_IO


@pytest.mark.parametrize("name", ["lum_static", "lum_itime"])
def test_luminescence_driver_files(name, tmp_path):
    """The nise driver's luminescence output: TD_Lum.dat (the total, no
    trailing blank, as luminescence.c:224 prints it) and the spectra of the
    total and of each dipole component, against the reference's files."""
    case = CASES[name]
    files = helpers.materialise(case, str(tmp_path))
    inp = synth.write_input(str(tmp_path / "input"), case["keywords"], files)
    exe = os.path.join(ROOT, "nise_2017_b200", "nise")
    r = subprocess.run([exe, inp], cwd=str(tmp_path), stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    g = helpers.golden(name)
    lines = open(str(tmp_path / "TD_Lum.dat")).read().splitlines()
    assert lines and not any(line.endswith(" ") for line in lines)
    td = np.loadtxt(str(tmp_path / "TD_Lum.dat"), ndmin=2)
    tol = 5e-4 if helpers.uses_eigen(case) else REF_FP32
    assert td.shape == g["td"][0].shape
    assert helpers.rel(td[:, 1:], g["td"][0][:, 1:]) < tol
    assert not (tmp_path / "TD_Lum_x.dat").exists()
    for k, (_, spf) in enumerate(oracle.LINEAR_FILES["Luminescence"]):
        sp = np.loadtxt(str(tmp_path / spf), ndmin=2)
        assert sp.shape == g["spec"][k].shape
        assert helpers.rel(sp[:, 1:], g["spec"][k][:, 1:]) < tol
    assert nise.linear_files("Luminescence") == [(td_, sp_) for td_, sp_ in oracle.LINEAR_FILES["Luminescence"]]
