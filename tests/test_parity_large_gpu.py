"""Parity at the benchmark sizes, against the reference's own CPU path.

Fixtures (tests/golden/make_golden_large.py, generated where the reference
builds; about 33 s of CPU per reference vector step at N = 1024):
  - the 1024-site lattice of the absorption benchmark: 8 vectors propagated
    2 steps by the reference's propagate_vector (Sparse, Threshold 0:
    propagate_vec_DIA, propagate.c:60-125), and by the FP64 exact propagator;
  - absorption on that lattice: 400 start points (1200 vectors: whole waves of
    8-vector CTAs plus 1-vector CTAs) with FP64 exact responses, and one start
    point run through the reference program (absorption.c:18-202);
  - 2DIR on the 64-site cluster of the 2DIR benchmark (calc_2DIR.c:22-629),
    t2 = 0 and t2 > 0, run through the reference program.

Criteria (errors are max |difference| / max |reference value|):
  - FP64 engine runs match the FP64 exact results to 1e-10;
  - FP32 engine runs are at least as close to the FP64 result as the
    reference's own single-precision run is, and within 1e-5 of the
    reference's output.
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

SPARSE_FP32 = 3e-6   # FP32 series vs the exact propagator, per vector over <= 16 steps
SUM_ORDER = 1e-10
T2_EIGEN = 1e-5


def fixture(name):
    d = np.load(os.path.join(helpers.GOLDEN, name + ".npz"))
    return {k: d[k] for k in d.files}, json.loads(str(d["meta"]))


def packed(M):
    n = M.shape[0]
    return M[np.triu_indices(n)].astype(np.float32)


def test_c1_lattice_vectors_match_reference_propagator(tmp_path):
    """nise_propagate (propagate_vector's batched form) on the benchmark
    lattice: FP64 = exact propagator, FP32 no further from it than the
    reference's own FP32 propagate_vector."""
    g, meta = fixture("large_c1_vectors")
    files = synth.write(synth.c1_spec(**meta["spec"]), str(tmp_path))
    kw = dict(meta["keywords"], RunTimes="1 0 0")  # single steps: no sample window to validate
    H, _ = oracle.read_frames(kw, files, [0])
    Hp = np.repeat(packed(H[0])[None], len(g["init"]), 0)
    exact = g["exact"][:, 0] + 1j * g["exact"][:, 1]
    ref = g["ref"][:, 0].astype(np.float64) + 1j * g["ref"][:, 1]
    err_ref = helpers.rel(ref, exact)
    for prec, tol in ((nise.FP64, 1e-10), (nise.FP32, None)):
        p = nise.params_from_keywords(kw, precision=prec)
        with nise.Context(p) as c:
            re, im = g["init"][:, 0], g["init"][:, 1]
            for _ in range(meta["steps"]):
                re, im = c.propagate(Hp, re, im, 1)
        got = re.astype(np.float64) + 1j * im
        err = helpers.rel(got, exact)
        if tol:
            assert err < tol, err
        else:
            print("N=1024 vectors: engine FP32 %.2e, reference %.2e of the FP64 exact result" % (err, err_ref))
            assert err <= err_ref and err < 1e-5
            assert helpers.rel(got, ref) < 1e-5 + err_ref


@pytest.mark.parametrize("cfg", [0, 8, 13])
def test_c1_lattice_absorption_matches_exact(cfg, tmp_path):
    """The benchmark's kernels on the 1024-site lattice with more vectors than
    one wave of 8-vector CTAs: the default (row-owner Chebyshev kernel for the
    whole waves, 1-vector Taylor CTAs for the rest), the row-owner Taylor
    kernel (8) and the sliced-ELL kernel (13), against the FP64 exact
    responses."""
    g, meta = fixture("large_c1_absorption")
    files = synth.write(synth.c1_spec(**meta["wide"]["spec"]), str(tmp_path))
    p = nise.params_from_keywords(meta["wide"]["keywords"], files, kernel_config=cfg)
    with nise.Context(p) as c:
        c.load_files()
        re, im, n = c.absorption()
    assert n == int(g["wide_samples"]) == 400
    ex = g["wide_exact"][0] + 1j * g["wide_exact"][1]
    err = helpers.rel(re + 1j * im, ex)
    print("N=1024 absorption, 1200 vectors, config %d: %.2e of the FP64 exact responses" % (cfg, err))
    assert err < SPARSE_FP32


def test_c1_lattice_absorption_matches_reference(tmp_path):
    """One start point on the 1024-site lattice, through the reference program:
    the engine's FP32 error against the FP64 exact responses is no larger
    than the reference's, and the two agree to 1e-5."""
    g, meta = fixture("large_c1_absorption")
    files = synth.write(synth.c1_spec(**meta["ref"]["spec"]), str(tmp_path))
    out = {}
    for prec in (nise.FP32, nise.FP64):
        p = nise.params_from_keywords(meta["ref"]["keywords"], files, precision=prec)
        with nise.Context(p) as c:
            c.load_files()
            re, im, n = c.absorption()
        out[prec] = (re + 1j * im) / n
    ex = (g["ref_exact"][0] + 1j * g["ref_exact"][1]) / int(g["ref_samples"])
    td = g["ref_td"][:, 1] + 1j * g["ref_td"][:, 2]
    err_ref = helpers.rel(td, ex)
    err32 = helpers.rel(out[nise.FP32], ex)
    print("N=1024 absorption, 1 start point: engine FP32 %.2e, reference %.2e of the FP64 exact responses; "
          "engine vs reference %.2e" % (err32, err_ref, helpers.rel(out[nise.FP32], td)))
    assert helpers.rel(out[nise.FP64], ex) < 1e-10
    assert err32 <= max(err_ref, 2e-7)  # 2e-7: the 7-digit print of TD_Absorption.dat
    assert helpers.rel(out[nise.FP32], td) < 1e-5


@pytest.mark.parametrize("case", ["t2_0", "t2_4"])
def test_c2_cluster_2dir_matches_oracle_and_reference(case, tmp_path):
    """2DIR on the 64-site cluster (N2 = 2080 doubles states).

    The reference propagates in FP32 and sums the response in float; at this
    size its result is only accurate to about 1e-2 of the largest response
    against FP64 (GB + SE + EA cancel).  The restatement with float sums
    reproduces the reference's R*.dat files (pinned on the CPU in
    test_oracle.py), so the checks are: the engine's FP32 run performs the
    same single-precision operations (equal to the FP32-propagation /
    FP64-sum restatement up to FP64 summation order; with t2 > 0 the
    eigenvectors come from another Jacobi ordering); its difference from the
    reference's files is the float summation alone (no larger than the
    restatement's); its error against FP64 is no larger than the
    reference's; and the FP64 engine equals the FP64 restatement."""
    g, meta = fixture("large_c2_2dir")
    spec = meta[case]
    files = synth.write(synth.c2_spec(**spec["spec"]), str(tmp_path))
    kw = spec["keywords"]
    po = oracle.params(kw, files)
    t2 = int(str(kw["RunTimes"]).split()[1])
    out = {}
    for prec in (nise.FP32, nise.FP64):
        p = nise.params_from_keywords(kw, files, precision=prec)
        with nise.Context(p) as c:
            c.load_files()
            out[prec] = c.twodir()
    R, n = out[nise.FP32]
    oR, on = oracle.twodir(po, "f32a64")
    oR64, _ = oracle.twodir(po, "f64")
    assert n == on == 2
    norm = lambda X: helpers.R12_to_files(oracle.normalize_2d(po, X, n, "f64"))  # noqa: E731
    ref = g[case]
    err_o = helpers.rel2d(R, oR)
    err_ref = helpers.rel2d(norm(R), ref)
    err_oref = helpers.rel2d(norm(oR), ref)
    err64 = helpers.rel2d(norm(R), norm(oR64))
    err_ref64 = helpers.rel2d(ref, norm(oR64))
    print("N=64 2DIR %s: engine vs restatement %.2e; vs reference files %.2e (restatement with FP64 sums %.2e); "
          "vs FP64 %.2e (reference %.2e)" % (case, err_o, err_ref, err_oref, err64, err_ref64))
    assert err_o < (T2_EIGEN if t2 > 0 else SUM_ORDER)
    assert err_ref <= err_oref + (T2_EIGEN if t2 > 0 else 1e-7)
    assert err64 <= err_ref64 * 1.01
    assert helpers.rel2d(out[nise.FP64][0], oR64) < (1e-9 if t2 > 0 else 1e-11)
