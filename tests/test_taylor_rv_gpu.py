"""The row-owner Taylor kernel (k_abs_taylor_rv: FP32, static couplings,
8 vectors per CTA, diagonal records staged by bulk copies) against the FP64
exact-propagator restatement (oracle.absorption_exact: absorption.c:119-145
with propagate_vec_DIA's U, propagate.c:60-125, in FP64) and against the
8-vector sliced-ELL kernel it replaces (kernel_config 13)."""
import numpy as np
import pytest

import helpers
import nise_2017_b200 as nise
import oracle
from nise_2017_b200 import synth

pytestmark = pytest.mark.gpu

SPARSE_FP32 = 3e-6  # FP32 Taylor series vs the exact propagator


def run(kw, files, shift=None, **engine):
    p = nise.params_from_keywords(kw, files, **engine)
    with nise.Context(p) as c:
        c.load_files()
        if shift:
            c.set_singleshift(*shift)
        re, im, n = c.absorption()
        _, _, launches = c.timing()
    return re, im, n, launches


# kernel_config: 0 default (row-owner Taylor, 768 threads), 14 (1024
# threads), 15 (row-owner Chebyshev)
@pytest.mark.parametrize("cfg", [0, 14, 15])
@pytest.mark.parametrize("n_sites", [101, 512])
def test_row_owner_kernel_matches_exact_fp64(n_sites, cfg, tmp_path):
    """300 vectors on 38 CTAs (the last holds 4), a site count that leaves
    padded rows in the last 8-row slice (101), and a half-size lattice."""
    s = synth.c1_spec(n_sites=n_sites, frames=112, seed=300 + n_sites)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Singles=n_sites, Length=112, RunTimes="12 0 0", Samplerate=1)
    re, im, n, _ = run(kw, files, kernel_config=cfg)
    ere, eim, en = oracle.absorption_exact(kw, files)
    assert n == en == 100
    assert helpers.rel(re + 1j * im, ere + 1j * eim) < SPARSE_FP32
    lre, lim, ln, _ = run(kw, files, kernel_config=13)
    assert ln == n
    assert helpers.rel(re + 1j * im, lre + 1j * lim) < SPARSE_FP32


@pytest.mark.parametrize("cfg", [0, 15])
def test_row_owner_kernel_whole_waves_and_tail(cfg, tmp_path):
    """More vectors than a wave of 8-vector CTAs: whole waves on the row-owner
    kernel, the rest on 1-vector CTAs (Taylor series in both forms); with
    SingleShift on the staged diagonal."""
    s = synth.c1_spec(n_sites=64, frames=520, seed=311)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Singles=64, Length=520, RunTimes="8 0 0", Samplerate=1)
    shift = ([3, 17, 40], [1.0, 1.01, 0.99], [4.0, -6.0, 2.5])
    re, im, n, launches = run(kw, files, shift=shift, kernel_config=cfg)
    assert n == 512 and launches >= 3  # 1536 vectors: 148 CTAs of 8, 352 vectors on 1-vector CTAs
    r64, i64, n64, _ = run(kw, files, shift=shift, precision=nise.FP64)
    assert n64 == n
    assert helpers.rel(re + 1j * im, r64 + 1j * i64) < SPARSE_FP32
    lre, lim, _, _ = run(kw, files, shift=shift, kernel_config=13)
    assert helpers.rel(re + 1j * im, lre + 1j * lim) < SPARSE_FP32
    # without the shift the result must move (the staged diagonal is shifted)
    ure, uim, _, _ = run(kw, files)
    assert helpers.rel(ure + 1j * uim, re + 1j * im) > 10 * SPARSE_FP32
