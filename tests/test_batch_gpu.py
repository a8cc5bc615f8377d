"""Level-scheduled Trotter rotations, the launch autotuner and the batch API.

The level-scheduled kernels apply the rotations of one level (disjoint site
pairs) in parallel, a CTA or a warp per vector; they must reproduce the
sequential lexicographic order, and the response sum order, bit for bit.  A batch runs many contexts' jobs as one CUDA graph and must return
exactly what the same contexts return one by one.
"""
import numpy as np
import pytest

import helpers
import nise_2017_b200 as nise
from nise_2017_b200 import synth

pytestmark = pytest.mark.gpu

CASES = helpers.cases()


def run(kw, files, **engine):
    p = nise.params_from_keywords(kw, files, **engine)
    with nise.Context(p) as c:
        c.load_files()
        re, im, n = c.absorption()
    return re, im, n


@pytest.mark.parametrize("cfg", [32, 33, 64, 128, 256])
@pytest.mark.parametrize("prec", [nise.FP32, nise.FP64])
def test_level_kernel_bitwise_equal_to_thread_per_vector(cfg, prec, tmp_path):
    case = CASES["abs_coupling_full"]
    files = helpers.materialise(case, str(tmp_path))
    r0 = run(case["keywords"], files, precision=prec, kernel_config=1)
    r1 = run(case["keywords"], files, precision=prec, kernel_config=cfg)
    assert r0[2] == r1[2]
    assert np.array_equal(r0[0], r1[0]) and np.array_equal(r0[1], r1[1])


def test_level_kernel_lattice_static_couplings(tmp_path):
    """N = 160 lattice with static couplings (many levels), against the oracle."""
    import oracle
    s = synth.c1_spec(n_sites=160, frames=260, seed=61)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Singles=160, Length=260, RunTimes="24 0 0", Samplerate=40, Propagation="Coupling",
                           Trotter=2)
    r0 = run(kw, files, kernel_config=1)
    r1 = run(kw, files, kernel_config=128)
    assert np.array_equal(r0[0], r1[0]) and np.array_equal(r0[1], r1[1])
    ore, oim, on = oracle.absorption(oracle.params(kw, files), "f32a64")
    assert helpers.rel(r1[0] + 1j * r1[1], ore + 1j * oim) < 1e-11


def same(r0, r1):
    return r0[2] == r1[2] and np.array_equal(r0[0], r1[0]) and np.array_equal(r0[1], r1[1])


def test_warp_kernel_levels_wider_than_a_warp(tmp_path):
    """Static couplings whose levels hold 40, 80 and 40 rotations (dimers (2i, 2i+1) and
    partners (i, i + 80) on 160 sites): lanes take several rotations of one level."""
    import oracle
    n = 160
    s = synth.c1_spec(n_sites=n, frames=260, seed=62)
    files = synth.write(s, str(tmp_path))
    rec = np.fromfile(files["coupling"], dtype=np.float32)
    h = rec[1:]  # int32 tag, then the packed upper triangle (index b + a(2n-a-1)/2)
    diag = np.array([h[a + a * (2 * n - a - 1) // 2] for a in range(n)])
    h[:] = 0
    for a in range(n):
        h[a + a * (2 * n - a - 1) // 2] = diag[a]
    for i in range(n // 2):
        a, b = 2 * i, 2 * i + 1
        h[b + a * (2 * n - a - 1) // 2] = 12.0
        h[i + n // 2 + i * (2 * n - i - 1) // 2] = -7.0
    rec.tofile(files["coupling"])
    kw = synth.c1_keywords(Singles=n, Length=260, RunTimes="24 0 0", Samplerate=40, Propagation="Coupling",
                           Trotter=2)
    r0 = run(kw, files, kernel_config=1)
    for cfg in (32, 33, 64):
        assert same(r0, run(kw, files, kernel_config=cfg)), cfg
    r1 = run(kw, files, kernel_config=32)
    ore, oim, on = oracle.absorption(oracle.params(kw, files), "f32a64")
    assert helpers.rel(r1[0] + 1j * r1[1], ore + 1j * oim) < 1e-11


@pytest.mark.parametrize("cfg", [32, 33])
@pytest.mark.parametrize("prec", [nise.FP32, nise.FP64])
def test_warp_kernel_lattice_static_couplings(cfg, prec, tmp_path):
    """300-site lattice (levels of ~20 rotations; the phases staged in shared memory)."""
    import oracle
    s = synth.c1_spec(n_sites=300, frames=260, seed=63)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Singles=300, Length=260, RunTimes="24 0 0", Samplerate=20, Propagation="Coupling",
                           Trotter=2)
    r0 = run(kw, files, precision=prec, kernel_config=1)
    r1 = run(kw, files, precision=prec, kernel_config=cfg)
    assert same(r0, r1)
    ore, oim, on = oracle.absorption(oracle.params(kw, files), "f32a64" if prec == nise.FP32 else "f64")
    assert helpers.rel(r1[0] + 1j * r1[1], ore + 1j * oim) < 1e-11


def test_autotune_keeps_results(tmp_path):
    case = CASES["abs_coupling_full"]
    files = helpers.materialise(case, str(tmp_path))
    r0 = run(case["keywords"], files)
    p = nise.params_from_keywords(case["keywords"], files)
    with nise.Context(p) as c:
        c.load_files()
        c.tune()
        re, im, n = c.absorption()
    assert np.array_equal(r0[0], re) and np.array_equal(r0[1], im)


def test_batch_equals_individual_runs(tmp_path):
    """Four schemes and sizes in one graph, run twice, against one-by-one runs."""
    names = ["abs_coupling_full", "abs_sparse_static", "abs_sparse_full", "abs_rk4_full"]
    ctxs, single = [], []
    try:
        for k, name in enumerate(names):
            case = CASES[name]
            files = helpers.materialise(case, str(tmp_path / str(k)))
            p = nise.params_from_keywords(case["keywords"], files)
            c = nise.Context(p)
            c.load_files()
            re, im, n = c.absorption()
            single.append((re, im, n, c.absorption_fft(re, im, n)))
            ctxs.append(c)
        s = synth.c1_spec(n_sites=140, frames=200, seed=62)
        files = synth.write(s, str(tmp_path / "lattice"))
        kw = synth.c1_keywords(Singles=140, Length=200, RunTimes="20 0 0", Samplerate=30, Propagation="Coupling",
                               Trotter=2)
        p = nise.params_from_keywords(kw, files)
        c = nise.Context(p)
        c.load_files()
        re, im, n = c.absorption()
        single.append((re, im, n, c.absorption_fft(re, im, n)))
        ctxs.append(c)
        with nise.Batch(ctxs) as b:
            for rep in range(2):
                b.run()
                ms, launches = b.timing()
                assert ms > 0 and launches >= 3 * len(ctxs)
                for i, (re, im, n, (w, sr, si)) in enumerate(single):
                    bre, bim, bn = b.result(i)
                    assert bn == n
                    assert np.array_equal(bre, re) and np.array_equal(bim, im), (i, rep)
                    bw, bsr, bsi = b.spectrum(i)
                    assert np.array_equal(bw, w) and np.allclose(bsr, sr, rtol=1e-12, atol=0)
    finally:
        for c in ctxs:
            c.close()


def test_batch_with_autotune(tmp_path):
    s = synth.c1_spec(n_sites=100, frames=200, seed=63)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Singles=100, Length=200, RunTimes="16 0 0", Samplerate=30, Propagation="Coupling",
                           Trotter=2)
    p = nise.params_from_keywords(kw, files)
    ref = run(kw, files, kernel_config=1)
    with nise.Context(p) as c:
        c.load_files()
        with nise.Batch([c], autotune=True) as b:
            b.run()
            re, im, n = b.result(0)
    assert np.array_equal(re, ref[0]) and np.array_equal(im, ref[1])

