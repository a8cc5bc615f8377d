"""The warp-per-two-vectors Trotter kernel (kernel_config 34, static
couplings): both vectors of a warp follow the one rotation schedule with the
same coefficients, each with its own start frame, phases and response, and
the float operations of the warp-per-vector kernel (kernel_config 32), so the
responses are bitwise equal."""
import numpy as np
import pytest

import nise_2017_b200 as nise
from nise_2017_b200 import synth

pytestmark = pytest.mark.gpu


def absorb(kw, files, **engine):
    p = nise.params_from_keywords(kw, files, **engine)
    with nise.Context(p) as c:
        c.load_files()
        re, im, n = c.absorption()
    return re, im, n


@pytest.mark.parametrize("n_sites, prec", [(300, nise.FP32), (300, nise.FP64), (1024, nise.FP32)])
def test_pair_kernel_is_bitwise_the_warp_kernel(n_sites, prec, tmp_path):
    frames = 431 if n_sites < 1024 else 260  # 37 and 21 start points: odd vector counts
    s = synth.c1_spec(n_sites=n_sites, frames=frames, seed=800 + n_sites)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Singles=n_sites, Length=frames, RunTimes="32 0 0", Samplerate=11, Propagation="Coupling")
    r2, i2, n2 = absorb(kw, files, precision=prec, kernel_config=34)
    r1, i1, n1 = absorb(kw, files, precision=prec, kernel_config=32)
    assert n1 == n2 and (3 * n1) % 2 == 1  # an odd vector count: the last warp has one vector
    assert np.array_equal(r1, r2) and np.array_equal(i1, i2)
    assert np.abs(r1).max() > 0


def test_pair_kernel_needs_static_couplings(tmp_path):
    s = synth.c0_spec(n_sites=12, frames=200, seed=810)
    files = synth.write(s, str(tmp_path))
    kw = synth.c0_keywords(Singles=12, Length=200, RunTimes="16 0 0", Samplerate=20)
    p = nise.params_from_keywords(kw, files, kernel_config=34)
    with nise.Context(p) as c:
        c.load_files()
        with pytest.raises(nise.NiseError):
            c.absorption()


def test_warp_kernels_over_several_cta_rounds(tmp_path):
    """A job of 4740 vectors on a 300-site lattice: more vectors than one round
    of the widest CTAs (16 warps on 148 SMs), so the launchers narrow the CTAs
    to spread the vectors evenly over the rounds (the warp kernel 3 rounds of
    11 warps, the two-vector kernel 2 rounds of 9).  Every configuration gives
    the thread-per-vector kernel's responses bitwise."""
    n, tmax, nsamp = 300, 8, 1580
    frames = nsamp + tmax
    s = synth.c1_spec(n_sites=n, frames=frames, seed=830)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Singles=n, Length=frames, RunTimes="%d 0 0" % tmax, Samplerate=1, Propagation="Coupling")
    r1, i1, n1 = absorb(kw, files, kernel_config=1)
    assert n1 == nsamp
    for cfg in (32, 34, 0):
        r, i, nn = absorb(kw, files, kernel_config=cfg)
        assert nn == n1
        assert np.array_equal(r, r1) and np.array_equal(i, i1), cfg
    assert np.abs(r1).max() > 0
