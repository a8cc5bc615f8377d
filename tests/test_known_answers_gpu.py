"""Known-answer tests from the physics of the path, independent of the oracle.

* Diagonal-only Hamiltonian: every site evolves alone, so NISE is exact,
  S(t1) = sum_s sum_x sum_i mu_x,i(ti+t1) mu_x,i(ti) exp(-i f sum_k e_i(ti+k))
  (absorption.c:119-145 with propagate_vector on a diagonal H), for every
  propagation scheme.
* Static Hamiltonian (no site noise, static couplings): the exact response is
  one matrix exponential, S(t1) = S * sum_x mu_x^T exp(-i H f t1) mu_x; the
  exact propagators (Sparse, Diagonal) reach it, and the Trotter scheme's
  error falls as 1/Trotter^2.
* Harmonic limit of 2DIR: with no anharmonicity and overtone dipoles sqrt(2)
  mu (NISE_subs.c:490-494) the ground-state bleach, stimulated emission and
  excited-state absorption cancel up to the Trotter error.
"""
import numpy as np
import pytest

import nise_2017_b200 as nise
from nise_2017_b200 import synth

pytestmark = pytest.mark.gpu

# the reference's constants are floats (types.h:5-12); FP64 mode promotes them
ICM2IFS, TWOPI = float(np.float32(2.99792458e-5)), float(np.float32(2 * 3.14159265359))


def absorb(kw, files, **engine):
    p = nise.params_from_keywords(kw, files, **engine)
    with nise.Context(p) as c:
        c.load_files()
        re, im, n = c.absorption()
    return np.asarray(re) + 1j * np.asarray(im), n


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def shift_of(kw):
    lo = np.float32(float(kw["MinFrequencies"].split()[0]))
    hi = np.float32(float(kw["MaxFrequencies"].split()[0]))
    return np.float32((lo + hi) / np.float32(2))


def sindex(a, b, n):
    return b + a * (2 * n - a - 1) // 2


def test_diagonal_hamiltonian_is_exact(tmp_path):
    """Chain with no couplings, OU site energies and per-frame dipoles."""
    n, frames = 12, 400
    s = synth.spec(n_sites=n, frames=frames, dt_fs=2.0, geometry=synth.CHAIN, j_nn=0.0, j_sigma=0.0, seed=1201)
    files = synth.write(s, str(tmp_path))
    kw = synth.c0_keywords(Singles=n, Length=frames, RunTimes="64 0 0", Samplerate=17)
    tmax, sample = 64, 17
    nn2 = n * (n + 1) // 2
    E = np.fromfile(files["energy"], dtype=np.float32).reshape(frames, 1 + nn2)[:, 1:]
    d = (E[:, [sindex(i, i, n) for i in range(n)]] - shift_of(kw)).astype(np.float64)  # float shift, as read_He
    M = np.fromfile(files["dipole"], dtype=np.float32).reshape(frames, 1 + 3 * n)[:, 1:].reshape(frames, 3, n)
    M = M.astype(np.float64)  # products of the float dipoles in double, as the FP64 engine forms them
    f = float(np.float32(2.0)) * ICM2IFS * TWOPI
    nsamp = (frames - tmax - 1) // sample + 1
    S = np.zeros(tmax, complex)
    for q in range(nsamp):
        ti = q * sample
        ph = np.concatenate([np.zeros((1, n)), np.cumsum(d[ti:ti + tmax - 1], axis=0)]) * f
        for x in range(3):
            S += (M[ti:ti + tmax, x, :] * M[ti, x, :] * np.exp(-1j * ph)).sum(axis=1)
    for prop, tol64 in (("Coupling", 1e-11), ("Sparse", 1e-11), ("Diagonal", 1e-11), ("RK4", 1e-9)):
        extra = dict(Threshold=0) if prop == "Sparse" else {}
        r64, n64 = absorb(dict(kw, Propagation=prop, **extra), files, precision=nise.FP64)
        r32, n32 = absorb(dict(kw, Propagation=prop, **extra), files)
        assert n64 == n32 == nsamp
        print("diagonal H, %s: FP64 %.2e, FP32 %.2e" % (prop, rel(r64, S), rel(r32, S)))
        assert rel(r64, S) < tol64
        assert rel(r32, S) < 2e-5


def test_static_hamiltonian_matrix_exponential(tmp_path):
    """Static chain (no site noise, static couplings, static dipoles)."""
    n, frames = 10, 300
    s = synth.spec(n_sites=n, frames=frames, dt_fs=2.0, geometry=synth.CHAIN, sigma=0.0, j_nn=-12.0,
                   ham_type=synth.COUPLING, dipole_frames=1, mu_jitter=0.0, seed=1202)
    files = synth.write(s, str(tmp_path))
    kw = synth.c0_keywords(Singles=n, Length=frames, RunTimes="96 0 0", Samplerate=20, HamiltonianType="Coupling")
    tmax, sample = 96, 20
    nn2 = n * (n + 1) // 2
    Hp = np.fromfile(files["coupling"], dtype=np.float32)[1:1 + nn2]
    e = np.fromfile(files["energy"], dtype=np.float32).reshape(frames, 1 + n)[0, 1:]
    H = np.zeros((n, n))
    for a in range(n):
        H[a, a] = np.float32(e[a] - shift_of(kw))
        for b in range(a + 1, n):
            J = Hp[sindex(a, b, n)]
            H[a, b] = H[b, a] = J if abs(J) >= float(kw["Couplingcut"]) else 0.0
    mu = np.fromfile(files["dipole"], dtype=np.float32)[1:1 + 3 * n].reshape(3, n).astype(np.float64)
    f = float(np.float32(2.0)) * ICM2IFS * TWOPI
    w, V = np.linalg.eigh(H)
    nsamp = (frames - tmax - 1) // sample + 1
    S = np.array([nsamp * sum(mu[x] @ (V * np.exp(-1j * w * f * t)) @ V.T @ mu[x] for x in range(3))
                  for t in range(tmax)])
    for prop in ("Sparse", "Diagonal"):
        extra = dict(Threshold=0) if prop == "Sparse" else {}
        r64, _ = absorb(dict(kw, Propagation=prop, **extra), files, precision=nise.FP64)
        r32, _ = absorb(dict(kw, Propagation=prop, **extra), files)
        print("static H, %s: FP64 %.2e, FP32 %.2e" % (prop, rel(r64, S), rel(r32, S)))
        assert rel(r64, S) < 1e-7
        assert rel(r32, S) < 3e-6
    errs = []
    for ts in (2, 4, 8):
        r64, _ = absorb(dict(kw, Propagation="Coupling", Trotter=ts), files, precision=nise.FP64)
        errs.append(rel(r64, S))
    print("static H, Trotter 2/4/8: %.2e %.2e %.2e" % tuple(errs))
    assert errs[0] < 1e-2
    # each halving of the sub-step f/Trotter divides the error by 4 or more
    # (measured 4.6 and 8.6: second order with cancellations)
    assert errs[0] / errs[1] > 3.0 and errs[1] / errs[2] > 3.0


def test_harmonic_limit_of_2dir(tmp_path):
    """2DIR (GB + SE + EA) against GB alone: the total nearly vanishes as the
    anharmonicity goes to zero and grows back with it."""
    n, frames = 5, 240
    s = synth.c2_spec(n_sites=n, frames=frames, seed=1203)
    files = synth.write(s, str(tmp_path))
    out = {}
    for tech, anh in (("GBIR", 16), ("2DIR", 16), ("2DIR", 0.001)):
        kw = synth.c2_keywords(Singles=n, Length=frames, RunTimes="16 0 16", Samplerate=40, Technique=tech,
                               Anharmonicity=anh, Trotter=20)
        p = nise.params_from_keywords(kw, files, precision=nise.FP64)
        with nise.Context(p) as c:
            c.load_files()
            R, count = c.twodir()
        out[(tech, anh)] = np.abs(np.asarray(R)).max()
    gb = out[("GBIR", 16)]
    anh16, harm = out[("2DIR", 16)] / gb, out[("2DIR", 0.001)] / gb
    print("2DIR / GB: anharmonicity 16: %.2e, 0.001: %.2e" % (anh16, harm))
    assert harm < 1e-4  # measured 5.8e-6
    assert anh16 > 1000 * harm  # measured 5.3e-2
