"""Host-side parts that need no GPU: the C ABI library, the keyword parser,
the output writers and the trajectory generator."""
import os
import re
import subprocess

import numpy as np
import pytest

import helpers
import nise_2017_b200 as nise
from nise_2017_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "nise_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*)\s*\*?(nise_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 18
    lib = nise.lib()
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(nise.EXPORTED) == syms


def test_params_default_follows_readinput():
    p = nise.default_params()
    assert (p.ts, p.tmax1, p.tmax2, p.tmax3, p.begin, p.end, p.fft) == (5, 256, 0, 256, 0, 0, 0)
    assert p.couplingcut == 0 and p.anharmonicity == 0 and p.window == 0
    assert p.hamiltonian == nise.HAM["Full"] and p.precision == nise.FP32


def write(tmp_path, text):
    path = tmp_path / "input"
    path.write_text(text)
    return str(path)


def test_keyword_parser_rules(tmp_path):
    p = nise.read_input(write(tmp_path, "\n".join([
        "Propagation Coupling", "Hamiltonianfile E.bin", "Dipolefile D.bin", "Length 1000", "Length 2000",
        "Samp 10", "Timestep 2.5", "RunTimes 64 3 7", "Singles 9", "Sing shifts.txt",
        "MinFrequencies 1500 1500 1500", "MaxFrequencies 1800 1800 1800", "Technique 2DIR",
        "Unknownkey 5", "Couplingcut 0.5", "Anharmonicity 14", "Trotter 3", "Window Hann"]) + "\n"))
    assert p.length == 2000  # last occurrence wins
    assert p.singles == 9 and p.sample == 10  # "Samp" is a prefix of Samplerate
    assert p.singleShiftFName == b"shifts.txt"  # "Sing" first matches SingleShiftfile
    assert (p.tmax1, p.tmax2, p.tmax3) == (64, 3, 64)  # tmax3 forced to tmax1 for 2D
    assert p.propagation == nise.PROP["Coupling"] and p.technique == nise.TECH["2DIR"]
    assert abs(p.deltat - 2.5) < 1e-7 and p.ts == 3 and p.window == 1
    assert p.energyFName == b"E.bin" and p.dipoleFName == b"D.bin"
    assert abs(p.couplingcut - 0.5) < 1e-7 and abs(p.anharmonicity - 14) < 1e-6


@pytest.mark.parametrize("prop,code", [("Sparse", 0), ("Coupling", 1), ("Diagonal", 2), ("RK4", 3), ("xyz", 0)])
def test_propagation_keyword_mapping(tmp_path, prop, code):
    p = nise.read_input(write(tmp_path, "Propagation %s\nLength 100\nRunTimes 10 0 0\n" % prop))
    assert p.propagation == code


def test_parser_errors(tmp_path):
    with pytest.raises(nise.NiseError) as e:
        nise.read_input(str(tmp_path / "missing"))
    assert e.value.code == -2
    with pytest.raises(nise.NiseError):
        nise.read_input(write(tmp_path, "Length 10\nRunTimes 64 0 0\n"))  # trajectory too short
    with pytest.raises(nise.NiseError):
        nise.read_input(write(tmp_path, "Length 100\nRunTimes 10 0 0\nTechnique 2DIR\nRunTimes 40 30 40\n"))
    with pytest.raises(nise.NiseError):
        nise.read_input(write(tmp_path, "Length 100\nRunTimes 10 0 0\nProjection 2\n"))


def test_writers_use_reference_formats(tmp_path):
    p = nise.default_params()
    p.tmax1, p.tmax3, p.tmax2, p.deltat = 4, 4, 2, 2.0
    re = np.array([4.0, 2.0, -1.0, 0.5])
    im = np.array([0.0, -0.25, 1.5, 2.0])
    nise.write_td_absorption(str(tmp_path / "td"), p, re, im, 2)
    lines = (tmp_path / "td").read_text().splitlines()
    assert lines[1] == "2.000000 1.000000e+00 -1.250000e-01 "
    R = np.arange(16.0).reshape(4, 4)
    nise.write_2d(str(tmp_path / "r2"), p, R, -R, 4)
    rows = (tmp_path / "r2").read_text().splitlines()
    assert len(rows) == 16
    # t1 = 0, t3 = 0 row is halved; t1 outer loop, t3 inner
    assert rows[0] == "0.000000 4.000000 0.000000 0.000000e+00 -0.000000e+00"
    assert rows[1] == "0.000000 4.000000 2.000000 1.000000e+00 -1.000000e+00"
    assert rows[4].startswith("2.000000 4.000000 0.000000 1.250000e-01")


def test_context_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    p = nise.default_params()
    p.singles, p.sample, p.deltat, p.length = 4, 10, 2.0, 100
    with pytest.raises(nise.NiseError) as e:
        nise.Context(p)
    assert e.value.code == -4


def test_generator_layout_and_determinism(tmp_path):
    s = synth.spec(n_sites=7, frames=50, seed=3)
    f1 = synth.write(s, str(tmp_path / "a"))
    f2 = synth.write(s, str(tmp_path / "b"))
    E1 = open(f1["energy"], "rb").read()
    assert E1 == open(f2["energy"], "rb").read()
    rec = 1 + 7 * 8 // 2
    arr = np.frombuffer(E1, dtype=np.int32).reshape(50, rec)
    assert (arr[:, 0] == np.arange(50)).all()
    h = np.frombuffer(E1, dtype=np.float32).reshape(50, rec)[:, 1:]
    diag = [i * 7 + i - i * (i + 1) // 2 for i in range(7)]
    assert abs(h[:, diag].mean() - 1650) < 10
    D = np.frombuffer(open(f1["dipole"], "rb").read(), dtype=np.float32).reshape(50, 1 + 21)
    assert D.shape == (50, 22)
    s2 = synth.spec(n_sites=64, frames=3, geometry=synth.LATTICE, spacing=8.0, jcut=2.0, ham_type=synth.COUPLING,
                    dipole_frames=1, seed=4)
    f3 = synth.write(s2, str(tmp_path / "c"))
    C = np.fromfile(f3["coupling"], dtype=np.float32)[1:]
    off = np.array([C[b + a * (128 - a - 1) // 2] for a in range(64) for b in range(a + 1, 64)])
    nz = off[off != 0]
    assert (np.abs(nz) >= 2.0).all() and 1 < len(nz) / 64 < 20


@pytest.mark.parametrize("ham,code", [("TransitionDipole", 2), ("ExtendedDipole", 3)])
def test_parser_onfly_coupling_types(tmp_path, ham, code):
    """HamiltonianType TransitionDipole / ExtendedDipole with the Positionfile
    and PBCfile keywords (readinput.c:94,100)."""
    path = tmp_path / "input"
    path.write_text("Hamiltonianfile E.bin\nDipolefile D.bin\nPositionfile P.bin\nPBCfile B.bin\n"
                    "HamiltonianType %s\nSingles 4\nLength 100\nSamplerate 10\nTimestep 2\nRunTimes 8 0 0\n"
                    "Technique Absorption\n" % ham)
    p = nise.read_input(str(path))
    assert p.hamiltonian == code
    assert p.positionFName == b"P.bin" and p.pbcFName == b"B.bin"


@pytest.mark.parametrize("tech,code", [("2DUVvis", 6), ("GBUVvis", 7), ("SEUVvis", 8), ("EAUVvis", 9),
                                       ("noEAUVvis", 10)])
def test_parser_uvvis_techniques(tmp_path, tech, code):
    """The calc_2DES technique names (NISE.c:296): a waiting-time technique,
    so tmax3 follows tmax1 and the length check covers t1 + t2 + t3
    (readinput.c:208-218)."""
    p = nise.read_input(write(tmp_path, "Technique %s\nLength 100\nRunTimes 20 5 3\n" % tech))
    assert p.technique == code == nise.TECH[tech]
    assert (p.tmax1, p.tmax2, p.tmax3) == (20, 5, 20)
    with pytest.raises(nise.NiseError):
        nise.read_input(write(tmp_path, "Technique %s\nLength 40\nRunTimes 20 5 3\n" % tech))
