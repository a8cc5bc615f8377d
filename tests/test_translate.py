"""Trajectory format translation against the reference's translate program.

The golden fixtures (tests/golden/translate_*.npz) hold seeded inputs in every
format the reference reads and the files its translate program wrote from
them.  The library's translation is host code, so these tests run without a
GPU and compare byte for byte.
"""
import base64
import json
import os
import subprocess

import numpy as np
import pytest

import nise_2017_b200 as nise

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
ROOT = os.path.dirname(HERE)

with open(os.path.join(GOLDEN, "translate_cases.json")) as f:
    CASES = json.load(f)


def load(name):
    d = np.load(os.path.join(GOLDEN, "translate_%s.npz" % name))
    dec = lambda s: {k: base64.b64decode(v) for k, v in json.loads(str(s)).items()}
    return dec(d["inputs"]), dec(d["outputs"])


def materialise(name, directory):
    ins, outs = load(name)
    for fn, data in ins.items():
        with open(os.path.join(directory, fn), "wb") as f:
            f.write(data)
    return ins, outs


@pytest.mark.parametrize("name", sorted(CASES))
def test_translation_is_byte_identical(name, tmp_path, monkeypatch):
    ins, outs = materialise(name, str(tmp_path))
    monkeypatch.chdir(tmp_path)
    nise.translate("input")
    written = sorted(fn for fn in os.listdir(tmp_path) if fn not in ins)
    assert written == sorted(outs)
    for fn, ref in outs.items():
        got = open(os.path.join(tmp_path, fn), "rb").read()
        assert got == ref, fn


def test_driver_executable(tmp_path):
    name = "groasc_grobin_doubles"
    ins, outs = materialise(name, str(tmp_path))
    exe = os.path.join(ROOT, "nise_2017_b200", "nise_translate")
    r = subprocess.run([exe, "input"], cwd=str(tmp_path), stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    for fn, ref in outs.items():
        assert open(os.path.join(tmp_path, fn), "rb").read() == ref


def test_doubles_block_matches_two_exciton_rules(tmp_path, monkeypatch):
    """GROASC -> GROBIN builds the pair-state block: energies e_a + e_b,
    2 e_a - anharmonicity on |aa>, sqrt2 couplings to |aa>, J_bd between
    pair states that share a site."""
    ins, outs = materialise("groasc_grobin_doubles", str(tmp_path))
    n, A = 4, np.float32(14)
    nd = n * (n + 1) // 2
    rec = np.frombuffer(outs["out_E.bin"], np.float32)[: 1 + nd + nd * (nd + 1) // 2]
    He, Hf = rec[1:1 + nd], rec[1 + nd:]
    pairs = [(a, b) for a in range(n) for b in range(a, n)]
    idx = lambda a, b, m: (b + a * (2 * m - a - 1) // 2) if a <= b else (a + b * (2 * m - b - 1) // 2)
    h = lambda a, b: He[idx(a, b, n)]
    s2 = np.float32(1.41421356237)
    for i, (a, b) in enumerate(pairs):
        for j in range(i, nd):
            c, d = pairs[j]
            w = Hf[idx(i, j, nd)]
            if i == j:
                assert w == (np.float32(2) * h(a, a) - A if a == b else h(a, a) + h(b, b))
            elif a == b and a in (c, d):
                assert w == s2 * h(c, d)
            elif c == d and c in (a, b):
                assert w == s2 * h(a, b)
            elif a != b and c != d and len({a, b} & {c, d}) == 1:
                (o1,), (o2,) = {a, b} - {c, d}, {c, d} - {a, b}
                assert w == h(o1, o2)
            else:
                assert w == 0


def test_errors(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    with pytest.raises(nise.NiseError) as e:
        nise.translate(str(tmp_path / "missing"))
    assert e.value.code == -2
    (tmp_path / "bad").write_text("InputFormat GROXYZ\nOutputFormat GROBIN\nSingles 2\n")
    with pytest.raises(nise.NiseError) as e:
        nise.translate(str(tmp_path / "bad"))
    assert "GROXYZ" in str(e.value)
    (tmp_path / "noin").write_text("InputFormat GROBIN\nOutputFormat GROASC\nSingles 2\n"
                                   "InputEnergy none.bin\nInputDipole none2.bin\nOutputEnergy o.txt\nOutputDipole d.txt\n")
    with pytest.raises(nise.NiseError) as e:
        nise.translate(str(tmp_path / "noin"))
    assert e.value.code == -2
    (tmp_path / "mod").write_text("InputFormat GROBIN\nOutputFormat GROASC\nSingles 2\nModify\nLabel\n")
    with pytest.raises(nise.NiseError) as e:
        nise.translate(str(tmp_path / "mod"))
    assert "Select" in str(e.value)
