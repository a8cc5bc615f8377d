"""The 2D FFT step (the reference's 2DFFT program) on the CPU side.

The restatement oracle/fft2d.py is pinned against the text files the
reference's own 2DFFT wrote for the golden cases, and the C ABI's argument
checks (which run before any device work) are exercised without a GPU.
"""
import os
import sys

import pytest

import helpers
import nise_2017_b200 as nise

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import fft2d  # noqa: E402

# numpy's FFT against the FP64 transform the reference was linked with
ORACLE_TOL = 1e-6


@pytest.mark.parametrize("name", helpers.fft2d_case_names())
def test_oracle_matches_reference_2dfft(name):
    ins, ref = helpers.fft2d_case(name)
    got = fft2d.run(ins)
    assert sorted(got) == sorted(ref)
    for fn in ref:
        helpers.compare_spectrum_text(got[fn], ref[fn], ORACLE_TOL)


def _write(dirpath, files):
    for fn, text in files.items():
        with open(os.path.join(dirpath, fn), "w") as f:
            f.write(text)


@pytest.mark.parametrize("edit,code", [
    (lambda t: t.replace("FFT 256\n", ""), -1),                                   # FFT keyword missing
    (lambda t: t.replace("MinFrequencies 1200", "MinFrequencies 2200"), -1),       # min > max
    (lambda t: t.replace("MinFrequencies 1200", "MinFrequencies -1200"), -1),      # negative frequency
    (lambda t: t.replace("Timestep 2\n", ""), -1),                                # no time step
])
def test_2dfft_argument_errors(tmp_path, monkeypatch, edit, code):
    ins, _ = helpers.fft2d_case("dislin")
    ins = dict(ins, input=edit(ins["input"]))
    _write(str(tmp_path), ins)
    monkeypatch.chdir(tmp_path)
    lib = nise.lib()
    assert lib.nise_2dfft_files(b"input", 0) == code
    assert lib.nise_global_error()


def test_2dfft_missing_input(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    assert nise.lib().nise_2dfft_files(b"no_such_input", 0) == -2
