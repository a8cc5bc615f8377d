"""The 2D FFT step on the GPU against the reference's 2DFFT output files.

Each golden case rebuilds the directory the reference's 2DFFT ran in (keyword
file, response files, Waitingtime.dat) and runs nise_2dfft_files there; every
file the reference wrote must be written, with identical frequency axes and
line layout and spectral values within the tolerances below.
"""
import os
import subprocess

import pytest

import helpers
import nise_2017_b200 as nise

pytestmark = pytest.mark.gpu

# Rw*/2D* values: both sides print 7 significant digits of FP64 transforms that
# differ by rounding only, so a printed value can move by one unit of its last
# digit (5e-7 relative) and the 2D sums of two such values by twice that.
VALUE_TOL = 2e-6
# PP*: float sums over up to a few hundred printed values.
PP_TOL = 2e-5


def _run_case(name, tmp_path, monkeypatch, runner):
    ins, ref = helpers.fft2d_case(name)
    for fn, text in ins.items():
        with open(os.path.join(str(tmp_path), fn), "w") as f:
            f.write(text)
    monkeypatch.chdir(tmp_path)
    runner()
    got = {fn: open(fn).read() for fn in os.listdir(".") if fn not in ins}
    assert sorted(got) == sorted(ref)
    for fn in ref:
        tol = PP_TOL if fn.startswith("PP") else VALUE_TOL
        helpers.compare_spectrum_text(got[fn], ref[fn], tol)


@pytest.mark.parametrize("name", helpers.fft2d_case_names())
def test_2dfft_matches_reference(name, tmp_path, monkeypatch):
    _run_case(name, tmp_path, monkeypatch, lambda: nise.fft2d_files("input"))


def test_nise2dfft_driver(tmp_path, monkeypatch):
    exe = os.path.join(os.path.dirname(nise.__file__), "nise2dfft")
    _run_case("gnuplot_apodised", tmp_path, monkeypatch,
              lambda: subprocess.run([exe, "input"], check=True, stdout=subprocess.DEVNULL))
