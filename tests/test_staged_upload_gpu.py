"""Trajectories from pinned host memory are copied in frame chunks on a copy
stream while the propagation runs wave by wave, each wave waiting for the
chunk that holds its last frame; the absorption plan of a context is reused
while its couplings and layout are unchanged.  Both must leave the results
bitwise unchanged."""
import ctypes

import numpy as np
import pytest

import nise_2017_b200 as nise
from nise_2017_b200 import synth

pytestmark = pytest.mark.gpu


def pinned_set(c, files):
    """nise_set_trajectory from pinned host copies of the files."""
    import torch
    bufs = []
    for key in ("energy", "dipole", "coupling"):
        raw = np.fromfile(files[key], dtype=np.uint8)
        t = torch.empty(raw.size, dtype=torch.uint8, pin_memory=True)
        t.numpy()[:] = raw
        bufs.append(t)
    E, D, C = bufs
    rc = nise.lib().nise_set_trajectory(c._h, E.data_ptr(), E.numel(), D.data_ptr(), D.numel(), C.data_ptr(),
                                        C.numel(), None, 0, None, 0)
    c._check(rc)
    return bufs


def test_chunked_upload_equals_resident(tmp_path):
    """16 400 frames of the 1024-site lattice (67 MB, 5 copy chunks), 1615
    start points: four waves of 8-vector CTAs and a tail."""
    s = synth.c1_spec(frames=16400, seed=501)
    files = synth.write(s, str(tmp_path))
    kw = synth.c1_keywords(Length=16400, Samplerate=10)
    p = nise.params_from_keywords(kw, files)
    with nise.Context(p) as c:
        c.load_files()  # pageable host memory: one synchronous copy
        r0, i0, n0 = c.absorption()
    with nise.Context(p) as c:
        keep = pinned_set(c, files)
        r1, i1, n1 = c.absorption()
        w1 = c.work()
        r2, i2, n2 = c.absorption()  # the cached plan
        w2 = c.work()
        del keep
    # the algorithmic counts are the plan's, reported again when it is reused
    assert w1 == w2 and w1[0] > 0 and w1[1] > 16000 * 1024 * 4
    assert n0 == n1 == n2 == 1615
    assert np.array_equal(r0, r1) and np.array_equal(i0, i1)
    assert np.array_equal(r1, r2) and np.array_equal(i1, i2)


def test_reused_plan_follows_new_data(tmp_path):
    """A second trajectory with the same couplings but other site energies
    reuses the plan; one with other couplings does not.  Each result equals a
    fresh context's."""
    def job(seed, d):
        s = synth.c1_spec(n_sites=96, frames=400, seed=seed)
        files = synth.write(s, str(d))
        kw = synth.c1_keywords(Singles=96, Length=400, RunTimes="16 0 0", Samplerate=1)
        return kw, files

    d1, d2, d3 = tmp_path / "a", tmp_path / "b", tmp_path / "c"
    for d in (d1, d2, d3):
        d.mkdir()
    kw, f1 = job(510, d1)
    _, f2 = job(511, d2)
    _, f3 = job(512, d3)
    # the same coupling frame, other diagonal records
    open(f2["coupling"], "wb").write(open(f1["coupling"], "rb").read())
    fresh = {}
    for name, f in (("a", f1), ("b", f2), ("c", f3)):
        with nise.Context(nise.params_from_keywords(kw, f)) as c:
            c.load_files()
            fresh[name] = c.absorption()
    with nise.Context(nise.params_from_keywords(kw, f1)) as c:
        for name, f in (("a", f1), ("b", f2), ("c", f3), ("a", f1)):
            keep = pinned_set(c, f)
            re, im, n = c.absorption()
            del keep
            assert np.array_equal(re, fresh[name][0]) and np.array_equal(im, fresh[name][1]), name
    assert not np.array_equal(fresh["a"][0], fresh["b"][0])
