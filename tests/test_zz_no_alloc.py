"""The allocation-free absorption entry point against the regular one.

nise_absorption_noalloc serves callers whose device memory is owned by their
own allocator (they hand the library device buffers and the library must not
call cudaMalloc/cudaFree itself).  Its intermediate tables live in the
library's static 32 MiB device scratch array.  This file is collected last so
that a stop-at-first-failure run has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import helpers
import nise_2017_b200 as nise

pytestmark = pytest.mark.gpu


def test_noalloc_matches_regular_entry_twice(tmp_path):
    import torch
    case = helpers.cases()["abs_coupling_full"]
    files = helpers.materialise(case, str(tmp_path))
    p = nise.params_from_keywords(case["keywords"], files)
    with nise.Context(p) as c:
        c.load_files()
        re_ref, im_ref, n_ref = c.absorption()
    energy = np.fromfile(files["energy"], dtype=np.uint8)
    dipole = np.fromfile(files["dipole"], dtype=np.uint8)
    d_e = torch.from_numpy(energy).cuda()
    d_d = torch.from_numpy(dipole).cuda()
    lib = nise.lib()
    fn = lib.nise_absorption_noalloc
    fn.argtypes = [ctypes.POINTER(nise.Params), ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        d_re = torch.full((p.tmax1,), float("nan"), dtype=torch.float64, device="cuda")
        d_im = torch.full((p.tmax1,), float("nan"), dtype=torch.float64, device="cuda")
        n = ctypes.c_int(0)
        rc = fn(ctypes.byref(p), d_e.data_ptr(), energy.nbytes, d_d.data_ptr(), dipole.nbytes, d_re.data_ptr(),
                d_im.data_ptr(), ctypes.byref(n), ctypes.c_void_p(stream))
        assert rc == 0, lib.nise_global_error().decode()
        torch.cuda.synchronize()
        re, im = d_re.cpu().numpy(), d_im.cpu().numpy()
        assert n.value == n_ref
        # same kernels and summation order as the regular entry point
        assert helpers.rel(re + 1j * im, re_ref + 1j * im_ref) < 1e-12, "call %d" % call


def test_noalloc_rejects_oversized_jobs(tmp_path):
    import torch
    from nise_2017_b200 import synth
    s = synth.spec(n_sites=200, frames=3000, seed=9)
    files = synth.write(s, str(tmp_path))
    kw = synth.c0_keywords(Singles=200, Length=3000, RunTimes="256 0 0", Samplerate=4)
    p = nise.params_from_keywords(kw, files)
    energy = np.fromfile(files["energy"], dtype=np.uint8)
    dipole = np.fromfile(files["dipole"], dtype=np.uint8)
    d_e = torch.from_numpy(energy).cuda()
    d_d = torch.from_numpy(dipole).cuda()
    d_out = torch.zeros(2 * p.tmax1, dtype=torch.float64, device="cuda")
    lib = nise.lib()
    fn = lib.nise_absorption_noalloc
    fn.argtypes = [ctypes.POINTER(nise.Params), ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]
    n = ctypes.c_int(0)
    rc = fn(ctypes.byref(p), d_e.data_ptr(), energy.nbytes, d_d.data_ptr(), dipole.nbytes, d_out.data_ptr(),
            d_out.data_ptr() + 8 * p.tmax1, ctypes.byref(n), None)
    assert rc == -3 and b"32 MiB" in lib.nise_global_error()
