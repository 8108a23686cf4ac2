"""The library's CTF filter against the reference's own `ctf` kernel on the GPU.

`ctf.cu` (src/EmSART/cuda_kernels/ctf.cu:82-240) is the one kernel of the
reference's EmSART path that CUDA 12 still compiles; oracle/ref_build.py
builds it unmodified for sm_100a into oracle/_ref/libref_ctf_gpu.so (with a
launcher that sets its constants as Kernels.cpp:1104-1131 does). Both filter
the same 1024^2 half-spectra (the C2 FFT size) in the forward (CTF), Wiener
and phase-flip modes; the results agree to 1e-5 relative L2 (both evaluate
the same expressions; the compilers' choices of fused multiply-adds may
differ), and the device time per launch of each is printed (CUDA events
around replays of 100 launches captured in a CUDA graph).
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

LIB = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "libref_ctf_gpu.so"
N = 1024
BETA = (200.0, 0.0, 0.008, 0.0)
TOL = 1e-5


def _ref():
    if not LIB.exists():
        pytest.skip("oracle/_ref/libref_ctf_gpu.so not built (needs the reference tree at build time)")
    lib = C.CDLL(str(LIB))
    F = C.c_float
    lib.ref_ctf_gpu.argtypes = [C.c_void_p, C.c_int, F, F, F, C.c_int, C.c_int, F, C.c_void_p, F, F, F, F, C.c_int,
                               C.c_void_p]
    lib.ref_ctf_gpu.restype = C.c_int
    return lib


@pytest.mark.parametrize("mode", ["fp", "wiener", "flip"])
def test_ctf_matches_reference_kernel(mode):
    import torch

    import artiatomi_b200 as E

    lib = _ref()
    rng = np.random.default_rng(11)
    spec = torch.from_numpy(rng.normal(size=(N, N // 2 + 1, 2)).astype(np.float32)).cuda()
    beta = np.asarray(BETA, np.float32)
    for_fp, flip = mode == "fp", mode == "flip"
    args = (2950.0, 3050.0, 37.0, for_fp, flip, 0.1)
    ours = spec.clone()
    E.ctf(ours, N, *args, beta_fac=BETA, cs_mm=2.7, voltage_kv=300.0, amp_contrast=0.07, pixel_size_nm=0.27)
    theirs = spec.clone()
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.ref_ctf_gpu(theirs.data_ptr(), N, args[0], args[1], args[2], int(for_fp), int(flip), args[5],
                         beta.ctypes.data, 2.7, 300.0, 0.07, 0.27, 1, stream)
    assert rc == 0
    torch.cuda.synchronize()
    e = rel_l2(ours.cpu().numpy(), theirs.cpu().numpy())
    print(f"CTF {mode}: library vs reference kernel rel-L2 {e:.2e}")
    assert e <= TOL, e

    def timed(fn, reps=100):
        # device time per launch: the launches are captured in a CUDA graph
        # and replayed, so host-side call overhead (ctypes) is not measured
        side = torch.cuda.Stream()
        with torch.cuda.stream(side):
            fn()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            for _ in range(reps):
                fn()
        g.replay()
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(5):
            g.replay()
        s1.record()
        torch.cuda.synchronize()
        return s0.elapsed_time(s1) / (5 * reps)

    t_ours = timed(lambda: E.ctf(ours, N, *args, beta_fac=BETA, cs_mm=2.7, voltage_kv=300.0, amp_contrast=0.07,
                                 pixel_size_nm=0.27))
    t_ref = timed(lambda: lib.ref_ctf_gpu(theirs.data_ptr(), N, args[0], args[1], args[2], int(for_fp), int(flip),
                                          args[5], beta.ctypes.data, 2.7, 300.0, 0.07, 0.27, 0,
                                          torch.cuda.current_stream().cuda_stream))
    nbytes = 2 * N * (N // 2 + 1) * 8
    print(f"CTF {mode} {N}^2 half-spectrum: library k_ctf {t_ours * 1e3:.1f} us ({nbytes / t_ours / 1e6:.0f} GB/s), "
          f"reference ctf.cu {t_ref * 1e3:.1f} us ({nbytes / t_ref / 1e6:.0f} GB/s) per launch")
