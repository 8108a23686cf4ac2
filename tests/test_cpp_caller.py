"""A compiled C++ caller of the C ABI: EmSart's SART run with libesb in place
of the reference's Reconstructor (oracle/cpp_caller/sart_caller.cpp).

The program reads emsart.cfg and the marker file with the reference's own
Configuration::Config and MarkerFile, derives the detector frames and the
volume placement with the reference's Projection and Volume, takes the
projection order from Projection::CreateProjectionIndexList, and runs
esb_reconstructor_create + esb_sart_run (EmSart.cpp:83-675 with the device
work replaced). Its volume is compared with the oracle's SART on the same
projections: the FAITHFUL kernels with the FP32 oracle (1e-5), the FAST
kernels with the FP64 oracle (2e-4), as the other SART tests do. The block of
the program between its begin/end markers is the C++ snippet of
INTEGRATION.md (checked on the CPU).
"""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests.helpers import rel_l2

ROOT = Path(__file__).resolve().parent.parent
EXE = ROOT / "oracle" / "_ref" / "sart_caller"
SRC = ROOT / "oracle" / "cpp_caller" / "sart_caller.cpp"

DIMS, W, H, N = (64, 64, 32), 64, 64, 9
ITERATIONS, SIRT, OS = 2, 3, 2
CFG = """ProjectionFile = {d}/ts.raw
OutVolumeFile = {d}/vol.raw
MarkerFile = {d}/markers.em
Lambda = 0.5
Iterations = {it}
RecDimesions = {nx} {ny} {nz}
UseFixPsiAngle = false
PsiAngle = 0
PhiAngle = 0
AddTiltAngle = 0
AddTiltXAngle = 0
VolumeShift = 0 0 0
ReferenceMarker = 0
OverSampling = {os}
VoxelSize = 1
DimLength = 3 3
CutLength = 1 1
Crop = 1 2 1 2
CropDim = 3 3 3 3
SkipFilter = false
fourFilterLP = 28
fourFilterLPS = 4
fourFilterHP = 0
fourFilterHPS = 0
SIRTCount = {sirt}
CtfMode = false
BadPixelValue = 10
CorrectBadPixels = true
ProjectionNormalization = std
WBP = false
WBPFilter = Ramp
CudaDeviceID = 0
ProjectionScaleFactor = 1
CtfFile = none
"""


def _snippet(text: str) -> str:
    a = text.index("// --- begin: libesb in place of the Reconstructor")
    b = text.index("// --- end ---", a)
    return text[a:b]


def _norm(s: str) -> str:
    return re.sub(r"\s+", " ", s).strip()


def test_integration_snippet_is_the_compiled_program():
    doc = (ROOT / "INTEGRATION.md").read_text()
    assert _norm(_snippet(SRC.read_text())) in _norm(doc)


def _blocks(text: str, begin: str):
    out, i = [], 0
    while True:
        a = text.find(begin, i)
        if a < 0:
            return out
        a = text.index("\n", a) + 1
        b = text.index("// --- end ---", a)
        out.append(text[a:b])
        i = b


def test_zslab_nccl_caller_compiles_and_is_documented(tmp_path):
    """The multi-GPU section's C++ (esb_sart_run_zslab with an NCCL
    all-reduce callback) compiles against include/esb.h and nccl.h and
    links against libesb and NCCL; INTEGRATION.md shows the same code."""
    import shutil

    src = ROOT / "oracle" / "cpp_caller" / "zslab_nccl.cpp"
    text = src.read_text()
    doc = _norm((ROOT / "INTEGRATION.md").read_text())
    blocks = _blocks(text, "// --- begin: z-slab SART")
    assert len(blocks) == 2
    for b in blocks:
        assert _norm(b) in doc
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    cuda = Path("/usr/local/cuda/include")
    r = subprocess.run(["g++", "-std=c++14", "-fPIC", "-shared", "-I", str(ROOT / "include"), "-I", str(cuda),
                        str(src), "-L", str(ROOT / "artiatomi_b200"), "-lesb", "-lnccl",
                        "-o", str(tmp_path / "libzslab.so")], capture_output=True, text=True)
    if r.returncode != 0 and ("nccl.h" in r.stderr or "-lnccl" in r.stderr):
        pytest.skip("NCCL headers or library not found: " + r.stderr.strip().splitlines()[-1])
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_cpp_caller_sart_matches_oracle(tmp_path):
    if not EXE.exists():
        pytest.skip("oracle/_ref/sart_caller not built (needs the reference tree at build time)")
    import artiatomi_b200 as E
    from artiatomi_b200 import fileio as F
    from artiatomi_b200 import phantom as PH
    from oracle import driver as D
    from oracle import geometry as G
    from oracle.driver import OracleReconstructor

    tilt = PH.tilt_series(N, -60, 60)
    xs, ys, psi = PH.alignment(N, seed=5, shift=1.0, psi_jitter=0.2)
    items = np.zeros((1, N, 10), np.float32)
    items[0, :, 0], items[0, :, 1:3], items[0, :, 4], items[0, :, 5] = tilt, 10.0, xs, ys
    items[0, :, 8], items[0, :, 9] = 1.0, psi
    F.write_markers(str(tmp_path / "markers.em"), items)
    og = G.projection_geometry(tilt, xs, ys, None, psi, W, H)
    vo = G.volume_geometry(DIMS)
    vol = PH.phantom_numpy(DIMS, 25, seed=9)
    projs = np.zeros((N, H, W), np.float32)
    rng = np.random.default_rng(4)
    for i in range(N):
        dist = np.zeros((H, W), np.float32)
        D.fp_march(G.orc_geom(og[i], vo), vol, 0, W, H, projs[i], dist)
        projs[i] += rng.normal(size=(H, W)).astype(np.float32) * 0.1 * projs[i].std()
    projs.tofile(tmp_path / "ts.raw")
    (tmp_path / "emsart.cfg").write_text(CFG.format(d=tmp_path, it=ITERATIONS, nx=DIMS[0], ny=DIMS[1], nz=DIMS[2],
                                                    os=OS, sirt=SIRT))
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, tilt)
    cfgd = dict(lambda_=0.5, oversampling=OS, cut_length=(1.0, 1.0), dim_length=(3.0, 3.0), crop=(1.0, 2.0, 1.0, 2.0),
                crop_dim=(3.0, 3.0, 3.0, 3.0))
    for variant, precision, tol in ((0, 0, 1e-5), (1, 1, 2e-4)):
        out = tmp_path / f"vol{variant}.raw"
        r = subprocess.run([str(EXE), str(tmp_path / "emsart.cfg"), str(tmp_path / "markers.em"),
                            str(tmp_path / "ts.raw"), str(W), str(H), str(out), str(variant)], capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        got = np.fromfile(out, np.float32).reshape(DIMS[::-1])
        orc = OracleReconstructor(cfgd, W, H, og, tilt, precision=precision)
        v = np.zeros(DIMS[::-1], np.float32)
        orc.sart(vo, v, 0, projs, il, ITERATIONS, SIRT)
        e = rel_l2(got, v)
        print(f"C++ caller, variant {variant}: rel-L2 vs {'FP32' if precision == 0 else 'FP64'} oracle {e:.2e}")
        assert e <= tol, (variant, e)
