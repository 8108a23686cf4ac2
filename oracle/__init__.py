"""CPU oracle of the EmSART reconstruction hot path (TEST INFRASTRUCTURE).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only as the reference the results are
compared with or as the timed CPU baseline. The product (``artiatomi_b200``) never imports it.

Layout:
  esb_oracle.cpp  - C++ restatement of the reference's device kernels
                    (march, slicer, volTraversalLength, compare, cropBorder,
                    backProjection[FP16], makeSquare, ctf, wbpWeighting,
                    fourierFilter, doseWeighting) and a radix-2 FFT
  geometry.py     - numpy restatement of Projection/Volume geometry
  driver.py       - restatement of Reconstructor's FP/compare/BP sequences,
                    the SART loop (EmSart.cpp) and the sub-volume loop
                    (EmSartSubVolumes.cpp)
"""
from .lib import olib, build_oracle  # noqa: F401
