"""Parameters of the synthetic benchmark workloads (data only).

This module imports nothing from the library, so that programs which only
need the parameters (the CPU baseline of bench.py, which must not load the
CUDA library) can read it by path. `workloads.build` turns an entry into
geometry, phantom and measured projections on the GPU.
"""

# name -> parameters; sizes are (x, y, z) voxels and W x H pixels
CONFIGS = {
    # Plain SART, no CTF: 256x256x128, 41 tilts of 256^2 in 3 degree steps,
    # lambda 0.5, one projection per ordered subset, oversampling 1.
    "c1_sart": dict(dims=(256, 256, 128), W=256, H=256, n_proj=41, n_ell=200, n_beads=0, ctf=False, os=1,
                    sirt=1, lam=0.5, iterations=3, shift=0.0, psi=0.0, noise_sigma_rel=0.1),
    # Full SART + 3D CTF: 1024x1024x256, 5000 ellipsoids + 300 beads, 61 tilts
    # of 1024^2 (2 degree steps), shifts U(+-2 px), psi jitter +-0.3 deg,
    # 300 kV, Cs 2.7 mm, pixel 0.27 nm, defocus 3000+-500 nm, astigmatism
    # 100 nm, 30 nm slabs, oversampling 2, 4 projections per subset.
    "c2_sart_ctf": dict(dims=(1024, 1024, 256), W=1024, H=1024, n_proj=61, n_ell=5000, n_beads=300, ctf=True, os=2,
                        sirt=4, lam=0.5, iterations=2, shift=2.0, psi=0.3, snr=0.1),
    # The same geometry with a 64-voxel-thick volume (256 MiB, still larger
    # than L2): the case on which kernels are profiled with ncu.
    # Precision at scale: 2048x2048x512, 20000 ellipsoids + 1000 beads, 61
    # tilts of 2048^2, CTF as above, oversampling 2, 8 projections per
    # subset, 5 iterations.
    "c5_precision": dict(dims=(2048, 2048, 512), W=2048, H=2048, n_proj=61, n_ell=20000, n_beads=1000, ctf=True,
                         os=2, sirt=8, lam=0.5, iterations=5, shift=2.0, psi=0.3, snr=0.1),
    # Its 256x256x64 crop-sized counterpart for the FP64 oracle (61 tilts of
    # 256^2, ellipsoid and bead counts scaled with the volume).
    "c5_crop": dict(dims=(256, 256, 64), W=256, H=256, n_proj=61, n_ell=40, n_beads=2, ctf=True, os=2, sirt=8,
                    lam=0.5, iterations=5, shift=2.0, psi=0.3, snr=0.1),
    # The C2 geometry cropped to 256x256x64 (61 tilts of 256^2, the same
    # angles, shifts, psi jitter, CTF, 30 nm slabs, oversampling 2, 4
    # projections per subset, 2 iterations; ellipsoid and bead counts scaled
    # with the volume): the size at which the FP32 and FP64 CPU oracles
    # reconstruct the C2 parameters in minutes.
    "c2_crop": dict(dims=(256, 256, 64), W=256, H=256, n_proj=61, n_ell=78, n_beads=5, ctf=True, os=2, sirt=4,
                    lam=0.5, iterations=2, shift=2.0, psi=0.3, snr=0.1),
    "c2_sart_ctf_z64": dict(dims=(1024, 1024, 64), W=1024, H=1024, n_proj=61, n_ell=1250, n_beads=75, ctf=True, os=2,
                            sirt=4, lam=0.5, iterations=2, shift=2.0, psi=0.3, snr=0.1),
}
