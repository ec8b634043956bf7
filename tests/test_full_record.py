"""The benchmark's accuracy condition on the benchmarked record itself.

The metric is RTM shots/s at an image error of at most 1e-3 relative L2 against FP64.  This
runs the benchmark's own shot (bench.setup: the 1601 x 801 PSF-RTM shot, nt = 6000, all 641
well receivers, PSF data of the 20 x 10 scatter lattice) through libswd and through the FP64
CPU oracle (the reference's strip reconstruction, imaging, illumination normalisation and
Laplacian filter, all in double) on the host cores, and checks the raw image, the source
illumination and the filtered image.  The FP32 reconstruction of the source wavefield runs
backwards over all 6000 steps here, the regime where its rounding accumulates most.

The oracle needs about two to four minutes of host time for this shot.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_IMAGE_VS_FP64 = 1e-3


def test_c2_full_record_images_vs_fp64_oracle(swd):
    import bench
    from swd_b200 import configs
    w = configs.c2()
    E, shot, rick, data, _ = bench.setup(swd, w, 0)
    assert shot.nt == 6000 and len(shot.r_ix) == 641
    par = bench.fp64_parity(swd, E, w, shot, rick, data)
    print(f"c2 full record vs FP64: I {par['image_rel_l2']:.2e}  S {par['illum_rel_l2']:.2e}  "
          f"filtered image {par['fimage_rel_l2']:.2e}  (oracle {par['oracle_s']} s)")
    assert par["record"] == "full"
    assert par["image_rel_l2"] < TOL_IMAGE_VS_FP64
    assert par["illum_rel_l2"] < TOL_IMAGE_VS_FP64
    assert par["fimage_rel_l2"] < TOL_IMAGE_VS_FP64
    E.close()
