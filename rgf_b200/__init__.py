"""rgf_b200 -- B200 (sm_100a) implementation of chiaweihsu/RGF's slice recursion.

The public functions mirror the reference's MATLAB entry points and run on
the GPU through the C ABI in ``include/rgf.h`` (``librgf.so``).
"""
from .api import (build_laplacian_1d, cal_smatrix_RGF, cal_smatrix_RGF_3D, setup_channels,
                  setup_channels_3D, smatrix_grad_RGF, smatrix_grad_RGF_3D, cal_smatrix_RGF_batch,
                  fields_RGF, fields_RGF_3D)

__all__ = ["cal_smatrix_RGF", "cal_smatrix_RGF_3D", "setup_channels", "setup_channels_3D",
           "build_laplacian_1d", "smatrix_grad_RGF", "smatrix_grad_RGF_3D",
           "cal_smatrix_RGF_batch", "fields_RGF", "fields_RGF_3D"]
__version__ = "0.1.0"
