"""B200-native Census+SGM stereo matcher with the interface of R3DMVS's
r3d::match_stereo (rhiestan/Regard3D_MVS, src/r3d/stereo/stereo_matcher.hpp).

The computation lives in the CUDA library ``_lib/libr3dgpu.so`` (C ABI in
include/r3dgpu.h); this package is its Python binding.
"""

from .types import DisparityMap, LabelRanges, StereoOptions, SubpixelMethod, INVALID_DISPARITY  # noqa: F401
from ._native import StereoError, NativeLibraryMissing  # noqa: F401
from .stereo import (Matcher, Server, census_transform, detail, lift_u8, match_stereo, match_stereo_batch,  # noqa: F401
                     median_filter_3x3, pyramid_down, remove_speckles)
