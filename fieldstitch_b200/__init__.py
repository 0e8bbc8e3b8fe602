"""fieldstitch_b200: B200-native (sm_100a) SIFT extraction + prior-guided descriptor matching.

A drop-in for the feature front end of PlaneSite (Edko01/FieldStitch): ``gsift.detect`` /
``gsift.describe``, ``features.sift_gpu`` and ``matching._ratio_match_bf`` / ``_guided`` /
``_unique``, with the same call signatures and OpenCV-compatible outputs, computed by hand-written
CUDA kernels in ``libfsb200.so`` behind a C ABI (include/fsb200.h). There is no CPU fallback.
"""
from . import features, frontend, gsift, matching, recon  # noqa: F401
from ._lib import LIB_PATH, context, load  # noqa: F401

__all__ = ["gsift", "features", "matching", "frontend", "context", "load", "LIB_PATH"]
