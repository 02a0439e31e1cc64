"""imageproc_b200: imageproc's template-matching path on NVIDIA B200 (sm_100a).

``imageproc_b200.template_matching`` mirrors ``imageproc::template_matching``
(match_template, match_template_parallel, match_template_with_mask,
match_template_with_mask_parallel, find_extremes). The compute runs in the
CUDA library ``libimageproc_b200.so`` through its C ABI
(``include/imageproc_b200.h``); ``imageproc_b200.device`` exposes the
device-resident forms on torch CUDA tensors.
"""

from . import template_matching  # noqa: F401
from ._lib import DeviceError, Panic  # noqa: F401
from .template_matching import (  # noqa: F401
    Extremes,
    MatchTemplateMethod,
    Precision,
    find_extremes,
    match_template,
    match_template_parallel,
    match_template_with_mask,
    match_template_with_mask_parallel,
)

__version__ = "0.1.0"
