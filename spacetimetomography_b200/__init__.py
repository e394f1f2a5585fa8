"""B200-native reconstruction hot path of SpaceTimeTomography.

The compute lives in ``libstt.so`` (hand-written sm_100a CUDA behind the C ABI
of ``include/stt.h``); this package is the Python side of that ABI, used by the
tests and the benchmark.  Tensors are torch CUDA tensors (device memory and
streams only); every operation is a call into libstt.
"""
from ._lib import STTError, lib  # noqa: F401  (loads libstt.so or raises)
from .api import (  # noqa: F401
    SOLVE_GRAPH,
    SOLVE_PERSISTENT,
    SOLVE_PLAIN,
    SOLVE_STREAMS,
    Batch,
    Context,
    Flow,
    PdParams,
    Solver,
    frame_order,
    image_gradient,
    lds_angles,
    permutation,
    views_from_rounds,
    warp,
    warp_box,
    warp_poll_status,
    warp_vjp,
)
from .api import FlowParams_ as FlowParams  # noqa: F401

__version__ = "0.1.0"
