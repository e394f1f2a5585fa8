"""The slab-staged forward projector (csrc/k_fp_slab.cu) against the gather
projector, bit for bit, through the C ABI.

stt_fp_correction projects the oblique views (central ray more than 25 degrees
off both x and z) with the TMA slab kernel whenever the volume's x and z
extents are multiples of 4; stt_fp always gathers.  Both add the same samples
in the same order with the same rounding, so the correction
c = (b - Ax) / (L + 1) must equal the one formed from stt_fp's projection and
ray lengths in float32, element for element, on every view: centred and
off-centre volumes, non-unit spacing, non-cubic extents, rays that miss, and
the non-zero boundary where the march re-walks samples before its entry."""
import math

import numpy as np
import pytest

import oracle_bind as ob
from test_gpu_kernels import _np, _t, make_ctx, phantom

pytestmark = pytest.mark.gpu

CASES = [  # dims (nx, ny, nz), detector (W, H), spacing, offset, zero boundary
    ((64, 64, 64), (96, 80), 1.0, (0.0, 0.0, 0.0), True),
    ((48, 40, 36), (72, 64), 1.3, (2.5, -1.5, 1.0), True),
    ((40, 24, 52), (60, 40), 0.9, (-1.0, 0.5, 2.0), False),
    ((32, 32, 32), (120, 96), 1.0, (0.0, 0.0, 0.0), True),  # many rays miss
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_slab_staged_fp_correction_equals_gather(cuda, case):
    import torch

    dims, det, sp, off, zb = CASES[case]
    scan = ob.Scan(dims, det, spacing=sp, off=off)
    # every octant, with views on both sides of the 25-degree line and at 45
    angles = np.array([0.05, 0.3, 0.45, 0.5, 0.785, 1.1, 1.3, 1.57, 2.0, 2.36, 2.9, 3.3, 3.93, 4.4, 5.5, 6.0])
    ctx = make_ctx(scan, angles)
    nx, ny, nz = dims
    W, H = det
    vol = phantom(dims, seed=11 + case, zero_boundary=zb) + np.float32(0.01)
    vol_d = _t(vol, cuda)
    rng = np.random.default_rng(case)
    b = rng.uniform(0, 30, (len(angles), H, W)).astype(np.float32)
    state = torch.zeros((H, W), device=cuda)
    corr = torch.zeros((H, W), device=cuda)
    ref_state = np.zeros((H, W), np.float32)
    staged = 0
    for v, a in enumerate(angles):
        ctx.fp_correction(vol_d, _t(b[v], cuda), state, corr, v)
        ax = torch.zeros((1, H, W), device=cuda)
        rl = torch.zeros((1, H, W), device=cuda)
        w = torch.zeros((1, H, W), device=cuda)
        ctx.fp(vol_d, ax, v, 1, raylen=rl, weight=w)
        torch.cuda.synchronize()
        hit = _np(w)[0] > 0
        ref_state = np.where(hit, _np(rl)[0], ref_state).astype(np.float32)
        c_ref = (b[v] - _np(ax)[0]) / (ref_state + np.float32(1.0))
        np.testing.assert_array_equal(_np(state), ref_state, err_msg=f"ray length, view {v}")
        np.testing.assert_array_equal(_np(corr), c_ref.astype(np.float32), err_msg=f"correction, view {v}")
        staged += min(abs(math.sin(a)), abs(math.cos(a))) > 0.4226
        assert hit.any()
    assert staged >= 6  # the slab kernel had views to project
    ctx.poll_status()  # no bounded wait of the staged kernel gave up
    ctx.close()
