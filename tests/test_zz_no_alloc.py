"""stt_bp_ray_noalloc: the ray-driven backprojector for callers that cannot
allocate device memory (a plugin whose host application owns all GPU memory,
a real-time loop that cannot take cudaMalloc's synchronisation).  Its scratch
is a fixed array inside libstt.so; this checks, through the C ABI, that two
calls in a row give what the allocating stt_bp_ray gives, and that a volume
larger than the fixed scratch is refused.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-4  # the tolerance of the other ray-BP parity tests (float atomics)
MAX_VOXELS = 1 << 21


def _bind():
    from spacetimetomography_b200._lib import lib

    lib.stt_bp_ray_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_void_p]
    lib.stt_bp_ray_noalloc.restype = C.c_int
    return lib


def _ctx(dims, det, angles):
    import spacetimetomography_b200 as stt

    ctx = stt.Context(0)
    ctx.set_geometry(dims, (1.0, 1.0, 1.0), det, 1.0, 600.0, 1000.0, angles)
    return ctx


def test_noalloc_matches_allocating_entry_point(cuda):
    import torch

    lib = _bind()
    dims, det = (48, 40, 44), (64, 56)
    angles = np.array([0.3, 1.7, 4.1])
    ctx = _ctx(dims, det, angles)
    rng = np.random.default_rng(3)
    nx, ny, nz = dims
    vol0 = torch.from_numpy(rng.uniform(0, 1, (nz, ny, nx)).astype(np.float32)).to(cuda)
    a, b = vol0.clone(), vol0.clone()
    gmax = 1.5
    stream = torch.cuda.current_stream().cuda_stream
    for call, view in enumerate((0, 2)):  # two calls in a row share the fixed scratch
        corr = torch.from_numpy(rng.normal(size=(det[1], det[0])).astype(np.float32)).to(cuda)
        ctx.bp_ray(corr, a, gmax, view)
        rc = lib.stt_bp_ray_noalloc(ctx._h, C.c_void_p(corr.data_ptr()), C.c_void_p(b.data_ptr()), gmax, view,
                                    C.c_void_p(stream) if stream else None)
        assert rc == 0, lib.stt_last_error(ctx._h)
        torch.cuda.synchronize()
        ref = a.double()
        err = float(torch.linalg.norm(b.double() - ref) / torch.linalg.norm(ref))
        assert err < TOL, (call, err)
    ctx.close()


def test_noalloc_rejects_volume_beyond_fixed_scratch(cuda):
    import torch

    lib = _bind()
    dims = (130, 130, 130)  # 2,197,000 voxels > 2^21
    assert np.prod(dims) > MAX_VOXELS
    ctx = _ctx(dims, (64, 64), np.array([0.0]))
    vol = torch.zeros((dims[2], dims[1], dims[0]), device=cuda)
    corr = torch.zeros((64, 64), device=cuda)
    rc = lib.stt_bp_ray_noalloc(ctx._h, C.c_void_p(corr.data_ptr()), C.c_void_p(vol.data_ptr()), 1.0, 0, None)
    assert rc == 1  # STT_ERR_INVALID
    msg = lib.stt_last_error(ctx._h).decode()
    assert "2097152" in msg and "scratch" in msg
    ctx.close()
