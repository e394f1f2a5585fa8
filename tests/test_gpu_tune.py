"""The autotuner's candidates (stt_autotune, stt_set_tuning through the C ABI)
give identical outputs: every launch variant of the gather projector, every
box of the slab-staged projector and every column length of the voxel
backprojection produce the same bits as the default, so the tuner only ever
changes the time.  The tuner's choice is valid and is cached per shape."""
import math

import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu


def _ctx(scan, angles):
    import spacetimetomography_b200 as stt

    c = stt.Context(0)
    c.set_geometry(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, angles, scan.off)
    return c


def _corrections(ctx, vol, b, views):
    import torch

    H, W = b.shape[1:]
    state = torch.zeros((H, W), device=vol.device)
    corr = torch.zeros((H, W), device=vol.device)
    out = []
    for v in views:
        ctx.fp_correction(vol, b[v], state, corr, v)
        out.append(corr.clone())
    out.append(state.clone())
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in out]


# every off-axis class: 0..45 degrees and their mirrors
ANGLES = np.deg2rad([0, 3, 8, 13, 17, 22, 27, 33, 38, 44, 47, 62, 88, 96, 133, 181, 228, 271, 313, 350])


@pytest.mark.parametrize("dims,det,off", [((48, 40, 44), (72, 60), (0.5, -0.3, 0.2)),
                                          ((64, 64, 64), (96, 80), (0.0, 0.0, 0.0))])
def test_every_projector_variant_gives_the_same_bits(cuda, dims, det, off):
    import torch

    from spacetimetomography_b200 import phantom as ph

    scan = ob.Scan(dims, det, off=off)
    ctx = _ctx(scan, ANGLES)
    vol = ph.ellipsoid_phantom(dims, 6, seed=4, semi=(3.0, 12.0)).to(cuda) + 0.01
    g = torch.Generator(device=cuda)
    g.manual_seed(1)
    b = torch.rand((len(ANGLES), det[1], det[0]), device=cuda, generator=g) * 30
    views = range(len(ANGLES))
    ctx.set_tuning(0, 0, 0, staged_bins=0)  # everything through the default gather variant
    base = _corrections(ctx, vol, b, views)
    # the tld4 variants must really bind the volume here, not run as loads
    assert ctx.fp_texture_ok(vol)
    for fv in range(1, 12):  # tiles, samples in flight, packed FP32x2 pairs, tld4 corners
        ctx.set_tuning(fv, 0, 0, staged_bins=0)
        for k, (a, c) in enumerate(zip(base, _corrections(ctx, vol, b, views))):
            np.testing.assert_array_equal(a, c, err_msg=f"gather variant {fv}, output {k}")
    for sv in range(8):  # every view through the slab-staged kernel with each box, scalar and packed
        ctx.set_tuning(0, sv, 0, staged_bins=0x1FF)
        for k, (a, c) in enumerate(zip(base, _corrections(ctx, vol, b, views))):
            np.testing.assert_array_equal(a, c, err_msg=f"slab box {sv}, output {k}")
    ctx.poll_status()
    ctx.close()


# a small scan, and a highly magnified one (sid 350 mm) where a column's
# detector rows move by up to three pixels per voxel
BP_SCANS = [dict(n=40, det=(64, 56), sid=600.0), dict(n=(160, 48, 96), det=(480, 160), sid=350.0)]


@pytest.mark.parametrize("sc", BP_SCANS)
def test_every_backprojection_variant_gives_the_same_bits(cuda, sc):
    """Column lengths 16, 8 and 32, with and without the L2 prefetch: the same solve bit for bit."""
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph

    V = 8
    scan = ob.Scan(sc["n"], sc["det"], sid=sc["sid"])
    nx, ny, nz = scan.dims
    W, H = scan.det
    angles = np.linspace(0, 2 * math.pi, V, endpoint=False) + 0.1
    truth = ph.ellipsoid_phantom(scan.dims, 5, seed=2, semi=(3.0, 10.0)).to(cuda)
    ctx = _ctx(scan, angles)
    proj = torch.zeros((V, H, W), device=cuda)
    ctx.fp(truth, proj)
    pd = stt.PdParams(gmax=float(proj.max()) / 4, tp_w=0.0, bc_w=0.0, cut=(3, 3, 3, 5, 3, 3, 6, 5))
    outs = []
    for bv in range(5):
        ctx.set_tuning(0, 0, bv)
        z = lambda *s: torch.zeros(s, device=cuda)  # noqa: E731
        st = dict(vol=z(2, nz, ny, nx), xbar=z(2, nz, ny, nx), xprev=z(1, nz, ny, nx), ytv=z(1, 3, nz, ny, nx),
                  ytp=z(1, nz, ny, nx), ybc=z(1, nz, ny, nx), flow=z(1, 3, nz, ny, nx), proj=proj[None].contiguous())
        s = stt.Solver(ctx, st, 1, V, pd, roi_cut=(3, 3, 3, 5, 3, 3, 6, 5), seed=3)
        s.iterate(2)
        torch.cuda.synchronize()
        outs.append(st["vol"][0].cpu().numpy())
        s.close()
    for bv in range(1, 5):
        np.testing.assert_array_equal(outs[0], outs[bv], err_msg=f"backprojection variant {bv}")
    assert np.abs(outs[0]).max() > 0
    ctx.close()


def test_autotune_picks_a_valid_choice_and_caches_it(cuda):
    import torch

    from spacetimetomography_b200 import phantom as ph

    dims, det = (64, 56, 60), (96, 80)
    scan = ob.Scan(dims, det)
    ctx = _ctx(scan, ANGLES)
    t = ctx.autotune()
    assert t["tuned"] and not t["from_cache"]
    assert 0 <= t["fp_variant"] < 12 and 0 <= t["slab_variant"] < 8 and 0 <= t["bp_variant"] < 5
    assert 0 <= t["ray_variant"] < 2
    assert 0 <= t["staged_bins"] < 512 and 0 <= t["staged_bins_bf16"] < 512
    assert all(x > 0 for x in t["fp_us"]) and all(x > 0 for x in t["bp_us"]) and all(x > 0 for x in t["ray_us"])
    assert t["fp"] and t["slab"] and t["bp"] and t["ray"]
    assert ctx.get_tuning()["fp_variant"] == t["fp_variant"]
    # a second context of the same shape takes the cached choice
    ctx2 = _ctx(scan, ANGLES)
    t2 = ctx2.autotune()
    assert t2["from_cache"] and t2["fp_variant"] == t["fp_variant"] and t2["staged_bins"] == t["staged_bins"]
    # and the tuned context projects what the default one does
    vol = ph.ellipsoid_phantom(dims, 6, seed=9, semi=(3.0, 12.0)).to(cuda)
    b = torch.rand((len(ANGLES), det[1], det[0]), device=cuda) * 10
    ctx3 = _ctx(scan, ANGLES)  # defaults
    for a, c in zip(_corrections(ctx3, vol, b, range(len(ANGLES))), _corrections(ctx, vol, b, range(len(ANGLES)))):
        np.testing.assert_array_equal(a, c)
    with pytest.raises(Exception):
        ctx.set_tuning(fp_variant=99)
    for c in (ctx, ctx2, ctx3):
        c.close()


def test_both_ray_backprojection_scatters_agree(cuda):
    """The two scatters of the ray-driven backprojection (global vector atomics;
    a shared-memory box per slab) add the same terms in different float
    orders: the same result within atomic-order rounding, on a geometry with
    oblique and axis views and rays that miss."""
    import torch

    import spacetimetomography_b200 as stt

    scan = ob.Scan((72, 64, 80), (120, 104), off=(0.6, -0.4, 1.1))
    ctx = _ctx(scan, ANGLES[:8])
    g = torch.Generator(device=cuda)
    g.manual_seed(4)
    corr = torch.randn((scan.det[1], scan.det[0]), device=cuda, generator=g)
    out = []
    for rv in (0, 1):
        ctx.set_tuning(0, 0, 0, ray_variant=rv)
        assert ctx.get_tuning()["ray_variant"] == rv
        c = torch.zeros(scan.dims[::-1], device=cuda)
        w = torch.zeros(scan.dims[::-1], device=cuda)
        for v in range(8):
            ctx.bp_ray_scatter(corr, c, w, v)
        torch.cuda.synchronize()
        out.append((c.cpu().numpy(), w.cpu().numpy()))
    assert ob.rel_l2(out[1][0], out[0][0]) < 1e-5 and ob.rel_l2(out[1][1], out[0][1]) < 1e-5
    assert float(np.abs(out[0][1]).sum()) > 0
    with pytest.raises(stt.STTError):
        ctx.set_tuning(0, 0, 0, ray_variant=2)
    ctx.close()


def test_batch_staging_choice_leaves_the_solve_unchanged(cuda):
    """A batch whose instances ask for tuning times its projector split both
    ways at creation (stt_batch_staging) without touching the callers' start
    volumes: after two iterations its volumes equal those of an untuned batch
    of the same instances bit for bit (voxel BP; every projector and
    backprojection variant gives the same bits)."""
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph

    shapes = [((48, 40, 48), (72, 64), 14), ((64, 48, 56), (96, 72), 11), ((40, 40, 40), (64, 64), 9)]
    cut = (2, 2, 2, 2, 2, 2, 3, 3)
    runs = []
    for tuned in (False, True):
        items = []
        for k, (dims, det, nv) in enumerate(shapes):
            ctx = stt.Context(0)
            ctx.set_geometry(dims, (1.0, 1.0, 1.0), det, 1.0, 600.0, 1000.0,
                             np.linspace(0, 2 * math.pi, nv, endpoint=False) + 0.2)
            truth = ph.ellipsoid_phantom(dims, 5, seed=20 + k, semi=(3.0, 10.0)).to(cuda)
            proj = torch.zeros((nv, det[1], det[0]), device=cuda)
            ctx.fp(truth, proj)
            pd = stt.PdParams(tv_w=0.02, tp_w=0.0, bc_w=0.0, huber_factor=0.9, gmax=float(proj.max()) / 4, cut=cut)
            items.append(dict(ctx=ctx, vol=(truth * 0.5).contiguous(), proj=proj, pd=pd, roi_cut=cut, seed=7 + k,
                              autotune=tuned))
        b = stt.Batch(items, mode=stt.SOLVE_GRAPH)
        info = b.staging()
        assert set(info) == {"timed", "all_gather", "ms_split", "ms_gather"}
        if tuned and info["timed"]:
            assert info["ms_split"] > 0 and info["ms_gather"] > 0
        b.iterate(2)
        torch.cuda.synchronize()
        b.poll_status()
        b.close()
        runs.append([d["vol"].cpu().numpy() for d in items])
        for d in items:
            d["ctx"].close()
    for a, c in zip(*runs):
        np.testing.assert_array_equal(a, c)
