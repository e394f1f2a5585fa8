"""The C++ drop-in layer on the GPU: code written against the reference's
interfaces (warping::warp, optical_flow::L1Huber_OF[_MultiScale3D],
TypicalRayProducer and the .core.h entry points; tests/facade_dropin_check.cpp)
and the ST-Tomography command line, checked against the oracle and against
the same pipeline driven through the Python side of the C ABI."""
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "spacetimetomography_b200"
CLI = PKG / "bin" / "st_tomography"


@pytest.fixture(scope="module")
def dropin(tmp_path_factory):
    exe = tmp_path_factory.mktemp("bin") / "facade_dropin_check"
    cmd = ["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", f"-I{ROOT / 'include' / 'reference'}",
           "-I/usr/local/cuda/include", str(ROOT / "tests" / "facade_dropin_check.cpp"), "-o", str(exe), f"-L{PKG}",
           "-L/usr/local/cuda/lib64", "-lstt_facade", "-lstt", "-lcudart", f"-Wl,-rpath,{PKG}",
           "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True)
    return exe


def run(exe, *args):
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r


def put(d, name, a):
    np.ascontiguousarray(a, np.float32).tofile(d / name)


def get(d, name, shape):
    return np.fromfile(d / name, np.float32).reshape(shape)


@pytest.mark.parametrize("box", [None, (21.0, 15.0, 13.0)])
def test_dropin_warp_equals_reference_arithmetic(cuda, dropin, tmp_path, box):
    rng = np.random.default_rng(21)
    nz, ny, nx = 11, 13, 17
    vel = (rng.normal(size=(3, nz, ny, nx)) * 1.4).astype(np.float32)
    src = rng.normal(size=(2, nz, ny, nx)).astype(np.float32)
    put(tmp_path, "vel.raw", vel)
    put(tmp_path, "src.raw", src)
    b = (nx, ny, nz) if box is None else box
    run(dropin, "warp", tmp_path, nx, ny, nz, 2, -1.0, *b)
    np.testing.assert_array_equal(get(tmp_path, "out.raw", src.shape), ob.warp_box32(vel, src, -1.0, b))


def test_dropin_flow_level_equals_oracle(cuda, dropin, tmp_path):
    rng = np.random.default_rng(22)
    shape = (12, 14, 16)
    i1 = ob.blur32(rng.uniform(0, 1, shape).astype(np.float32), 1.2)
    i2 = ob.blur32(rng.uniform(0, 1, shape).astype(np.float32), 1.2)
    v0 = (rng.normal(size=(3,) + shape) * 0.3).astype(np.float32)
    y0 = (rng.normal(size=(10,) + shape) * 0.05).astype(np.float32)
    for name, a in (("I1.raw", i1), ("I2.raw", i2), ("V.raw", v0), ("Y.raw", y0)):
        put(tmp_path, name, a)
    roi, box = (2, 1, 1, 2, 1, 1), (20.0, 14.0, 15.0)
    run(dropin, "flowlevel", tmp_path, 16, 14, 12, *box, *roi, 0.0, 1.2, 45, 4, 2, 1.0)
    vo, yo, _ = ob.flow_level32(i1, i2, v0, y0, roi, box=box, tol=0.0, lam=1.2, max_iter=45, n_warps=2)
    np.testing.assert_array_equal(get(tmp_path, "V_out.raw", v0.shape), vo)
    np.testing.assert_array_equal(get(tmp_path, "Y_out.raw", y0.shape), yo)


def test_dropin_flow_multiscale_equals_oracle(cuda, dropin, tmp_path):
    rng = np.random.default_rng(23)
    shape = (24, 26, 28)
    i1 = ob.blur32(rng.uniform(0, 1, shape).astype(np.float32), 2.0)
    i2 = ob.blur32(rng.uniform(0, 1, shape).astype(np.float32), 2.0)
    v0 = (rng.normal(size=(3,) + shape) * 0.2).astype(np.float32)
    for name, a in (("I1.raw", i1), ("I2.raw", i2), ("V.raw", v0)):
        put(tmp_path, name, a)
    cut = (3, 2, 2, 4, 1, 3)
    run(dropin, "flowms", tmp_path, 28, 26, 24, *cut, 0.0, 1.2, 30, 4, 2, 0.65, 0.5, 3, 1.0)
    ref = ob.flow_multiscale32(i1, i2, v0, cut, tol=0.0, max_iter=30, n_warps=2, eta=0.65, sigma=0.5, scales=3)
    np.testing.assert_array_equal(get(tmp_path, "V_out.raw", v0.shape), ref)


G = np.load(Path(__file__).resolve().parent / "golden" / "reference_golden.npz")


@pytest.mark.parametrize("v", [0, 1, 2])
def test_dropin_projector_from_scene_matrices(cuda, dropin, tmp_path, v):
    """The view is handed over as the reference hands it: the scene's view and
    projection matrices, here the ones the reference itself composed for the
    fixture views (an off-centre scan with 1.1 mm voxels).  The image is
    compared with the reference's own image of the same volume."""
    scan = ob.Scan((20, 18, 16), (24, 20), spacing=1.1, off=(0.5, -0.3, 0.8))
    nz, ny, nx = 16, 18, 20
    vol = G["fp_vol"]
    mats = G["fp_mats"][v].reshape(-1, 16)
    put(tmp_path, "vol.raw", vol)
    put(tmp_path, "view.raw", mats[4])
    put(tmp_path, "proj.raw", mats[5])
    corr = np.random.default_rng(24 + v).normal(size=(20, 24)).astype(np.float32)
    put(tmp_path, "corr.raw", corr)
    run(dropin, "project", tmp_path, nx, ny, nz, 1.1, 1.1, 1.1, 24, 20)
    sd, k = G["fp_views"][v]
    view = ob.view_round(float(sd), int(k))
    angle = float(get(tmp_path, "angle.raw", (1,))[0])
    assert abs(math.remainder(angle - view.angle, 2 * math.pi)) < 1e-5
    img = get(tmp_path, "img.raw", (20, 24))
    assert ob.rel_l2(img, G["fp_img"][v]) < 1e-4
    hit = G["fp_raylen"][v] > 0
    np.testing.assert_allclose(get(tmp_path, "rl.raw", (20, 24))[hit], G["fp_raylen"][v][hit], atol=2e-3)
    assert np.abs(get(tmp_path, "wt.raw", (20, 24)) - G["fp_weight"][v]).max() <= 1.0
    c, w = ob.bp_ray_scatter32(scan, view, corr, gmode=1)
    assert ob.rel_l2(get(tmp_path, "contrib.raw", vol.shape), c) < 1e-4
    assert ob.rel_l2(get(tmp_path, "wsum.raw", vol.shape), w) < 1e-4


def _write_tiff(path, a):
    import ctypes as C

    lib = C.CDLL(str(PKG / "libstt_facade.so"))
    lib.stt_tiff_write.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
    a = np.ascontiguousarray(a, np.float32)
    assert lib.stt_tiff_write(str(path).encode(), a.shape[-1], a.shape[-2], int(np.prod(a.shape[:-2])),
                              a.ctypes.data_as(C.c_void_p)) == 0


def _read_tiff(path):
    import ctypes as C

    lib = C.CDLL(str(PKG / "libstt_facade.so"))
    lib.stt_tiff_read.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                  C.POINTER(C.POINTER(C.c_float))]
    w, h, d = C.c_int(), C.c_int(), C.c_int()
    p = C.POINTER(C.c_float)()
    assert lib.stt_tiff_read(str(path).encode(), C.byref(w), C.byref(h), C.byref(d), C.byref(p)) == 0
    out = np.ctypeslib.as_array(p, shape=(d.value, h.value, w.value)).copy()
    lib.stt_host_free(C.cast(p, C.c_void_p))
    return out


def test_cli_end_to_end_matches_the_c_abi_pipeline(cuda, tmp_path):
    """ST-Tomography on a 2-frame 64^3 scan (10 views each): the files it
    writes, and its volumes against the same joint loop driven through the
    Python side of the C ABI (Flow + Solver with the same parameters)."""
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph

    n, det, F, V = 64, 112, 2, 10
    dims = (n, n, n)
    starts = [5.0, 23.0]
    (tmp_path / "lds.txt").write_text("\n".join(str(s) for s in starts) + "\n")
    ang = np.concatenate([stt.views_from_rounds([s], 10) for s in starts])
    ctx = stt.Context(0)
    ctx.set_geometry(dims, (1.0, 1.0, 1.0), (det, det), 1.0, 600.0, 1000.0, ang)
    params = ph.ellipsoid_params(8, dims, seed=5, semi=(4.0, 14.0))
    proj = torch.zeros((F, V, det, det), device=cuda)
    for f in range(F):
        truth = ph.rasterize(ph.displaced_params(params, f, 4, 2.0, 2 * math.pi / n, 0.3), dims, cuda)
        ctx.fp(truth, proj[f], view0=f * V, nviews=V)
    torch.cuda.synchronize()
    pj = proj.cpu().numpy()
    _write_tiff(tmp_path / "proj.tif", pj.reshape(F * V, det, det))
    (tmp_path / "Input").mkdir()
    for f in range(F):
        _write_tiff(tmp_path / "Input" / f"rose.-{f:03d}-frame-9iter.tiff", np.zeros(dims, np.float32))
    args = [str(CLI), "-i", "proj.tif", "-f", str(n), "-f", str(n), "-f", str(n), "-u", str(det), "-u", str(det),
            "-v", str(F), "-r", "1", "-g", "600", "-j", "1000", "-a", "0.3", "-l", "0.01", "-k", "0.1", "-e", "0.05",
            "--huber", "0.01", "--joint-iters", "3", "--pd-passes", "2", "--flow-iters", "30", "--seed", "7",
            "-o", "out/test"]
    r = subprocess.run(args, cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    for f in range(F):
        for it in range(1, 5):
            assert (tmp_path / "out" / f"test-{f:03d}-frame-{it}iter.tiff").exists()
    for it in range(3):
        base = tmp_path / "FlowOutput" / f"064.064.064.frame00.iter{it:02d}"
        assert Path(str(base) + ".tiff").exists() and Path(str(base) + ".field.hdr").exists()
    cli_vol = [_read_tiff(tmp_path / "out" / f"test-{f:03d}-frame-4iter.tiff") for f in range(F)]

    # the same loop through the C ABI (ST_Tomography::Render, ST_Tomography.cpp:398-611)
    hf = float(np.float32(1) / (np.float32(1) + np.float32(0.9) / np.float32(8) * np.float32(0.01) / np.float32(0.01)))
    gmax = float(np.float32(pj[0].max()) / np.float32(4))
    pd = stt.PdParams(sigma=float(np.float32(0.9) / np.float32(8)), tau=1.0, tv_w=0.01, tp_w=0.1, bc_w=0.05,
                      huber_factor=hf, gmax=gmax)
    st = dict(vol=torch.zeros((F + 1,) + dims, device=cuda), xbar=torch.zeros((F + 1,) + dims, device=cuda),
              xprev=torch.zeros((F,) + dims, device=cuda), ytv=torch.zeros((F, 3) + dims, device=cuda),
              ytp=torch.zeros((F,) + dims, device=cuda), ybc=torch.zeros((F,) + dims, device=cuda),
              flow=torch.zeros((F, 3) + dims, device=cuda), proj=proj)
    solver = stt.Solver(ctx, st, F, V, pd, alpha=0.3, bp_mode=0, seed=7, mode=stt.SOLVE_GRAPH)
    flow = stt.Flow(dims, stt.FlowParams(max_iter=30))
    for out_iter in range(3):
        flow.multiscale(st["vol"][0], st["vol"][1], st["flow"][0])
        torch.cuda.synchronize()
        if out_iter == 0:
            continue
        for p in range(2):
            if out_iter == 1 and p == 0:
                st["xbar"].copy_(st["vol"])
            torch.cuda.synchronize()
            solver.iterate(1)
    torch.cuda.synchronize()
    for f in range(F):
        mine = st["vol"][f].cpu().numpy()
        assert np.abs(mine).max() > 0
        np.testing.assert_allclose(cli_vol[f], mine, rtol=1e-5, atol=1e-6)
    solver.close()
    flow.close()
