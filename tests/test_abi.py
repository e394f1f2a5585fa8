"""The C ABI: libstt.so loads, exports every entry point of include/stt.h, and
its host-only helpers and argument checks behave (no GPU needed)."""
import ctypes as C
import math
import re
from pathlib import Path

import numpy as np
import pytest

import oracle_bind as ob

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def lib():
    from spacetimetomography_b200 import build

    build.build_libstt()
    from spacetimetomography_b200._lib import lib as L

    return L


def declared_symbols():
    """Entry points of include/stt.h, the C ABI of libstt.so (include/stt_host.h
    is libstt_facade.so's, checked in test_facade_io.py)."""
    names = set()
    for h in [ROOT / "include" / "stt.h"]:
        text = h.read_text()
        names |= set(re.findall(r"^\s*(?:stt_status|const char \*|void|int)\s*\*?\s*(stt_\w+)\s*\(", text, re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("stt_create", "stt_fp", "stt_fp_vjp", "stt_bp_voxel", "stt_bp_ray", "stt_sart_sweep",
                 "stt_pd_dual", "stt_pd_primal", "stt_warp", "stt_warp_vjp"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, f"libstt.so lacks {missing}"


def test_views_from_rounds_matches_reference_composition(lib):
    from spacetimetomography_b200 import views_from_rounds

    starts = [0.0, 17.3, 200.5]
    ang = views_from_rounds(starts, 10)
    assert ang.shape == (30,)
    for r, s in enumerate(starts):
        for k in range(10):
            v = ob.view_round(s, k)
            # the reference composes float quaternions; the FP64 angle is the exact sum
            assert abs(ang[r * 10 + k] - v.angle) < 1e-12
            half = ang[r * 10 + k] / 2
            assert abs(math.cos(half) - v.quat[3]) < 2e-6 and abs(math.sin(half) - v.quat[1]) < 2e-6


def test_permutation_matches_oracle(lib):
    from spacetimetomography_b200 import permutation

    for seed, n in [(0, 1), (1, 10), (1234, 360), (2**63 + 5, 97)]:
        p = permutation(seed, n)
        np.testing.assert_array_equal(p, ob.permutation(seed, n))
        assert sorted(p.tolist()) == list(range(n))


def test_lds_angles_known_values(lib):
    from spacetimetomography_b200 import lds_angles

    # van der Corput base 2: 0, 1/2, 1/4, 3/4, 1/8 -> scaled to one 36-degree segment
    a = lds_angles(50, segments=10, base=2)
    starts = a[::10]
    np.testing.assert_allclose(starts, [0.0, 18.0, 9.0, 27.0, 4.5])
    np.testing.assert_allclose(a[:10], np.arange(10) * 36.0)
    z = lds_angles(25, segments=10, base=2, zero_every=10)
    # the reference angle is inserted only when the length is a multiple of Nz
    # at the top of an outer iteration (Low_discrepency_squence.m:44-46)
    assert z[10] == 0.0 and z[11] == 18.0 and z[21] == 9.0


def test_argument_errors_without_gpu(lib):
    from spacetimetomography_b200._lib import Geometry

    assert lib.stt_fp(None, None, None, None, None, 0, 1, None) != 0
    assert lib.stt_set_geometry(None, None) != 0
    assert lib.stt_views_from_rounds(-1, None, 10, 36.0, None) == 1
    assert lib.stt_warp(None, None, None, 1, 1.0, None, None) == 1
    msg = lib.stt_last_error(None)
    assert msg and b"null" in msg
    assert lib.stt_version().startswith(b"stt ")
    assert C.sizeof(Geometry) == 112  # LP64 layout of stt_geometry


def test_flow_argument_checks_without_gpu(lib):
    """stt_flow_create validates its arguments before touching the device."""
    from spacetimetomography_b200._lib import FlowParams

    h = C.c_void_p()
    dims = (C.c_int * 3)(32, 32, 32)
    bad = [FlowParams(0.1, 1.2, 1.0, 0.65, 0.5, 3000, 4, 3, 0, (C.c_int * 6)(*[0] * 6)),     # scales 0
           FlowParams(0.1, 0.0, 1.0, 0.65, 0.5, 3000, 4, 3, 3, (C.c_int * 6)(*[0] * 6)),     # lambda 0
           FlowParams(0.1, 1.2, 1.0, 1.5, 0.5, 3000, 4, 3, 3, (C.c_int * 6)(*[0] * 6)),      # eta > 1
           FlowParams(0.1, 1.2, 1.0, 0.65, 0.5, 3000, 4, 3, 3, (C.c_int * 6)(-1, 0, 0, 0, 0, 0)),  # cut < 0
           FlowParams(0.1, 1.2, 1.0, 0.2, 0.5, 3000, 4, 3, 4, (C.c_int * 6)(*[0] * 6))]      # level < 3 voxels
    for p in bad:
        assert lib.stt_flow_create(0, dims, C.byref(p), C.byref(h)) == 1
        assert h.value is None
        assert lib.stt_last_error(None)
    assert lib.stt_flow_create(0, (C.c_int * 3)(2, 32, 32), C.byref(FlowParams(
        0.1, 1.2, 1.0, 0.65, 0.5, 30, 4, 3, 1, (C.c_int * 6)(*[0] * 6))), C.byref(h)) == 1


def test_tuning_variant_names_and_struct_layout(lib):
    """stt_tuning_variant_name names every variant of the five tuned kernels
    and returns NULL past them; the ctypes stt_tuning matches the header's
    layout (the host reads the tuner's report through it)."""
    from spacetimetomography_b200._lib import SolveCfg, Instance, Tuning

    # gather projector, slab projector, voxel BP, ray-BP scatter, BF16 gather projector
    counts = {0: 12, 1: 8, 2: 5, 3: 2, 4: 2}
    for kernel, n in counts.items():
        names = [lib.stt_tuning_variant_name(kernel, v) for v in range(n)]
        assert all(names) and len(set(names)) == n, (kernel, names)
        assert lib.stt_tuning_variant_name(kernel, n) is None
        assert lib.stt_tuning_variant_name(kernel, -1) is None
    assert lib.stt_tuning_variant_name(5, 0) is None
    # int fp, slab, bp; unsigned bins; int tuned, from_cache; float fp_us[12], slab_us[8], bp_us[8];
    # int ray_variant; float ray_us[2]; unsigned staged_bins_bf16; int fp_variant_bf16; float fp16_us[2]
    assert C.sizeof(Tuning) == 6 * 4 + (12 + 8 + 8) * 4 + 4 + 2 * 4 + 4 + 4 + 2 * 4
    assert Tuning.ray_variant.offset == 6 * 4 + 28 * 4
    assert SolveCfg.storage.offset > SolveCfg.autotune.offset and Instance.storage.offset > Instance.autotune.offset


def test_typed_entry_points_reject_bad_dtypes_without_gpu(lib):
    """The BF16-storage entry points check their dtype before touching the device."""
    assert lib.stt_warp_typed(None, None, None, 7, 1, 1.0, None, None) == 1
    assert lib.stt_sart_sweep_typed(None, None, 7, None, None, 0, 0, 0.3, 1.0, 0, None, None, None) != 0
    assert lib.stt_bp_voxel_typed(None, None, None, 7, 0.3, 1.0, 0, None) != 0
    assert lib.stt_bp_ray_typed(None, None, None, 7, 1.0, 0, None) != 0


def test_solver_modes_and_persistent_info_without_gpu(lib):
    """The solver modes of stt_solve_mode as the Python side numbers them, and
    the persistent form's report refusing a null solver (no device touched)."""
    import spacetimetomography_b200 as stt

    text = (ROOT / "include" / "stt.h").read_text()
    for name, value in (("PLAIN", stt.SOLVE_PLAIN), ("STREAMS", stt.SOLVE_STREAMS), ("GRAPH", stt.SOLVE_GRAPH),
                        ("PERSISTENT", stt.SOLVE_PERSISTENT)):
        assert re.search(rf"STT_SOLVE_{name}\s*=\s*{value}\b", text), name
    b, g = C.c_int(7), C.c_int(7)
    assert lib.stt_solver_persistent_info(None, C.byref(b), C.byref(g)) == 1  # STT_ERR_INVALID
    assert lib.stt_solver_stats(None, None, None) == 1
