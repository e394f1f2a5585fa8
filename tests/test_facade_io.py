"""The C++ drop-in layer without a GPU: libstt_facade.so loads and exports
include/stt_host.h; the TIFF and Analyze codec reads files written here by an
independent writer (struct-packed TIFF 6.0 in either byte order, several
strips, integer and float samples) and round-trips its own output; the
ST-Tomography command line parses the reference's options."""
import ctypes as C
import re
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "spacetimetomography_b200"
FACADE = PKG / "libstt_facade.so"
CLI = PKG / "bin" / "st_tomography"


@pytest.fixture(scope="module")
def fl():
    import importlib.util

    spec = importlib.util.spec_from_file_location("stt_build", PKG / "build.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    b.build_all()
    lib = C.CDLL(str(FACADE))
    vp, i = C.c_void_p, C.c_int
    lib.stt_tiff_read.argtypes = [C.c_char_p, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(C.POINTER(C.c_float))]
    lib.stt_tiff_write.argtypes = [C.c_char_p, i, i, i, vp]
    lib.stt_analyze_write.argtypes = [C.c_char_p, i, i, i, i, vp]
    lib.stt_analyze_read.argtypes = [C.c_char_p, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i),
                                     C.POINTER(C.POINTER(C.c_float))]
    lib.stt_host_free.argtypes = [vp]
    lib.stt_host_last_error.restype = C.c_char_p
    return lib


def read_tiff(lib, path):
    w, h, d = C.c_int(), C.c_int(), C.c_int()
    p = C.POINTER(C.c_float)()
    rc = lib.stt_tiff_read(str(path).encode(), C.byref(w), C.byref(h), C.byref(d), C.byref(p))
    if rc != 0:
        raise RuntimeError(lib.stt_host_last_error().decode())
    out = np.ctypeslib.as_array(p, shape=(d.value, h.value, w.value)).copy()
    lib.stt_host_free(C.cast(p, C.c_void_p))
    return out


def tiff_bytes(pages, dtype, big_endian=False, rows_per_strip=None):
    """An uncompressed TIFF 6.0 file, one page per array, written from the spec."""
    e = ">" if big_endian else "<"
    dt = np.dtype(dtype).newbyteorder(e)
    fmt = {"f": 3, "i": 2, "u": 1}[dt.kind]
    out = bytearray(b"MM\x00\x2a" if big_endian else b"II\x2a\x00")
    out += struct.pack(e + "I", 8)
    for k, a in enumerate(pages):
        h, w = a.shape
        rps = rows_per_strip or h
        strips = [a[r:r + rps] for r in range(0, h, rps)]
        nent = 11
        ifd_at = len(out)
        data_at = ifd_at + 2 + 12 * nent + 4 + 8 * len(strips)
        offs, counts, at = [], [], data_at
        for s in strips:
            offs.append(at)
            counts.append(s.size * dt.itemsize)
            at += s.size * dt.itemsize
        table_at = ifd_at + 2 + 12 * nent + 4
        ents = [(256, 4, 1, w), (257, 4, 1, h), (258, 3, 1, dt.itemsize * 8), (259, 3, 1, 1), (262, 3, 1, 1),
                (273, 4, len(strips), offs[0] if len(strips) == 1 else table_at), (277, 3, 1, 1),
                (278, 4, 1, rps), (279, 4, len(strips), counts[0] if len(strips) == 1 else table_at + 4 * len(strips)),
                (284, 3, 1, 1), (339, 3, 1, fmt)]
        out += struct.pack(e + "H", nent)
        for tag, typ, cnt, val in ents:
            if typ == 3 and cnt == 1:
                out += struct.pack(e + "HHIHH", tag, typ, cnt, val, 0)
            else:
                out += struct.pack(e + "HHII", tag, typ, cnt, val)
        nxt = at if k + 1 < len(pages) else 0
        out += struct.pack(e + "I", nxt)
        out += struct.pack(e + "%dI" % len(strips), *offs) + struct.pack(e + "%dI" % len(strips), *counts)
        for s in strips:
            out += s.astype(dt).tobytes()
    return bytes(out)


@pytest.mark.parametrize("dtype,be,rps", [("<f4", False, None), (">f4", True, 3), ("<u2", False, 2), (">i2", True, 1),
                                          ("u1", False, 4), ("<f8", False, 5), ("<i4", False, None)])
def test_tiff_reader_reads_spec_written_files(fl, tmp_path, dtype, be, rps):
    rng = np.random.default_rng(3)
    d = np.dtype(dtype)
    if d.kind == "f":
        pages = [rng.normal(size=(7, 9)).astype(d) for _ in range(3)]
    else:
        info = np.iinfo(d)
        pages = [rng.integers(max(info.min, -1000), min(info.max, 1000), size=(7, 9)).astype(d) for _ in range(3)]
    path = tmp_path / "t.tif"
    path.write_bytes(tiff_bytes(pages, d, big_endian=be, rows_per_strip=rps))
    got = read_tiff(fl, path)
    np.testing.assert_array_equal(got, np.stack(pages).astype(np.float32))


def test_tiff_write_round_trip(fl, tmp_path):
    a = np.random.default_rng(4).normal(size=(5, 6, 7)).astype(np.float32)
    a[0, 0, 0] = np.nan
    a[1, 2, 3] = -np.inf
    path = tmp_path / "vol.tiff"
    assert fl.stt_tiff_write(str(path).encode(), 7, 6, 5, a.ctypes.data_as(C.c_void_p)) == 0
    got = read_tiff(fl, path)
    np.testing.assert_array_equal(got, a)
    raw = path.read_bytes()
    assert raw[:4] == b"II*\x00" and len(raw) > a.nbytes


def test_tiff_reader_rejects_bad_files(fl, tmp_path):
    p = tmp_path / "bad.tif"
    p.write_bytes(b"not a tiff at all")
    with pytest.raises(RuntimeError, match="not a TIFF"):
        read_tiff(fl, p)
    with pytest.raises(RuntimeError, match="cannot open"):
        read_tiff(fl, tmp_path / "missing.tif")
    good = tiff_bytes([np.zeros((4, 4), np.float32)], np.float32)
    p.write_bytes(good[:60])
    with pytest.raises(RuntimeError):
        read_tiff(fl, p)


def test_analyze_round_trip_and_header(fl, tmp_path):
    a = np.random.default_rng(5).normal(size=(3, 4, 5, 6)).astype(np.float32)  # c, z, y, x
    hdr = tmp_path / "flow.field.hdr"
    assert fl.stt_analyze_write(str(hdr).encode(), 6, 5, 4, 3, a.ctypes.data_as(C.c_void_p)) == 0
    raw = hdr.read_bytes()
    assert len(raw) == 348
    assert struct.unpack("<i", raw[:4])[0] == 348
    assert struct.unpack("<5h", raw[40:50]) == (4, 6, 5, 4, 3)
    assert struct.unpack("<hh", raw[70:74]) == (16, 32)
    np.testing.assert_array_equal(np.fromfile(tmp_path / "flow.field.img", np.float32).reshape(a.shape), a)
    w, h, d, c = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    p = C.POINTER(C.c_float)()
    assert fl.stt_analyze_read(str(hdr).encode(), C.byref(w), C.byref(h), C.byref(d), C.byref(c), C.byref(p)) == 0
    got = np.ctypeslib.as_array(p, shape=(c.value, d.value, h.value, w.value)).copy()
    fl.stt_host_free(C.cast(p, C.c_void_p))
    np.testing.assert_array_equal(got, a)


def test_facade_exports_every_host_symbol(fl):
    text = (ROOT / "include" / "stt_host.h").read_text()
    names = re.findall(r"^\s*(?:int|const char \*|void)\s*\*?\s*(stt_\w+)\s*\(", text, re.M)
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(fl, n)]
    assert not missing


def _cli(*args):
    return subprocess.run([str(CLI), *args], capture_output=True, text=True, timeout=60)


def test_cli_help_lists_the_reference_options(fl):
    r = _cli("--help")
    assert r.returncode == 0
    for opt in ("-s|--Sigma", "-t|--Tau", "-l|--Lambda", "-k|--TemporalPrior", "--huber", "-a|--Alpha", "-o <output>",
                "-i|--projsvolume", "-f|--XYZ", "-u|--imgUV", "-c|--voxelspacing", "-g|--sid", "-j|--sdd", "--oxyz",
                "--sdg", "-v|--nframes", "-r|--nrounds", "-b|--AlgorithmIter", "-p|--SartIter", "--prior", "--bp"):
        assert opt in r.stdout, opt


def test_cli_reports_argument_errors(fl):
    r = _cli("-f", "32")
    assert r.returncode == 1
    assert "missing option -i|--projsvolume" in r.stdout and "missing option -u|--imgUV" in r.stdout
    r = _cli("-i", "p.tif", "-f", "32", "-u", "48", "-s", "abc")
    assert r.returncode == 1 and 'invalid argument "abc"' in r.stdout
    r = _cli("-i", "p.tif", "-f", "32", "-f", "32", "-f", "32", "-f", "32", "-u", "48")
    assert r.returncode == 1 and "excess option -f|--XYZ" in r.stdout
    r = _cli("--nosuch")
    assert r.returncode == 1 and 'invalid option "--nosuch"' in r.stdout
    r = _cli("--version")
    assert r.returncode == 0 and "sm_100a" in r.stdout


def test_cli_fails_cleanly_on_missing_input(fl, tmp_path):
    """No GPU is needed to reach the missing-file error of ReadStructuredFile."""
    r = subprocess.run([str(CLI), "-i", "proj.tif", "-f", "32", "-u", "48", "--input-dir", str(tmp_path / "none")],
                       capture_output=True, text=True, timeout=60, cwd=tmp_path)
    assert r.returncode == 2
    assert "cannot open" in r.stderr or "cudaSetDevice" in r.stderr or "CUDA" in r.stderr
