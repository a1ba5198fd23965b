"""Checkpoint files and the restart set-up, on the CPU.

The reference writes checkpoints with the HDF5 library (src/IO/io_hdf5.c);
the library writes them without one.  The pins:
  - a file written by the HDF5 library itself (scipy's MATLAB 7.3 test file,
    an HDF5 file behind a 512-byte user block) read by the library's C
    reader and by an independent Python walk of the format (hdf5_walk.py);
  - the library's files walked by that second reader: every structure at the
    version the HDF5 library writes by default;
  - the restart state against the reference's own restart branch
    (tests/golden/ckpt_*.npz, make_golden.py --checkpoint).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from disco2_b200 import lib
from hdf5_walk import H5

SCIPY_H5 = None
try:
    import scipy.io.matlab as _m

    _p = os.path.join(os.path.dirname(_m.__file__), "tests", "data", "testhdf5_7.4_GLNX86.mat")
    SCIPY_H5 = _p if os.path.exists(_p) else None
except ImportError:
    pass

needs_scipy_file = pytest.mark.skipif(SCIPY_H5 is None, reason="scipy's HDF5 test file is not installed")
CASES = ("gresho16", "kepler24", "cbd32", "torus3d16", "vortex16dye")


def ckpt(name):
    with np.load(os.path.join(GOLDEN, f"ckpt_{name}.npz")) as z:
        return {k: z[k] for k in z.files}


@needs_scipy_file
def test_reads_a_file_the_hdf5_library_wrote():
    want = np.linspace(0.0, 2 * np.pi, 9)
    got = lib.hdf5_dataset(SCIPY_H5, "testdouble")
    assert got.shape == (9, 1)
    assert np.array_equal(got.ravel(), want)
    # the independent walk agrees, and sees the library's own structures
    f = H5(SCIPY_H5)
    assert f.sb_off == 512 and f.base == 512 and f.sb_version == 0
    data, h = f.dataset("testdouble")
    assert np.array_equal(data.ravel(), want)
    types = [t for t, _, _ in h["messages"]]
    assert {1, 3, 8} <= set(types)


def test_written_file_structure(tmp_path):
    path = str(tmp_path / "ck.h5")
    rng = np.random.default_rng(7)
    data = rng.standard_normal((37, 8))
    gm = rng.standard_normal((2, 4))
    lib.hdf5_out(path, 0.125, gm, data)
    f = H5(path)
    # superblock 0 at byte 0, 8-byte offsets and lengths, K 4 / 16, no base
    # offset, the end-of-file address equal to the file's size
    assert f.sb_off == 0 and f.sb_version == 0 and f.base == 0
    assert (f.leaf_k, f.internal_k, f.flags) == (4, 16, 0)
    assert f.eof == os.path.getsize(path)
    assert f.freespace == 0xFFFFFFFFFFFFFFFF and f.driver == 0xFFFFFFFFFFFFFFFF
    # root entry: cache type 1, scratch pad = the symbol table message's
    assert f.root_cache == 1 and f.root_scratch == (f.btree, f.heap_addr)
    assert f.name(f.root_name_off) == ""
    # one symbol-table node, names sorted, B-tree keys bracket them
    assert len(f.snods) == 1
    assert f.snods[0]["names"] == ["Data", "GravMass", "T"]
    assert f.snods[0]["keys"] == ["", "T"]
    assert f.heap["free"] == 1  # no free block
    want = {"T": (np.array([0.125]), 1), "GravMass": (gm, 2), "Data": (data, 2)}
    for name, (w, rank) in want.items():
        got, h = f.dataset(name)
        assert np.array_equal(got, w), name
        # dataspace v1, datatype v1 (class 1, 8 bytes), fill value v2, layout v3
        versions = {t: body[0] for t, _, body in h["messages"]}
        assert versions == {1: 1, 3: 0x11, 5: 2, 8: 3}, name
        assert h["nmsg"] == len(h["messages"]) == 4
        assert h["size"] == sum(8 + len(b) for _, _, b in h["messages"])
        sp = [b for t, _, b in h["messages"] if t == 1][0]
        assert sp[1] == rank


def test_round_trip_is_bit_exact(tmp_path):
    path = str(tmp_path / "ck.h5")
    data = np.random.default_rng(3).standard_normal((101, 9))
    specials = [np.nan, -0.0, np.inf, -np.inf, 5e-324, np.finfo(float).max]
    data.ravel()[:len(specials)] = specials
    gm = np.arange(8.0).reshape(2, 4) - 3.5
    lib.hdf5_out(path, -2.5, gm, data)
    r = lib.hdf5_in(path)
    assert r["t"] == -2.5
    assert np.array_equal(r["gravmass"], gm)
    assert np.array_equal(r["data"].view(np.uint64), data.view(np.uint64))
    # hyperslabs of rows, as io_hdf5_in reads at sim_offset on each rank
    for row0, n in ((0, 101), (17, 40), (100, 1), (101, 0)):
        assert np.array_equal(lib.hdf5_in(path, row0, n)["data"].view(np.uint64),
                              data[row0:row0 + n].view(np.uint64))


def test_empty_and_single_row(tmp_path):
    for rows in (0, 1):
        path = str(tmp_path / f"ck{rows}.h5")
        data = np.ones((rows, 8))
        lib.hdf5_out(path, 1.0, np.zeros((2, 4)), data)
        r = lib.hdf5_in(path)
        assert r["data"].shape == (rows, 8)
        assert H5(path).dataset("Data")[0].shape == (rows, 8)


def test_errors(tmp_path):
    path = str(tmp_path / "ck.h5")
    lib.hdf5_out(path, 1.0, np.zeros((2, 4)), np.ones((10, 8)))
    with pytest.raises(lib.DiscoError, match="IO"):
        lib.hdf5_in(str(tmp_path / "missing.h5"))
    with pytest.raises(lib.DiscoError, match="outside"):
        lib.hdf5_in(path, 5, 6)
    # a column count other than the file's
    L = lib.load()
    buf = np.zeros((10, 7))
    assert L.dgpu_hdf5_in(path.encode(), 0, 10, 7, None, None, lib._dptr(buf)) == -8
    # not HDF5, truncated, no such dataset
    bad = tmp_path / "bad.h5"
    bad.write_bytes(b"not an hdf5 file" * 64)
    with pytest.raises(lib.DiscoError, match="superblock"):
        lib.hdf5_in(str(bad))
    raw = open(path, "rb").read()
    trunc = tmp_path / "trunc.h5"
    trunc.write_bytes(raw[:len(raw) - 100])
    with pytest.raises(lib.DiscoError):
        lib.hdf5_in(str(trunc))
    with pytest.raises(lib.DiscoError, match="no dataset"):
        lib.hdf5_dataset(path, "Nope")
    with pytest.raises(lib.DiscoError, match="ARG"):
        lib.hdf5_out(path, 1.0, np.zeros((2, 4)), np.ones((3, 0)))


@pytest.mark.parametrize("name", CASES)
def test_restart_state_matches_the_reference_restart(name, tmp_path):
    """dgpu_sim_restart_state against the reference's restart branch
    (main.c:95-117, io_readbuf) from the same 5-step checkpoint buffer:
    prim, tiph, dphi, the GravMasses and t, bit for bit."""
    g = ckpt(name)
    path = str(tmp_path / "input.h5")
    lib.hdf5_out(path, float(g["ck5_t"]), g["ck5_gm"], g["ck5_data"])
    sim = lib.Sim(str(g["parfile"]))
    rs = sim.restart_state(path)
    assert rs["t"] == g["rs_t"]
    for k in ("prim", "tiph", "dphi"):
        assert np.array_equal(rs[k], g["rs_" + k]), k
    assert np.array_equal(rs["gm"][:, :4], g["rs_gm"][:, :4])
    assert np.all(rs["gm"][:, 4:] == 0.0)


def test_restart_state_refuses_another_grid(tmp_path):
    g = ckpt("kepler24")
    path = str(tmp_path / "input.h5")
    lib.hdf5_out(path, 0.0, g["ck5_gm"], g["ck5_data"][:-1])
    with pytest.raises(lib.DiscoError, match="IO"):
        lib.Sim(str(g["parfile"])).restart_state(path)


# ---------------------------------------------------------------------------
# The reader's wider formats, on a file laid out here by hand from the format
# specification: a 512-byte user block, superblock version 1, a root group
# whose B-tree has an internal node over two leaves (two symbol-table nodes),
# a NIL message in the root header, a dataset header split by a continuation
# message, layout versions 1 (contiguous) and 3 (compact), dataspace
# version 2.
# ---------------------------------------------------------------------------
def _crafted(path):
    import struct

    UB, UND = 512, 0xFFFFFFFFFFFFFFFF
    buf = bytearray(8192)

    def put(at, fmt, *v):
        struct.pack_into("<" + fmt, buf, UB + at, *v)

    def msg(at, typ, body, flags=0):
        body = body + b"\0" * (-len(body) % 8)
        put(at, "HHB3x", typ, len(body), flags)
        buf[UB + at + 8:UB + at + 8 + len(body)] = body
        return at + 8 + len(body)

    def header(at, msgs, size):
        put(at, "BxHII4x", 1, len(msgs), 1, size)
        m = at + 16
        for typ, body in msgs:
            m = msg(m, typ, body)
        assert m - at - 16 <= size

    f64 = bytes([0x11, 0x20, 63, 0]) + struct.pack("<IHHBBBBI", 8, 0, 64, 52, 11, 0, 52, 1023)
    a_vals = np.arange(6.0).reshape(3, 2) + 0.5
    b_vals = np.array([2.0, -3.0, 4.25])
    c_vals = np.array([[7.0, 8.0]])
    # names in the local heap
    names = {"": 0, "A": 8, "B": 16, "C": 24}
    heap, heap_data = 200, 240
    put(heap, "4sB3xQQQ", b"HEAP", 0, 32, 1, heap_data)
    for nm, off in names.items():
        raw = nm.encode() + b"\0"
        buf[UB + heap_data + off:UB + heap_data + off + len(raw)] = raw
    # B-tree: an internal node (level 1) over two leaves, each with one SNOD
    root_bt, leaf1, leaf2, snod1, snod2 = 300, 900, 1500, 2100, 2500
    put(root_bt, "4sBBHQQ", b"TREE", 0, 1, 2, UND, UND)
    put(root_bt + 24, "QQQQQ", 0, leaf1, names["B"], leaf2, names["C"])
    put(leaf1, "4sBBHQQ", b"TREE", 0, 0, 1, UND, leaf2)
    put(leaf1 + 24, "QQQ", 0, snod1, names["B"])
    put(leaf2, "4sBBHQQ", b"TREE", 0, 0, 1, leaf1, UND)
    put(leaf2 + 24, "QQQ", names["B"], snod2, names["C"])
    oh_a, oh_b, oh_b2, oh_c = 3000, 3300, 3600, 3900
    put(snod1, "4sBxH", b"SNOD", 1, 2)
    put(snod1 + 8, "QQI4x16x", names["A"], oh_a, 0)
    put(snod1 + 48, "QQI4x16x", names["B"], oh_b, 0)
    put(snod2, "4sBxH", b"SNOD", 1, 1)
    put(snod2 + 8, "QQI4x16x", names["C"], oh_c, 0)
    # root group header: a NIL message, then the symbol table message
    root = 100
    header(root, [(0x0000, b"\0" * 8), (0x0011, struct.pack("<QQ", root_bt, heap))], 48)
    # A: dataspace v1 (3 x 2), datatype, layout v1 contiguous
    a_data = 4200
    header(oh_a, [(0x0001, struct.pack("<BBBx4xQQ", 1, 2, 0, 3, 2)), (0x0003, f64),
                  (0x0008, struct.pack("<BBB5xQIII", 1, 3, 1, a_data, 3, 2, 8))], 120)
    buf[UB + a_data:UB + a_data + 48] = a_vals.astype("<f8").tobytes()
    # B: dataspace in the first block, then a continuation to a second block
    # holding the datatype and a layout v3 contiguous
    b_data = 4300
    header(oh_b, [(0x0001, struct.pack("<BBBx4xQ", 1, 1, 0, 3)), (0x0010, struct.pack("<QQ", oh_b2, 64))], 48)
    m = msg(oh_b2, 0x0003, f64)
    msg(m, 0x0008, struct.pack("<BBQQ", 3, 1, b_data, 24))
    put(oh_b, "BxHII4x", 1, 4, 1, 48)  # four messages over both blocks
    buf[UB + b_data:UB + b_data + 24] = b_vals.astype("<f8").tobytes()
    # C: dataspace v2, compact layout v3 holding the values
    header(oh_c, [(0x0001, struct.pack("<BBBBQQ", 2, 2, 0, 1, 1, 2)), (0x0003, f64),
                  (0x0008, struct.pack("<BBH", 3, 0, 16) + c_vals.astype("<f8").tobytes())], 96)
    eof = 4400
    # superblock version 1 at the end of the user block, base address 512
    sb = b"\x89HDF\r\n\x1a\n" + struct.pack("<BBBBBBBBHHIHH", 1, 0, 0, 0, 0, 8, 8, 0, 4, 16, 0, 32, 0)
    sb += struct.pack("<QQQQ", UB, UND, eof, UND)
    sb += struct.pack("<QQI4x16x", 0, root, 0)
    buf[UB:UB + len(sb)] = sb
    buf[:16] = b"user block here\0"
    with open(path, "wb") as f:
        f.write(bytes(buf[:UB + eof]))
    return {"A": a_vals, "B": b_vals, "C": c_vals}


def test_reader_formats_beyond_the_writer(tmp_path):
    path = str(tmp_path / "crafted.h5")
    want = _crafted(path)
    for name, w in want.items():
        got = lib.hdf5_dataset(path, name)
        assert np.array_equal(got.reshape(w.shape), w), name
    # the independent walk reads the contiguous ones the same way
    f = H5(path)
    assert f.sb_version == 1 and f.base == 512 and len(f.snods) == 2
    assert np.array_equal(f.dataset("A")[0], want["A"])
    assert np.array_equal(f.dataset("B")[0], want["B"])


def test_corrupted_files_are_errors_not_crashes(tmp_path):
    """Seeded byte corruptions and truncations of a checkpoint: each read
    either succeeds or raises DiscoError; the reading process never crashes
    (run in a child process, so a fault would show as its exit status)."""
    import random
    import subprocess
    import sys

    good = str(tmp_path / "ck.h5")
    lib.hdf5_out(good, 1.0, np.zeros((2, 4)), np.arange(80.0).reshape(10, 8))
    raw = open(good, "rb").read()
    rng = random.Random(20251204)
    files = []
    for k in range(200):
        b = bytearray(raw)
        for _ in range(rng.randint(1, 8)):
            b[rng.randrange(len(b))] = rng.randrange(256)
        if rng.random() < 0.2:
            b = b[:rng.randrange(len(b))]
        q = tmp_path / f"c{k}.h5"
        q.write_bytes(bytes(b))
        files.append(str(q))
    code = ("import sys\nsys.path.insert(0, sys.argv[1])\nfrom disco2_b200 import lib\n"
            "for f in sys.argv[2:]:\n    try:\n        lib.hdf5_in(f)\n    except lib.DiscoError:\n        pass\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code, root] + files, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
