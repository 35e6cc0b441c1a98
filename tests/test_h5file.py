"""The library's HDF5 container code (csrc/h5file.cpp) on the CPU: a fixed file written
through it parses under an independent reader written from the file format specification
(tests/h5spec.py, which asserts the structural rules a libhdf5 reader relies on), with
every value where it was put, and the library's own reader reads it back by path and
member name.  Groups hold up to 64 entries in one symbol-table node (12 here)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import h5spec

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "ch4-project_b200", "csrc")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    exe = str(tmp_path_factory.mktemp("h5") / "h5_driver")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", CSRC, os.path.join(HERE, "h5_driver.cpp"),
                    os.path.join(CSRC, "h5file.cpp"), "-o", exe], check=True)
    return exe


@pytest.fixture(scope="module")
def written(driver, tmp_path_factory):
    path = str(tmp_path_factory.mktemp("h5f") / "t.h5")
    subprocess.run([driver, "write", path], check=True)
    return path


def test_structure_and_values_under_the_spec_reader(written):
    got = h5spec.read(written)
    names = ["velocity_x", "velocity_y", "velocity_z", "density", "temperature", "scalar", "position_x",
             "position_y", "position_z", "extra_a", "extra_b", "extra_c"]
    for d, nm in enumerate(names):
        a = got["/euler/" + nm]
        assert a.shape == (3, 4, 5) and a.dtype == np.float64
        assert np.array_equal(a.ravel(), d * 1000.0 + np.arange(60) + 0.25), nm
    pop = got["/population/velocity"]
    assert pop.shape == (2, 3, 4) and pop.dtype.names == tuple("p%d" % q for q in range(19))
    flat = np.stack([pop["p%d" % q].ravel() for q in range(19)], axis=1).ravel()
    assert np.array_equal(flat, 0.5 * np.arange(19 * 24) - 7)
    assert got["/forcing@number of modes (nk)"].item() == 6
    phi = got["/forcing@phi_u"]
    assert phi.shape == (6,) and phi.dtype.names == ("x", "y", "z")
    assert np.array_equal(np.stack([phi["x"], phi["y"], phi["z"]], 1).ravel(), 0.1 * np.arange(18))


def test_library_reader_by_path_and_member(driver, written):
    out = subprocess.run([driver, "read", written, "/euler/extra_b"], check=True, capture_output=True, text=True)
    assert np.array_equal(np.array(out.stdout.split(), float), 10 * 1000.0 + np.arange(60) + 0.25)
    out = subprocess.run([driver, "read", written, "/population/velocity", "p3", "p18", "p0"], check=True,
                         capture_output=True, text=True)
    v = np.array(out.stdout.split(), float).reshape(24, 3)
    full = (0.5 * np.arange(19 * 24) - 7).reshape(24, 19)
    assert np.array_equal(v, full[:, [3, 18, 0]])
    out = subprocess.run([driver, "attrs", written, "/forcing"], check=True, capture_output=True, text=True)
    assert out.stdout.splitlines() == ["number of modes (nk) 4", "phi_u 144"]


def test_reader_refuses_what_it_cannot_read(driver, written, tmp_path):
    bad = subprocess.run([driver, "read", written, "/euler/nothing"], capture_output=True, text=True)
    assert bad.returncode != 0 and "no object named nothing" in bad.stderr
    bad = subprocess.run([driver, "read", written, "/population/velocity", "p19"], capture_output=True, text=True)
    assert bad.returncode != 0 and "no member p19" in bad.stderr
    junk = tmp_path / "junk.h5"
    junk.write_bytes(b"not an hdf5 file at all" * 40)
    bad = subprocess.run([driver, "read", str(junk), "/x"], capture_output=True, text=True)
    assert bad.returncode != 0 and "signature" in bad.stderr


def _libhdf5_style_file(path):
    """A file laid out the way libhdf5 writes with its default settings, in the forms the
    library's own writer never uses: symbol-table nodes of 8 entries (leaf K = 4) so one
    group spans two nodes under one B-tree, an object header split by a continuation
    message with a NIL message before it, fill-value and modification-time messages,
    dataspaces with maximum dimensions, and compounds with a float member after a double
    at non-packed offsets.  /population/d0 .. d9: 2 x 3 elements {p0: f8 at 0, p1: f4 at 8}
    of 16 bytes, element e of dataset d has p0 = 100 d + e and p1 = -(d + e / 4)."""
    import struct as S
    buf = bytearray(8192)
    U = 0xFFFFFFFFFFFFFFFF

    def put(at, b):
        buf[at:at + len(b)] = b

    def msg(t, body):
        body = body + b"\0" * (-len(body) % 8)
        return S.pack("<HHB3x", t, len(body), 0) + body

    def header(msgs, at, continued=0):
        # the message count includes the messages of continuation blocks
        body = b"".join(msgs)
        put(at, S.pack("<BBHII4x", 1, 0, len(msgs) + continued, 1, len(body)) + body)

    def fdt(size):
        if size == 8:
            return bytes([0x11, 0x20, 63, 0]) + S.pack("<IHHBBBBI", 8, 0, 64, 52, 11, 0, 52, 1023)
        return bytes([0x11, 0x20, 31, 0]) + S.pack("<IHHBBBBI", 4, 0, 32, 23, 8, 0, 23, 127)

    def member(name, off, t):
        n = name.encode() + b"\0"
        return n + b"\0" * (-len(n) % 8) + S.pack("<IB3xII16x", off, 0, 0, 0) + t

    names = ["d%d" % i for i in range(10)]
    heap_names = b"\0" * 8
    offs = []
    for n in names:
        offs.append(len(heap_names))
        heap_names += n.encode() + b"\0" * (8 - len(n))
    # addresses
    ROOT, ROOT_CONT, ROOT_BT, ROOT_SN, ROOT_HP = 96, 160, 200, 744, 1072
    GRP, GRP_BT, SN0, SN1, GRP_HP, DS0, DATA0 = 1136, 1200, 1744, 2072, 2400, 2528, 5248
    STRIDE = 272  # one dataset header
    # root group: NIL, then a continuation to the block holding the symbol-table message
    header([msg(0, b"\0" * 8), msg(0x10, S.pack("<QQ", ROOT_CONT, 24))], ROOT, continued=1)
    put(ROOT_CONT, msg(0x11, S.pack("<QQ", ROOT_BT, ROOT_HP)))
    put(ROOT_HP, b"HEAP" + bytes(4) + S.pack("<QQQ", 24, 1, ROOT_HP + 32) + b"\0" * 8 + b"population\0" + bytes(5))
    put(ROOT_BT, b"TREE" + bytes([0, 0]) + S.pack("<HQQQQQ", 1, U, U, 0, ROOT_SN, 8))
    put(ROOT_SN, b"SNOD" + bytes([1, 0]) + S.pack("<HQQII QQ".replace(" ", ""), 1, 8, GRP, 1, 0, GRP_BT, GRP_HP))
    # /population: two symbol-table nodes under one leaf B-tree node
    header([msg(0x11, S.pack("<QQ", GRP_BT, GRP_HP))], GRP)
    put(GRP_HP, b"HEAP" + bytes(4) + S.pack("<QQQ", len(heap_names), 1, GRP_HP + 32) + heap_names)
    put(GRP_BT, b"TREE" + bytes([0, 0]) + S.pack("<HQQ", 2, U, U) + S.pack("<QQQQQ", 0, SN0, offs[4], SN1, offs[9]))
    for sn, part in ((SN0, range(0, 5)), (SN1, range(5, 10))):
        ent = b"".join(S.pack("<QQII16x", offs[i], DS0 + STRIDE * i, 0, 0) for i in part)
        put(sn, b"SNOD" + bytes([1, 0]) + S.pack("<H", len(part)) + ent)
    ctype = bytes([0x16, 2, 0, 0]) + S.pack("<I", 16) + member("p0", 0, fdt(8)) + member("p1", 8, fdt(4))
    for d in range(10):
        space = S.pack("<BBBxI", 1, 2, 1, 0) + S.pack("<QQ", 2, 3) + S.pack("<QQ", 2, 3)
        hdr = [msg(1, space), msg(3, ctype), msg(5, bytes([2, 2, 0, 0])), msg(0x12, S.pack("<B3xI", 1, 0)),
               msg(8, S.pack("<BBQQ", 3, 1, DATA0 + 96 * d, 96))]
        body = b"".join(hdr)
        hb = S.pack("<BBHII4x", 1, 0, len(hdr), 1, len(body)) + body
        assert len(hb) <= STRIDE and DS0 + 10 * STRIDE <= DATA0
        put(DS0 + STRIDE * d, hb)
        for e in range(6):
            put(DATA0 + 96 * d + 16 * e, S.pack("<df4x", 100.0 * d + e, -(d + e / 4)))
    eof = DATA0 + 960
    put(0, b"\x89HDF\r\n\x1a\n" + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + S.pack("<HHI", 4, 16, 0)
        + S.pack("<QQQQ", 0, U, eof, U) + S.pack("<QQII QQ".replace(" ", ""), 0, ROOT, 1, 0, ROOT_BT, ROOT_HP))
    with open(path, "wb") as f:
        f.write(bytes(buf[:eof]))


def test_reader_takes_libhdf5_default_forms(driver, tmp_path):
    path = str(tmp_path / "lib.h5")
    _libhdf5_style_file(path)
    for d in (0, 4, 5, 9):
        out = subprocess.run([driver, "read", path, "/population/d%d" % d, "p1", "p0"], check=True,
                             capture_output=True, text=True)
        v = np.array(out.stdout.split(), float).reshape(6, 2)
        e = np.arange(6)
        assert np.array_equal(v[:, 0], np.float32(-(d + e / 4)).astype(float)), d
        assert np.array_equal(v[:, 1], 100.0 * d + e), d
