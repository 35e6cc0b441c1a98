"""The library's HDF5 container code (csrc/h5file.cpp) on the CPU: a fixed file written
through it parses under an independent reader written from the file format specification
(tests/h5spec.py, which asserts the structural rules a libhdf5 reader relies on), with
every value where it was put, and the library's own reader reads it back by path and
member name.  Groups hold up to 32 entries in one symbol-table node (12 here)."""
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
