"""Matrix Market ingest and the drivers' CSV line (CPU only).

The fixtures in tests/golden/mm/ were read by the reference's own
io::mm::read_system + io::CSR (tests/golden/gen_golden.py, recorded in
tests/golden/mm.npz); the library reader (f3r_mm_read / f3r_mm_read_rhs) and
the oracle's restatement (oracle/mm.py) must reproduce them bit for bit.
"""
import os
import subprocess

import numpy as np
import pytest

import f3r_b200 as F
from oracle import mm as OM

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
G = os.path.join(ROOT, "tests", "golden")
MM = os.path.join(G, "mm")
NAMES = ["sym_mixed", "gen_int", "rect", "hpcg_3_4_3", "hpgmp_4_3_3"]


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(G, "mm.npz")))


@pytest.mark.parametrize("name", NAMES)
def test_reader_matches_reference(gold, name):
    path = os.path.join(MM, name + ".mtx")
    want = (gold[name + "_rptr"], gold[name + "_idx"], gold[name + "_val"])
    A, b, from_file = F.read_system(path)
    assert all(same(x, y) for x, y in zip(A.arrays(), want)), name
    assert same(b, gold[name + "_b"])
    assert from_file == (name == "sym_mixed")
    # the oracle's restatement agrees too
    nrow, ncol, r, i, v = OM.read_matrix(path)
    assert all(same(x, y) for x, y in zip((r, i, v), want)), name
    assert same(OM.read_rhs(path, nrow), gold[name + "_b"])
    if name == "rect":
        assert A.shape == (3, 5)


def test_random_rhs_is_the_drivers_init():
    # v.random<0, 1>(std::mt19937_64(0)): the restated MT19937-64 and the library agree
    assert same(OM.uniform01(0, 5000), F.random_uniform(0, 0.0, 1.0, 5000))


def test_round_trip_and_thread_independence(tmp_path):
    """write -> read is exact (%.17g), also for a file large enough to be
    parsed in several chunks by several threads"""
    A = F.stencil27(24, 24, 24, 2, 0.5).scale()  # ~350k entries, ~10 MB of text
    p = str(tmp_path / "half24.mtx")
    A.write_mm(p)
    B = F.read_matrix(p)
    assert all(same(x, y) for x, y in zip(A.arrays(), B.arrays()))
    # a one-thread parse gives the same arrays
    code = ("import f3r_b200 as F, numpy as np, sys; A = F.read_matrix(sys.argv[1]); "
            "np.savez(sys.argv[2], *A.arrays())")
    out = str(tmp_path / "one.npz")
    env = dict(os.environ, OMP_NUM_THREADS="1", PYTHONPATH=ROOT)
    subprocess.run(["python", "-c", code, p, out], check=True, env=env, cwd=ROOT)
    one = np.load(out)
    assert all(same(one[f"arr_{k}"], x) for k, x in enumerate(B.arrays()))
    x = np.random.default_rng(1).standard_normal(A.shape[0])
    write = str(tmp_path / "half24_b.mtx")
    F.write_vector(write, x)
    _, b, ff = F.read_system(p)
    assert ff and same(b, x)


def test_symmetric_expansion_and_duplicates(tmp_path):
    p = str(tmp_path / "dup.mtx")
    with open(p, "w") as f:
        # a duplicated (2,1) entry: both copies are kept, in file order, as
        # the reference's reader keeps them (io.hpp:165-189 never merges)
        f.write("%%MatrixMarket matrix coordinate real symmetric\n3 3 5\n1 1 2\n2 1 -1\n2 1 -0.5\n2 2 3\n3 3 1\n")
    A = F.read_matrix(p)
    r, i, v = A.arrays()
    assert list(r) == [0, 3, 6, 7]
    assert list(i) == [0, 1, 1, 0, 0, 1, 2]
    assert list(v) == [2, -1, -0.5, -1, -0.5, 3, 1]
    # the solver-side entry points want strictly increasing columns and say so
    with pytest.raises(F.F3RError, match="strictly increasing"):
        A.spmv(np.ones(3))


def _bad(tmp_path, text, name="bad.mtx"):
    p = str(tmp_path / name)
    with open(p, "w") as f:
        f.write(text)
    return p


@pytest.mark.parametrize("text", [
    "not a banner\n2 2 1\n1 1 1\n",
    "%%MatrixMarket matrix coordinate real\n2 2 1\n1 1 1\n",                       # four banner tokens
    "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n",                # dense matrix
    "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n3 1 1\n",        # row out of range
    "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n0 1 1\n",        # 0 is not a 1-based index
    "%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n2 2 1\n",        # fewer entries than announced
    "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1\n2 2 1\n",          # short line
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n1.5 1 1\n",             # fractional index
    "%%MatrixMarket matrix coordinate real general\n2 x 1\n1 1 1\n",               # bad size line
])
def test_malformed_files_are_errors(tmp_path, text):
    with pytest.raises(F.F3RError):
        F.read_matrix(_bad(tmp_path, text))


@pytest.mark.parametrize("kind", ["pattern general", "complex general", "real skew-symmetric",
                                  "real hermitian"])
def test_unsupported_kinds_are_refused(tmp_path, kind):
    p = _bad(tmp_path, f"%%MatrixMarket matrix coordinate {kind}\n2 2 1\n1 1 1 0\n")
    with pytest.raises(F.F3RError, match="UNSUPPORTED|unsupported|only"):
        F.read_matrix(p)


def test_rhs_file_errors(tmp_path):
    p = _bad(tmp_path, "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n2 2 1\n", "m.mtx")
    _bad(tmp_path, "%%MatrixMarket matrix array real general\n3 1\n1\n2\n3\n", "m_b.mtx")
    with pytest.raises(F.F3RError):  # 3 values for 2 rows (the reference exits, io.hpp:123-124)
        F.read_system(p)
    _bad(tmp_path, "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", "m_b.mtx")
    with pytest.raises(F.F3RError):  # not n x 1
        F.read_system(p)
    with pytest.raises(F.F3RError):
        F.read_matrix(str(tmp_path / "missing.mtx"))


def test_uppercase_keywords_and_crlf(tmp_path):
    p = _bad(tmp_path, "%%MatrixMarket MATRIX Coordinate REAL General\r\n% c\r\n2 2 2\r\n1 1 1.5\r\n2 2 -2\r\n")
    r, i, v = F.read_matrix(p).arrays()
    assert list(r) == [0, 1, 2] and list(i) == [0, 1] and list(v) == [1.5, -2]


def test_csv_row_format():
    # the drivers' printf formats (f3r-gpu.cpp:94-103, 267-272)
    row = F.csv_row("hpcg_8_8_8", "F3R", "__half", 8, 4, 2, 64, "SDAINV", "1.0", 0.0123, 2048, 3.2e-9, 4.1e-9)
    assert row == "hpcg_8_8_8,F3R,__half,8,4,2,64,SDAINV,1.0,1.230000e-02,2048,3.200000e-09,4.100000e-09"
    assert F.CSV_HEADER.split(",") == ["Problem", "Method", "Prec", "M2", "M3", "M4", "W", "Precond", "ACC", "Time",
                                       "Iter", "ImplRes", "ExplRes"]


def test_driver_argument_errors():
    """the command-line driver rejects bad arguments before touching a GPU"""
    exe = os.path.join(ROOT, "f3r_b200", "bin", "f3r-run")
    assert os.path.exists(exe), "python -m f3r_b200.build builds bin/f3r-run"
    for args in ([], ["a.mtx", "1.0"], ["--method", "F5", "a.mtx", "1.0", "1", "8", "4", "2", "64", "3"],
                 ["--method", "F3R-Static", "a.mtx", "1.0", "1", "8", "4", "2", "64", "3"]):
        r = subprocess.run([exe] + args, capture_output=True, text=True)
        assert r.returncode == 2 and "usage" in r.stderr
