"""CPU tests of the C ABI and of the .bin file format.

- The native library loads and exports every function include/*.h declares
  (no compute call is made: there is no GPU here).
- The .bin writer is byte-identical to the reference's own writebin
  (oracle/_ref) for dense arrays of several types, keyword headers, cells
  with empty members and a sparse matrix; files the reference writes read
  back exactly, and files written here read back through the reference's
  dread; gzip files and several top-level arrays read as the reference's
  readbin does.
"""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in sorted(os.listdir(inc)):
        if f.endswith(".h"):
            text = open(os.path.join(inc, f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(shwfs_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_function():
    import ctypes
    from maos_b200 import shwfs
    lib = ctypes.CDLL(shwfs.LIB_PATH)
    names = _declared()
    assert len(names) > 40
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string():
    from maos_b200 import shwfs
    assert shwfs.lib().shwfs_version().decode()


def _bytes(p):
    with open(p, "rb") as f:
        return f.read()


def test_dense_bytes_match_reference_writer(ref_lib, tmp_path):
    import ctypes as C
    from maos_b200.binio import write_bin, read_bin
    L = ref_lib.lib()
    rng = np.random.default_rng(3)
    a = rng.standard_normal((7, 5))
    for kw in (None, "", "wvl=5e-7\nsa=1", "x" * 23):
        ref, mine = str(tmp_path / "ref.bin"), str(tmp_path / "mine.bin")
        fa = np.asfortranarray(a)
        L.oref_writebin_d(ref.encode(), fa.ctypes.data_as(C.c_void_p), C.c_long(7), C.c_long(5),
                          kw.encode() if kw is not None else None)
        write_bin(mine, a, keywords=kw)
        assert _bytes(ref) == _bytes(mine), kw
        back, kw2 = read_bin(ref, keywords=True)
        assert np.array_equal(back, a) and back.dtype == np.float64
        assert (kw2 or None) == (kw or None)
    # float32 and complex128
    f = rng.standard_normal((4, 6)).astype(np.float32)
    ref, mine = str(tmp_path / "rf.bin"), str(tmp_path / "mf.bin")
    ff = np.asfortranarray(f)
    L.oref_writebin_f(ref.encode(), ff.ctypes.data_as(C.c_void_p), C.c_long(4), C.c_long(6), None)
    write_bin(mine, f)
    assert _bytes(ref) == _bytes(mine)
    z = rng.standard_normal((3, 2)) + 1j * rng.standard_normal((3, 2))
    ref, mine = str(tmp_path / "rc.bin"), str(tmp_path / "mc.bin")
    fz = np.asfortranarray(z)
    L.oref_writebin_c(ref.encode(), fz.ctypes.data_as(C.c_void_p), C.c_long(3), C.c_long(2))
    write_bin(mine, z)
    assert _bytes(ref) == _bytes(mine)
    assert np.array_equal(read_bin(ref), z)


def test_cell_with_empty_member_matches_reference(ref_lib, tmp_path):
    import ctypes as C
    from maos_b200.binio import write_bin, read_bin
    L = ref_lib.lib()
    m = [np.arange(6.0).reshape(3, 2, order="F"), None, np.linspace(0, 1, 4).reshape(4, 1)]
    nx = (C.c_long * 3)(3, 0, 4)
    ny = (C.c_long * 3)(2, 0, 1)
    keep = [np.asfortranarray(x) if x is not None else np.zeros(1) for x in m]
    ptrs = (C.c_void_p * 3)(*[k.ctypes.data for k in keep])
    ref, mine = str(tmp_path / "ref.bin"), str(tmp_path / "mine.bin")
    L.oref_writebin_dcell(ref.encode(), 3, nx, ny, ptrs, b"cell header")
    write_bin(mine, m, keywords="cell header")
    assert _bytes(ref) == _bytes(mine)
    c = read_bin(ref)
    assert c.shape == (3, 1) and c[1, 0] is None
    assert np.array_equal(c[0, 0], m[0]) and np.array_equal(c[2, 0], m[2])


def test_sparse_matches_reference(ref_lib, tmp_path):
    from maos_b200.binio import write_bin, read_bin
    from maos_b200.configs import NGS8
    import scipy.sparse as sp
    r = ref_lib.RefPowfs(NGS8)
    nrow, ncol, pp, pi, px = r.gs0()
    ref, mine = str(tmp_path / "gs0_ref.bin"), str(tmp_path / "gs0.bin")
    ref_lib.lib().oref_writebin_gs0(ref.encode())
    write_bin(mine, sp.csc_matrix((px, pi, pp), shape=(nrow, ncol)))
    assert _bytes(ref) == _bytes(mine)
    g = read_bin(ref)
    assert g.shape == (nrow, ncol) and np.array_equal(g.indptr, pp) and np.array_equal(g.data, px)


def test_written_files_read_by_reference(ref_lib, tmp_path):
    import ctypes as C
    from maos_b200.binio import write_bin
    a = np.random.default_rng(5).standard_normal((9, 4))
    for name in ("w.bin", "w.bin.gz"):
        p = str(tmp_path / name)
        write_bin(p, a, keywords="k=1")
        out = np.zeros(36)
        nx, ny = C.c_long(), C.c_long()
        n = ref_lib.lib().oref_readbin_d(p.encode(), out.ctypes.data_as(C.c_void_p), C.c_long(36), C.byref(nx),
                                         C.byref(ny))
        assert (n, nx.value, ny.value) == (36, 9, 4)
        assert np.array_equal(out.reshape(9, 4, order="F"), a)


def test_gzip_and_multiple_arrays(tmp_path):
    import gzip
    from maos_b200.binio import write_bin, read_bin, read_bin_all
    a, b = np.arange(5.0), np.arange(6, dtype=np.int32).reshape(2, 3)
    pa, pb = str(tmp_path / "a.bin"), str(tmp_path / "b.bin")
    write_bin(pa, a)
    write_bin(pb, b)
    both = str(tmp_path / "ab.bin.gz")
    with gzip.open(both, "wb") as f:
        f.write(_bytes(pa) + _bytes(pb))
    assert np.array_equal(read_bin(both).ravel(), a)
    al = read_bin_all(both)
    assert len(al) == 2 and np.array_equal(al[1], b) and al[1].dtype == np.int32
    # a truncated file is an error, not a short array
    with open(str(tmp_path / "t.bin"), "wb") as f:
        f.write(_bytes(pa)[:-3])
    from maos_b200.binio import BinError
    with pytest.raises(BinError):
        read_bin(str(tmp_path / "t.bin"))


def test_reference_data_file_reads(ref_lib):
    """A data file shipped with the reference, when its tree is present."""
    from oracle import REF_TREE
    p = os.path.join(REF_TREE, "config", "maos", "bin", "NapMean.bin")
    if not os.path.exists(p):
        pytest.skip("reference tree absent")
    from maos_b200.binio import read_bin
    a = read_bin(p)
    assert a is not None and np.isfinite(np.asarray(a, dtype=float)).all() and a.size > 10
