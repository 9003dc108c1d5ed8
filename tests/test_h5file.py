"""The checkpoint file layer (astr_h5*, the library's HDF5 reader and writer; no GPU needed) against
the oracle's restatement of the HDF5 file format (oracle/h5format.py).

Pin: the only file in this image written by the HDF5 library itself, a MATLAB 7.3 test file that
ships with scipy (512-byte user block, superblock version 0, symbol-table root group, one
contiguous double dataset with an attribute). Both readers return its dataset; the library's
writer emits the same message encodings (fill value, datatype, dataspace) as that file.

Then: files of the library's writer read by the oracle (bit-exact), files of the oracle's writer
in variants the library's writer does not make (user block, layout version 2, big-endian, float32
and integer elements, compact storage, several symbol table nodes, the version-2 superblock and
object headers with compact links) read by the library, the
read-write mode that h5srite uses (src/hdf5io.F90:1015-1100), hyperslab and stream reads
(h5ra3d_r8_struct / h5ra3d_r8_stream, src/hdf5io.F90:204-348), and the refusals."""
import os

import numpy as np
import pytest

from oracle import h5format

ag = pytest.importorskip("astr_gpu_b200")

ASTR_ERR_ARG, ASTR_ERR_STATE, ASTR_ERR_UNSUPPORTED = -1, -3, -4


def _library_file():
    try:
        import scipy.io.matlab as m
    except ImportError:
        return None
    p = os.path.join(os.path.dirname(m.__file__), "tests", "data", "testhdf5_7.4_GLNX86.mat")
    return p if os.path.exists(p) else None


LIB_FILE = _library_file()
needs_lib_file = pytest.mark.skipif(LIB_FILE is None, reason="scipy's HDF5 test file is not installed")


def _flowfield_arrays(shape, seed):
    rng = np.random.default_rng(seed)
    return {n: np.asfortranarray(rng.standard_normal(shape)) for n in ("ro", "u1", "u2", "u3", "p", "t")}


@needs_lib_file
def test_oracle_reads_the_library_written_file():
    info = h5format.read(LIB_FILE)
    assert info.superblock_version == 0 and info.base == 512 and info.group_kind == "symbol_table"
    e = info.entries["testdouble"]
    assert e.kind == "dataset" and e.dims == (9, 1) and e.dtype == np.dtype("<f8") and e.layout == "contiguous"
    assert np.abs(e.data.ravel() - np.linspace(0.0, 2.0 * np.pi, 9)).max() <= 1e-15
    assert e.attrs["MATLAB_class"].tobytes() == b"double"


@needs_lib_file
def test_library_reads_the_library_written_file():
    ref = h5format.read(LIB_FILE).entries["testdouble"].data
    with ag.h5io_init(LIB_FILE) as f:
        assert f.names() == ["testdouble"]
        assert f.info("testdouble") == ((1, 9), 1, 8)
        got = f.read("testdouble")
    assert got.shape == (1, 9)
    assert np.array_equal(got, ref.T)


@needs_lib_file
def test_writer_emits_the_library_encodings(tmp_path):
    """The datatype and fill value messages of a real(8) dataset equal the HDF5 library's bytes,
    and the dataspace is a version-1 message as the library writes it."""
    fn = tmp_path / "w.h5"
    with ag.h5io_init(fn, "write") as f:
        f.write("x", np.arange(9.0).reshape(1, 9))
    ours = {t: (v, raw) for t, v, _f, raw in h5format.read(fn).entries["x"].messages}
    lib = {t: (v, raw) for t, v, _f, raw in h5format.read(LIB_FILE).entries["testdouble"].messages}
    assert ours[0x03] == lib[0x03]
    assert ours[0x05] == lib[0x05]
    assert ours[0x01] == lib[0x01]     # the same (9, 1) dataspace
    assert ours[0x08][0] == 3          # layout version 3, contiguous


@needs_lib_file
def test_rdwr_adds_to_the_library_written_file(tmp_path):
    """h5srite's read-write step on a file the HDF5 library wrote (user block, its own heap with a
    free block, its symbol table node): the existing dataset and its attribute stay readable and
    the new dataset is found by both readers."""
    import shutil
    fn = tmp_path / "copy.mat"
    shutil.copyfile(LIB_FILE, fn)
    with ag.h5io_init(fn, "rdwr") as f:
        f.write("nstep", np.array([12], dtype=np.int32))
        f.write("time", np.array([0.25]))
    info = h5format.read(fn)
    assert sorted(info.entries) == ["nstep", "testdouble", "time"]
    ref = h5format.read(LIB_FILE).entries["testdouble"]
    assert np.array_equal(info.entries["testdouble"].data, ref.data)
    assert info.entries["testdouble"].attrs["MATLAB_class"].tobytes() == b"double"
    assert info.eof == os.path.getsize(fn)
    with ag.h5io_init(fn) as f:
        assert f.names() == ["nstep", "testdouble", "time"]
        assert f.read("nstep", dtype=np.int32).tolist() == [12] and f.read("time").tolist() == [0.25]
        assert np.array_equal(f.read("testdouble"), ref.data.T)


def test_flowfield_file_written_by_the_library_matches_the_oracle(tmp_path):
    fn = tmp_path / "flowfield.h5"
    arrays = _flowfield_arrays((9, 7, 5), 1)
    with ag.h5io_init(fn, "write") as f:
        for n, a in arrays.items():
            f.write(n, a)
        f.write("nstep", np.array([1200], dtype=np.int32))
        f.write("time", np.array([12.375]))
    info = h5format.read(fn)
    assert info.superblock_version == 0 and info.group_kind == "symbol_table"
    assert sorted(info.entries) == sorted(list(arrays) + ["nstep", "time"])
    for n, a in arrays.items():
        e = info.entries[n]
        assert e.dims == (5, 7, 9) and e.dtype == np.dtype("<f8")
        assert np.array_equal(e.data, a.T)           # Fortran order: the reversed dataspace
    assert info.entries["nstep"].dtype == np.dtype("<i4") and info.entries["nstep"].data.tolist() == [1200]
    assert info.entries["time"].data.tolist() == [12.375]
    assert info.eof == os.path.getsize(fn)


@pytest.mark.parametrize("user_block,layout_version,byte_order,snod", [
    (0, 3, "<", 8), (512, 2, "<", 8), (0, 3, ">", 2), (1024, 2, ">", 4)])
def test_library_reads_oracle_written_files(tmp_path, user_block, layout_version, byte_order, snod):
    rng = np.random.default_rng(user_block + snod)
    items = [(f"v{k:02d}", rng.standard_normal((3, 4, 5))) for k in range(11)]
    items += [("f32", rng.standard_normal((6, 2)).astype(np.float32)),
              ("i32", rng.integers(-2**31, 2**31, (5, 3)).astype(np.int32)),
              ("i64", rng.integers(-2**40, 2**40, 7).astype(np.int64)),
              ("u16", rng.integers(0, 2**16, 4).astype(np.uint16)),
              ("small", np.array([2.5, -1.0])),
              ("scalar", np.array(3.25)),
              ("empty", np.zeros((0, 3)))]
    fn = tmp_path / "o.h5"
    h5format.write(fn, items, user_block=user_block, layout_version=layout_version, snod_capacity=snod,
                   byte_order=byte_order, compact=("small",))
    with ag.h5io_init(fn) as f:
        assert f.names() == sorted(n for n, _ in items)
        for n, a in items:
            shape = a.shape[::-1]
            assert f.info(n)[0] == shape
            if a.dtype.kind == "f":
                assert np.array_equal(f.read(n), a.T.astype(np.float64)), n
            else:
                if a.dtype != np.int64:
                    assert np.array_equal(f.read(n, dtype=np.int32), a.T.astype(np.int64)), n
                assert np.array_equal(f.read(n), a.T.astype(np.float64)), n
        with pytest.raises(ag.AstrError) as e:
            f.read("i64", dtype=np.int32)            # values beyond int32
        assert e.value.code == ASTR_ERR_ARG


def test_lookup3_known_answers():
    """The checksum of the format's version-2 structures: lookup3's published test values."""
    assert h5format.lookup3(b"") == 0xDEADBEEF
    assert h5format.lookup3(b"", 0xDEADBEEF) == 0xBD5B7DDE
    assert h5format.lookup3(b"Four score and seven years ago") == 0x17770551
    assert h5format.lookup3(b"Four score and seven years ago", 1) == 0xCD628161


def test_library_reads_version2_files(tmp_path):
    """Superblock version 2, version-2 object headers and a compact-link root group (the HDF5
    library's output with its latest format bounds); the library reads them but does not add to
    them (read-write needs a version-0 file)."""
    rng = np.random.default_rng(5)
    items = [("ro", rng.standard_normal((4, 5, 6))), ("nstep", np.array([7], dtype=np.int32)),
             ("f32be", rng.standard_normal(9).astype(">f4")), ("empty", np.zeros((0, 2))),
             ("a" * 200, np.array([1.5]))]
    fn = tmp_path / "v2.h5"
    h5format.write_v2(fn, items)
    info = h5format.read(fn)        # checks the checksums
    assert info.superblock_version == 2 and info.group_kind == "links"
    with ag.h5io_init(fn) as f:
        assert f.names() == [n for n, _ in items]
        for n, a in items:
            assert f.info(n)[0] == a.shape[::-1]
            assert np.array_equal(f.read(n), a.T.astype(np.float64)), n
        assert f.read("nstep", dtype=np.int32).tolist() == [7]
    with pytest.raises(ag.AstrError) as e:
        ag.h5io_init(fn, "rdwr")
    assert e.value.code == ASTR_ERR_UNSUPPORTED


def test_hyperslab_and_stream_reads(tmp_path):
    """h5ra3d_r8_struct reads a rank's block at (ig0, jg0, kg0); h5ra3d_r8_stream reads a rank's
    run of a 1-D dataset at its element offset."""
    fn = tmp_path / "h.h5"
    a = np.asfortranarray(np.random.default_rng(3).standard_normal((10, 8, 6)))
    with ag.h5io_init(fn, "write") as f:
        f.write("ro", a)
        f.write("ro_stream", a.ravel(order="F"))
    with ag.h5io_init(fn) as f:
        for off, shp in [((0, 0, 0), (10, 8, 6)), ((0, 0, 2), (10, 8, 3)), ((0, 3, 1), (10, 4, 5)),
                         ((2, 1, 1), (5, 6, 4)), ((9, 7, 5), (1, 1, 1))]:
            sl = tuple(slice(o, o + s) for o, s in zip(off, shp))
            assert np.array_equal(f.read("ro", shape=shp, offset=off), a[sl])
        assert np.array_equal(f.read("ro_stream", shape=(10, 8, 6), mode="s"), a)
        assert np.array_equal(f.read("ro_stream", shape=(7, 3), offset=(55,), mode="s"),
                              a.ravel(order="F")[55:76].reshape((7, 3), order="F"))
        with pytest.raises(ag.AstrError):
            f.read("ro", shape=(10, 8, 6), mode="s")        # not one-dimensional
        with pytest.raises(ag.AstrError):
            f.read("ro", shape=(6, 8, 6), offset=(5, 0, 0))  # past the dataset
        with pytest.raises(ag.AstrError):
            f.read("ro_stream", shape=(10, 8, 7), mode="s")  # more elements than stored


def test_rdwr_adds_datasets_as_h5srite_does(tmp_path):
    """writeflfed's sequence: write_io_tree creates the file with the six fields, then h5srite
    opens it read-write twice to add nstep and time (src/readwrite.F90:1774-1835)."""
    fn = tmp_path / "flowfield.h5"
    arrays = _flowfield_arrays((5, 6, 7), 2)
    with ag.h5io_init(fn, "write") as f:
        for n, a in arrays.items():
            f.write(n, a)
    with ag.h5io_init(fn, "rdwr") as f:
        f.write("nstep", np.array([77], dtype=np.int32))
    with ag.h5io_init(fn, "rdwr") as f:
        f.write("time", np.array([0.5]))
    info = h5format.read(fn)
    assert sorted(info.entries) == ["nstep", "p", "ro", "t", "time", "u1", "u2", "u3"]
    for n, a in arrays.items():
        assert np.array_equal(info.entries[n].data, a.T)
    with ag.h5io_init(fn) as f:
        assert f.read("nstep", dtype=np.int32).tolist() == [77] and f.read("time").tolist() == [0.5]
        assert np.array_equal(f.read("u3"), arrays["u3"])


def test_rdwr_on_an_oracle_file_with_a_user_block(tmp_path):
    """Adding to a file the library did not write: base address 512, eight members filling one
    symbol table node, so the ninth needs a second node."""
    fn = tmp_path / "u.h5"
    items = [(f"a{k}", np.full((2, 3), float(k))) for k in range(8)]
    h5format.write(fn, items, user_block=512)
    with ag.h5io_init(fn, "rdwr") as f:
        f.write("nstep", np.array([5], dtype=np.int32))
    info = h5format.read(fn)
    assert info.base == 512 and len(info.entries) == 9
    for n, a in items:
        assert np.array_equal(info.entries[n].data, a)
    assert info.entries["nstep"].data.tolist() == [5]


def test_many_datasets_and_long_names(tmp_path):
    fn = tmp_path / "m.h5"
    names = [f"sp{k:03d}" for k in range(200)] + ["a" * 300]
    with ag.h5io_init(fn, "write") as f:
        for k, n in enumerate(names):
            f.write(n, np.array([float(k)]))
    info = h5format.read(fn)
    assert sorted(info.entries) == sorted(names)
    assert all(info.entries[n].data.tolist() == [float(k)] for k, n in enumerate(names))


def test_refusals(tmp_path):
    fn = tmp_path / "r.h5"
    h5format.write(fn, [("c", np.ones((4, 4))), ("z", np.ones(3)), ("ok", np.ones(2)), ("s", np.ones(2))],
                   chunked=("c",), filtered=("z",), shared_type=("s",))
    with ag.h5io_init(fn) as f:
        with pytest.raises(ag.AstrError) as e:
            f.read("s")                             # a committed (shared) datatype
        assert e.value.code == ASTR_ERR_UNSUPPORTED
        with pytest.raises(ag.AstrError) as e:
            f.read("c")
        assert e.value.code == ASTR_ERR_UNSUPPORTED
        with pytest.raises(ag.AstrError) as e:
            f.read("z")
        assert e.value.code == ASTR_ERR_UNSUPPORTED
        with pytest.raises(ag.AstrError) as e:
            f.read("missing")
        assert e.value.code == ASTR_ERR_ARG
        with pytest.raises(ag.AstrError) as e:
            f.read("ok", dtype=np.int32)            # a float dataset read as integers
        assert e.value.code == ASTR_ERR_UNSUPPORTED
        with pytest.raises(ag.AstrError) as e:
            f.read("ok", shape=(2, 1))              # rank differs
        assert e.value.code == ASTR_ERR_ARG
        with pytest.raises(ag.AstrError) as e:
            f.write("new", np.ones(2))              # opened for reading
        assert e.value.code == ASTR_ERR_ARG
    with ag.h5io_init(tmp_path / "d.h5", "write") as f:
        f.write("x", np.ones(2))
        with pytest.raises(ag.AstrError):
            f.write("x", np.ones(2))                # duplicate name
        with pytest.raises(ag.AstrError):
            f.write("a/b", np.ones(2))              # not a name in the root group
    (tmp_path / "not.h5").write_bytes(b"plain text, not HDF5" * 40)
    with pytest.raises(ag.AstrError) as e:
        ag.h5io_init(tmp_path / "not.h5")
    assert e.value.code == ASTR_ERR_STATE and "not an HDF5 file" in str(e.value)
    good = (tmp_path / "d.h5").read_bytes()
    (tmp_path / "cut.h5").write_bytes(good[: len(good) // 2])
    with pytest.raises(ag.AstrError) as e:
        ag.h5io_init(tmp_path / "cut.h5")
    assert e.value.code == ASTR_ERR_STATE
    with pytest.raises(ag.AstrError) as e:
        ag.h5io_init(tmp_path / "missing.h5")
    assert e.value.code == ASTR_ERR_STATE
    with pytest.raises(ag.AstrError) as e:
        ag.h5io_init(fn, "append")
    assert e.value.code == ASTR_ERR_ARG
