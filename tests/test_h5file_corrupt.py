"""The checkpoint reader (astr_h5*) on damaged files: seeded random bytes, bit flips and truncations
of three valid files -- one from the library's writer, one from the oracle's version-0 writer with
a user block and several symbol table nodes, one from the oracle's version-2 writer. Every open,
listing and read either succeeds or returns an error code: none may crash, hang or allocate without
bound (a restart reads whatever file it is given). The loop runs in a child process, so that a crash
shows as the child's exit status instead of ending the test run. No GPU is needed."""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import h5format

ag = pytest.importorskip("astr_gpu_b200")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from astr_gpu_b200 import _lib
L = _lib.load()
rng = np.random.default_rng(int(sys.argv[2]))
opened = refused = read_ok = read_err = 0
for path in sys.argv[3:]:
    good = open(path, "rb").read()
    for trial in range(150):
        b = bytearray(good)
        kind = trial % 3
        if kind == 2:
            b = b[: int(rng.integers(0, len(b)))]
        else:
            for _ in range(int(rng.integers(1, 5))):
                pos = int(rng.integers(0, len(b)))
                b[pos] = int(rng.integers(0, 256)) if kind == 0 else b[pos] ^ (1 << int(rng.integers(0, 8)))
        bad = path + ".bad"
        with open(bad, "wb") as fh:
            fh.write(bytes(b))
        h = ctypes.c_void_p()
        if L.astr_h5io_init(bad.encode(), b"read", ctypes.byref(h)) != 0:
            refused += 1
            continue
        opened += 1
        n = ctypes.c_int()
        L.astr_h5_count(h, ctypes.byref(n))
        for i in range(n.value):
            name = ctypes.create_string_buffer(4096)
            if L.astr_h5_name(h, i, name, 4096) != 0:
                continue
            rank, cls, size = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            dims = (ctypes.c_int64 * 32)()
            if L.astr_h5_dataset_info(h, name.value, ctypes.byref(rank), dims, ctypes.byref(cls),
                                      ctypes.byref(size)) != 0:
                read_err += 1
                continue
            shape = [dims[d] for d in range(rank.value)] or [1]
            total = 1
            for d in shape:
                total *= max(d, 0)
            if total > 100000:          # a corrupted dataspace: ask for a small block instead
                shape = [1] * len(shape)
                total = 1
            out = np.zeros(max(total, 1))
            rc = L.astr_h5read_r8(h, name.value, len(shape), (ctypes.c_int64 * len(shape))(*shape), None,
                                  b"h", ctypes.c_void_p(out.ctypes.data))
            if rc == 0:
                read_ok += 1
            else:
                read_err += 1
        L.astr_h5io_end(h)
print(opened, refused, read_ok, read_err)
"""


def test_damaged_files_give_errors_not_crashes(tmp_path):
    rng = np.random.default_rng(11)
    small = [(k, rng.standard_normal(s)) for k, s in
             (("ro", (3, 4, 5)), ("u1", (3, 4, 5)), ("p", (2, 6)), ("t", (7,)))]
    lib_fn = str(tmp_path / "lib.h5")
    with ag.h5io_init(lib_fn, "write") as f:
        for k, a in small:
            f.write(k, np.asfortranarray(a))
        f.write("nstep", np.array([5], dtype=np.int32))
        f.write("time", np.array([0.5]))
    v0_fn = str(tmp_path / "v0.h5")
    items = [(f"d{k}", rng.standard_normal((2, 3))) for k in range(9)] + [("i", np.arange(4, dtype=np.int32)),
                                                                         ("c", np.array([1.0, 2.0]))]
    h5format.write(v0_fn, items, user_block=512, snod_capacity=2, layout_version=2, compact=("c",))
    v2_fn = str(tmp_path / "v2.h5")
    h5format.write_v2(v2_fn, small + [("nstep", np.array([5], dtype=np.int32))])
    res = subprocess.run([sys.executable, "-c", CHILD, ROOT, "2024", lib_fn, v0_fn, v2_fn], capture_output=True,
                         text=True, timeout=600)
    assert res.returncode == 0, (res.returncode, res.stderr[-2000:])
    opened, refused, read_ok, read_err = map(int, res.stdout.split())
    assert opened + refused == 450
    # the damage is spread over data and metadata: some files still read, some are refused
    assert refused > 0 and read_ok > 0
