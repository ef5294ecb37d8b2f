"""C-ABI library and host-side logic, without a GPU: symbols, argument checking, and the index
reader/validator (which runs before any device is touched)."""
import ctypes
import os
import shutil
import struct

import numpy as np
import pytest

import nmslib_b200 as nmslib
from nmslib_b200 import _capi
from nmslib_b200.build import build

from conftest import golden_path


@pytest.fixture(scope="module")
def lib():
    build()
    return _capi.load()


def test_library_exports_every_declared_symbol(lib):
    names = _capi.header_symbols()
    assert "nmsg_knn_batch" in names and "nmsg_index_load" in names
    for name in names:
        assert hasattr(lib, name), name


def _load_rc(lib, path, space=0):
    h = ctypes.c_void_p()
    rc = lib.nmsg_index_load(os.fsencode(path), space, 0, ctypes.byref(h))
    if h:
        lib.nmsg_index_free(h)
    return rc, _capi.last_error()


def _header(path):
    with open(path, "rb") as f:
        raw = bytearray(f.read())
    return raw


@pytest.mark.parametrize("name,space", [("c1_l2_d128", _capi.SPACE_L2), ("cos_d100", _capi.SPACE_COSINE),
                                        ("negdot_d960", _capi.SPACE_NEGDOT), ("l1_d22", _capi.SPACE_L1),
                                        ("linf_d37", _capi.SPACE_LINF)])
def test_valid_file_reaches_device_check(lib, name, space):
    rc, msg = _load_rc(lib, golden_path(name), space=space)
    # no GPU in this container: the file passes validation and the device check answers
    import torch
    if torch.cuda.is_available():
        assert rc == _capi.OK
    else:
        assert rc == _capi.ERR_DEVICE, msg


def test_missing_and_truncated_files(lib, tmp_path):
    rc, msg = _load_rc(lib, str(tmp_path / "nope.hnsw"))
    assert rc == _capi.ERR_BAD_FILE and "Cannot open" in msg
    raw = _header(golden_path("c1_l2_d128"))
    for cut in (2, 40, 68 + 1000, len(raw) - 3):
        p = tmp_path / f"cut{cut}.hnsw"
        p.write_bytes(bytes(raw[:cut]))
        rc, msg = _load_rc(lib, str(p))
        assert rc == _capi.ERR_BAD_FILE, (cut, msg)


def test_corrupt_neighbour_ids_are_rejected(lib, tmp_path):
    raw = _header(golden_path("c1_l2_d128"))
    n, mpo, off_l0 = struct.unpack_from("<IQQ", raw, 4)
    # node 7's first level-0 neighbour -> out of range
    pos = 68 + 7 * mpo + off_l0 + 4
    bad = bytearray(raw)
    struct.pack_into("<i", bad, pos, n + 5)
    p = tmp_path / "badid.hnsw"
    p.write_bytes(bytes(bad))
    rc, msg = _load_rc(lib, str(p))
    assert rc == _capi.ERR_CORRUPT_GRAPH and "out of range" in msg
    # neighbour count above maxM0
    bad = bytearray(raw)
    struct.pack_into("<i", bad, 68 + 3 * mpo + off_l0, 1000)
    p.write_bytes(bytes(bad))
    rc, msg = _load_rc(lib, str(p))
    assert rc == _capi.ERR_CORRUPT_GRAPH


def test_unsupported_files(lib, tmp_path):
    raw = _header(golden_path("c1_l2_d128"))
    bad = bytearray(raw)
    struct.pack_into("<i", bad, 4 + 4 + 8 * 3 + 4 + 4 + 8 + 8, 5)  # dist_func_type := L1
    p = tmp_path / "l1.hnsw"
    p.write_bytes(bytes(bad))
    assert _load_rc(lib, str(p))[0] == _capi.ERR_BAD_ARG  # an L1 index opened as l2
    struct.pack_into("<i", bad, 4 + 4 + 8 * 3 + 4 + 4 + 8 + 8, 9)  # no such distance code
    p.write_bytes(bytes(bad))
    assert _load_rc(lib, str(p))[0] == _capi.ERR_BAD_FILE
    p.write_bytes(struct.pack("<II", 0, 10) + b"\0" * 64)  # regular format with elements
    assert _load_rc(lib, str(p))[0] == _capi.ERR_UNSUPPORTED
    # wrong space for the file
    assert _load_rc(lib, golden_path("c1_l2_d128"), space=1)[0] == _capi.ERR_BAD_ARG


def test_python_surface_errors():
    with pytest.raises(ValueError):
        nmslib.init(method="sw-graph", space="l2")
    with pytest.raises(ValueError):
        nmslib.init(method="hnsw", space="l3")
    nmslib.init(method="hnsw", space="l1")  # the optimized index's L1 / LInf codes are served
    nmslib.init(method="hnsw", space="linf")
    idx = nmslib.init(method="hnsw", space="l2")
    with pytest.raises(ValueError, match="Must call createIndex or loadIndex"):
        idx.knnQueryBatch(np.zeros((2, 4), np.float32))
    with pytest.raises(ValueError, match="Must call createIndex or loadIndex"):
        idx.setQueryTimeParams({"efSearch": 10})


def test_param_parsing():
    from nmslib_b200 import _load_params
    assert _load_params({"efSearch": 100, "algoType": "old"}) == {"efSearch": "100", "algoType": "old"}
    assert _load_params(["ef=5", "algoType=v1merge"]) == {"ef": "5", "algoType": "v1merge"}
    assert _load_params(None) == {}
    with pytest.raises(ValueError):
        _load_params({"ef": [1]})
