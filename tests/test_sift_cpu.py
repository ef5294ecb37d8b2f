"""l2sqr_sift in the engine, host side (no GPU): the regular graph file and the objects file are
read and validated by nmsg_index_load_with_data before any device is touched, and the Python
mirror of IndexWrapper<int> checks its arguments as the reference does."""
import ctypes
import os
import struct

import numpy as np
import pytest

import nmslib_b200 as nmslib
from nmslib_b200 import _capi
from nmslib_b200.build import build

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def lib():
    build()
    return _capi.load()


def _gpath(name):
    return os.path.join(GOLDEN, name + ".hnsw")


def _load_rc(lib, graph, data):
    h = ctypes.c_void_p()
    rc = lib.nmsg_index_load_with_data(os.fsencode(str(graph)), os.fsencode(str(data)), _capi.SPACE_L2SQR_SIFT, 0,
                                       ctypes.byref(h))
    if h:
        lib.nmsg_index_free(h)
    return rc, _capi.last_error()


@pytest.mark.parametrize("name", ["sift_u8_d128", "sift_u8_ties", "sift_u8_tiny"])
def test_valid_files_reach_the_device_check(lib, name):
    import torch
    rc, msg = _load_rc(lib, _gpath(name), _gpath(name) + ".dat")
    assert rc == (_capi.OK if torch.cuda.is_available() else _capi.ERR_DEVICE), msg


def _graph_lists(path):
    """(header bytes, [(level, [list, ...]) per node]) of a regular graph file."""
    raw = open(path, "rb").read()
    head = raw[:40]
    n = struct.unpack_from("<I", raw, 4)[0]
    pos, nodes = 40, []
    for _ in range(n):
        (lev,) = struct.unpack_from("<I", raw, pos)
        pos += 4
        lists = []
        for _ in range(lev + 1):
            (c,) = struct.unpack_from("<I", raw, pos)
            lists.append(list(struct.unpack_from(f"<{c}i", raw, pos + 4)))
            pos += 4 + 4 * c
        nodes.append((lev, lists))
    return head, nodes


def _write_graph(path, head, nodes):
    out = bytearray(head)
    for lev, lists in nodes:
        out += struct.pack("<I", lev)
        for lst in lists:
            out += struct.pack("<I", len(lst)) + struct.pack(f"<{len(lst)}i", *lst)
    open(path, "wb").write(bytes(out))


def test_corrupt_graphs_are_rejected(lib, tmp_path):
    name = "sift_u8_d128"
    data = _gpath(name) + ".dat"
    head, nodes = _graph_lists(_gpath(name))
    n = len(nodes)
    g = tmp_path / "g.hnsw"
    # a level-0 neighbour id out of range (the reference's own check, hnsw.cc:982-984)
    bad = [(lev, [list(x) for x in lists]) for lev, lists in nodes]
    bad[5][1][0][0] = n + 3
    _write_graph(g, head, bad)
    rc, msg = _load_rc(lib, g, data)
    assert rc == _capi.ERR_CORRUPT_GRAPH and "Invalid friendId" in msg
    # an upper-level neighbour that has no list at that level
    up = next(i for i, (lev, _) in enumerate(nodes) if lev >= 1 and nodes[i][1][1])
    low = next(i for i, (lev, _) in enumerate(nodes) if lev == 0)
    bad = [(lev, [list(x) for x in lists]) for lev, lists in nodes]
    bad[up][1][1][0] = low
    _write_graph(g, head, bad)
    rc, msg = _load_rc(lib, g, data)
    assert rc == _capi.ERR_CORRUPT_GRAPH and "does not exist at level 1" in msg
    # truncated graph file
    raw = open(_gpath(name), "rb").read()
    g.write_bytes(raw[:len(raw) - 7])
    assert _load_rc(lib, g, data)[0] == _capi.ERR_BAD_FILE
    # an optimized (float) index file given as the graph
    rc, msg = _load_rc(lib, _gpath("c1_l2_d128"), data)
    assert rc == _capi.ERR_BAD_FILE and "regular format" in msg


def test_object_file_errors(lib, tmp_path):
    name = "sift_u8_tiny"
    graph = _gpath(name)
    raw = open(graph + ".dat", "rb").read()
    d = tmp_path / "o.dat"
    d.write_bytes(raw[:len(raw) - 10])  # truncated
    assert _load_rc(lib, graph, d)[0] == _capi.ERR_BAD_FILE
    d.write_bytes(struct.pack("<Q", 1 << 40) + raw[8:])  # a count the file cannot hold
    rc, msg = _load_rc(lib, graph, d)
    assert rc == _capi.ERR_BAD_FILE and "does not fit" in msg
    d.write_bytes(struct.pack("<Q", 3) + raw[8:8 + 3 * 156])  # fewer objects than graph nodes
    rc, msg = _load_rc(lib, graph, d)
    assert rc == _capi.ERR_BAD_FILE and "Did you forget to re-load data?" in msg
    bad = bytearray(raw)
    struct.pack_into("<Q", bad, 8 + 16, 100)  # an object whose data length is not 132
    d.write_bytes(bytes(bad))
    assert _load_rc(lib, graph, d)[0] == _capi.ERR_BAD_FILE
    rc = lib.nmsg_index_load_with_data(os.fsencode(graph), os.fsencode(graph + ".dat"), _capi.SPACE_L2, 0,
                                       ctypes.byref(ctypes.c_void_p()))
    assert rc == _capi.ERR_UNSUPPORTED


def test_python_surface_of_the_int_index():
    idx = nmslib.init(method="hnsw", space="l2sqr_sift", data_type=nmslib.DataType.DENSE_UINT8_VECTOR,
                      dtype=nmslib.DistType.INT)
    assert isinstance(idx, nmslib.IntIndex)
    with pytest.raises(ValueError):
        nmslib.init(method="hnsw", space="l2sqr_sift", data_type=nmslib.DataType.DENSE_VECTOR,
                    dtype=nmslib.DistType.INT)
    with pytest.raises(ValueError):
        nmslib.init(method="hnsw", space="l2", data_type=nmslib.DataType.DENSE_UINT8_VECTOR,
                    dtype=nmslib.DistType.INT)
    with pytest.raises(ValueError, match="Must call createIndex or loadIndex"):
        idx.knnQueryBatch(np.zeros((2, 128), np.uint8))
    with pytest.raises(RuntimeError):
        idx.addDataPointBatch(np.zeros((2, 64), np.uint8))
    with pytest.raises(RuntimeError):
        idx.createIndex({"M": 8})


def test_objects_file_from_added_rows_matches_the_reference_layout(tmp_path):
    """Rows added with addDataPointBatch are written in the reference's objects-file layout (the
    committed fixture's objects file reproduced byte for byte from its own rows)."""
    raw = open(_gpath("sift_u8_tiny") + ".dat", "rb").read()
    n = struct.unpack_from("<Q", raw, 0)[0]
    rows = np.stack([np.frombuffer(raw, np.uint8, 128, 8 + i * 156 + 24) for i in range(n)])
    ids = [struct.unpack_from("<i", raw, 8 + i * 156 + 8)[0] for i in range(n)]
    labels = [struct.unpack_from("<i", raw, 8 + i * 156 + 12)[0] for i in range(n)]
    idx = nmslib.init(method="hnsw", space="l2sqr_sift", data_type=nmslib.DataType.DENSE_UINT8_VECTOR,
                      dtype=nmslib.DistType.INT)
    idx.addDataPointBatch(rows, ids=ids)
    out = tmp_path / "o.dat"
    idx._objects_file(str(out))
    if set(labels) == {-1}:
        assert out.read_bytes() == raw
    else:  # labels are not part of addDataPointBatch; compare everything else
        assert len(out.read_bytes()) == len(raw)
