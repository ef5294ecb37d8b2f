"""The Thrift query server in front of a loaded index: NMSLIB's QueryService
(query_server/protocol.thrift; the reference's server is query_server/cpp_client_server/
QueryService_server.cpp), served by the engine's C ABI (nmsg_query_server_*), so the reference's
C++, Java and Python clients connect to it unchanged.

    server = QueryServer(index, port=10000, max_connections=8)   # port=0: any free port
    ...                                                            # clients connect to server.port
    server.stop()

or from the command line, with the reference server's option names:

    python -m nmslib_b200.query_server -m hnsw -s l2 -L index.hnsw -p 10000 [-t efSearch=64] \\
        [--threadQty 8] [--distType float|int] [-D]

(``--distType int`` with ``-s l2sqr_sift`` loads the regular graph file and its ``.dat`` objects.)
"""
from __future__ import annotations

import argparse
import ctypes
import signal
import threading

from . import _capi


class QueryServer:
    """Serves `index` (a loaded FloatIndex or IntIndex) on a TCP port until stop()."""

    def __init__(self, index, port=0, max_connections=8, debug=False):
        self._lib = _capi.load()
        self._index = index  # keeps the index alive while the server runs
        self._h = ctypes.c_void_p()
        _capi.check(self._lib.nmsg_query_server_start(index._require(), int(port), int(max_connections),
                                                      1 if debug else 0, ctypes.byref(self._h)))

    @property
    def port(self) -> int:
        return self._lib.nmsg_query_server_port(self._h)

    def stop(self):
        if self._h:
            self._lib.nmsg_query_server_stop(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


def main(argv=None):
    import nmslib_b200 as nmslib
    ap = argparse.ArgumentParser(description="NMSLIB QueryService on the B200 engine")
    ap.add_argument("-m", "--method", default="hnsw")
    ap.add_argument("-s", "--spaceType", required=True)
    ap.add_argument("--distType", default="float", choices=["float", "int"])
    ap.add_argument("-L", "--loadIndex", required=True)
    ap.add_argument("-p", "--port", type=int, required=True)
    ap.add_argument("--threadQty", type=int, default=8)
    ap.add_argument("-t", "--queryTimeParams", default="")
    ap.add_argument("-D", "--debug", action="store_true")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    if args.distType == "int":
        index = nmslib.init(method=args.method, space=args.spaceType, data_type=nmslib.DataType.DENSE_UINT8_VECTOR,
                            dtype=nmslib.DistType.INT, device=args.device)
        index.loadIndex(args.loadIndex, load_data=True)
    else:
        index = nmslib.init(method=args.method, space=args.spaceType, device=args.device)
        index.loadIndex(args.loadIndex)
    if args.queryTimeParams:
        index.setQueryTimeParams(args.queryTimeParams.split(","))
    server = QueryServer(index, args.port, args.threadQty, args.debug)
    print(f"Started a server on port {server.port} with up to {args.threadQty} connections.", flush=True)
    done = threading.Event()
    signal.signal(signal.SIGINT, lambda *a: done.set())
    signal.signal(signal.SIGTERM, lambda *a: done.set())
    done.wait()
    server.stop()


if __name__ == "__main__":
    main()
