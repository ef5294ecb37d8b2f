"""A small client of NMSLIB's Thrift QueryService (query_server/protocol.thrift) speaking the binary
protocol over a plain TCP stream, as the reference's clients do with TBinaryProtocol over a
TBufferedTransport. Test helper: it lets the tests drive the engine's query server without the
Thrift library."""
import socket
import struct

T_STOP, T_BOOL, T_DOUBLE, T_I32, T_STRING, T_STRUCT, T_LIST = 0, 2, 4, 8, 11, 12, 15
CALL, REPLY, EXCEPTION = 1, 2, 3


class QueryException(Exception):
    pass


class ApplicationException(Exception):
    def __init__(self, message, kind):
        super().__init__(message)
        self.kind = kind


class _Reader:
    def __init__(self, sock):
        self.sock = sock
        self.buf = b""

    def take(self, n):
        while len(self.buf) < n:
            chunk = self.sock.recv(1 << 16)
            if not chunk:
                raise ConnectionError("server closed the connection")
            self.buf += chunk
        out, self.buf = self.buf[:n], self.buf[n:]
        return out

    def i8(self):
        return struct.unpack(">b", self.take(1))[0]

    def i16(self):
        return struct.unpack(">h", self.take(2))[0]

    def i32(self):
        return struct.unpack(">i", self.take(4))[0]

    def dbl(self):
        return struct.unpack(">d", self.take(8))[0]

    def string(self):
        return self.take(self.i32())

    def value(self, t):
        if t == T_BOOL:
            return self.i8() != 0
        if t == T_I32:
            return self.i32()
        if t == T_DOUBLE:
            return self.dbl()
        if t == T_STRING:
            return self.string()
        if t == T_STRUCT:
            fields = {}
            while True:
                ft = self.i8()
                if ft == T_STOP:
                    return fields
                fid = self.i16()
                fields[fid] = self.value(ft)
        if t == T_LIST:
            et = self.i8()
            return [self.value(et) for _ in range(self.i32())]
        raise ValueError(f"unexpected type {t}")


def _s(v):
    b = v if isinstance(v, bytes) else v.encode()
    return struct.pack(">i", len(b)) + b


class QueryClient:
    def __init__(self, host, port, strict=True):
        self.sock = socket.create_connection((host, port))
        self.sock.setsockopt(socket.IPPROTO_TCP, socket.TCP_NODELAY, 1)
        self.reader = _Reader(self.sock)
        self.seq = 0
        self.strict = strict

    def close(self):
        self.sock.close()

    def _call(self, name, args):
        self.seq += 1
        if self.strict:
            msg = struct.pack(">i", -2147418112 | CALL) + _s(name) + struct.pack(">i", self.seq)
        else:
            msg = _s(name) + struct.pack(">bi", CALL, self.seq)
        self.sock.sendall(msg + args + bytes([T_STOP]))
        r = self.reader
        first = r.i32()
        if first < 0:
            mtype = first & 0xFF
            rname = r.string().decode()
        else:
            rname = r.take(first).decode()
            mtype = r.i8()
        seq = r.i32()
        assert seq == self.seq and rname == name
        result = r.value(T_STRUCT)
        if mtype == EXCEPTION:
            raise ApplicationException(result.get(1, b"").decode(), result.get(2))
        assert mtype == REPLY
        if 1 in result:
            raise QueryException(result[1].get(1, b"").decode())
        return result.get(0)

    @staticmethod
    def _entries(lst):
        return [{"id": e[1], "dist": e[2], "externId": e.get(3, b"").decode() if 3 in e else None,
                 "obj": e.get(4) if 4 in e else None} for e in lst]

    def setQueryTimeParams(self, params):
        self._call("setQueryTimeParams", bytes([T_STRING]) + struct.pack(">h", 1) + _s(params))

    def knnQuery(self, k, obj, retExternId=False, retObj=False):
        args = (bytes([T_I32]) + struct.pack(">hi", 1, k) + bytes([T_STRING]) + struct.pack(">h", 2) + _s(obj) +
                bytes([T_BOOL]) + struct.pack(">hb", 3, retExternId) + bytes([T_BOOL]) + struct.pack(">hb", 4, retObj))
        return self._entries(self._call("knnQuery", args))

    def knnQueryBatch(self, k, objs, retExternId=False, retObj=False, numThreads=4):
        lst = bytes([T_STRING]) + struct.pack(">i", len(objs)) + b"".join(_s(o) for o in objs)
        args = (bytes([T_I32]) + struct.pack(">hi", 1, k) + bytes([T_LIST]) + struct.pack(">h", 2) + lst +
                bytes([T_BOOL]) + struct.pack(">hb", 3, retExternId) + bytes([T_BOOL]) + struct.pack(">hb", 4, retObj) +
                bytes([T_I32]) + struct.pack(">hi", 5, numThreads))
        return [self._entries(x) for x in self._call("knnQueryBatch", args)]

    def rangeQuery(self, r, obj, retExternId=False, retObj=False):
        args = (bytes([T_DOUBLE]) + struct.pack(">hd", 1, r) + bytes([T_STRING]) + struct.pack(">h", 2) + _s(obj) +
                bytes([T_BOOL]) + struct.pack(">hb", 3, retExternId) + bytes([T_BOOL]) + struct.pack(">hb", 4, retObj))
        return self._entries(self._call("rangeQuery", args))

    def getDistance(self, a, b):
        args = bytes([T_STRING]) + struct.pack(">h", 1) + _s(a) + bytes([T_STRING]) + struct.pack(">h", 2) + _s(b)
        return self._call("getDistance", args)

    def call_unknown(self, name):
        return self._call(name, b"")
