"""Client of harmony_serve, speaking the reference's TCP protocol
(src/client.cpp, src/master_server.h:5-8): the same bytes the reference's
harmony_client sends, so either client works with either server.

    c = ServeClient("127.0.0.1", 7777)
    c.insert(x)            # [u8 1][u64 n][n*d f32] -> [u8 status]
    c.build_done()         # [u8 2] -> [u8 status]; the server then serves queries
    c.reconnect()          # the insert connection is closed after BUILD_DONE
    D, I = c.query(q, k)   # [u64 nq][u64 k][nq*d f32] -> [nq*k f32][nq*k i64]
    c.shutdown()           # [u64 0][u64 0]
"""
import socket
import struct
import time

import numpy as np

OP_SHUTDOWN, OP_INSERT, OP_BUILD_DONE = 0, 1, 2
STATUS_OK = 0


class ServeError(RuntimeError):
    pass


class ServeClient:
    def __init__(self, host="127.0.0.1", port=7777, timeout=600.0, retries=50):
        self.addr = (host, port)
        self.timeout = timeout
        self.retries = retries
        self.sock = None
        self.connect()

    def connect(self):
        """Connects, retrying while the server is not listening yet."""
        last = None
        for _ in range(self.retries):
            try:
                s = socket.create_connection(self.addr, timeout=self.timeout)
                s.setsockopt(socket.IPPROTO_TCP, socket.TCP_NODELAY, 1)
                self.sock = s
                return
            except OSError as e:
                last = e
                time.sleep(0.2)
        raise ServeError(f"cannot connect to {self.addr}: {last}")

    def reconnect(self):
        self.close()
        self.connect()

    def close(self):
        if self.sock is not None:
            self.sock.close()
            self.sock = None

    def _recv(self, n):
        buf = bytearray(n)
        view = memoryview(buf)
        got = 0
        while got < n:
            r = self.sock.recv_into(view[got:], n - got)
            if r == 0:
                raise ServeError("server closed the connection")
            got += r
        return bytes(buf)

    def _status(self, what):
        st = self._recv(1)[0]
        if st != STATUS_OK:
            raise ServeError(f"{what}: status {st}")

    def insert(self, x, batch=100_000):
        """OP_INSERT batches of float32 rows."""
        x = np.ascontiguousarray(x, np.float32)
        for s in range(0, x.shape[0], batch):
            part = x[s:s + batch]
            self.sock.sendall(struct.pack("<BQ", OP_INSERT, part.shape[0]) + part.tobytes())
            self._status("insert")

    def build_done(self):
        self.sock.sendall(struct.pack("<B", OP_BUILD_DONE))
        self._status("build")

    def query(self, q, k):
        q = np.ascontiguousarray(q, np.float32)
        nq = q.shape[0]
        self.sock.sendall(struct.pack("<QQ", nq, k) + q.tobytes())
        D = np.frombuffer(self._recv(nq * k * 4), np.float32).reshape(nq, k)
        I = np.frombuffer(self._recv(nq * k * 8), np.int64).reshape(nq, k)
        return D.copy(), I.copy()

    def shutdown(self):
        """Ends the query server (a header with nq = 0)."""
        self.sock.sendall(struct.pack("<QQ", 0, 0))
        self.close()
