"""Network front end and write-ahead log (rg_frontend_*, rg_wal_*): the
reference's ClientUpdateRequest / ClientUpdateResponse structs
(core/rpc.hpp:19-38) over TCP, the clock-sync handshake of
src/all_inc_rpc.cpp:277-290, and the 4 KB group-commit log blocks of
src/all_inc_rpc.cpp:306-335.  The CPU test reads a log written by hand in the
documented format; the GPU test serves updates from socket clients, checks the
responses, the values against the oracle, and that replaying the log on a
fresh graph gives the same values."""
import socket
import struct
import time

import numpy as np
import pytest

import risgraph_b200 as rg
from risgraph_b200 import gen

from helpers import gpu_graph, oracle_graph

REQ = rg.CLIENT_REQUEST_DTYPE
RESP = rg.CLIENT_RESPONSE_DTYPE


def write_block(f, version, records):
    blk = bytearray(4096)
    struct.pack_into("<QQ", blk, 0, version, len(records))
    rec = np.array(records, dtype=rg.WAL_RECORD_DTYPE)
    blk[16:16 + rec.nbytes] = rec.tobytes()
    f.write(bytes(blk))


def test_wal_read_follows_the_block_format(tmp_path):
    """Blocks 1 and 2 are read in order; block 3 carries the wrong version, so
    reading stops there (the log ends at the first block out of sequence)."""
    p = str(tmp_path / "wal")
    a = [(0, 1, 5, 6, 7), (1, 2, 8, 9, 10)]
    b = [(0, 3, 11, 12, 1 << 40)] * 127
    with open(p, "wb") as f:
        write_block(f, 1, a)
        write_block(f, 2, b)
        write_block(f, 7, [(0, 4, 1, 2, 3)])
    got = rg.wal_read(p)
    assert len(got) == 2 + 127
    np.testing.assert_array_equal(got[:2], np.array(a, dtype=rg.WAL_RECORD_DTYPE))
    assert (got["data"][2:] == 1 << 40).all()


class Client:
    """A socket client speaking the reference's wire structs."""

    def __init__(self, port):
        self.s = socket.create_connection(("127.0.0.1", port))
        self.s.setsockopt(socket.IPPROTO_TCP, socket.TCP_NODELAY, 1)
        self.s.settimeout(120)

    def send(self, reqs):
        self.s.sendall(np.ascontiguousarray(reqs, dtype=REQ).tobytes())

    def recv(self, n):
        buf = b""
        while len(buf) < n * RESP.itemsize:
            chunk = self.s.recv(n * RESP.itemsize - len(buf))
            assert chunk, "connection closed early"
            buf += chunk
        return np.frombuffer(buf, dtype=RESP)

    def close(self):
        self.s.close()


def requests(client_id, kinds, edges):
    r = np.zeros(len(kinds), REQ)
    r["client_id"] = client_id
    r["type"] = kinds
    r["src"], r["dst"], r["data"] = edges["src"], edges["dst"], edges["data"]
    r["request_time_ns"] = time.time_ns()
    return r


@pytest.mark.gpu
@pytest.mark.parametrize("use_wal", [True, False])
def test_frontend_serves_reference_clients(tmp_path, use_wal):
    scale = 12
    pairs = gen.rmat(scale, seed=81)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    root = gen.max_out_degree_vertex(pairs, V)
    g = gpu_graph("sssp", V, pairs[:imported], hint=len(pairs), inc_mode=True)
    g.build_tree("sssp", root)
    e = gen.edges_with_weights(pairs, True)
    n = 2000                                     # updates per connection
    wal = str(tmp_path / "wal") if use_wal else None
    with rg.Server(max_epoch=512) as srv:
        k = srv.attach(g)
        fe = rg.Frontend(srv, k, wal_path=wal, sync_requests=16)
        c1 = Client(fe.port)
        # clock synchronisation on the first connection: 16 requests, each answered {0, 0}
        for _ in range(16):
            c1.send(requests(0, [2], np.zeros(1, rg.EDGE_DTYPE)))
            z = c1.recv(1)
            assert z["client_id"][0] == 0 and z["version_id"][0] == 0
        c2 = Client(fe.port)
        # connection 1: clients 1 and 2 alternate; connection 2: client 3 (inserts, then deletes)
        adds1, dels1 = e[imported:imported + n // 2], e[:n // 2]
        ed = np.zeros(n, rg.EDGE_DTYPE)
        ed[0::2], ed[1::2] = adds1, dels1
        r1 = requests(1, np.tile([0, 1], n // 2), ed)
        r1["client_id"][1::2] = 2
        adds2, dels2 = e[imported + n // 2:imported + n], e[n // 2:n]
        r2 = requests(3, np.r_[np.zeros(n // 2, np.uint32), np.ones(n // 2, np.uint32)], np.r_[adds2, dels2])
        bad = requests(4, [0], np.array([(V, 1, 1)], rg.EDGE_DTYPE))  # vertex id out of range
        c1.send(r1)
        c2.send(np.r_[r2, bad])
        got1, got2 = c1.recv(n), c2.recv(n + 1)
        # responses come back in request order, one per update, with versions that never decrease
        np.testing.assert_array_equal(got1["client_id"], r1["client_id"])
        np.testing.assert_array_equal(got2["client_id"][:n], r2["client_id"])
        assert (np.diff(got1["version_id"].astype(np.int64)) >= 0).all()
        assert got2["version_id"][n] == np.iinfo(np.uint64).max   # refused, never applied
        # End: answered after the client's updates
        c1.send(requests(1, [2], np.zeros(1, rg.EDGE_DTYPE)))
        end = c1.recv(1)
        assert end["client_id"][0] == 1 and end["version_id"][0] >= got1["version_id"].max()
        c1.close()
        c2.close()
        st = fe.stats()
        fe.stop()
        srv.detach(k)
    assert st["sync_requests"] == 16 and st["updates"] == 2 * n + 1 and st["failed"] == 1
    assert st["connections"] == 2 and st["p99_us"] > 0
    # values: the loaded window, minus the deleted, plus the inserted edges
    final = np.concatenate([pairs[n:imported], pairs[imported:imported + n]])
    og = oracle_graph("sssp", V, final)
    og.build_tree(root)
    served = g.values()
    np.testing.assert_array_equal(served, og.labels()[0])
    if use_wal:
        assert st["wal_blocks"] >= 2 * n // 127
        recs = rg.wal_read(wal)
        assert len(recs) == 2 * n                      # the refused update is not logged
        assert (recs["src"] < V).all()
        # replay on a fresh graph with the same initial load gives the served values
        h = gpu_graph("sssp", V, pairs[:imported], hint=len(pairs), inc_mode=True)
        h.build_tree("sssp", root)
        assert rg.wal_replay(h, "sssp", wal) == 2 * n
        np.testing.assert_array_equal(h.values(), served)
        h.close()
    g.close()
