"""Checkpoints, snapshots and trajectories in the reference's HDF5 layouts
(src/checkpoint.jl, src/io.jl) written and read by libbsn's own HDF5 code,
on host arrays (no GPU).  The files are checked twice: round trips through
the library's reader, and an independent walk of the HDF5 structures in this
file (superblock v2, version-2 object headers with their lookup3 checksums,
link / attribute / dataspace / datatype / layout messages) against the
reference's group, dataset and attribute names and shapes."""
import os
import struct
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "binary-supernova_b200"))
NG = 3


def lookup3(data: bytes, init: int = 0) -> int:
    """Bob Jenkins' lookup3 hashlittle (the HDF5 metadata checksum)."""
    M = 0xFFFFFFFF
    rot = lambda x, k: ((x << k) | (x >> (32 - k))) & M
    n = len(data)
    a = b = c = (0xDEADBEEF + n + init) & M
    i = 0
    w = lambda j: int.from_bytes(data[j:j + 4].ljust(4, b"\0"), "little")
    while n > 12:
        a, b, c = (a + w(i)) & M, (b + w(i + 4)) & M, (c + w(i + 8)) & M
        a = (a - c) & M; a ^= rot(c, 4); c = (c + b) & M
        b = (b - a) & M; b ^= rot(a, 6); a = (a + c) & M
        c = (c - b) & M; c ^= rot(b, 8); b = (b + a) & M
        a = (a - c) & M; a ^= rot(c, 16); c = (c + b) & M
        b = (b - a) & M; b ^= rot(a, 19); a = (a + c) & M
        c = (c - b) & M; c ^= rot(b, 4); b = (b + a) & M
        n -= 12
        i += 12
    if n == 0:
        return c
    tail = data[i:i + n] + bytes(12 - n)
    a = (a + int.from_bytes(tail[0:4], "little")) & M
    b = (b + int.from_bytes(tail[4:8], "little")) & M
    c = (c + int.from_bytes(tail[8:12], "little")) & M
    c ^= b; c = (c - rot(b, 14)) & M
    a ^= c; a = (a - rot(c, 11)) & M
    b ^= a; b = (b - rot(a, 25)) & M
    c ^= b; c = (c - rot(b, 16)) & M
    a ^= c; a = (a - rot(c, 4)) & M
    b ^= a; b = (b - rot(a, 14)) & M
    c ^= b; c = (c - rot(b, 24)) & M
    return c


def test_lookup3_known_answers():
    # the test vectors published with lookup3.c
    assert lookup3(b"") == 0xDEADBEEF
    assert lookup3(b"Four score and seven years ago") == 0x17770551
    assert lookup3(b"Four score and seven years ago", 1) == 0xCD628161


def walk(path):
    """Independent reader of the version-2 structures: {name: node}, node =
    ('group', attrs, children) or ('dataset', attrs, dims, kind, addr, size)."""
    raw = open(path, "rb").read()
    assert raw[:8] == b"\x89HDF\r\n\x1a\n"
    assert raw[8] == 2 and raw[9] == 8 and raw[10] == 8
    assert struct.unpack_from("<I", raw, 44)[0] == lookup3(raw[:44])
    base, ext, eof, root = struct.unpack_from("<QQQQ", raw, 12)
    assert base == 0 and ext == 2 ** 64 - 1 and eof == len(raw)

    def dtype(b, o):
        cls = b[o] & 0x0F
        size = struct.unpack_from("<I", b, o + 4)[0]
        return {0: "i64", 1: "f64", 3: "str"}[cls], size

    def space(b, o):
        ver, rank = b[o], b[o + 1]
        assert ver == 2
        return [struct.unpack_from("<Q", b, o + 4 + 8 * k)[0] for k in range(rank)]

    def obj(addr):
        assert raw[addr:addr + 4] == b"OHDR" and raw[addr + 4] == 2
        flags = raw[addr + 5]
        assert flags & 3 == 2 and not flags & 0x34
        chunk = struct.unpack_from("<I", raw, addr + 6)[0]
        end = addr + 10 + chunk
        assert struct.unpack_from("<I", raw, end)[0] == lookup3(raw[addr:end])
        o, attrs, links, layout, dims, kind = addr + 10, {}, {}, None, None, None
        while o < end:
            t, sz, _ = raw[o], struct.unpack_from("<H", raw, o + 1)[0], raw[o + 3]
            b = o + 4
            if t == 0x06:
                assert raw[b] == 1 and raw[b + 1] == 0
                ln = raw[b + 2]
                links[raw[b + 3:b + 3 + ln].decode()] = struct.unpack_from("<Q", raw, b + 3 + ln)[0]
            elif t == 0x0C:
                assert raw[b] == 3
                ns, ts, ss = struct.unpack_from("<HHH", raw, b + 2)
                name = raw[b + 9:b + 9 + ns - 1].decode()
                k, size = dtype(raw, b + 9 + ns)
                assert space(raw, b + 9 + ns + ts) == []
                d = b + 9 + ns + ts + ss
                attrs[name] = {"f64": lambda: struct.unpack_from("<d", raw, d)[0],
                               "i64": lambda: struct.unpack_from("<q", raw, d)[0],
                               "str": lambda: raw[d:d + size].split(b"\0")[0].decode()}[k]()
            elif t == 0x01:
                dims = space(raw, b)
            elif t == 0x03:
                kind = dtype(raw, b)
            elif t == 0x08:
                assert raw[b] == 3 and raw[b + 1] == 1
                layout = struct.unpack_from("<QQ", raw, b + 2)
            o = b + sz
        assert o == end
        if layout is not None:
            return ("dataset", attrs, dims, kind, layout[0], layout[1])
        return ("group", attrs, {n: obj(a) for n, a in links.items()})

    return raw, obj(root)


def data_of(raw, node):
    _, _, dims, kind, addr, size = node
    assert kind == ("f64", 8) and size == 8 * int(np.prod(dims))
    return np.frombuffer(raw, dtype="<f8", count=size // 8, offset=addr)


@pytest.fixture(scope="module")
def bsn():
    import bsn
    return bsn


def _state(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal((5, nx + 2 * NG, ny + 2 * NG, nz + 2 * NG)))


def _bhs(bsn):
    return [bsn.BlackHole((1.5, 0.25, -0.125), (0.0, 0.9128709, 0.01), 5.0, 0.0625, 1e6, 0.125),
            bsn.BlackHole((-1.5, -0.25, 0.0), (0.0, -0.9128709, 0.0), 4.75, 0.0625, 1e6, 0.125)]


GRID = dict(nx=6, ny=5, nz=4, dx=0.5, dy=0.25, dz=0.125, gamma=4 / 3, x0=-1.5, y0=-0.625, z0=-0.25,
            rho_floor=1e-8, P_floor=1e-10)
META = dict(t=0.5907709947988187, step=1000, dt_last=5.2e-4, t_snap=0.5, t_bh2_sink_on=0.0125)


def test_uniform_checkpoint_round_trip_and_layout(bsn, tmp_path):
    U = _state(6, 5, 4, 1)
    p = tmp_path / "ckpt.h5"
    bsn.save_checkpoint_uniform(p, U, _bhs(bsn), **META, **GRID)
    V, bhs, grid, meta = bsn.load_checkpoint_uniform(p, device="cpu")
    assert np.array_equal(U, V) and V.flags.f_contiguous
    assert grid == GRID
    assert {k: meta[k] for k in META} == META and meta["format_version"] == 1
    for a, b in zip(bhs, _bhs(bsn)):
        assert list(a.pos) == list(b.pos) and list(a.vel) == list(b.vel)
        assert (a.mass, a.eps, a.c_code, a.r_floor) == (b.mass, b.eps, b.c_code, b.r_floor)
    # the reference's layout, read by the independent walker
    raw, root = walk(p)
    g = root[2]
    assert set(g) == {"manifest", "grid", "bhs"}
    man = g["manifest"][1]
    assert man == {"format_version": 1, "kind": "uniform", **META}
    grid_attrs = g["grid"][1]
    assert grid_attrs == GRID
    Unode = g["grid"][2]["U"]
    assert Unode[2] == [4 + 2 * NG, 5 + 2 * NG, 6 + 2 * NG, 5]   # HDF5 order of Julia (5, nx+6, ny+6, nz+6)
    assert np.array_equal(data_of(raw, Unode), U.ravel(order="F"))
    b = g["bhs"]
    assert b[1] == {"n": 2}
    assert b[2]["pos"][2] == [2, 3] and b[2]["mass"][2] == [2]   # Julia (3, n) and (n,)
    assert list(data_of(raw, b[2]["pos"])) == [1.5, 0.25, -0.125, -1.5, -0.25, 0.0]
    assert list(data_of(raw, b[2]["mass"])) == [5.0, 4.75]


def test_checkpoint_rejections(bsn, tmp_path):
    U = _state(6, 5, 4, 2)
    p = tmp_path / "c.h5"
    bsn.save_checkpoint_uniform(p, U, [], **META, **GRID)
    _, bhs, _, _ = bsn.load_checkpoint_uniform(p, device="cpu")
    assert bhs == []
    raw = bytearray(open(p, "rb").read())
    # a flipped byte inside an object header fails its checksum
    bad = bytearray(raw)
    bad[60] ^= 0x40
    q = tmp_path / "bad.h5"
    q.write_bytes(bytes(bad))
    with pytest.raises(bsn.BSNError):
        bsn.load_checkpoint_uniform(q, device="cpu")
    # not HDF5 at all
    r = tmp_path / "not.h5"
    r.write_bytes(b"plain text, not a checkpoint")
    with pytest.raises(bsn.BSNError):
        bsn.load_checkpoint_uniform(r, device="cpu")
    # a snapshot is not a checkpoint
    s = tmp_path / "snap.h5"
    bsn.write_snapshot(s, U, 6, 5, 4, 0.5, 0.25, 0.125, 0.1, 5 / 3)
    with pytest.raises(bsn.BSNError):
        bsn.load_checkpoint_uniform(s, device="cpu")


def test_snapshot_round_trip_and_layout(bsn, tmp_path):
    U = _state(6, 5, 4, 3)
    p = tmp_path / "snap_0001.h5"
    bsn.write_snapshot(p, U, 6, 5, 4, 0.5, 0.25, 0.125, 0.375, 5 / 3)
    A, nx, ny, nz, dx, dy, dz, t, g = bsn.read_snapshot(p)
    assert (nx, ny, nz, dx, dy, dz, t, g) == (6, 5, 4, 0.5, 0.25, 0.125, 0.375, 5 / 3)
    assert np.array_equal(A, U[:, NG:-NG, NG:-NG, NG:-NG])
    raw, root = walk(p)
    assert root[1] == dict(t=0.375, nx=6, ny=5, nz=4, dx=0.5, dy=0.25, dz=0.125, gamma=5 / 3)
    gas = root[2]["gas"][2]
    assert set(gas) == {"rho", "rhovx", "rhovy", "rhovz", "E"}
    for q, name in enumerate(["rho", "rhovx", "rhovy", "rhovz", "E"]):
        assert gas[name][2] == [4, 5, 6]
        assert np.array_equal(data_of(raw, gas[name]), U[q, NG:-NG, NG:-NG, NG:-NG].ravel(order="F"))


def test_trajectory_records(bsn, tmp_path):
    p = tmp_path / "traj.h5"
    bsn.init_trajectory_file(p, 2)
    t0, rec0 = bsn.read_trajectory(p)
    assert len(t0) == 0 and len(rec0) == 2
    bhs = _bhs(bsn)
    for k in range(3):
        bhs[0].pos[0] += 0.1
        bhs[1].mass += 0.25
        bsn.append_trajectory(p, 0.1 * k, bhs)
    t, rec = bsn.read_trajectory(p)
    assert list(t) == [0.0, 0.1, 0.2]
    assert list(rec[1]["mass"]) == [5.0, 5.25, 5.5]
    assert rec[0]["pos"].shape == (3, 3) and list(rec[0]["pos"][:, 0]) == [1.6, 1.7000000000000002, 1.8000000000000003]
    assert list(rec[0]["rsink"]) == [0.125] * 3       # r_sink = max(6 M / c^2, r_floor)
    raw, root = walk(p)
    assert set(root[2]) == {"time", "bh1", "bh2"}
    assert root[2]["bh1"][2]["pos"][2] == [3, 3]        # Julia (N, 3)


# ---- the reference's own checkpoint tests (test/test_checkpoint.jl), restated


def _fmr_host(bsn, U_c, U_f):
    """bsn_fmr2 over host arrays: 8^3 coarse, dx 1/8, refined box 4:5 in every
    axis at ratio 4 (8^3 fine), gamma 5/3, outflow, floors 1e-12."""
    from bsn._lib import bsn_fmr2
    import ctypes as C
    return bsn_fmr2(C.c_void_p(U_c.ctypes.data), 8, 8, 8, 1 / 8, 1 / 8, 1 / 8, C.c_void_p(U_f.ctypes.data), 8, 8, 8,
                    1 / 32, 1 / 32, 1 / 32, 4, 4, 5, 4, 5, 4, 5, 5 / 3, 0, 1e-12, 1e-12)


def test_reference_checkpoint_round_trip_fmr_grid_and_bhs(bsn, tmp_path):
    """"Checkpoint round-trip: FMR grid + BHs" (test/test_checkpoint.jl:4-67)
    and "Checkpoint with empty BH list" (:69-82): every field bit for bit,
    the fine level as saved."""
    import ctypes as C
    g = 5 / 3
    Uc = np.zeros((5, 14, 14, 14), order="F")
    for k in range(NG, NG + 8):
        for j in range(NG, NG + 8):
            for i in range(NG, NG + 8):
                xc, yc, zc = ((i - NG + 0.5) / 8 - 0.5, (j - NG + 0.5) / 8 - 0.5, (k - NG + 0.5) / 8 - 0.5)
                Uc[0, i, j, k] = 1.0 + 0.1 * (xc * xc + yc * yc + zc * zc)
                Uc[4, i, j, k] = 1.0 / (g - 1.0)
    Uf = np.asfortranarray(np.random.default_rng(8).random((5, 14, 14, 14)) * 1.01)
    G = _fmr_host(bsn, Uc, Uf)
    bhs = [bsn.BlackHole((-0.5, 0.0, 0.0), (0.0, -0.5, 0.0), 0.5, 1e-3, 1431.6, 1e-3),
           bsn.BlackHole((0.5, 0.1, 0.0), (0.0, 0.5, 0.0), 0.5, 1e-3, 1431.6, 1e-3)]
    L = bsn._lib.load()
    p = str(tmp_path / "ckpt.h5").encode()
    assert L.bsn_save_checkpoint_fmr(None, p, C.byref(G), 0, bsn.api._bh_array(bhs), 2, 0.25, 42, 0.001) == 0
    Vc, Vf = np.zeros_like(Uc, order="F"), np.zeros_like(Uf, order="F")
    H = _fmr_host(bsn, Vc, Vf)
    for f in ("ratio", "ci_lo", "gamma", "rho_floor", "ncx", "nfx", "dxc", "dxf"):
        setattr(H, f, 0)
    arr = (bsn._lib.bsn_bh * 2)()
    nb, t, step, dtl = C.c_int(), C.c_double(), C.c_longlong(), C.c_double()
    assert L.bsn_load_checkpoint_fmr(None, p, C.byref(H), 0, arr, 2, C.byref(nb), C.byref(t), C.byref(step),
                                     C.byref(dtl)) == 0
    assert (t.value, step.value, dtl.value, nb.value) == (0.25, 42, 0.001, 2)
    for f, _ in G._fields_:
        if f not in ("Uc", "Uf"):
            assert getattr(H, f) == getattr(G, f), f
    assert np.array_equal(Vc, Uc) and np.array_equal(Vf, Uf)
    for b, b2 in zip(bhs, arr):
        assert list(b2.pos) == list(b.pos) and list(b2.vel) == list(b.vel)
        assert (b2.mass, b2.eps, b2.c_code, b2.r_floor) == (b.mass, b.eps, b.c_code, b.r_floor)
    # empty BH list, default t / step
    q = str(tmp_path / "ckpt_empty.h5").encode()
    assert L.bsn_save_checkpoint_fmr(None, q, C.byref(G), 0, None, 0, 0.0, 0, 0.0) == 0
    assert L.bsn_load_checkpoint_fmr(None, q, C.byref(H), 0, arr, 2, C.byref(nb), C.byref(t), C.byref(step),
                                     C.byref(dtl)) == 0
    assert (nb.value, t.value, step.value) == (0, 0.0, 0)
    # the two checkpoint kinds are not cross-loadable (test/test_checkpoint.jl:139-140)
    with pytest.raises(bsn.BSNError):
        bsn.load_checkpoint_uniform(q.decode(), device="cpu")


def test_reference_uniform_checkpoint_round_trip(bsn, tmp_path):
    """"Uniform checkpoint round-trip: U + BHs + meta" (test/test_checkpoint.jl:86-141)."""
    import ctypes as C
    nx = ny = nz = 6
    U = np.asfortranarray((0.5 + 1.0e-3 * np.arange(1, 5 * 12 ** 3 + 1)).reshape((5, 12, 12, 12), order="F"))
    bhs = [bsn.BlackHole((-0.3, 0.0, 0.0), (0.0, -0.7, 0.0), 0.6, 2e-3, 1431.6, 2e-3),
           bsn.BlackHole((0.3, 0.05, -0.1), (0.01, 0.7, 0.0), 0.4, 2e-3, 1431.6, 2e-3)]
    p = tmp_path / "ckpt_uniform.h5"
    bsn.save_checkpoint_uniform(p, U, bhs, t=7.5, step=12345, dt_last=2.5e-3, t_snap=8.0, t_bh2_sink_on=5.0,
                                nx=nx, ny=ny, nz=nz, dx=0.2, dy=0.2, dz=0.2, gamma=4 / 3, x0=-1.0, y0=-1.0, z0=-1.0,
                                rho_floor=3e-4, P_floor=1e-5)
    U2, bhs2, grid, meta = bsn.load_checkpoint_uniform(p, device="cpu")
    assert U2.shape == U.shape and np.array_equal(U2, U)
    assert (meta["t"], meta["step"], meta["dt_last"], meta["t_snap"], meta["t_bh2_sink_on"]) == \
        (7.5, 12345, 2.5e-3, 8.0, 5.0)
    assert meta["format_version"] == 1
    assert (grid["nx"], grid["ny"], grid["nz"], grid["dx"], grid["gamma"]) == (6, 6, 6, 0.2, 4 / 3)
    assert (grid["x0"], grid["y0"], grid["z0"], grid["rho_floor"], grid["P_floor"]) == (-1.0, -1.0, -1.0, 3e-4, 1e-5)
    for b, b2 in zip(bhs, bhs2):
        assert list(b2.pos) == list(b.pos) and list(b2.vel) == list(b.vel)
        assert (b2.mass, b2.eps, b2.c_code, b2.r_floor) == (b.mass, b.eps, b.c_code, b.r_floor)
    # the FMR loader on a uniform file fails
    L = bsn._lib.load()
    H = _fmr_host(bsn, np.zeros((5, 14, 14, 14), order="F"), np.zeros((5, 14, 14, 14), order="F"))
    nb, t, step, dtl = C.c_int(), C.c_double(), C.c_longlong(), C.c_double()
    assert L.bsn_load_checkpoint_fmr(None, str(p).encode(), C.byref(H), 0, None, 0, C.byref(nb), C.byref(t),
                                     C.byref(step), C.byref(dtl)) == 7
