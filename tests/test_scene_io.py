"""The persistent scene format (blazert_b200/csrc/scene_io.cpp) on the CPU, through the
emulator that links the same code: a scene written and read back has the same trees node for
node and answers rays and distance queries bit for bit as the original, re-encoding gives the
same bytes, and damaged or inconsistent data is refused with a reason (checksum, truncation,
magic, a tampered node box, a broken DFS link, a leaf list that is not a permutation)."""
import struct

import numpy as np
import pytest

from blazert_b200 import workloads as W
from tests.emu.emu import EmuScene
from tests.helpers import bits_equal
from tests.scenes import distance_queries, edge_case_scenes

KINDS = ("mesh", "spheres", "planes", "cylinders")


def fnv1a(b: bytes) -> int:
    h = 1469598103934665603
    for x in b:
        h = ((h ^ x) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def block_hash(b: bytes, block=1 << 20) -> int:
    """The version-2 hash: FNV-1a of each 2^20-byte block, then FNV-1a over the block hashes
    as little-endian u64."""
    return fnv1a(b"".join(struct.pack("<Q", fnv1a(b[i:i + block]))
                          for i in range(0, len(b), block)))


def reseal(body: bytes) -> bytes:
    """body (without the hash) followed by the hash its version field names: FNV-1a over the
    whole body for version 1, the block hash otherwise."""
    version = struct.unpack_from("<I", body, 8)[0] if len(body) >= 12 else 0
    return body + struct.pack("<Q", fnv1a(body) if version == 1 else block_hash(body))


def _scenes():
    out = [("mixed", W.mixed_primitives(n_rays=3000, n_spheres=700, n_cylinders=150, n_planes=40,
                                        seed=8)),
           ("icosphere", W.icosphere_pinhole(n_rays=4000)),
           ("adjoint", W.adjoint_scene(n_rays=3000))]
    out += [(name, W.Workload(name, spec, R, {})) for name, spec, R in edge_case_scenes()]
    return out


def same_trees(a, b, spec):
    for kind in spec.order:
        ta, tb = a.tree(kind), b.tree(kind)
        for key in ("leaf", "axis", "children", "prim_cnt", "prim_ids", "bmin", "bmax"):
            if not np.array_equal(np.asarray(ta[key]).view(np.uint8), np.asarray(tb[key]).view(np.uint8)):
                return f"{kind}: {key}"
    return None


@pytest.mark.parametrize("name,wl", _scenes(), ids=lambda x: x if isinstance(x, str) else "")
def test_round_trip(name, wl):
    spec, R = wl.scene, wl.rays
    a = EmuScene(spec)
    data = a.encode()
    b = EmuScene.decode(data)
    assert same_trees(a, b, spec) is None
    assert b.encode() == data
    ra = a.intersect(R.origins, R.directions, R.tmin, R.tmax)
    rb = b.intersect(R.origins, R.directions, R.tmin, R.tmax)
    for k in ("t", "uv", "normal", "prim", "geom", "hit"):
        assert np.array_equal(np.asarray(ra[k]).view(np.uint8), np.asarray(rb[k]).view(np.uint8)), k
    rng = np.random.default_rng(3)
    for kind in spec.order:
        ids, pts = distance_queries(spec, kind, rng, 500)
        assert bits_equal(a.distance_to_surface(kind, ids, pts)[0], b.distance_to_surface(kind, ids, pts)[0])


def test_build_options_and_deep_trees_round_trip():
    n = 90
    c = np.stack([2.0 ** np.arange(n), np.zeros(n), np.zeros(n)], 1)
    spec = W.SceneSpec().add_spheres(c, np.full(n, 0.25)).add_mesh(*W.icosphere(2))
    for kw in (dict(min_leaf=1, max_depth=200, bins=2), dict(min_leaf=8, max_depth=3, bins=16)):
        a = EmuScene(spec, **kw)
        b = EmuScene.decode(a.encode())
        assert same_trees(a, b, spec) is None
        assert b.encode() == a.encode()


def _spheres_file(n=5):
    rng = np.random.default_rng(1)
    spec = W.SceneSpec().add_spheres(rng.uniform(-5, 5, (n, 3)), rng.uniform(0.1, 1, n))
    return EmuScene(spec, min_leaf=1).encode(), n


def test_damaged_data_is_refused():
    data, n = _spheres_file()
    bad = bytearray(data)
    bad[40] ^= 1
    with pytest.raises(ValueError, match="checksum"):
        EmuScene.decode(bytes(bad))
    with pytest.raises(ValueError):
        EmuScene.decode(data[:-20])
    with pytest.raises(ValueError, match="not a scene file"):
        EmuScene.decode(b"XXXXXXXX" + data[8:])
    with pytest.raises(ValueError):
        EmuScene.decode(b"")
    with pytest.raises(ValueError, match="version"):
        EmuScene.decode(reseal(data[:8] + struct.pack("<I", 3) + data[12:-8]))


def test_hash_is_the_block_hash_and_version_1_files_still_load():
    """Files are written as version 2 with the block hash (blocks of 2^20 bytes, so a scene of
    a few MB spans several); a version-1 file, the same bytes hashed with one FNV-1a over the
    whole body, loads to the same scene, which is written back as version 2."""
    spec = W.adjoint_scene(n_rays=16).scene
    a = EmuScene(spec)
    data = a.encode()
    body = data[:-8]
    assert len(body) > 3 << 20
    assert struct.unpack_from("<I", body, 8)[0] == 2
    assert struct.unpack("<Q", data[-8:])[0] == block_hash(body)
    v1 = reseal(body[:8] + struct.pack("<I", 1) + body[12:])
    b = EmuScene.decode(v1)
    assert same_trees(a, b, spec) is None
    assert b.encode() == data
    with pytest.raises(ValueError, match="checksum"):
        EmuScene.decode(v1[:-8] + data[-8:])  # version 1 with a version-2 hash


def test_inconsistent_trees_are_refused():
    data, n = _spheres_file()
    body = bytearray(data[:-8])
    node0 = 8 + 4 + 12 + 4 + 16 + 32 * n + 8  # first node record (72 bytes each)
    # a node box that is not the union of its primitives' boxes
    b = bytearray(body)
    struct.pack_into("<d", b, node0, struct.unpack_from("<d", b, node0)[0] - 1.0)
    with pytest.raises(ValueError, match="box"):
        EmuScene.decode(reseal(bytes(b)))
    # the root's right child moved off the DFS pre-order
    b = bytearray(body)
    c1 = struct.unpack_from("<I", b, node0 + 48 + 12)[0]
    struct.pack_into("<I", b, node0 + 48 + 12, c1 + 1)
    with pytest.raises(ValueError, match="DFS|outside"):
        EmuScene.decode(reseal(bytes(b)))
    # a leaf list that repeats a primitive
    nn = struct.unpack_from("<Q", body, node0 - 8)[0]
    leaves = node0 + 72 * nn + 8
    b = bytearray(body)
    struct.pack_into("<I", b, leaves, struct.unpack_from("<I", b, leaves + 4)[0])
    with pytest.raises(ValueError, match="permutation"):
        EmuScene.decode(reseal(bytes(b)))
    # a face index outside the vertices
    v, f = W.icosphere(1)
    mdata = EmuScene(W.SceneSpec().add_mesh(v, f)).encode()
    mb = bytearray(mdata[:-8])
    at = 8 + 4 + 12 + 4 + 16 + 8 + 24 * len(v)
    struct.pack_into("<I", mb, at, len(v) + 5)
    with pytest.raises(ValueError, match="face index"):
        EmuScene.decode(reseal(bytes(mb)))


@pytest.mark.parametrize("seed", range(4))
def test_fuzzed_files_are_refused_or_safe(seed):
    """Random byte changes, insertions and cuts, with the checksum recomputed so that the
    parser goes past it: every result is a refusal with a reason or a scene whose trees passed
    the checks and that traces rays without a bounds error."""
    rng = np.random.default_rng(seed)
    wl = W.mixed_primitives(n_rays=64, n_spheres=40, n_cylinders=12, n_planes=6, seed=seed)
    spec = W.SceneSpec()
    spec.add_mesh(*W.icosphere(1))
    for kind in wl.scene.order:
        getattr(spec, "add_" + kind)(*getattr(wl.scene, kind).values())
    body = EmuScene(spec, min_leaf=2).encode()[:-8]
    refused = loaded = 0
    for _ in range(150):
        b = bytearray(body)
        op = rng.integers(3)
        if op == 0:
            for _ in range(int(rng.integers(1, 4))):
                b[int(rng.integers(len(b)))] = int(rng.integers(256))
        elif op == 1:
            at = int(rng.integers(len(b)))
            b[at:at] = bytes(rng.integers(0, 256, int(rng.integers(1, 16)), dtype=np.uint8))
        else:
            del b[int(rng.integers(len(b))):]
        try:
            s = EmuScene.decode(reseal(bytes(b)))
        except ValueError as e:
            assert str(e)
            refused += 1
            continue
        loaded += 1
        R = wl.rays
        out = s.intersect(R.origins, R.directions)
        assert out["error_word"] == 0
    assert refused > 0
