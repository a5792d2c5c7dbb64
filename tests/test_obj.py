"""Mesh ingestion (bzr_obj_load, blazert_b200/csrc/obj.cpp) against the reference's own OBJ path
-- its vendored tiny_obj_loader 0.9.14 with the scene_mesh example's assembly, compiled here as
oracle/_ref/libref_obj.so -- bit for bit on vertices and faces: index forms (i, i/j, i//k,
i/j/k, negative), polygons, shapes ended by g and o, vertices duplicated per (v, vt, vn) triple,
the loader's number grammar and its float rounding, comments, CRLF, tabs, ignored statements;
plus seeded random files.  Runs on the CPU (the loader is host code)."""
import os

import numpy as np
import pytest

import blazert_b200 as B
from oracle.oracle import ref_load_obj

HAVE_REF = os.path.exists(os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref",
                                       "libref_obj.so"))
needs_ref = pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref/libref_obj.so not built")

HANDWRITTEN = {
    "cube_quads": """# a cube of quads with texcoords and normals
mtllib cube.mtl
o cube
v -1 -1 -1
v 1 -1 -1
v 1 1 -1
v -1 1 -1
v -1 -1 1
v 1 -1 1
v 1 1 1
v -1 1 1
vt 0 0
vt 1 0
vt 1 1
vn 0 0 -1
vn 0 0 1
usemtl red
f 1/1/1 2/2/1 3/3/1 4/1/1
f 5/1/2 8/2/2 7/3/2 6/1/2
f 1//1 5//1 6//1 2//1
f 2/1 6/2 7/3 3/2
f 3 7 8 4
f -8 -4 -1 -5
""",
    "groups_and_relative": "v 0 0 0\r\nv 1 0 0\r\nv 0 1 0\r\ng first\r\nf 1 2 3\r\n"
                           "v 0 0 1\r\n\tv\t1\t0\t1\r\nv 0 1 1\r\ng second extra\r\nf -3 -2 -1\r\n"
                           "f 1 2 3\r\no third\r\nf 4 5 6 1 2\r\n",
    "numbers": "v 1e3 -0.0E-3 +3.1417e+2\nv .5 1. -7\nv 123456789.123456789 1e-40 3.4e39\n"
               "v 0.1 0.2 0.3\nv 1e 2 3\nv -1.5e-3x 7 8\nf 1 2 3\nf 2 3 4 5 6\n",
    "same_position_other_attributes": "v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 1\nvn 0 0 -1\nvt 0 0\n"
                                      "f 1//1 2//1 3//1\nf 1//2 3//2 2//2\nf 1/1 2/1 3/1\nf 1 2 3\n",
    "degenerate_faces_and_blank_lines": "\n\n# nothing yet\nv 0 0 0\nv 1 1 1\nv 2 2 2\nf 1 2\n"
                                        "   \nf 1 2 3\ng\nf 3 2 1\n",
}


def _write(tmp_path, name, text):
    p = tmp_path / f"{name}.obj"
    p.write_bytes(text.encode())
    return p


@needs_ref
@pytest.mark.parametrize("name", sorted(HANDWRITTEN))
def test_handwritten_files(tmp_path, name):
    p = _write(tmp_path, name, HANDWRITTEN[name])
    v, f = B.load_obj(p)
    rv, rf = ref_load_obj(p)
    assert v.shape == rv.shape and f.shape == rf.shape
    assert np.array_equal(v.view(np.uint64), rv.view(np.uint64))
    assert np.array_equal(f, rf)


def _random_obj(rng):
    lines, nv, nvt, nvn = [], 0, 0, 0
    fmt = ["{:.17g}", "{:.6f}", "{:.3e}", "{:+.9g}", "{:g}"]
    for _ in range(int(rng.integers(3, 9))):
        for _ in range(int(rng.integers(3, 40))):
            x = rng.normal(scale=10.0 ** int(rng.integers(-3, 4)), size=3)
            lines.append("v " + " ".join(fmt[int(rng.integers(len(fmt)))].format(c) for c in x))
            nv += 1
        for _ in range(int(rng.integers(0, 5))):
            lines.append("vn 0 0 1")
            nvn += 1
            lines.append("vt 0.5 0.5")
            nvt += 1
        for _ in range(int(rng.integers(1, 30))):
            k = int(rng.integers(3, 7))
            corners = []
            for _ in range(k):
                i = int(rng.integers(1, nv + 1))
                ref = str(i) if rng.random() < 0.7 else str(i - nv - 1)  # absolute or relative
                form = int(rng.integers(4))
                if form == 1 and nvt:
                    ref += f"/{int(rng.integers(1, nvt + 1))}"
                elif form == 2 and nvn:
                    ref += f"//{int(rng.integers(1, nvn + 1))}"
                elif form == 3 and nvt and nvn:
                    ref += f"/{int(rng.integers(1, nvt + 1))}/{int(rng.integers(1, nvn + 1))}"
                corners.append(ref)
            lines.append("f " + " ".join(corners))
        lines.append(["g part", "o obj", "usemtl m", "s 1", "# c"][int(rng.integers(5))])
    return "\n".join(lines) + "\n"


@needs_ref
@pytest.mark.parametrize("seed", range(12))
def test_random_files(tmp_path, seed):
    p = _write(tmp_path, f"r{seed}", _random_obj(np.random.default_rng(seed)))
    v, f = B.load_obj(p)
    rv, rf = ref_load_obj(p)
    assert np.array_equal(v.view(np.uint64), rv.view(np.uint64)) and np.array_equal(f, rf)


def test_errors(tmp_path):
    with pytest.raises(B.BlazertError) as e:
        B.load_obj(tmp_path / "missing.obj")
    assert e.value.code == B.EINVAL
    p = _write(tmp_path, "bad_index", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 9\n")
    with pytest.raises(B.BlazertError, match="face index"):
        B.load_obj(p)
    v, f = B.load_obj(_write(tmp_path, "empty", "# no geometry\n"))
    assert v.shape == (0, 3) and f.shape == (0, 3)


@pytest.mark.parametrize("seed", range(3))
def test_fuzzed_files_load_or_are_refused(tmp_path, seed):
    """Random edits of valid files (bytes replaced, inserted, lines cut): every one either
    loads, with faces inside the vertices, or is refused with BZR_EINVAL; never a crash.
    Where the reference's loader accepts the same file without an out-of-range index, the
    meshes are equal."""
    rng = np.random.default_rng(100 + seed)
    base = _random_obj(np.random.default_rng(seed)).encode()
    alphabet = np.frombuffer(b"0123456789 -+./eEvfgot\\n#\\t\\r", np.uint8)
    for k in range(60):
        b = bytearray(base)
        for _ in range(int(rng.integers(1, 6))):
            at = int(rng.integers(len(b)))
            if rng.random() < 0.5:
                b[at] = int(alphabet[rng.integers(len(alphabet))])
            else:
                b[at:at] = bytes(alphabet[rng.integers(0, len(alphabet), int(rng.integers(1, 8)))])
        p = tmp_path / f"f{k}.obj"
        p.write_bytes(bytes(b))
        try:
            v, f = B.load_obj(p)
        except B.BlazertError as e:
            assert e.code == B.EINVAL
            continue
        assert f.size == 0 or int(f.max()) < len(v)
        if HAVE_REF:
            rv, rf = ref_load_obj(p)
            assert np.array_equal(v.view(np.uint64), rv.view(np.uint64)) and np.array_equal(f, rf)
