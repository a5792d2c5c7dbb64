"""The C-ABI library: it loads, exports every function include/blazert_b200.h declares, and keeps
the reference's add/commit state rules (blazert/scene.h:227-346) without touching a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import blazert_b200 as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(bzr_[A-Za-z0-9_]+)\s*\(", text, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = B.library()
    names = declared_functions()
    assert "bzr_intersectN" in names and "bzr_commit" in names
    for n in names:
        assert hasattr(lib, n), n


def test_add_rules_without_gpu():
    s = B.Scene()
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float64)
    f = np.array([[0, 1, 2]], np.uint32)
    assert s.add_mesh(v, f) == 0
    assert s.add_mesh(v, f) == B.INVALID_ID  # second add of a kind
    assert s.add_spheres(np.zeros((1, 3)), np.ones(1)) == 1
    assert s.add_cylinders(np.zeros((1, 3)), np.ones(1), np.ones(1), np.ones(1), np.eye(3)[None]) == 2
    assert s.add_planes(np.zeros((1, 3)), np.ones(1), np.ones(1), np.eye(3)[None]) == 3
    s.close()


def test_errors_are_reported():
    s = B.Scene()
    with pytest.raises(B.BlazertError) as e:
        s.add_mesh(np.zeros((3, 3)), np.array([[0, 1, 5]], np.uint32))  # index out of range
    assert e.value.code == B.EINVAL
    with pytest.raises(B.BlazertError) as e:  # query before commit
        s.intersectN(np.zeros((1, 3)), np.ones((1, 3)))
    assert e.value.code == B.ESTATE
    lib = B.library()
    assert lib.bzr_add_spheres(None, None, None, 0, None) == B.EINVAL
    s.close()


def test_commit_without_device_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    s = B.Scene()
    s.add_spheres(np.zeros((1, 3)), np.ones(1))
    with pytest.raises(B.BlazertError) as e:
        s.commit()
    assert e.value.code == B.ENODEV
    s.close()


FACADE_APP = r"""
#include <blazert_b200/scene.hpp>
#include <cstdio>
using namespace blazert_b200;

int main(int argc, char **) {
  // reference-style call sites (blazert/scene.h, blazert/ray.h)
  Vec3rList<double> centers{{0.0, 0.0, 0.0}, {3.0, 0.0, 0.0}};
  std::vector<double> radii{1.0, 0.5};
  Vec3rList<double> vertices{{0.0, 0.0, 2.0}, {1.0, 0.0, 2.0}, {0.0, 1.0, 2.0}};
  Vec3iList triangles{{0, 1, 2}};
  Mat3rList<double> rot{Mat3r<double>::identity()};
  Scene<double> scene;
  const unsigned mesh_id = scene.add_mesh(vertices, triangles);
  const unsigned sph_id = scene.add_spheres(centers, radii);
  scene.add_cylinders(Vec3rList<double>{{0.0, 5.0, 0.0}}, {0.5}, {0.5}, {2.0}, rot);
  scene.add_planes(Vec3rList<double>{{0.0, -5.0, 0.0}}, {2.0}, {2.0}, rot);
  if (scene.add_spheres(centers, radii) != static_cast<unsigned>(-1)) return 2;
  if (argc > 1) {  // needs a GPU
    scene.commit();
    Ray<double> ray{{0.2, 0.2, 5.0}, {0.0, 0.0, -1.0}};
    Ray<double> shadow{{0.2, 0.2, 5.0}, {0.0, 0.0, -1.0}, 0.0, 10.0,
                       Ray<double>::CullBackFace::no, Ray<double>::AnyHit::yes};
    RayHit<double> rh, rh2;
    const bool hit = intersect1(scene, ray, rh);
    const bool hit2 = intersect1(scene, shadow, rh2);
    std::printf("%d %u %u %.17g %d\n", hit, rh.geom_id, rh.prim_id, rh.hit_distance, hit2);
  }
  return mesh_id == 0 && sph_id == 1 ? 0 : 1;
}
"""


EMBREE_APP = r"""
#include <blazert_b200/embree_scene.hpp>
#include <cstdio>
using namespace blazert_b200;

int main(int argc, char **argv) {
  // call sites written for the reference's Embree backend (blazert/embree/scene.h)
  EmbreeScene<float> fs;
  EmbreeScene<double> ds;
  const unsigned a = fs.add_spheres(Vec3rList<float>{{0.f, 0.f, 0.f}, {3.f, 0.f, 0.f}}, {1.f, 0.5f});
  const unsigned b = ds.add_spheres(Vec3rList<double>{{0.0, 0.0, 0.0}, {3.0, 0.0, 0.0}}, {1.0, 0.5});
  if (a != 0 || b != 0) return 1;
  Scene<float> sf;  // the reference's float call sites (blazert::Scene<float>)
  if (sf.add_spheres(Vec3rList<float>{{0.f, 0.f, 0.f}}, {1.f}) != 0) return 1;
  if (argc > 1) {  // needs a GPU; argv[1]: a scene file to write
    fs.commit();
    ds.commit();
    Ray<float> rf{{3.f, 0.f, 5.f}, {0.f, 0.f, -1.f}};
    RayHit<float> hf;
    const bool h1 = intersect1(fs, rf, hf);
    Ray<double> rd{{3.0, 0.0, 5.0}, {0.0, 0.0, -1.0}};
    RayHit<double> hd;
    const bool h2 = intersect1(ds, rd, hd);
    const std::vector<uint32_t> ids{0, 1};
    const std::vector<double> pts{0.0, 0.0, 3.0, 3.0, 0.0, 3.0};
    std::vector<double> dist(2);
    ds.blazertscene.distance_to_surface(1, 2, ids.data(), pts.data(), dist.data());
    ds.blazertscene.save(argv[1]);
    auto loaded = Scene<double>::load(argv[1]);
    RayHit<double> h3;
    const bool h3hit = intersect1(*loaded, rd, h3);
    sf.commit();
    RayHit<float> hs;
    const bool h4 = intersect1(sf, Ray<float>{{0.f, 0.f, 5.f}, {0.f, 0.f, -1.f}}, hs);
    std::printf("%d %u %.9g %d %u %.17g %.17g %.17g %d %.17g %d %.9g\n", h1, hf.prim_id,
                hf.hit_distance, h2, hd.prim_id, hd.hit_distance, dist[0], dist[1], h3hit,
                h3.hit_distance, h4, hs.hit_distance);
  }
  return 0;
}
"""


def _compile(src_text, tmp_path, name):
    import subprocess

    src = tmp_path / f"{name}.cpp"
    src.write_text(src_text)
    exe = tmp_path / name
    lib = os.path.join(ROOT, "blazert_b200", "_lib")
    cxx = os.environ.get("BZR_CXX", "g++")
    subprocess.run([cxx, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src),
                    "-L", lib, "-lblazert_b200", f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True)
    return exe


def test_embree_facade_compiles_and_links(tmp_path):
    """include/blazert_b200/embree_scene.hpp: EmbreeScene<float> / <double> call sites, the
    distance and save/load members compile and link; the add rules run without a GPU."""
    import subprocess

    subprocess.run([str(_compile(EMBREE_APP, tmp_path, "embree_app"))], check=True)


def test_cpp_facade_compiles_links_and_keeps_add_rules(tmp_path):
    """include/blazert_b200/scene.hpp: reference-style C++ (Scene<double>, add_*, Ray with the
    reference's CullBackFace / AnyHit enums, RayHit, intersect1) compiles against the header,
    links against the library, and runs the add rules without a GPU."""
    import subprocess

    src = tmp_path / "app.cpp"
    src.write_text(FACADE_APP)
    exe = tmp_path / "app"
    lib = os.path.join(ROOT, "blazert_b200", "_lib")
    cxx = os.environ.get("BZR_CXX", "g++")
    subprocess.run([cxx, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src),
                    "-L", lib, "-lblazert_b200", f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True)
    subprocess.run([str(exe)], check=True)


C_APP = r"""
#include "blazert_b200.h"
#include <stdio.h>

int main(void) {
  bzr_scene *s = NULL;
  uint32_t gid = 0;
  const double c[3] = {0.0, 0.0, 0.0}, r[1] = {1.0};
  if (bzr_scene_create(&s) != BZR_OK) return 1;
  if (bzr_add_spheres(s, c, r, 1, &gid) != BZR_OK || gid != 0) return 2;
  if (bzr_add_spheres(s, c, r, 1, &gid) != BZR_ESTATE || gid != BZR_INVALID_ID) return 3;
  /* queries before commit are refused with a reason */
  double d = 0.0;
  const uint32_t id = 0;
  if (bzr_distance_to_surface(s, 1, 1, &id, c, &d, NULL, NULL) != BZR_ESTATE) return 4;
  if (bzr_scene_serialize(s, NULL, 0) != BZR_ESTATE) return 5;
  if (bzr_last_error_string()[0] == 0) return 6;
  bzr_scene_destroy(s);
  return 0;
}
"""


def test_c_header_compiles_as_c_and_headers_are_warning_free(tmp_path):
    """include/blazert_b200.h is plain C (C99, -Wall -Wextra -Werror) and the C++ facade
    headers compile without warnings; the C program runs the add and state rules without a
    GPU."""
    import subprocess

    lib = os.path.join(ROOT, "blazert_b200", "_lib")
    inc = os.path.join(ROOT, "include")
    src = tmp_path / "app.c"
    src.write_text(C_APP)
    exe = tmp_path / "app_c"
    subprocess.run([os.environ.get("BZR_CC", "gcc"), "-std=c99", "-Wall", "-Wextra", "-Werror",
                    "-pedantic", "-I", inc,
                    str(src), "-L", lib, "-lblazert_b200", f"-Wl,-rpath,{lib}", "-o", str(exe)],
                   check=True)
    subprocess.run([str(exe)], check=True)
    cpp = tmp_path / "headers.cpp"
    cpp.write_text("#include <blazert_b200/scene.hpp>\n#include <blazert_b200/embree_scene.hpp>\n"
                   "#include <sstream>\n"
                   "int main() { blazert_b200::Scene<double> a; blazert_b200::Scene<float> b;"
                   " blazert_b200::EmbreeScene<float> c; (void)a; (void)b; (void)c;"
                   " std::ostringstream o; o << blazert_b200::Ray<double>{{0, 0, 0}, {1, 2, -2}}"
                   " << blazert_b200::RayHit<float>{};"
                   " blazert_b200::BVHBuildStatistics<double> st = a.handle() ? a.build_statistics(1)"
                   " : blazert_b200::BVHBuildStatistics<double>{}; (void)st;"
                   " return o.str().empty(); }\n")
    subprocess.run([os.environ.get("BZR_CXX", "g++"), "-std=c++17", "-Wall", "-Wextra", "-Werror",
                    "-fsyntax-only", "-I", inc, str(cpp)], check=True)


def test_python_inputs_are_checked_not_reshaped():
    """Arrays whose rows do not hold 3 values (9 for rotations) are refused instead of being
    silently reshaped; flat arrays and one 3 x 3 rotation are accepted; shape mismatches between
    arrays and out-of-range faces are reported."""
    import numpy as np

    import blazert_b200 as B

    with pytest.raises(ValueError):
        B.Scene().add_spheres(np.zeros((6, 2)), np.ones(4))  # would reshape to 4 x 3
    with pytest.raises(ValueError):
        B.Scene().add_planes(np.zeros((2, 3)), np.ones(2), np.ones(2), np.zeros((2, 3, 2)))
    with pytest.raises(ValueError):
        B.Scene().add_mesh(np.zeros(7), np.zeros((1, 3), np.uint32))
    with pytest.raises(B.BlazertError):
        B.Scene().add_spheres(np.zeros((3, 3)), np.ones(2))
    with pytest.raises(B.BlazertError):
        B.Scene().add_mesh(np.zeros((4, 3)), np.array([[0, 1, 9]], np.uint32))
    assert B.Scene().add_spheres(np.zeros(6), np.ones(2)) == 0  # flat centres
    assert B.Scene().add_cylinders(np.zeros((1, 3)), [1.0], [1.0], [2.0], np.eye(3)) == 0
    assert B.Scene().add_planes(np.zeros((2, 3)), [1.0, 1.0], [1.0, 1.0], np.zeros((2, 9))) == 0


def test_scene_file_reading_without_gpu(tmp_path):
    """bzr_scene_load reads the whole file (in one read, or in pieces from a pipe) and checks it
    before the commit, which is the step that needs a device: a valid file gets as far as
    BZR_ENODEV here, a damaged, empty or missing one is refused with its reason."""
    import threading

    from blazert_b200 import workloads as W
    from tests.emu.emu import EmuScene

    lib = B.library()
    lib.bzr_scene_load.argtypes = [C.POINTER(C.c_void_p), C.c_char_p]
    lib.bzr_last_error_string.restype = C.c_char_p
    data = EmuScene(W.mixed_primitives(n_rays=16).scene).encode()

    def load(path):
        out = C.c_void_p()
        rc = lib.bzr_scene_load(C.byref(out), str(path).encode())
        assert not out.value
        return rc, lib.bzr_last_error_string().decode()

    good = tmp_path / "good.bzrscene"
    good.write_bytes(data)
    assert load(good)[0] == B.ENODEV
    bad = tmp_path / "bad.bzrscene"
    bad.write_bytes(data[:100] + bytes([data[100] ^ 1]) + data[101:])
    assert load(bad)[0] == B.EINVAL and "checksum" in load(bad)[1]
    empty = tmp_path / "empty.bzrscene"
    empty.write_bytes(b"")
    assert load(empty)[0] == B.EINVAL and "empty" in load(empty)[1]
    assert load(tmp_path / "missing.bzrscene")[0] == B.EINVAL
    if hasattr(os, "mkfifo"):
        fifo = tmp_path / "pipe.bzrscene"
        os.mkfifo(fifo)
        writer = threading.Thread(target=lambda: fifo.write_bytes(data))
        writer.start()
        assert load(fifo)[0] == B.ENODEV
        writer.join(timeout=60)
