"""A program written against the reference's C++ API (BVHGPUBuilder,
OnesweepSort, intersect_stackfree / intersect_escape_link called from the
caller's own kernel), compiled against include/minimum_lbvh.h and linked
with libmlbvh_b200.so, gives the oracle's tree and hits bit for bit."""
import os
import subprocess

import numpy as np
import pytest

import _oracle as O
from minimumlbvh_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "_build")


def compile_drop_in():
    os.makedirs(BUILD, exist_ok=True)
    exe = os.path.join(BUILD, "drop_in")
    lib = os.path.join(ROOT, "minimumlbvh_b200")
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "-fmad=false",
                    "-I", os.path.join(ROOT, "include"), "-o", exe, os.path.join(ROOT, "tests", "cpp", "drop_in.cu"),
                    "-L", lib, "-lmlbvh_b200", "-Xlinker", "-rpath," + lib], check=True, capture_output=True)
    return exe


def compile_cpu_builder():
    """tests/cpp/cpu_builder.cpp: host-only C++ (g++), linked with the library
    and cudart."""
    os.makedirs(BUILD, exist_ok=True)
    exe = os.path.join(BUILD, "cpu_builder")
    lib = os.path.join(ROOT, "minimumlbvh_b200")
    cuda = "/usr/local/cuda"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", cuda + "/include", "-o",
                    exe, os.path.join(ROOT, "tests", "cpp", "cpu_builder.cpp"), "-L", lib, "-lmlbvh_b200",
                    "-Wl,-rpath," + lib, "-L", cuda + "/lib64", "-lcudart", "-Wl,-rpath," + cuda + "/lib64"],
                   check=True, capture_output=True)
    return exe


def test_cpu_builder_program_compiles():
    """A program written against the reference's BVHCPUBuilder (build when
    empty, validate, read m_internals on the host: main.cpp:246-249) compiles
    and links unchanged against include/minimum_lbvh.h."""
    assert os.path.exists(compile_cpu_builder())


def test_header_compiles_host_only(tmp_path):
    """include/minimum_lbvh.h is usable from a plain C++ translation unit."""
    src = tmp_path / "host.cpp"
    src.write_text('#include "minimum_lbvh.h"\nint main() { minimum_lbvh::Hit h; return h.triangleIndex == 0xFFFFFFFFu ? 0 : 1; }\n')
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), "-I",
                    "/usr/local/cuda/include", str(src)], check=True)


@pytest.mark.gpu
def test_drop_in_program(cuda, tmp_path):
    exe = compile_drop_in()
    tris = scenes.heightfield_icospheres(seed=3, quads=64, spheres=16, level=2)
    rays = scenes.random_rays(20000, tris.reshape(-1, 3).min(0), tris.reshape(-1, 3).max(0), seed=5)
    rays[::2, 7] = 0.2
    (tmp_path / "t.bin").write_bytes(tris.tobytes())
    (tmp_path / "r.bin").write_bytes(rays.tobytes())
    subprocess.run([exe, str(tmp_path / "t.bin"), str(tmp_path / "r.bin"), str(tmp_path / "o.bin")], check=True)
    out = np.frombuffer((tmp_path / "o.bin").read_bytes(), dtype=np.uint32)
    n, m = len(tris), len(rays)
    ref = O.build(tris)
    assert int(out[0]) == ref["root"]
    nodes = out[1:1 + 16 * (n - 1)].reshape(n - 1, 16)
    np.testing.assert_array_equal(nodes, ref["nodes"])
    hits = out[1 + 16 * (n - 1):1 + 16 * (n - 1) + 8 * m].reshape(m, 8)
    anyh = out[1 + 16 * (n - 1) + 8 * m:].reshape(m, 8)
    exp = O.trace(ref["nodes"], tris, ref["root"], rays, 0, 0)
    cols = [0, 2, 3, 4, 5, 6, 7]  # the Hit padding word is not written by the reference's code either
    np.testing.assert_array_equal(hits[:, cols], exp[:, cols])
    exp_any = O.trace(ref["nodes"], tris, ref["root"], rays, 1, 1)
    np.testing.assert_array_equal(anyh[:, cols], exp_any[:, cols])


@pytest.mark.gpu
def test_drop_in_program_ploc(cuda, tmp_path):
    """The same program with the tree from BVHGPUBuilder::buildByPLOC
    (radius 8): the oracle's PLOC tree and the oracle's Hit records over it
    from the caller's own kernel."""
    exe = compile_drop_in()
    tris = scenes.heightfield_icospheres(seed=3, quads=64, spheres=16, level=2)
    rays = scenes.random_rays(20000, tris.reshape(-1, 3).min(0), tris.reshape(-1, 3).max(0), seed=5)
    (tmp_path / "t.bin").write_bytes(tris.tobytes())
    (tmp_path / "r.bin").write_bytes(rays.tobytes())
    subprocess.run([exe, str(tmp_path / "t.bin"), str(tmp_path / "r.bin"), str(tmp_path / "o.bin"), "8"], check=True)
    out = np.frombuffer((tmp_path / "o.bin").read_bytes(), dtype=np.uint32)
    n, m = len(tris), len(rays)
    ref = O.build_ploc(tris, 0, 8)
    assert int(out[0]) == ref["root"]
    np.testing.assert_array_equal(out[1:1 + 16 * (n - 1)].reshape(n - 1, 16), ref["nodes"])
    hits = out[1 + 16 * (n - 1):1 + 16 * (n - 1) + 8 * m].reshape(m, 8)
    exp = O.trace(ref["nodes"], tris, ref["root"], rays, 0, 0)
    cols = [0, 2, 3, 4, 5, 6, 7]
    np.testing.assert_array_equal(hits[:, cols], exp[:, cols])


@pytest.mark.gpu
@pytest.mark.parametrize("option", [2, 1])
def test_cpu_builder_program(cuda, tmp_path, option):
    """BVHCPUBuilder's host vectors (nodes, deltas, root) are the oracle's
    tree; its validate() passes and a host walk over m_internals reaches every
    leaf. Option 2 is BUILD_OPTION_CPU_PARALLEL (no effect here), 1 normal keys."""
    exe = compile_cpu_builder()
    tris = scenes.heightfield_icospheres(seed=4, quads=64, spheres=16, level=2)
    (tmp_path / "t.bin").write_bytes(tris.tobytes())
    subprocess.run([exe, str(tmp_path / "t.bin"), str(tmp_path / "o.bin"), str(option)], check=True)
    raw = (tmp_path / "o.bin").read_bytes()
    n = len(tris)
    ref = O.build(tris, option & 1)
    root = int(np.frombuffer(raw[:4], np.uint32)[0])
    nodes = np.frombuffer(raw[4:4 + 64 * (n - 1)], np.uint32).reshape(n - 1, 16)
    deltas = np.frombuffer(raw[4 + 64 * (n - 1):4 + 65 * (n - 1)], np.uint8)
    leaves = int(np.frombuffer(raw[-4:], np.uint32)[0])
    assert root == ref["root"]
    np.testing.assert_array_equal(nodes, ref["nodes"])
    np.testing.assert_array_equal(deltas, ref["deltas"])
    assert leaves == n


@pytest.mark.gpu
@pytest.mark.parametrize("ploc", [0, 8])
def test_drop_in_status_reports_timeout(cuda, tmp_path, ploc):
    """BVHGPUBuilder::status makes a bounded wait that gave up visible to a C++
    caller: with one-poll waits (mlbvh_set_spin_limit) at least one of three
    builds of a million triangles reports MLBVH_ERR_TIMEOUT, and the next
    build with the default limit is the oracle's tree, with the oracle's hits
    from the caller's kernel."""
    import re
    exe = compile_drop_in()
    tris = scenes.gaussian_soup(1 << 20, clusters=16, seed=31)
    rays = scenes.random_rays(4096, tris.reshape(-1, 3).min(0), tris.reshape(-1, 3).max(0), seed=6)
    (tmp_path / "t.bin").write_bytes(tris.tobytes())
    (tmp_path / "r.bin").write_bytes(rays.tobytes())
    r = subprocess.run([exe, str(tmp_path / "t.bin"), str(tmp_path / "r.bin"), str(tmp_path / "o.bin"), str(ploc),
                        "timeout"], check=True, capture_output=True, text=True)
    m_ = re.search(r"(\d) of 3 builds", r.stdout)
    assert m_ and int(m_.group(1)) >= 1, r.stdout
    out = np.frombuffer((tmp_path / "o.bin").read_bytes(), dtype=np.uint32)
    n, m = len(tris), len(rays)
    ref = O.build_ploc(tris, 0, ploc) if ploc else O.build(tris)
    assert int(out[0]) == ref["root"]
    np.testing.assert_array_equal(out[1:1 + 16 * (n - 1)].reshape(n - 1, 16), ref["nodes"])
    hits = out[1 + 16 * (n - 1):1 + 16 * (n - 1) + 8 * m].reshape(m, 8)
    exp = O.trace(ref["nodes"], tris, ref["root"], rays, 0, 0)
    cols = [0, 2, 3, 4, 5, 6, 7]
    np.testing.assert_array_equal(hits[:, cols], exp[:, cols])
