"""The host BVH builder on the CPU (no GPU): its SAH-optimal 8-wide collapse
gives a tree that traversal can trust.  The builder's source is compiled with
a small dump program (tests/c_abi/bvh_host_dump.cpp) and the tree checked
with the structure rules of the device-builder tests: every node reached
once, every triangle in exactly one leaf slot and inside every slot box on
its path (decoded in FP32 as traversal decodes them), at most 32 levels;
and the collapse fills nodes with more than two children on average."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from test_bvh_gpu import check_tree, decode_nodes, tiny_soups

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def dump_tool(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    out = tmp_path_factory.mktemp("bvh") / "bvh_host_dump"
    src = ROOT / "raymond_b200" / "csrc"
    subprocess.run([cxx, "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-I", str(src),
                    str(ROOT / "tests" / "c_abi" / "bvh_host_dump.cpp"), str(src / "bvh_build.cpp"), "-o", str(out)],
                   check=True)
    return out


def build(tool, tmp_path, tris):
    inp = tmp_path / "in.f32"
    np.asarray(tris, np.float32).reshape(-1, 9).tofile(inp)
    subprocess.run([str(tool), str(inp), str(tmp_path / "nodes.bin"), str(tmp_path / "tris.bin")], check=True)
    nodes = np.fromfile(tmp_path / "nodes.bin", np.uint8).reshape(-1, 80)
    out = np.fromfile(tmp_path / "tris.bin", np.float32).reshape(-1, 12)
    return nodes, out


def slots_per_node(nodes):
    n = decode_nodes(nodes)
    used = (n["meta"] != 0) | ((n["imask"][:, None] >> np.arange(8)) & 1).astype(bool)
    return used.sum(axis=1)


@pytest.mark.parametrize("name", list(tiny_soups()))
def test_host_bvh_soups(dump_tool, tmp_path, name):
    v = tiny_soups()[name]
    nodes, tris = build(dump_tool, tmp_path, v)
    assert len(tris) == len(v)
    check_tree(nodes, tris)
    # the leaf-ordered triangles are the input's, each once (primitive index in v1.w)
    prims = np.sort(tris[:, 7].view(np.uint32))
    np.testing.assert_array_equal(prims, np.arange(len(v), dtype=np.uint32))


def test_host_bvh_fills_nodes(dump_tool, tmp_path):
    """On 20,000 random triangles the optimal collapse uses more than 4 of a
    node's 8 slots on average (a binary tree would use 2)."""
    rng = np.random.default_rng(11)
    c = rng.uniform(0, 10, (20000, 1, 3))
    v = c + rng.normal(0, 0.05, (20000, 3, 3))
    nodes, tris = build(dump_tool, tmp_path, v)
    depth = check_tree(nodes, tris)
    assert slots_per_node(nodes).mean() > 4.0
    assert depth <= 12
