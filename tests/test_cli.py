"""The `wos` command line against the reference's own launcher (src/main.cpp,
compiled with its one-rank MPI shim as oracle/_ref/wos_ref): the same exit
codes, messages and overwrite protection on every path that ends before a
solve.  CPU only: none of these runs reaches the GPU."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

from walk_on_spheres_b200 import meshes

ROOT = Path(__file__).resolve().parents[1]
WOS = ROOT / "walk_on_spheres_b200" / "bin" / "wos"
REF = ROOT / "oracle" / "_ref" / "wos_ref"


def _run(binary: Path, args: list[str], cwd: Path) -> subprocess.CompletedProcess:
    return subprocess.run([str(binary)] + args, capture_output=True, text=True, cwd=cwd,
                          timeout=60)


@pytest.fixture(scope="module")
def ref_cli():
    if not REF.exists():
        pytest.skip("oracle/_ref is not built (the reference sources are not on this machine)")
    return REF


def test_cli_is_built():
    assert WOS.exists(), "walk_on_spheres_b200/bin/wos is built with the library"


# argument vectors that end before a solve; a fixed seed keeps stdout comparable
FAILING = [
    ["--walks"], ["--walks", "0"], ["--walks", "12x"], ["--walks", "99999999999"],
    ["--seed"], ["--seed", "-1"], ["--seed", "18446744073709551616"], ["--seed", "0x10"],
    ["--epsilon", "0"], ["--epsilon", "nan"], ["--epsilon", "inf"], ["--epsilon", " 1"],
    ["--epsilon", "1e999"], ["--max-steps", "0"], ["--max-ray-attempts", "2"],
    ["--alpha", "-1"], ["--alpha"], ["--source-mode", "mis"], ["--source-mode"],
    ["--output"], ["--bogus"], ["-x"],
    ["--seed", "1", "laplace", "16"],
    ["--seed", "1", "laplace", "a", "b"],
    ["--seed", "1", "laplace", "0", "4"],
    ["--seed", "1", "laplace", "4", "4", "x", "y.obj"],
    ["--seed", "1", "a", "1", "2", "3", "4", "5"],
    ["--seed", "1", "nosuch"],
    ["--seed", "1", "nosuch", "4", "4"],
    ["--seed", "1", "laplace", "4", "4", "missing.obj"],
    ["--seed", "1", "laplace", "4", "4", "4", "missing.obj"],
    ["--seed", "1", "--alpha", "3", "laplace", "4", "4", "missing.obj"],
    ["--seed", "1", "--source-mode", "green", "helmholtz", "4", "4", "missing.obj"],
]


@pytest.mark.parametrize("args", FAILING, ids=[" ".join(a) or "none" for a in FAILING])
def test_failing_arguments_match_reference(tmp_path, ref_cli, args):
    a = _run(WOS, args, tmp_path)
    b = _run(ref_cli, args, tmp_path)
    assert a.returncode == b.returncode == 1
    assert a.stderr and a.stderr == b.stderr
    if "--seed" in args and "1" in args:
        assert a.stdout == b.stdout


def test_overwrite_protection_matches_reference(tmp_path, ref_cli):
    (tmp_path / "taken.h5").write_bytes(b"x")
    args = ["--seed", "5", "-o", "taken.h5", "laplace", "4", "4", "missing.obj"]
    a, b = _run(WOS, args, tmp_path), _run(ref_cli, args, tmp_path)
    assert a.returncode == b.returncode == 1
    assert a.stderr == b.stderr and "Refusing to overwrite" in a.stderr
    assert (tmp_path / "taken.h5").read_bytes() == b"x"
    # --force goes on to the mesh (which is missing here)
    args = ["--force"] + args
    a, b = _run(WOS, args, tmp_path), _run(ref_cli, args, tmp_path)
    assert a.returncode == b.returncode == 1 and a.stderr == b.stderr


def test_bad_mesh_messages_match_reference(tmp_path, ref_cli):
    (tmp_path / "bad.obj").write_text("v 0 0 0\nq 1 2\n")
    (tmp_path / "empty.obj").write_text("")
    for mesh in ("bad.obj", "empty.obj", "."):
        args = ["--seed", "2", "poisson", "4", "4", mesh]
        a, b = _run(WOS, args, tmp_path), _run(ref_cli, args, tmp_path)
        assert a.returncode == b.returncode == 1, mesh
        assert a.stderr == b.stderr, mesh


def test_help_contains_the_reference_help(tmp_path, ref_cli):
    a, b = _run(WOS, ["--help"], tmp_path), _run(ref_cli, ["-h"], tmp_path)
    assert a.returncode == b.returncode == 0
    ours = a.stdout.replace(str(WOS), "PROG").splitlines()
    theirs = b.stdout.replace(str(ref_cli), "PROG").splitlines()
    it = iter(ours)
    assert all(line in it for line in theirs), "reference help lines missing or out of order"
    assert any("--method" in line for line in ours)


def test_generated_seed_line(tmp_path, ref_cli):
    a = _run(WOS, ["nosuch"], tmp_path)
    b = _run(ref_cli, ["nosuch"], tmp_path)
    assert a.returncode == b.returncode == 1
    for r in (a, b):
        assert r.stdout.startswith("Random seed: ")
        assert r.stdout.rstrip().endswith("(generated from current time)")


def test_mesh_dimension_peek(tmp_path):
    """wos_peek_mesh_dim: 2 for `l` records, 3 for `f` records (src/mesh.cpp:51-74)."""
    from walk_on_spheres_b200 import peek_mesh_dim
    p2 = meshes.write_obj(meshes.annulus(segments=8), tmp_path / "a.obj")
    p3 = meshes.write_obj(meshes.uv_sphere(lon=8, lat=4), tmp_path / "s.obj")
    assert peek_mesh_dim(str(p2)) == 2 and peek_mesh_dim(str(p3)) == 3
