"""PLY reading and writing (src/ply.rs) and the `poisson-recon` command (src/main.rs).  The
library's PLY code is host-only: these tests need no GPU, except the end-to-end CLI run."""
import os
import struct
import subprocess

import numpy as np
import pytest

import poissonreconstruction_b200 as prb
from poissonreconstruction_b200 import synthetic

HEADER = ("ply\nformat ascii 1.0\nelement vertex {nv}\nproperty float x\nproperty float y\nproperty float z\n"
          "element face {nf}\nproperty list uchar int vertex_indices\nend_header\n")


def rust_display(x):
    """Rust's `{}` for a finite f64: shortest round-trip digits, positional, no exponent."""
    return np.format_float_positional(x, unique=True, trim="-")


def crate_mesh_text(v, t):
    """The bytes ply::write_mesh (src/ply.rs:73-107) writes."""
    out = [HEADER.format(nv=len(v), nf=len(t))]
    out += ["%s %s %s\n" % tuple(rust_display(c) for c in row) for row in v]
    out += ["3 %d %d %d\n" % tuple(int(c) for c in row) for row in t]
    return "".join(out).encode()


def test_ascii_writer_matches_the_crate_byte_for_byte(tmp_path):
    rng = np.random.default_rng(3)
    special = [0.0, -0.0, 1.0, -1.0, 0.1, 1e-7, 1e21, 123456789.125, 5e-324, 1.7976931348623157e308,
               0.30000000000000004, 2.5e-310, -3.14159265358979, 1e16, 9007199254740993.0]
    v = np.concatenate([np.array(special[:15]).reshape(5, 3), rng.normal(size=(3000, 3)) * 10.0 ** rng.integers(
        -12, 12, size=(3000, 1))])
    t = rng.integers(0, len(v), size=(5000, 3)).astype(np.uint64)
    t[0] = [2 ** 40, 0, 7]
    path = tmp_path / "m.ply"
    prb.write_ply(path, prb.Mesh(v, t))
    assert path.read_bytes() == crate_mesh_text(v, t)


def test_empty_mesh_writes_a_header_only(tmp_path):
    path = tmp_path / "e.ply"
    prb.write_ply(path, prb.Mesh(np.zeros((0, 3)), np.zeros((0, 3), np.uint64)))
    assert path.read_bytes() == HEADER.format(nv=0, nf=0).encode()


def test_binary_writer_round_trips(tmp_path):
    rng = np.random.default_rng(4)
    v, t = rng.normal(size=(1000, 3)), rng.integers(0, 1000, size=(1500, 3)).astype(np.uint64)
    path = tmp_path / "b.ply"
    prb.write_ply(path, prb.Mesh(v, t), binary=True)
    data = path.read_bytes()
    head, body = data.split(b"end_header\n", 1)
    assert b"format binary_little_endian 1.0" in head and b"element vertex 1000" in head
    assert np.array_equal(np.frombuffer(body[:24000], "<f8").reshape(-1, 3), v)
    faces = np.frombuffer(body[24000:], dtype=[("n", "u1"), ("i", "<u4", 3)])
    assert (faces["n"] == 3).all() and np.array_equal(faces["i"], t)


def _write(path, text):
    path.write_bytes(text.encode() if isinstance(text, str) else text)
    return path


POINT_HEADER = ("ply\nformat ascii 1.0\nelement vertex {n}\nproperty float x\nproperty float y\nproperty float z\n"
                "property float nx\nproperty float ny\nproperty float nz\nend_header\n")


def test_ascii_reader_follows_the_crate(tmp_path):
    """src/ply.rs:47-67: lines with < 6 tokens are skipped, unparsable tokens read as 0.0, extra
    tokens ignored, and every line after the header counts (not just `element vertex` lines)."""
    body = ("1 2 3 0 0 1\n"
            "short line\n"
            "\n"
            "  4.5\t-5e-1 +6 1e400 -inf NaN 99 100\r\n"
            "7 abc 9 0x10 1. .5\n"
            "3 0 1 2 4 5\n")
    pts = prb.read_ply(_write(tmp_path / "p.ply", POINT_HEADER.format(n=2) + body))
    expect = np.array([[1, 2, 3, 0, 0, 1], [4.5, -0.5, 6, np.inf, -np.inf, np.nan], [7, 0, 9, 0, 1, 0.5],
                       [3, 0, 1, 2, 4, 5]])
    assert pts.shape == (4, 6)
    assert np.array_equal(pts, expect, equal_nan=True)


def test_reader_errors_carry_the_crate_messages(tmp_path):
    with pytest.raises(prb.ReconstructError, match="does not contain normal data"):
        prb.read_ply(_write(tmp_path / "a.ply", "ply\nelement vertex 1\nproperty float x\nend_header\n1 2 3 4 5 6\n"))
    with pytest.raises(prb.ReconstructError, match="Unexpected end of file"):
        prb.read_ply(_write(tmp_path / "b.ply", "ply\nproperty float nx\n"))
    with pytest.raises(prb.ReconstructError, match="Invalid vertex count"):
        prb.read_ply(_write(tmp_path / "c.ply", "ply\nelement vertex 12 \nproperty float nx\nend_header\n"))
    with pytest.raises(prb.ReconstructError, match=r"Cannot open .*nope.ply: No such file or directory \(os error 2\)"):
        prb.read_ply(tmp_path / "nope.ply")
    # normals marked by normal_x, CRLF header
    pts = prb.read_ply(_write(tmp_path / "d.ply", "ply\r\nproperty float normal_x\r\nend_header\r\n1 2 3 4 5 6\r\n"))
    assert np.array_equal(pts, [[1, 2, 3, 4, 5, 6]])


def test_binary_reader_by_property_name(tmp_path):
    rng = np.random.default_rng(9)
    n = 5000
    pos, nrm = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    rec = np.zeros(n, dtype=[("nz", "<f4"), ("x", "<f8"), ("red", "u1"), ("y", "<f8"), ("z", "<f8"),
                             ("nx", "<f4"), ("ny", "<f4")])
    rec["x"], rec["y"], rec["z"] = pos.T
    rec["nx"], rec["ny"], rec["nz"] = nrm.T
    head = ("ply\nformat binary_little_endian 1.0\ncomment made by a test\nelement vertex %d\nproperty float nz\n"
            "property double x\nproperty uchar red\nproperty double y\nproperty double z\nproperty float nx\n"
            "property float ny\nelement face 0\nproperty list uchar int vertex_indices\nend_header\n" % n)
    pts = prb.read_ply(_write(tmp_path / "b.ply", head.encode() + rec.tobytes()))
    expect = np.hstack([pos, nrm.astype(np.float32).astype(np.float64)])
    assert np.array_equal(pts, expect)


def test_ascii_reader_large_file_matches_numpy(tmp_path):
    pts = synthetic.sphere(200_000, seed=11)
    path = tmp_path / "big.ply"
    with open(path, "w") as f:
        f.write(POINT_HEADER.format(n=len(pts)))
        np.savetxt(f, pts, fmt="%.17g")
    assert np.array_equal(prb.read_ply(path), pts)


def _cli(*args, **kw):
    return subprocess.run([prb.CLI_PATH, *map(str, args)], capture_output=True, text=True, timeout=600, **kw)


def test_cli_flags_and_errors(tmp_path):
    assert os.path.exists(prb.CLI_PATH)
    r = _cli("--version")
    assert r.returncode == 0 and r.stdout.strip() == "poisson-recon 0.1.0"
    assert _cli("--help").returncode == 0
    r = _cli()
    assert r.returncode == 2 and "--input <INPUT>" in r.stderr
    assert _cli("-i", "x.ply", "--bogus").returncode == 2
    assert _cli("-i", "x.ply", "--depth", "abc").returncode == 2
    r = _cli("-i", tmp_path / "missing.ply")
    assert r.returncode == 1 and r.stderr.startswith("Error: Cannot open ")
    r = _cli("--input", _write(tmp_path / "nn.ply", "ply\nend_header\n1 2 3 4 5 6\n"))
    assert r.returncode == 1 and r.stderr == "Error: PLY file does not contain normal data (nx, ny, nz)\n"
    r = _cli("-i", _write(tmp_path / "empty.ply", POINT_HEADER.format(n=0)))
    assert r.returncode == 1 and r.stderr == "No points found.\n"


@pytest.mark.gpu
def test_cli_end_to_end_matches_the_library(tmp_path):
    pts = synthetic.sphere(20_000, seed=5)
    src = tmp_path / "in.ply"
    with open(src, "w") as f:
        f.write(POINT_HEADER.format(n=len(pts)))
        np.savetxt(f, pts, fmt="%.17g")
    out = tmp_path / "out.ply"
    r = _cli("-i", src, "-o", out, "-d", 6, "--point-weight", 4, "-v")
    assert r.returncode == 0, r.stderr
    lines = r.stderr.splitlines()
    assert lines[0] == "Read 20000 oriented points" and lines[1].startswith("Timing [s]: xform=")
    assert lines[2] == "FEM nodes=262144, matrix NNZ=0" and lines[-1] == "Wrote %s" % out
    mesh, st = prb.reconstruct(prb.read_ply(src), prb.ReconstructParams(depth=6, point_weight=4.0))
    ref = tmp_path / "ref.ply"
    prb.write_ply(ref, mesh)
    assert out.read_bytes() == ref.read_bytes()
    assert lines[3] == "Mesh: %d verts, %d tris, iso=%.6f" % (st.mesh_vertices, st.mesh_triangles, st.iso_value)
