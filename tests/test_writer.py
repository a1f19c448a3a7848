"""On-disk output in the reference's formats: GridWrite (Common/Serialize.c:
23-55), LevelSetWriteIrregularNodeList (LevelSetMethod/IrregularNodes.c:
145-246), the particle ArrayWrite (Common/Array.c:133-150).

Pinning: the reference's own reader of .Real64 files
(Visualization/DCellVTK.py: skip two int32 header words, read big-endian
FP64) reads our grids back exactly; the header is PETSc's binary Vec header
(class id 1211214, length); node rows follow the reference's row layouts
field by field; the particle file is the Array's raw records.  The host forms
run here; the device forms must write the same bytes (GPU tests), including
when the caller overwrites the device data right after the call."""
import os

import numpy as np
import pytest

from dcell_b200 import _lib
from dcell_b200.writer import FILE_COUNT_START, Writer, read_real64


def _dcellvtk_read(path):
    # the reference's reader, restated: 2 * sizeof(int) header, then '>f8'
    with open(path, "rb") as f:
        f.read(2 * 4)
        return np.fromfile(f, dtype=">f8")


def _nodes(n, dim, seed=3):
    rng = np.random.default_rng(seed)
    a = np.zeros(n, dtype=_lib.NODE_DTYPE)
    a["pos"] = rng.integers(-5, 40, size=(n, 3))
    a["axis"] = rng.integers(-1, dim, size=n)
    a["X"] = rng.uniform(-3, 40, size=(n, 3))
    a["op"] = rng.uniform(-1, 1, size=(n, 3))
    a["n"] = rng.uniform(-1, 1, size=(n, 3))
    a["k"] = rng.uniform(-2, 2, size=n)
    a["d"] = rng.uniform(0, 1, size=n)
    return a


def test_grid_files(tmp_path):
    d = str(tmp_path)
    rng = np.random.default_rng(1)
    phi3 = rng.standard_normal((5, 6, 7))
    vel2 = rng.standard_normal((4, 9, 2))
    with Writer(d, tmpdir=d) as w:
        w.grid("phi", 0, phi3, 0.1, (3, -2, 5))
        w.grid("phi", 1, phi3 * 2, 0.1, (4, -2, 5))
        w.grid("vel", 7, vel2, 0.1, (1, 2), dof=2)
    cid, n, vals = read_real64(os.path.join(d, f"phi.{FILE_COUNT_START}.Real64"))
    assert cid == 1211214 and n == phi3.size and np.array_equal(vals, phi3.ravel())
    assert np.array_equal(_dcellvtk_read(os.path.join(d, f"phi.{FILE_COUNT_START + 1}.Real64")), 2 * phi3.ravel())
    assert open(os.path.join(d, "phi.pos")).read() == "3 -2 5\n4 -2 5\n"
    assert open(os.path.join(d, "phi.size")).read() == "7 6 5\n7 6 5\n"
    assert open(os.path.join(d, f"phi.{FILE_COUNT_START}.Real64.info")).read() == ""
    assert open(os.path.join(d, f"vel.{FILE_COUNT_START + 7}.Real64.info")).read() == "-vecload_block_size 2\n"
    assert np.array_equal(_dcellvtk_read(os.path.join(d, f"vel.{FILE_COUNT_START + 7}.Real64")), vel2.ravel())
    assert open(os.path.join(d, "vel.pos")).read() == "1 2\n" and open(os.path.join(d, "vel.size")).read() == "9 4\n"
    # a new writer truncates .pos/.size on its first write
    with Writer(d, tmpdir=d) as w:
        w.grid("phi", 2, phi3, 0.1, (0, 0, 0))
    assert open(os.path.join(d, "phi.pos")).read() == "0 0 0\n"


def test_irregular_node_rows(tmp_path):
    d = str(tmp_path)
    a2, a3 = _nodes(40, 2), _nodes(25, 3)
    with Writer(d) as w:
        w.irregular_nodes("phi2", 3, a2, len(a2), dim=2)
        w.irregular_nodes("phi3", -1, a3, len(a3), dim=3)
    r2 = np.fromfile(os.path.join(d, f"phi2.irregNode.{FILE_COUNT_START + 3}.array"), dtype=">f8").reshape(-1, 11)
    keep = a2[a2["axis"] != -1]
    assert r2.shape[0] == len(keep)
    want2 = np.zeros((len(keep), 11))
    want2[:, 0:2], want2[:, 2:4], want2[:, 4:6], want2[:, 8] = keep["X"][:, :2], keep["pos"][:, :2], \
        keep["n"][:, :2], keep["k"]
    assert np.array_equal(r2, want2)
    r3 = np.fromfile(os.path.join(d, f"phi3.irregNode.{FILE_COUNT_START - 1}.array"), dtype=">f8").reshape(-1, 23)
    want3 = np.zeros((len(a3), 23))
    want3[:, 0:3], want3[:, 3:6], want3[:, 6:9], want3[:, 9] = a3["X"], a3["pos"], a3["n"], a3["k"]
    assert np.array_equal(r3, want3)


def test_particle_array_and_errors(tmp_path):
    d = str(tmp_path)
    parts = np.random.default_rng(2).uniform(-1, 30, size=(33, 4))
    with Writer(str(tmp_path / "grids"), tmpdir=d) as w:
        w.particles("particles", 4, parts)
        w.particles("empty", 0, np.zeros((0, 4)))
    raw = np.fromfile(os.path.join(d, f"particles.{FILE_COUNT_START + 4}.array"), dtype="<f8").reshape(-1, 4)
    assert np.array_equal(raw, parts)
    assert os.path.getsize(os.path.join(d, f"empty.{FILE_COUNT_START}.array")) == 0
    w = Writer(str(tmp_path / "g2"), tmpdir=str(tmp_path / "missing" / "dir"))
    w.particles("p", 0, parts)
    with pytest.raises(_lib.DcellError):
        w.flush()  # the unwritable directory surfaces at the flush
    w.close()
    with pytest.raises(_lib.DcellError):
        Writer(d).grid("a/b", 0, np.zeros((2, 2)), 1.0)


# ---------------------------------------------------------------------------
# GPU: device snapshots write the same bytes

@pytest.mark.gpu
def test_gpu_device_writes_equal_host_writes(tmp_path, cuda):
    import torch

    from dcell_b200 import fields
    from dcell_b200 import levelset as L
    N = 48
    phi = (fields.sphere_sdf(N, device=cuda) * N).contiguous()
    band = fields.band_of(phi, 6.0, margin=3).to(cuda)
    raw, count = L.irregular_nodes(phi, 1.0 / N, band)
    parts = torch.rand((1000, 4), dtype=torch.float64, device=cuda)
    dev_dir, host_dir = str(tmp_path / "dev"), str(tmp_path / "host")
    with Writer(dev_dir, tmpdir=dev_dir) as w:
        w.grid("phi", 0, phi, 1.0 / N)
        phi.fill_(123.0)     # overwritten right after the call: the snapshot stands
        w.irregular_nodes("phi", 0, raw, count, dim=3)
        w.particles("particles", 0, parts)
        w.grid("phi32", 0, (fields.sphere_sdf(N, device=cuda) * N).float(), 1.0 / N)
    phi_host = (fields.sphere_sdf(N, device=cuda) * N).cpu().numpy()
    nodes = L.nodes_to_numpy(raw, count)
    with Writer(host_dir, tmpdir=host_dir) as w:
        w.grid("phi", 0, phi_host, 1.0 / N)
        w.irregular_nodes("phi", 0, nodes, len(nodes), dim=3)
        w.particles("particles", 0, parts.cpu().numpy())
    for f in (f"phi.{FILE_COUNT_START}.Real64", f"phi.irregNode.{FILE_COUNT_START}.array",
              f"particles.{FILE_COUNT_START}.array", "phi.pos", "phi.size"):
        assert open(os.path.join(dev_dir, f), "rb").read() == open(os.path.join(host_dir, f), "rb").read(), f
    _, _, v32 = read_real64(os.path.join(dev_dir, f"phi32.{FILE_COUNT_START}.Real64"))
    assert np.array_equal(v32, phi_host.astype(np.float32).astype(np.float64).ravel())
