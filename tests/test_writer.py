"""On-disk output in the reference's formats: GridWrite (Common/Serialize.c:
23-55), LevelSetWriteIrregularNodeList (LevelSetMethod/IrregularNodes.c:
145-246), the particle ArrayWrite (Common/Array.c:133-150).

Pinning: tests/golden/writer.npz holds the bytes of every file the
reference's OWN writers produced (run by tests/golden/make_golden.py through
oracle/_ref; PETSc's binary viewer, absent here, is its documented format in
the shim: big-endian values, Vec class id 1211214 and length, `.info` with
the block size) together with their inputs -- the writer must reproduce each
file byte for byte from the same inputs, host forms here and device forms on
the GPU.  The reference's own reader of .Real64 files
(Visualization/DCellVTK.py: skip two int32 header words, read big-endian
FP64) also reads the grids back exactly.  The device forms must write the
same bytes even when the caller overwrites the device data right after the
call."""
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


def _rows_to_nodes(rows):
    """18-column node rows (pos, axis, shift, signCenter, signFace, d, X, op,
    n, k) -> NODE_DTYPE records."""
    a = np.zeros(len(rows), dtype=_lib.NODE_DTYPE)
    a["pos"], a["axis"], a["shift"] = rows[:, 0:3], rows[:, 3], rows[:, 4]
    a["signCenter"], a["signFace"], a["d"] = rows[:, 5], rows[:, 6], rows[:, 7]
    a["X"], a["op"], a["n"], a["k"] = rows[:, 8:11], rows[:, 11:14], rows[:, 14:17], rows[:, 17]
    return a


def _write_like_reference(w, g, arrays):
    """The golden sequence of writes (tests/golden/make_golden.py
    run_writer) through writer `w`; `arrays(x)` makes each input the form to
    write (numpy here, device tensors on the GPU)."""
    w.grid("ls3", 0, arrays(g["phi3"]), 0.1, (-3, 2, 1))
    w.grid("ls3", 1, arrays(g["phi3"] * 0.5), 0.1, (-3, 2, 1))
    w.irregular_nodes("ls3", 2, *_nodes_arg(arrays, g["nodes3"]), dim=3)
    w.grid("vel3", 4, arrays(g["vel3"]), 0.1, (-3, 2, 1), dof=3)
    w.grid("ls2", 7, arrays(g["phi2"]), 0.1, (5, -4))
    w.irregular_nodes("ls2", 0, *_nodes_arg(arrays, g["nodes2"]), dim=2)
    w.grid("vel2", 1, arrays(g["vel2"]), 0.1, (5, -4), dof=2)
    w.particles("particles", 3, arrays(g["particles"]))


def _nodes_arg(arrays, rows):
    nodes = _rows_to_nodes(rows)
    a = arrays(nodes)
    if isinstance(a, np.ndarray):
        return a, len(nodes)
    import torch
    return a, torch.tensor([len(nodes)], dtype=torch.int32, device=a.device)


def _compare_with_reference_files(g, wd, tmp):
    files = [k for k in g if k.startswith("file:")]
    assert len(files) == 23
    for k in files:
        sub, name = k[5:].split("/", 1)
        path = os.path.join(wd if sub == "wd" else tmp, name)
        assert os.path.exists(path), name
        assert open(path, "rb").read() == g[k].tobytes(), name


def test_files_equal_the_reference_writers_bytes(golden, tmp_path):
    """Host forms: every file of the reference's own writers, byte for byte."""
    g = golden("writer")
    wd, tmp = str(tmp_path / "wd"), str(tmp_path / "tmp")
    os.makedirs(tmp)
    with Writer(wd, tmpdir=tmp) as w:
        _write_like_reference(w, g, lambda x: x)
    _compare_with_reference_files(g, wd, tmp)


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
def test_gpu_device_files_equal_the_reference_writers_bytes(golden, tmp_path, cuda):
    """Device forms (FP64 device grids, node records and particles on the
    device): every file of the reference's own writers, byte for byte."""
    import torch
    g = golden("writer")
    wd, tmp = str(tmp_path / "wd"), str(tmp_path / "tmp")
    os.makedirs(tmp)

    def dev(x):
        if x.dtype.names:  # node records: raw bytes on the device
            return torch.from_numpy(np.frombuffer(x.tobytes(), dtype=np.uint8).copy()).to(cuda)
        return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=cuda)
    with Writer(wd, tmpdir=tmp) as w:
        _write_like_reference(w, g, dev)
    _compare_with_reference_files(g, wd, tmp)


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
