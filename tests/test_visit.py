"""Graphics output of the driver (the reference's visit(), tealeaf_2d/visit.f90:23-112,
tealeaf_3d/visit.f90), written when the deck sets visit_frequency: the tea.visit index
and one legacy-VTK rectilinear grid per rank and call, with the cells' density, energy
and temperature read through tea_read_field_.  Runs on the CPU against the oracle port;
the GPU case checks the CUDA library writes the same files."""
import json
import os
import socket

import numpy as np
import pytest

from conftest import SUM_COMPENSATED, SUM_SEQUENTIAL, port_lib, rel, tea


def _deck(dim, cells, end_step, freq, solver="cg"):
    spec = tea.DeckSpec(dim=dim, cells=cells, states=5, seed=11, solver=solver, end_step=end_step, eps=1e-15,
                        max_iters=5000, summary_frequency=1, check_result=False)
    return tea.seeded_deck(spec).replace("*endtea", f"visit_frequency={freq}\n*endtea")


def _parse_vtk(path):
    """The legacy-VTK file as a dict: header lines, dims, coordinates, cell arrays."""
    lines = path.read_text().splitlines()
    out = {"header": lines[:4]}
    i = 4
    assert lines[i].startswith("DIMENSIONS")
    out["dims"] = [int(v) for v in lines[i][len("DIMENSIONS"):].split()]
    i += 1
    for axis in "XYZ":
        name, n, kind = lines[i].split()
        assert (name, kind) == (f"{axis}_COORDINATES", "double")
        n = int(n)
        out[axis] = np.array([float(v) for v in lines[i + 1:i + 1 + n]])
        assert all(len(v) == 12 for v in lines[i + 1:i + 1 + n])  # Fortran E12.4
        i += 1 + n
    assert lines[i].split()[0] == "CELL_DATA"
    ncells = int(lines[i].split()[1])
    assert lines[i + 1] == "FIELD FieldData 3"
    i += 2
    for _ in range(3):
        name, one, n, kind = lines[i].split()
        assert (one, int(n), kind) == ("1", ncells, "double")
        out[name] = np.array([float(v) for v in lines[i + 1:i + 1 + ncells]])
        i += 1 + ncells
    assert i == len(lines)
    out["ncells"] = ncells
    return out


@pytest.mark.parametrize("dim,cells", [(2, 20), (3, 8)])
def test_visit_files(tmp_path, monkeypatch, dim, cells):
    monkeypatch.chdir(tmp_path)
    summary, recs = tea.run_deck(_deck(dim, cells, end_step=4, freq=2), dim,
                                 backend=port_lib(dim, SUM_SEQUENTIAL))
    # Written at steps 2 and 4, and again at the end (diffuse.f90 calls visit() once more
    # after the last step, so step 4 is listed twice, as the reference lists it).
    assert (tmp_path / "tea.visit").read_text().splitlines() == [
        "!NBLOCKS     1", "tea.00001.00002.vtk", "tea.00001.00004.vtk", "tea.00001.00004.vtk"]
    assert sorted(p.name for p in tmp_path.glob("*.vtk")) == ["tea.00001.00002.vtk", "tea.00001.00004.vtk"]
    v = _parse_vtk(tmp_path / "tea.00001.00004.vtk")
    assert v["header"] == ["# vtk DataFile Version 3.0", "vtk output", "ASCII", "DATASET RECTILINEAR_GRID"]
    assert v["dims"] == [cells + 1, cells + 1, cells + 1 if dim == 3 else 1]
    edges = np.linspace(0.0, 10.0, cells + 1)
    for axis in "XY" + ("Z" if dim == 3 else ""):
        np.testing.assert_allclose(v[axis], edges, rtol=5e-4, atol=1e-12)
    if dim == 2:
        assert list(v["Z"]) == [0.0]
    assert v["ncells"] == cells ** dim
    # Against the field summary of the same step (4 significant digits per value):
    # mass = sum vol*density, temp = sum vol*density*u; energy1 = u / density.
    vol = (10.0 / cells) ** dim
    last = recs[-1]
    assert rel(vol * v["density"].sum(), last["mass"]) < 1e-3
    assert rel(vol * (v["density"] * v["temperature"]).sum(), last["temp"]) < 2e-3
    np.testing.assert_allclose(v["energy"], v["temperature"] / v["density"], rtol=2e-3)


def test_no_visit_files_without_the_keyword(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    tea.run_deck(_deck(2, 12, end_step=2, freq=0), 2, backend=port_lib(2, SUM_SEQUENTIAL))
    assert list(tmp_path.iterdir()) == []


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, size, port, out_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.chdir(out_dir)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        _, recs = tea.run_deck_dist(_deck(2, 16, end_step=2, freq=1), 2, port_lib(2, SUM_COMPENSATED))
        with open(f"recs{rank}.json", "w") as f:
            json.dump(recs, f)
    finally:
        dist.destroy_process_group()


def test_visit_files_of_two_ranks(tmp_path, monkeypatch):
    """Two gloo ranks: each writes its slab (rows 1-8 and 9-16), rank 0 lists both files."""
    import torch.multiprocessing as mp

    mp.start_processes(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    assert (tmp_path / "tea.visit").read_text().splitlines() == [
        "!NBLOCKS     2", "tea.00001.00001.vtk", "tea.00002.00001.vtk",
        "tea.00001.00002.vtk", "tea.00002.00002.vtk", "tea.00001.00002.vtk", "tea.00002.00002.vtk"]
    lo, hi = (_parse_vtk(tmp_path / f"tea.0000{r}.00002.vtk") for r in (1, 2))
    assert lo["dims"] == [17, 9, 1] and hi["dims"] == [17, 9, 1]
    np.testing.assert_allclose(np.concatenate([lo["Y"], hi["Y"][1:]]), np.linspace(0.0, 10.0, 17), rtol=5e-4)
    # The slabs together against a single-rank run of the same deck.
    one = tmp_path / "one"
    one.mkdir()
    monkeypatch.chdir(one)
    tea.run_deck(_deck(2, 16, end_step=2, freq=1), 2, backend=port_lib(2, SUM_COMPENSATED))
    whole = _parse_vtk(one / "tea.00001.00002.vtk")
    np.testing.assert_array_equal(np.concatenate([lo["density"], hi["density"]]), whole["density"])
    # Sums over ranks may differ from the one-rank sums in the last bit, which can move a
    # value across a rounding boundary of its 4 printed digits (at most 1e-3 relative).
    np.testing.assert_allclose(np.concatenate([lo["temperature"], hi["temperature"]]), whole["temperature"],
                               rtol=1.1e-3)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,cells", [(2, 20), (3, 8)])
def test_visit_files_of_the_cuda_library(tmp_path, monkeypatch, dim, cells):
    """The CUDA library's fields are bit-identical to the compensated port's, so the files
    are byte-identical."""
    for name, backend in (("port", port_lib(dim, SUM_COMPENSATED)), ("cuda", None)):
        (tmp_path / name).mkdir()
        monkeypatch.chdir(tmp_path / name)
        tea.run_deck(_deck(dim, cells, end_step=3, freq=3), dim, backend=backend)
    for f in ("tea.visit", "tea.00001.00003.vtk"):
        assert (tmp_path / "cuda" / f).read_bytes() == (tmp_path / "port" / f).read_bytes()
