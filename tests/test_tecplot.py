"""Tecplot solution files (the reference's SolTecplotPrinter): the oracle's
restatement and the library's writer (lsg_tecplot_sol_write, host code, no
device work) against the file the reference printed for the state after one
step of the 16^3 sphere flow (tests/golden/tecplot16.npz), byte for byte."""
import numpy as np

from conftest import load_golden

import lsg_oracle as lo


def _case():
    t = load_golden("tecplot16")
    g = load_golden("flow16_steps")
    dims = tuple(int(v) for v in g["dims"])
    return t, g, dims


def test_oracle_matches_reference_file():
    t, g, dims = _case()
    ref = bytes(np.asarray(t["sol"], dtype=np.uint8))
    mine = lo.tecplot_sol(*dims, t["nodes"], g["delta"], g["theta"], g["celltype"], t["u"], t["v"], t["w"], t["p"],
                          g["u_w"], g["bc"], True)
    assert len(ref) == 365065 and ref.startswith(b'TITLE     = "Velocity Vectors" \n')
    assert mine == ref


def test_library_writer_matches_reference_file(tmp_path):
    from lsstag_b200 import tecplot
    t, g, dims = _case()
    path = tmp_path / "sol.dat"
    tecplot.write_sol(path, dims, t["nodes"], g, t["u"], t["v"], t["w"], t["p"], flow=True)
    assert path.read_bytes() == bytes(np.asarray(t["sol"], dtype=np.uint8))


def test_library_writer_matches_oracle_without_outflow(tmp_path):
    """The non-flow branches (wall planes at the bottom and top, the east
    boundary value U_E), with perturbed boundary velocities and no inflow
    profile: the library's writer and the oracle agree byte for byte."""
    from lsstag_b200 import tecplot
    t, g, dims = _case()
    bc = np.linspace(-0.4, 0.9, 18)
    geom = dict(g, bc=bc, u_w=None)
    path = tmp_path / "sol.dat"
    tecplot.write_sol(path, dims, t["nodes"], geom, t["u"], t["v"], t["w"], t["p"], flow=False)
    mine = lo.tecplot_sol(*dims, t["nodes"], g["delta"], g["theta"], g["celltype"], t["u"], t["v"], t["w"], t["p"],
                          None, bc, False)
    assert path.read_bytes() == mine


def test_cell_centres_are_the_reference_nodes():
    from lsstag_b200 import tecplot
    t, g, dims = _case()
    assert np.array_equal(tecplot.cell_centres(dims, (1 / 16, 1 / 16, 1 / 16)), t["nodes"])


def test_threaded_writer_at_full_size(tmp_path):
    """The 128x64x64 flow case's initial state: the library formats the 66
    layers on several threads from a dry walk's running indices; the bytes
    equal the oracle's single walk (19 MB)."""
    from lsstag_b200 import cases, tecplot
    g, dims, par, (u, v, w, p) = cases.load_flow_case()
    nodes = tecplot.cell_centres(dims, (1 / 16, 1 / 16, 1 / 16))
    path = tmp_path / "sol.dat"
    tecplot.write_sol(path, dims, nodes, g, u, v, w, p, flow=True)
    ref = lo.tecplot_sol(*dims, nodes, g["delta"], g["theta"], g["celltype"], u, v, w, p, g["u_w"], g["bc"], True)
    assert len(ref) > 18_000_000
    assert path.read_bytes() == ref
