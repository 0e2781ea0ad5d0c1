"""The asynchronous Tecplot writer (lsg_tecplot_sol_async): device fields of
the state after one step of the 16^3 sphere flow, copied to pinned host
memory and formatted on a host thread, give the reference's file byte for
byte; the fields may be overwritten as soon as the call returns."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_async_writer_matches_reference_file(tmp_path):
    import torch
    from lsstag_b200 import solver as S
    from lsstag_b200 import tecplot
    t = load_golden("tecplot16")
    g = load_golden("flow16_steps")
    dims = tuple(int(v) for v in g["dims"])
    pres = S.MGFGMRES()
    pres.set_geometry({k: g[k] for k in ("celltype", "theta", "delta", "inv_mx", "inv_my", "inv_mz")}, dims,
                      g["pins"], setup=False)
    wr = tecplot.SolWriter(pres, t["nodes"], g, flow=True)
    fields = [torch.as_tensor(np.asarray(t[k], dtype=np.float64), device="cuda:0").contiguous() for k in "uvwp"]
    torch.cuda.synchronize()
    path = tmp_path / "sol_async.dat"
    wr.write_async(path, *fields)
    for f in fields:
        f.fill_(12345.0)                    # overwritten while the host thread formats
    wr.wait()
    assert path.read_bytes() == bytes(np.asarray(t["sol"], dtype=np.uint8))
    pres.close()
