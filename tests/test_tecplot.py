"""The checkpoint plot file (mhd_tecplot_write) against the one the
reference's own writer (IOModule::WriteTecplotBinFile,
src/6_io/IOModule_Tecplot.cpp:749-1017, AllNode as MercurySolver selects it)
produced from the same state: the reference's dumped fields (PV_H, PV_Na,
B_cell, Bind_cell, Na, J_cell with their ghost layers, Jac, the nodes) are
written by the library and the two files must be equal byte for byte."""
import numpy as np
import pytest

N = 4
FIELDS = "PV_H PV_Na B_cell Bind_cell Na J_cell"


def _reference_plot(ref_oracle, tmp_path, extra):
    path = str(tmp_path / "ref.plt")
    job = dict(ref_oracle.CUBE_JOB)
    job.update(n=N, steps=2, dump_at="2", write_tecplot=path, dump_fields=FIELDS, dump_static="Jac", dump_grid=1,
               **extra)
    return path, ref_oracle.run_job(job, workdir=str(tmp_path / "job"))


@pytest.mark.parametrize("extra,nblock", [({}, 1), ({"case": "lattice", "nb": "2 1 2"}, 4)])
def test_plot_file_matches_reference(ref_oracle, tmp_path, extra, nblock):
    from mpcns_mercury_b200 import capi

    ref_path, d = _reference_plot(ref_oracle, tmp_path, extra)
    nodes, jac = [], []
    for b in range(nblock):
        rec = d[("node_x", b)]
        sl = tuple(slice(-lo, -lo + N + 1) for lo in rec.lo)
        nodes.append(np.stack([d[("node_" + a, b)].data[..., 0][sl] for a in "xyz"], axis=-1))
        jac.append(d[("static:Jac", b)].data)
    jac_ghost = -d[("static:Jac", 0)].lo[0]
    cell_ghost = -d[("step2:PV_H", 0)].lo[0]
    fields = {f: [d[("step2:" + f, b)].data for b in range(nblock)] for f in capi.TECPLOT_FIELDS}
    time = float(d[("step2:dt_time", -1)].data.ravel()[1])
    ours = str(tmp_path / "ours.plt")
    capi.tecplot_write(ours, [(N, N, N)] * nblock, ["Fluid"] * nblock, time, nodes, jac, jac_ghost, fields,
                       cell_ghost)
    a, b = open(ref_path, "rb").read(), open(ours, "rb").read()
    assert len(a) == len(b)
    assert a == b


def test_bad_image_is_rejected(tmp_path):
    from mpcns_mercury_b200 import capi

    with pytest.raises(capi.MhdError):
        capi.tecplot_write(str(tmp_path / "x.plt"), [(N, N, N)], ["Fluid"], 0.0, [np.zeros((N + 1,) * 3 + (3,))],
                           [np.zeros((N + 2,) * 3 + (1,))], 0, {f: [np.zeros(1)] for f in capi.TECPLOT_FIELDS}, 4)
