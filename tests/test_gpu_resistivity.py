"""Artificial resistivity on the GPU against the reference build: the
current-dependent term E += eta_art(|J|/|dr|) J (its smooth ramp exercised by
a window inside the run's |J| range) and the local term E += eta_local J
(eta_local from the reference's own per-edge arrays), 20 steps of a 16^3
periodic curvilinear Orszag-Tang cube.  FP64 tolerance 1e-12 per field."""
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

ARTI = dict(arti_eta_max=1e-3, arti_J_start=0.2, arti_J_on=0.8, local_arti=1, local_arti_eta_max=0.05,
            local_arti_x0=0.5, local_arti_y0=0.5, local_arti_z0=0.5, local_arti_r_decay=0.2,
            local_arti_r_cutoff=0.4)


def test_artificial_resistivity_matches_reference(ref_oracle):
    if not has_gpu():
        pytest.skip("no GPU")
    import mercury_oracle as mo
    from gpu_helpers import compare, context_from_dump
    from mpcns_mercury_b200 import reference_constants

    dump = ref_oracle.cube_run(n=16, steps=20, dump_at=[0, 20], extra=ARTI)
    k = reference_constants(cfl=0.4, arti_eta_max=ARTI["arti_eta_max"], arti_J_start=ARTI["arti_J_start"],
                            arti_J_on=ARTI["arti_J_on"], local_arti=True)
    ctx = context_from_dump(dump, 16, constants=k)
    ctx.prepare()
    ctx.step(20)
    worst, bad = compare(ctx, dump, "step20:", mo.STATE_FIELDS + mo.DERIVED_FIELDS, 1e-12)
    assert not bad, worst
    # the terms are active: the run differs from one without them
    plain = ref_oracle.cube_run(n=16, steps=20, dump_at=[20])
    import numpy as np

    a = dump[("step20:B_xi", 0)].data
    b = plain[("step20:B_xi", 0)].data
    assert float(np.abs(a - b).max()) > 1e-8
