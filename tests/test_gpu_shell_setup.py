"""The magnetosphere case set up on the device from its parameters
(mpcns_mercury_b200.magnetosphere: mhd_shell_grid nodes,
mhd_setup_geometry_bg, Sync(Badd), the initial state, Sync(Ucell),
Sync(Bface)) against the reference's own setup of the same case (the oracle
harness's shell job, oracle/_ref built from the reference sources).

Static fields: bit for bit where they involve only +, -, *, / and sqrt (the
metric, the edge and face Hodge ratios, the background field, the cell
centres); within 1e-13 relative where the device's transcendental functions
enter (the reconstruction weights' Jacobi rotations, the photo rate, the Hall
taper's tanh).  The state after the steps: 1e-12 relative L2 per field."""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

NA, NR, STEPS = 8, 12, 5
EXACT = ["Jac", "JDxi", "JDet", "JDze", "Area_xi", "Area_eta", "Area_zeta", "dl_xi", "dl_eta", "dl_zeta",
         "dr_xi", "dr_eta", "dr_zeta", "Hodge_star_2form_to_1form_face_xi_lumped",
         "Hodge_star_2form_to_1form_face_eta_lumped", "Hodge_star_2form_to_1form_face_zeta_lumped",
         "Hodge_star_inverse_2form_to_1form_edge_xi_lumped", "Hodge_star_inverse_2form_to_1form_edge_eta_lumped",
         "Hodge_star_inverse_2form_to_1form_edge_zeta_lumped", "Badd_xi", "Badd_eta", "Badd_zeta"]
CLOSE = ["Bcell_from_Bface_w", "Jcell_from_Jedge_w", "Photo_rate"]


@pytest.fixture(scope="module")
def ref(ref_oracle):
    if not has_gpu():
        pytest.skip("no GPU")
    return ref_oracle.shell_run(na=NA, nr=NR, steps=STEPS, dump_at=[0, STEPS])


@pytest.fixture(scope="module")
def dev(ref):
    from mpcns_mercury_b200 import magnetosphere as M

    case = M.ShellCase(na=NA, nr=NR)
    ctx = M.context(case)
    yield ctx
    ctx.close()


@pytest.mark.parametrize("name", EXACT + CLOSE)
def test_static_fields_match_reference(ref, dev, name):
    """Every position the reference fills and the step can read: the owned
    range widened by the ghost layers the device setup writes."""
    from mpcns_mercury_b200.capi import REF_FIELD

    field = REF_FIELD[name]
    worst = 0.0
    for b in range(6):
        r = ref[("static:" + name, b)]
        got = dev.download(field, r.lo, r.hi, block=b)
        want = r.data
        # compare where the device setup writes: [-(g-1), n + 1 + (g-1)) covers every field's written range
        g = [-v for v in r.lo]
        sl = tuple(slice(1, r.hi[a] - r.lo[a] - 1) for a in range(3))
        a, w = got[sl], want[sl]
        if name in EXACT:
            bad = np.argwhere(a != w)
            assert len(bad) == 0, (name, b, [tuple(int(v) - g[q] for q, v in enumerate(p[:3])) for p in bad[:5]],
                                   float(np.abs(a - w).max()))
        else:
            scale = float(np.abs(w).max()) or 1.0
            worst = max(worst, float(np.abs(a - w).max()) / scale)
    assert worst <= 1e-13, (name, worst)


def test_taper_matches_reference(ref, dev):
    worst = 0.0
    for ax, field in (("xi", "TAPER_XI"), ("eta", "TAPER_ETA"), ("zeta", "TAPER_ZETA"), ("cell", "TAPER_CELL")):
        for b in range(6):
            r = ref[("static:taper_" + ax, b)]
            got = dev.download(field, r.lo, r.hi, block=b)
            worst = max(worst, float(np.abs(got - r.data).max()))
    assert worst <= 1e-13, worst


def test_initial_state_matches_reference(ref, dev):
    """The state after the setup's syncs and the derived refresh of
    mhd_prepare, against the reference's step 0."""
    import mercury_oracle as mo
    from gpu_helpers import compare

    worst, bad = compare(dev, ref, "step0:", mo.STATE_FIELDS + mo.DERIVED_FIELDS, 1e-13)
    print("magnetosphere setup, step 0: max rel L2", max(worst.values()))
    assert not bad, bad


def test_steps_from_device_setup_match_reference(ref):
    import mercury_oracle as mo
    from gpu_helpers import compare
    from mpcns_mercury_b200 import magnetosphere as M

    ctx = M.context(M.ShellCase(na=NA, nr=NR))
    ctx.step(STEPS)
    worst, bad = compare(ctx, ref, f"step{STEPS}:", mo.STATE_FIELDS, 1e-12)
    print(f"magnetosphere setup, {STEPS} steps: max rel L2", max(worst.values()))
    assert not bad, bad
    assert ctx.info().status == 0
    ctx.close()
