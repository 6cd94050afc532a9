"""Per-solve setup on the device (mhd_setup_geometry): the static fields the
step reads, computed from the block's nodes, against the host setup
(mpcns_mercury_b200/setup.py, pinned against the reference build in
test_setup.py), and a solve set up this way stepped against the reference.

Tolerances: fields without transcendental functions are bitwise equal (same
formulas and operation order, no FMA contraction, IEEE division and square
root); the reconstruction weights (Jacobi rotations: atan2, sin, cos) and
the photo rate (acos, exp) agree to 1e-13 of the field's magnitude; the
step after 20 steps to the parity tolerance, 1e-12 relative L2."""
import time

import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

TRANSCENDENTAL = {"Bcell_from_Bface_w", "Jcell_from_Jedge_w", "Photo_rate"}


def _static_names():
    from mpcns_mercury_b200 import workloads as W

    return [n for n in W.UPLOAD_FIELDS if n not in W.STATE_FIELDS]


@pytest.fixture(scope="module")
def gpu():
    if not has_gpu():
        pytest.skip("no GPU")


@pytest.mark.parametrize("precision", [0, 1])
def test_device_static_fields_match_host(gpu, precision):
    from mpcns_mercury_b200 import reference_constants
    from mpcns_mercury_b200 import setup as S
    from mpcns_mercury_b200 import workloads as W
    from mpcns_mercury_b200.capi import Batch, SolveDesc

    cells = (10, 12, 14)
    t0 = time.perf_counter()
    geom, host = S.cube_case(cells, solve_id=1)
    t_host = time.perf_counter() - t0
    b = Batch(1, precision)
    d = SolveDesc([cells], W.NGHOST, reference_constants(cfl=0.4), precision=precision)
    slot = b.add(d)
    t0 = time.perf_counter()
    b.setup_geometry(slot, geom.aos())
    t_dev = time.perf_counter() - t0
    worst = {}
    for name in _static_names():
        a = host[name]
        dev = b.download(slot, W.capi_field(name), a.lo, a.hi)
        metric = name in ("Jac", "JDxi", "JDet", "JDze")  # double in every precision
        ref = a.data if precision == 0 or metric else a.data.astype(np.float32).astype(np.float64)
        if name in TRANSCENDENTAL:
            scale = max(float(np.abs(ref).max()), 1e-300)
            err = float(np.abs(dev - ref).max()) / scale
            worst[name] = err
            assert err <= 1e-13 if precision == 0 else err <= 1e-6, (name, err)
        else:
            assert np.array_equal(dev, ref), name
    print(f"host setup {t_host:.3f} s, device setup {t_dev:.3f} s; transcendental fields {worst}")
    b.close()
    d.close()


REF_STATIC = {"beta_xi": "Hodge_star_2form_to_1form_face_xi_lumped",
              "beta_eta": "Hodge_star_2form_to_1form_face_eta_lumped",
              "beta_zeta": "Hodge_star_2form_to_1form_face_zeta_lumped",
              "alpha_xi": "Hodge_star_inverse_2form_to_1form_edge_xi_lumped",
              "alpha_eta": "Hodge_star_inverse_2form_to_1form_edge_eta_lumped",
              "alpha_zeta": "Hodge_star_inverse_2form_to_1form_edge_zeta_lumped"}


@pytest.fixture(scope="module")
def cube16(gpu, ref_oracle):
    return ref_oracle.cube_run(n=16, steps=20, dump_at=[0, 20])


def _ref_nodes(dump):
    """The reference's own node coordinates (its ghost-corner treatment included)."""
    return np.ascontiguousarray(np.concatenate([dump[(k, 0)].data for k in ("node_x", "node_y", "node_z")], axis=-1))


def test_device_static_fields_match_reference(cube16):
    """From the reference's nodes, the device setup reproduces the reference's
    static fields over the whole range it uploads, ghosts included."""
    from gpu_helpers import NGHOST
    from mpcns_mercury_b200 import Context, reference_constants
    from mpcns_mercury_b200 import workloads as W

    ctx = Context([(16, 16, 16)], NGHOST, reference_constants(cfl=0.4))
    ctx.setup_geometry(_ref_nodes(cube16))
    checked = 0
    for name in _static_names():
        key = ("static:" + REF_STATIC.get(name, name), 0)
        if key not in cube16:
            continue
        r = cube16[key]
        dev = ctx.download(W.capi_field(name), r.lo, r.hi)
        if name in TRANSCENDENTAL:
            scale = max(float(np.abs(r.data).max()), 1e-300)
            assert float(np.abs(dev - r.data).max()) <= 1e-13 * scale, name
        else:
            assert np.array_equal(dev, r.data), name
        checked += 1
    assert checked >= 20
    ctx.close()


def test_device_setup_steps_like_the_reference(cube16):
    import mercury_oracle as mo
    from gpu_helpers import NGHOST, compare
    from mpcns_mercury_b200 import Context, reference_constants
    from mpcns_mercury_b200.capi import REF_FIELD

    ctx = Context([(16, 16, 16)], NGHOST, reference_constants(cfl=0.4))
    ctx.setup_geometry(_ref_nodes(cube16))
    for name in mo.STATE_FIELDS:  # the reference's own initial state
        r = cube16[("step0:" + name, 0)]
        ctx.upload(REF_FIELD[name], r.data, r.lo, r.hi)
    ctx.prepare()
    ctx.step(20)
    worst, bad = compare(ctx, cube16, "step20:", mo.STATE_FIELDS + mo.DERIVED_FIELDS, 1e-12)
    assert not bad, worst
    ctx.close()
