"""The package's host setup (mpcns_mercury_b200.setup) against the
reference's own setup: static geometry, reconstruction weights, photo rate
and the seeded Orszag-Tang state on the owned DOFs."""
import numpy as np
import pytest

# Fields whose owned values depend only on owned + face-ghost nodes; the
# edge inverse Hodge of boundary edges also reads corner-ghost cell centres,
# which the reference builds with its own corner treatment.
EXACT = ["JDxi", "JDet", "JDze", "Jac", "Area_xi", "Area_eta", "Area_zeta", "dl_xi", "dl_eta", "dl_zeta",
         "dr_xi", "dr_eta", "dr_zeta", "Badd_xi", "Badd_eta", "Badd_zeta"]
CLOSE = ["Hodge_star_2form_to_1form_face_xi_lumped", "Bcell_from_Bface_w", "Jcell_from_Jedge_w", "Photo_rate"]
SETUP_NAME = {"Hodge_star_2form_to_1form_face_xi_lumped": "beta_xi"}


def _owned(arr, lo, hi):
    g = [-v for v in lo]
    return arr[g[0]:hi[0], g[1]:hi[1], g[2]:hi[2]]


@pytest.fixture(scope="module", params=[6, (5, 7, 9)], ids=["cube6", "box5x7x9"])
def both(ref_oracle, request):
    """The 6^3 cube and a non-cubic periodic box (per-axis cell counts, the
    ensemble's block shapes) set up by both sides."""
    from mpcns_mercury_b200 import setup as S

    n = request.param
    d = ref_oracle.cube_run(n=n if isinstance(n, int) else " ".join(map(str, n)), steps=0, dump_at=[0])
    _, f = S.cube_case(n)
    return d, f


@pytest.mark.parametrize("name", EXACT)
def test_static_exact(both, name):
    d, f = both
    r = d[("static:" + name, 0)]
    a = f[SETUP_NAME.get(name, name)]
    assert (tuple(a.lo), tuple(a.hi)) == (tuple(r.lo), tuple(r.hi))
    assert np.array_equal(_owned(a.data, a.lo, a.hi), _owned(r.data, r.lo, r.hi))


@pytest.mark.parametrize("name", CLOSE)
def test_static_close(both, name):
    d, f = both
    r = d[("static:" + name, 0)]
    a = f[SETUP_NAME.get(name, name)]
    x, y = _owned(a.data, a.lo, a.hi), _owned(r.data, r.lo, r.hi)
    assert np.max(np.abs(x - y)) <= 1e-14 * max(1.0, np.max(np.abs(y)))


@pytest.mark.parametrize("name", ["U_H", "U_Na", "B_xi", "B_eta", "B_zeta"])
def test_seeded_initial_state_matches(both, name):
    """Same seed, same draw order, same formulas: identical bytes on owned DOFs."""
    d, f = both
    r = d[("step0:" + name, 0)]
    a = f[name]
    assert np.array_equal(_owned(a.data, a.lo, a.hi), _owned(r.data, r.lo, r.hi))


def test_resistivity_eta_matches_reference(ref_oracle):
    """Edge eta of the implicit substep against the reference's own
    ImplicitResistiveEtaAtEdge_ (eta_max_mercury 1.25e7, window 0.84..1.04)."""
    from mpcns_mercury_b200 import reference_constants
    from mpcns_mercury_b200 import setup as S

    n = 6
    d = ref_oracle.cube_run(n=n, steps=0, dump_at=[0], extra=dict(resistive=1))
    geom, _ = S.cube_case(n)
    eta = S.resistivity_eta(geom, reference_constants())
    nonzero = 0
    for name, a in eta.items():
        r = d[("static:" + name, 0)]
        x, y = _owned(a.data, a.lo, a.hi), _owned(r.data, r.lo, r.hi)
        assert x.shape == y.shape
        assert np.array_equal(x == 0.0, y == 0.0), name
        assert np.max(np.abs(x - y)) <= 1e-14 * np.max(np.abs(y)), name
        nonzero += int(np.count_nonzero(y))
    assert nonzero > 0
