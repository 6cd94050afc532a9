"""Host side of the magnetosphere case (no GPU): the seeded ensemble and
request stream, the case's constants and background record, the initial
state, and the reference arm's jobs for the same members."""
import math

import numpy as np
import pytest


def test_ensemble_is_seeded_and_in_range():
    from mpcns_mercury_b200 import magnetosphere as M

    a, b = M.ensemble(64), M.ensemble(64)
    assert [(c.na, c.nr, c.upstream, c.na_fraction) for c in a] == [(c.na, c.nr, c.upstream, c.na_fraction) for c in b]
    for c in a:
        assert 24 <= c.na <= 64 and 24 <= c.nr <= 128
        U, T, n, Mm, cy, cz, Bx, By, Bz = c.upstream
        assert 2.0 * 4.031e5 <= U <= 6.0 * 4.031e5 and 0.5 * 4e7 <= n <= 3.0 * 4e7
        assert abs(Bz) <= 0.4e-9 and Bx == By == 0.0 and cy == cz == 0.0
        assert 1e-4 <= c.na_fraction <= 1e-2
    total = sum(c.cell_count() for c in a)
    assert 20e6 < total < 60e6
    assert M.ensemble(8, stream=300001)[0].na != a[0].na or M.ensemble(8, stream=300001)[0].nr != a[0].nr


def test_request_stream():
    from mpcns_mercury_b200 import magnetosphere as M

    s = M.request_stream(100, 20.0, shapes=16)
    t = [x[0] for x in s]
    assert all(t1 > t0 for t0, t1 in zip(t, t[1:]))
    assert 2.0 < t[-1] < 10.0  # 100 arrivals at 20/s
    grids = {(c.na, c.nr) for _, c, _ in s}
    assert len(grids) <= 16
    for _, c, st in s:
        assert 24 <= c.na <= 96 and 24 <= c.nr <= 192 and 50 <= st <= 500


def test_initial_state_and_background():
    from mpcns_mercury_b200 import magnetosphere as M

    case = M.ShellCase(na=8, nr=12)
    k = M.constants(case)
    uh, un = M.initial_state(case, k)
    assert np.array_equal(uh, [k.bc[q] for q in range(5)])
    g = k.gamma
    rho = uh[0]
    p = (g - 1.0) * (uh[4] - 0.5 * rho * ((uh[1] / rho) ** 2 + (uh[2] / rho) ** 2 + (uh[3] / rho) ** 2))
    assert math.isclose(un[0], 1e-3 * (k.M_Na / k.M_H) * rho, rel_tol=1e-15)
    pn = (g - 1.0) * (un[4] - 0.5 * un[0] * ((un[1] / un[0]) ** 2 + (un[2] / un[0]) ** 2 + (un[3] / un[0]) ** 2))
    assert math.isclose(pn, 1e-3 * p, rel_tol=1e-12)
    bg = M.background(case, k)
    assert bg.n_dipoles == 1 and bg.dipole[0][5] == M.DIPOLE[5]
    assert bg.B_imf[2] == M.UPSTREAM[8] and bg.L_ref == k.L_ref and bg.inver_Rem == 0.0
    res = M.ShellCase(na=8, nr=12, resistive=True)
    kr = M.constants(res)
    assert M.background(res, kr).inver_Rem == pytest.approx(1.25e7 / (kr.mu0 * kr.U_ref * kr.L_ref), rel=1e-15)


def test_reference_jobs_match_the_members():
    """The reference arm's harness jobs carry each member's size and upstream."""
    import bench
    from mpcns_mercury_b200 import magnetosphere as M

    class A:
        workload = "shells"
        solves = 5

    members = bench.reference_members(A())
    for (job, cells), c in zip(members, M.ensemble(5)):
        assert job["na"] == c.na and job["nr"] == c.nr and cells == c.cell_count()
        assert [float(v) for v in job["initial_line"].split()] == [float(v) for v in c.upstream]
        assert float(job["farfield_line"].split()[0]) == float(c.upstream[0])
        assert job["na_fraction"] == c.na_fraction
        # the configuration's implicit resistivity, solved to the same tolerance
        assert c.resistive and job["resistive"] == 1 and job["ksp_rtol"] == c.res_rtol == 1e-10
        assert (job["eta_r_inner"], job["eta_r_outer"], job["eta_width"]) == (0.0, 1.0, 0.4)
        assert job["eta_max"] == pytest.approx(1e-3 * 1.256637061e-6 * 4.031e5 * 2.44e6, rel=1e-15)


def test_resistivity_window_follows_the_stated_profile():
    """The tanh window of ETA_CONFIG against eta = 1e-3 exp(-(r - 1) / 0.2):
    within 1.5 % for r >= 2, 9 % at r = 1.5, half of it at the surface."""
    from mpcns_mercury_b200 import magnetosphere as M

    c = M.ETA_CONFIG
    k = M.constants(M.ShellCase(resistive=True, **c))
    inver_Rem = c["eta_max"] / (k.mu0 * k.U_ref * k.L_ref)
    assert inver_Rem == pytest.approx(1e-3, rel=1e-12)
    w, r0, r1 = c["eta_width"], c["eta_r_inner"], c["eta_r_outer"]
    for r in np.linspace(1.5, 4.0, 11):
        eta = inver_Rem * 0.5 * (math.tanh((r - r0) / w) - math.tanh((r - r1) / w))
        assert eta == pytest.approx(1e-3 * math.exp(-(r - 1.0) / 0.2), rel=1.5e-2 if r >= 2.0 else 9e-2)
    eta1 = inver_Rem * 0.5 * (math.tanh((1.0 - r0) / w) - math.tanh(0.0))
    assert eta1 == pytest.approx(0.5e-3, rel=2e-2)


def test_fluid_tile_shapes_and_shape_classes():
    from mpcns_mercury_b200 import autotune, capi

    shapes = [capi.fluid_tile_shape(v) for v in range(capi.NUM_FLUID_TILES)]
    assert shapes[0] == (16, 4, 4, 3)
    assert all(k * j * i == 256 and ctas in (2, 3, 4) for k, j, i, ctas in shapes)
    # variant 6 is variant 0's tile with its cells staged by TMA tensor copies
    assert len(set(shapes[:6])) == 6 and shapes[6] == shapes[0]
    with pytest.raises(capi.MhdError):
        capi.fluid_tile_shape(capi.NUM_FLUID_TILES)
    assert autotune.shape_class([(24, 24, 30)] * 6) == "k<=32-j<=32"
    assert autotune.shape_class([(48, 48, 96)] * 6) == "k<=128-j<=64"
