"""Implicit resistive substep on the GPU against the reference build.

The reference (is_Mercury_resistance on, eta = eta_max_mercury / (mu0 U L)
times its radial tanh window 0.84 < r < 1.04, which crosses the unit cube)
solves (I + dt eta alpha C^T beta C) E = eta J(B*) with GMRES (no
preconditioner) after every explicit update; the GPU solves the same system
with preconditioned CG in the 1/(eta alpha)-weighted inner product.  Both run
to a relative residual of 1e-14, so the states agree to the solvers'
tolerance, not bitwise: tolerance 1e-10 relative L2 per field after 10 steps
of the 16^3 periodic curvilinear Orszag-Tang cube (the substep changes B by
O(1) relative to a run without it).

Mixed precision: the residual and its norms in FP64 on an FP64 companion of
the solve, corrections by FP32 CG, refined to 1e-10; the state after 10 steps
within the mixed path's tolerance of the FP64 reference, 1e-5 relative L2 per
field."""
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

TOL = 1e-10
MIXED_TOL = 1e-5
EXTRA = dict(resistive=1, ksp_rtol=1e-14, ksp_atol=1e-300, ksp_max_it=4000)


@pytest.fixture(scope="module")
def res_dump(ref_oracle):
    if not has_gpu():
        pytest.skip("no GPU")
    return ref_oracle.cube_run(n=16, steps=10, dump_at=[0, 10], extra=EXTRA)


def test_implicit_resistivity_matches_reference(ref_oracle, res_dump):
    import numpy as np

    import mercury_oracle as mo
    from gpu_helpers import compare, context_from_dump
    from mpcns_mercury_b200 import reference_constants

    dump = res_dump
    k = reference_constants(cfl=0.4, resistive=True, res_rtol=1e-14, res_max_it=2000)
    ctx = context_from_dump(dump, 16, constants=k)
    ctx.prepare()
    ctx.step(10)
    worst, bad = compare(ctx, dump, "step10:", mo.STATE_FIELDS, TOL)
    assert not bad, worst
    info = ctx.info()
    assert info.res_relres <= 1e-14 and info.res_iters > 0 and info.res_refinements == 0
    ref_dt, ref_time = dump[("step10:dt_time", -1)].data.ravel()
    assert info.step == 10 and abs(info.time - ref_time) <= 1e-10 * ref_time
    # the substep is active: B differs from a run without it
    plain = ref_oracle.cube_run(n=16, steps=10, dump_at=[10])
    a = dump[("step10:B_xi", 0)].data
    b = plain[("step10:B_xi", 0)].data
    assert float(np.abs(a - b).max()) > 1e-6
    print("implicit resistivity rel L2 vs reference:", worst)


def _mixed_constants(direct=0):
    from mpcns_mercury_b200 import reference_constants

    return reference_constants(cfl=0.4, resistive=True, res_rtol=1e-10, res_max_it=500, res_direct_iters=direct)


def test_mixed_precision_implicit_direct(res_dump):
    """The mixed form's solve as FP64 CG on the companion (no refinement), to
    1e-10: every substep under a threshold above its iteration count (1000);
    under the default threshold (20) the first substep only, the next ones
    switch to iterative refinement (this case takes ~100 iterations)."""
    import mercury_oracle as mo
    from gpu_helpers import compare, context_from_dump

    for direct in (1000, 0):
        ctx = context_from_dump(res_dump, 16, precision=1, constants=_mixed_constants(direct))
        ctx.prepare()
        refinements, iters = [], []
        for _ in range(10):
            ctx.step(1)
            info = ctx.info()
            assert info.status == 0
            assert info.res_relres <= 1e-10, info.res_relres
            refinements.append(info.res_refinements)
            iters.append(info.res_iters)
        assert refinements[0] == 0 and iters[0] > 20
        if direct == 1000:
            assert max(refinements) == 0
        else:
            assert min(refinements[1:]) >= 1
        worst, bad = compare(ctx, res_dump, "step10:", mo.STATE_FIELDS, MIXED_TOL)
        assert not bad, worst
        ctx.close()
        print("mixed implicit, direct threshold", direct, ": refinements", refinements, "CG iterations", iters,
              "rel L2 vs reference", worst)


def test_mixed_precision_implicit_resistivity(res_dump):
    import mercury_oracle as mo
    from gpu_helpers import compare, context_from_dump

    ctx = context_from_dump(res_dump, 16, precision=1, constants=_mixed_constants(direct=-1))
    ctx.prepare()
    refinements, iters = [], []
    for _ in range(10):
        ctx.step(1)
        info = ctx.info()
        assert info.status == 0
        assert info.res_relres <= 1e-10, info.res_relres
        refinements.append(info.res_refinements)
        iters.append(info.res_iters)
    # FP32 CG alone stops near 1e-7: every substep needed FP64-refined corrections
    assert min(refinements) >= 2
    worst, bad = compare(ctx, res_dump, "step10:", mo.STATE_FIELDS, MIXED_TOL)
    assert not bad, worst
    ctx.close()
    print("mixed implicit: refinements", refinements, "CG iterations", iters, "rel L2 vs reference", worst)


def test_mixed_precision_implicit_in_a_batch(res_dump):
    """Companion solves follow their solves through add, add_like and remove."""
    import numpy as np

    import mercury_oracle as mo
    from gpu_helpers import NGHOST, upload_from_dump
    from mpcns_mercury_b200.capi import REF_FIELD, Batch, SolveDesc

    k = _mixed_constants()
    d = SolveDesc([(16, 16, 16)], NGHOST, k, precision=1)
    b = Batch(3, 1)
    s0 = b.add(d)
    upload_from_dump(lambda f, a, lo, hi: b.upload(s0, f, a, lo, hi), res_dump)
    b.prepare(s0)
    s1 = b.add_like(s0)  # the template's fields: the same inputs
    b.prepare(s1)
    infos = b.poll()
    assert infos[s0].device_bytes == infos[s1].device_bytes
    fp64 = SolveDesc([(16, 16, 16)], NGHOST, k, precision=0)
    assert infos[s0].device_bytes > fp64.device_bytes()  # the FP64 companion is counted
    fp64.close()
    for s in (s0, s1):
        b.request(s, 4)
    b.run(4)
    infos = b.poll()
    for s in (s0, s1):
        assert infos[s].status == 0 and infos[s].step == 4 and infos[s].res_relres <= 1e-10
    for name in mo.STATE_FIELDS:
        r = res_dump[("step10:" + name, 0)]
        x0 = b.download(s0, REF_FIELD[name], r.lo, r.hi)
        x1 = b.download(s1, REF_FIELD[name], r.lo, r.hi)
        assert mo.rel_l2(x1, x0) <= 1e-6, name  # dot products sum in another order in each slot
    b.remove(s1)
    b.request(s0, 2)
    b.run(2)
    assert b.poll()[s0].step == 6 and b.poll()[s0].res_relres <= 1e-10
    b.remove(s0)
    b.close()
    d.close()


@pytest.mark.parametrize("precision,direct", [(0, 0), (1, 0), (1, -1)], ids=["fp64", "mixed-direct", "mixed-refined"])
def test_unconverged_substep_reports_solve_status(res_dump, precision, direct):
    """A solve capped below convergence ends its device loop at res_max_it
    and the step returns MHD_ERR_SOLVE (the reference throws there)."""
    from gpu_helpers import context_from_dump
    from mpcns_mercury_b200 import reference_constants
    from mpcns_mercury_b200.capi import MhdError

    # one CG iteration per solve: the operator needs about 200 to reach 1e-10
    k = reference_constants(cfl=0.4, resistive=True, res_rtol=1e-14, res_max_it=1, res_direct_iters=direct)
    ctx = context_from_dump(res_dump, 16, precision=precision, constants=k)
    ctx.prepare()
    with pytest.raises(MhdError):
        ctx.step(1)
    info = ctx.info()
    assert info.status == 6  # MHD_ERR_SOLVE
    if direct == 0:  # FP64 CG (on the FP64 companion in mixed precision)
        assert info.res_iters == 1 and info.res_refinements == 0
    else:  # 30 refinements of one FP32 iteration each
        assert info.res_refinements == 30 and info.res_iters == 30
    assert info.res_relres > 1e-14
    ctx.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_host_driven_cg_loop_matches_the_device_loop(res_dump, precision):
    """The substep's CG iterations launched from the host (for profilers)
    give the device loop's results bit for bit: the same kernels and the
    same fixed-order sums."""
    import mercury_oracle as mo
    from gpu_helpers import NGHOST, upload_from_dump
    from mpcns_mercury_b200.capi import REF_FIELD, Batch, SolveDesc

    import numpy as np

    k = _mixed_constants()
    k.res_rtol = 1e-12 if precision == 0 else 1e-10
    out = []
    for host in (False, True):
        d = SolveDesc([(16, 16, 16)], NGHOST, k, precision=precision)
        b = Batch(1, precision)
        s = b.add(d)
        if host:
            b.cg_host_loop(True)
        upload_from_dump(lambda f, a, lo, hi: b.upload(s, f, a, lo, hi), res_dump)
        b.prepare(s)
        b.request(s, 3)
        b.run(3)
        inf = b.poll()[s]
        assert inf.status == 0 and inf.step == 3 and inf.res_iters > 0
        out.append({n: b.download(s, REF_FIELD[n], res_dump[("step10:" + n, 0)].lo, res_dump[("step10:" + n, 0)].hi)
                    for n in mo.STATE_FIELDS})
        b.close()
        d.close()
    for n in mo.STATE_FIELDS:
        assert np.array_equal(out[0][n], out[1][n]), n
