"""The GPU step on the 6-panel cubed-sphere shell (the magnetosphere
configuration: inner solid wall, outer Farfield, eight valence-3 radial
lines, a centred dipole background field, two ion fluids with Na+ at 1e-3,
Hall with the reference's radial taper, electron pressure) against the
reference built from its own sources (oracle/_ref) on identical inputs,
through the C ABI.  The sync tables come from the library's own builder
(mhd_topology_cubed_sphere), the static inputs from the reference's setup.

Tolerance: FP64 <= 1e-12 relative L2 per field over the owned DOFs (the path
is built without FMA contraction, in the reference's operation order, and is
expected to be bitwise equal)."""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

TOL = 1e-12
NA, NR, STEPS = 8, 12, 5


@pytest.fixture(scope="module")
def shell(ref_oracle):
    if not has_gpu():
        pytest.skip("no GPU")
    return ref_oracle.shell_run(na=NA, nr=NR, steps=STEPS, dump_at=[0, 1, STEPS])


def test_shell_prepare_reproduces_derived_fields(shell):
    import mercury_oracle as mo
    from gpu_helpers import compare, shell_context

    ctx = shell_context(shell, NA, NR)
    ctx.prepare()
    worst, bad = compare(ctx, shell, "step0:", mo.DERIVED_FIELDS, TOL)
    print("shell prepare: max rel L2", max(worst.values()))
    assert not bad, {k: v for k, v in worst.items() if v > TOL}
    ctx.close()


@pytest.mark.parametrize("steps", [1, STEPS])
def test_shell_step_matches_reference(shell, steps):
    import mercury_oracle as mo
    from gpu_helpers import compare, shell_context

    ctx = shell_context(shell, NA, NR)
    ctx.prepare()
    ctx.step(steps)
    worst, bad = compare(ctx, shell, f"step{steps}:", mo.STATE_FIELDS + mo.DERIVED_FIELDS, TOL)
    print(f"shell {steps} steps: max rel L2", max(worst.values()))
    assert not bad, {k: v for k, v in worst.items() if v > TOL}
    ref_dt, ref_time = shell[(f"step{steps}:dt_time", -1)].data.ravel()
    info = ctx.info()
    assert info.status == 0 and info.step == steps
    assert abs(info.dt - ref_dt) <= 1e-14 * ref_dt
    ctx.close()


def test_shell_mixed_precision(shell):
    """The shell in mixed precision (FP32 state/flux/EMF/update, FP64 metric):
    per-field relative L2 <= 1e-5 against the reference's FP64 step."""
    import mercury_oracle as mo
    from gpu_helpers import compare, shell_context

    ctx = shell_context(shell, NA, NR, precision=1)
    ctx.prepare()
    ctx.step(STEPS)
    worst, bad = compare(ctx, shell, f"step{STEPS}:", mo.STATE_FIELDS, 1e-5)
    print(f"shell mixed {STEPS} steps: max rel L2", max(worst.values()))
    assert not bad, {k: v for k, v in worst.items() if v > 1e-5}
    ctx.close()


def test_shell_div_b_matches_reference(ref_oracle):
    """div B of the induced face flux after the steps, against the
    reference's own calc_divB on the shell (no Pole patches, so no zeroed
    shell): bit for bit on the owned cells, and at roundoff."""
    if not has_gpu():
        pytest.skip("no GPU")
    from gpu_helpers import shell_context

    dump = ref_oracle.shell_run(na=NA, nr=NR, steps=STEPS, dump_at=[0, STEPS],
                                extra={"calc_divb": 1, "dump_fields": "U_H U_Na B_xi B_eta B_zeta divB"})
    ctx = shell_context(dump, NA, NR)
    ctx.prepare()
    ctx.step(STEPS)
    m = ctx.div_b()
    worst = 0.0
    for b in range(6):
        r = dump[(f"step{STEPS}:divB", b)]
        dev = ctx.download("DIVB", r.lo, r.hi, block=b)
        g = [-v for v in r.lo]
        sl = (slice(g[0], g[0] + NA), slice(g[1], g[1] + NA), slice(g[2], g[2] + NR))
        assert np.array_equal(dev[sl], r.data[sl]), b
        worst = max(worst, float(np.abs(r.data[sl]).max()))
    assert m == worst
    assert m < 1e-10
    ctx.close()


@pytest.fixture(scope="module")
def config2(ref_oracle):
    """The configuration's own shell: 6 panels of 48 x 48 x 96 cells
    (r_k = 8^(k/96)), 10 steps on the reference."""
    if not has_gpu():
        pytest.skip("no GPU")
    return ref_oracle.shell_run(na=48, nr=96, steps=10, dump_at=[0, 10],
                                extra={"dump_fields": "U_H U_Na B_xi B_eta B_zeta"})


@pytest.mark.parametrize("precision,tol", [(0, TOL), (1, 1e-5)], ids=["fp64", "mixed"])
def test_config2_shell_matches_reference(config2, precision, tol):
    import mercury_oracle as mo
    from gpu_helpers import compare, shell_context

    ctx = shell_context(config2, 48, 96, precision=precision)
    ctx.prepare()
    ctx.step(10)
    worst, bad = compare(ctx, config2, "step10:", mo.STATE_FIELDS, tol)
    print("6 x 48x48x96 shell, 10 steps, precision", precision, "max rel L2", max(worst.values()))
    assert not bad, {k: v for k, v in worst.items() if v > tol}
    assert ctx.info().status == 0
    ctx.close()


RES_EXTRA = dict(resistive=1, ksp_rtol=1e-14, ksp_atol=1e-300, ksp_max_it=4000)


@pytest.fixture(scope="module")
def res_shell(ref_oracle):
    """The shell with the implicit resistive substep (the reference's radial
    tanh window of eta around the inner wall), solved to 1e-14 by the
    reference's GMRES."""
    if not has_gpu():
        pytest.skip("no GPU")
    return ref_oracle.shell_run(na=NA, nr=NR, steps=STEPS, dump_at=[0, STEPS], extra=RES_EXTRA)


def test_shell_implicit_resistivity_matches_reference(ref_oracle, res_shell):
    """Sync(Eres)/Sync(dB)/Sync(dJ) with the shell's physical boundaries and
    the singular edges' current inside the operator, B* restore and update:
    the state after the steps within 1e-10 relative L2 per field (CG in the
    1/(eta alpha)-weighted product against the reference's GMRES, both to a
    relative residual of 1e-14)."""
    import mercury_oracle as mo
    from gpu_helpers import compare, shell_constants, shell_context

    k = shell_constants(resistive=True, res_rtol=1e-14, res_max_it=2000)
    ctx = shell_context(res_shell, NA, NR, constants=k)
    ctx.prepare()
    ctx.step(STEPS)
    worst, bad = compare(ctx, res_shell, f"step{STEPS}:", mo.STATE_FIELDS, 1e-10)
    print("shell implicit resistivity: max rel L2", max(worst.values()))
    assert not bad, {k: v for k, v in worst.items() if v > 1e-10}
    info = ctx.info()
    assert info.status == 0 and info.res_iters > 0 and info.res_relres <= 1e-14
    # the substep is active: B differs from the run without it
    a = res_shell[(f"step{STEPS}:B_xi", 0)].data
    plain = ref_oracle.shell_run(na=NA, nr=NR, steps=STEPS, dump_at=[STEPS], extra={"dump_fields": "B_xi"})
    b = plain[(f"step{STEPS}:B_xi", 0)].data
    assert float(np.abs(a - b).max()) > 1e-9
    ctx.close()


def test_shell_implicit_resistivity_mixed(res_shell):
    """The mixed form on the shell: residual and its norms in FP64 on the
    solve's FP64 companion (with the singular edges' geometry), FP32 CG
    corrections, refined to 1e-10; the state within 1e-5 relative L2."""
    import mercury_oracle as mo
    from gpu_helpers import compare, shell_constants, shell_context

    k = shell_constants(resistive=True, res_rtol=1e-10, res_max_it=2000)
    ctx = shell_context(res_shell, NA, NR, precision=1, constants=k)
    ctx.prepare()
    ctx.step(STEPS)
    worst, bad = compare(ctx, res_shell, f"step{STEPS}:", mo.STATE_FIELDS, 1e-5)
    info = ctx.info()
    print("shell mixed implicit: refinements", info.res_refinements, "CG iterations", info.res_iters,
          "max rel L2", max(worst.values()))
    assert not bad, {k: v for k, v in worst.items() if v > 1e-5}
    assert info.status == 0 and info.res_relres <= 1e-10
    ctx.close()


def test_config2_shell_implicit_resistivity(ref_oracle):
    """The configuration's shell (6 x 48x48x96) with the implicit resistive
    substep, 3 steps, FP64: within 1e-10 relative L2 of the reference (CG
    against GMRES, both to 1e-14)."""
    if not has_gpu():
        pytest.skip("no GPU")
    import mercury_oracle as mo
    from gpu_helpers import compare, shell_constants, shell_context

    extra = dict(RES_EXTRA, dump_fields="U_H U_Na B_xi B_eta B_zeta")
    dump = ref_oracle.shell_run(na=48, nr=96, steps=3, dump_at=[0, 3], extra=extra)
    k = shell_constants(resistive=True, res_rtol=1e-14, res_max_it=4000)
    ctx = shell_context(dump, 48, 96, constants=k)
    ctx.prepare()
    ctx.step(3)
    worst, bad = compare(ctx, dump, "step3:", mo.STATE_FIELDS, 1e-10)
    info = ctx.info()
    print("6 x 48x48x96 shell, implicit resistivity, 3 steps: max rel L2", max(worst.values()),
          "CG iterations of the last substep", info.res_iters)
    assert not bad, {k: v for k, v in worst.items() if v > 1e-10}
    assert info.status == 0 and info.res_relres <= 1e-14
    ctx.close()
