"""Mixed precision (FP32 state, work fields and flux/EMF/update arithmetic;
FP64 metric Jac/JD) against the reference's FP64 step, on the periodic
curvilinear Orszag-Tang cube (32^3, 100 steps).

Tolerance: per-field relative L2 <= 1e-5 over the owned DOFs of the state
(U_H, U_Na, B faces) after 100 steps; div B (max |sum of face fluxes| over
max |B face|) stays at FP32 roundoff (<= 1e-5) while the FP64 path keeps it
at FP64 roundoff (<= 1e-12)."""
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def cube32(ref_oracle):
    if not has_gpu():
        pytest.skip("no GPU")
    return ref_oracle.cube_run(n=32, steps=100, dump_at=[0, 100])


def test_mixed_precision_error_vs_reference(cube32):
    import mercury_oracle as mo
    from gpu_helpers import compare, context_from_dump, div_b

    ctx = context_from_dump(cube32, 32, precision=1)
    ctx.prepare()
    d0 = div_b(ctx, 32)
    ctx.step(100)
    worst, bad = compare(ctx, cube32, "step100:", mo.STATE_FIELDS, TOL)
    print("mixed precision rel L2 after 100 steps:", worst, "div B before/after:", d0, div_b(ctx, 32))
    assert not bad, worst
    assert div_b(ctx, 32) <= 1e-5
    info = ctx.info()
    ref_dt, ref_time = cube32[("step100:dt_time", -1)].data.ravel()
    assert info.step == 100 and abs(info.time - ref_time) <= 1e-5 * ref_time


def test_fp64_div_b_roundoff(cube32):
    from gpu_helpers import context_from_dump, div_b

    ctx = context_from_dump(cube32, 32)
    ctx.prepare()
    ctx.step(100)
    assert div_b(ctx, 32) <= 1e-12
