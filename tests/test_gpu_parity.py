"""FP64 GPU step vs the reference built from its own sources (oracle/_ref),
on the periodic curvilinear Orszag-Tang cube (32^3, two ion
fluids, Hall + electron pressure), through the C ABI.

Tolerance: the FP64 path must match to <= 1e-12 relative L2 per field after
the stated steps (it is built without FMA contraction, in the reference's
operation order, and is expected to be bitwise equal)."""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def cube16(ref_oracle):
    if not has_gpu():
        pytest.skip("no GPU")
    return ref_oracle.cube_run(n=16, steps=20, dump_at=[0, 1, 20])


def test_prepare_reproduces_derived_fields(cube16):
    import mercury_oracle as mo
    from gpu_helpers import compare, context_from_dump

    ctx = context_from_dump(cube16, 16)
    ctx.prepare()
    worst, bad = compare(ctx, cube16, "step0:", mo.DERIVED_FIELDS, 0.0)
    assert not bad, worst


@pytest.mark.parametrize("steps", [1, 20])
def test_step_matches_reference(cube16, steps):
    import mercury_oracle as mo
    from gpu_helpers import compare, context_from_dump

    ctx = context_from_dump(cube16, 16)
    ctx.prepare()
    ctx.step(steps)
    worst, bad = compare(ctx, cube16, f"step{steps}:", mo.STATE_FIELDS + mo.DERIVED_FIELDS, TOL)
    assert not bad, worst
    ref_dt, ref_time = cube16[(f"step{steps}:dt_time", -1)].data.ravel()
    info = ctx.info()
    assert abs(info.dt - ref_dt) <= 1e-14 * ref_dt
    assert abs(info.time - ref_time) <= 1e-13 * ref_time
    assert info.step == steps


def test_cube32_100_steps(ref_oracle):
    """The full 32^3 cube, 100 steps."""
    if not has_gpu():
        pytest.skip("no GPU")
    import mercury_oracle as mo
    from gpu_helpers import compare, context_from_dump

    dump = ref_oracle.cube_run(n=32, steps=100, dump_at=[0, 100])
    ctx = context_from_dump(dump, 32)
    ctx.prepare()
    ctx.step(100)
    worst, bad = compare(ctx, dump, "step100:", mo.STATE_FIELDS, TOL)
    assert not bad, worst
