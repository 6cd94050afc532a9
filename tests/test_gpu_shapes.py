"""The GPU step on non-cubic periodic boxes (shapes of the ensemble's size
distribution, one z-elongated) and on a periodic box cut into a 2 x 2 x 2
lattice of blocks, against the reference built from its own sources
(oracle/_ref) on identical seeded inputs, through the C ABI.

Tolerances, per field, relative L2 over the owned DOFs:
  FP64 path   <= 1e-12 (built without FMA contraction in the reference's
              operation order; expected bitwise)
  mixed path  <= 1e-5  (FP32 state/flux/EMF/update, FP64 metric)
Block shapes that are not cubes exercise the per-axis extents of every
kernel's index arithmetic (a transposed axis would pass on a cube); the
lattice exercises the multi-block halo, owner and edge-alias tables on the
device (inner patches between blocks, periodic ones where a patch wraps)."""
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-5
STEPS = 20

# (cells per axis): two members of the ensemble's distribution and a
# z-elongated block (24 x 40 x 128, the long axis is the contiguous one)
SHAPES = [(10, 14, 18), (26, 20, 33), (24, 40, 128)]


def _box_run(ref_oracle, cells, steps, extra=None):
    job_n = " ".join(map(str, cells))
    return ref_oracle.cube_run(n=job_n, steps=steps, dump_at=[0, steps], extra=extra)


@pytest.fixture(scope="module", params=SHAPES, ids=lambda c: "x".join(map(str, c)))
def box(ref_oracle, request):
    if not has_gpu():
        pytest.skip("no GPU")
    return request.param, _box_run(ref_oracle, request.param, STEPS)


@pytest.mark.parametrize("precision,tol", [(0, FP64_TOL), (1, MIXED_TOL)], ids=["fp64", "mixed"])
def test_box_matches_reference(box, precision, tol):
    import mercury_oracle as mo
    from gpu_helpers import compare, context_from_dump

    cells, dump = box
    ctx = context_from_dump(dump, cells, precision=precision)
    ctx.prepare()
    ctx.step(STEPS)
    names = mo.STATE_FIELDS + (mo.DERIVED_FIELDS if precision == 0 else [])
    worst, bad = compare(ctx, dump, f"step{STEPS}:", names, tol)
    print(cells, "precision", precision, "rel L2:", worst)
    assert not bad, worst
    ref_dt, ref_time = dump[(f"step{STEPS}:dt_time", -1)].data.ravel()
    info = ctx.info()
    assert info.step == STEPS
    assert abs(info.time - ref_time) <= (1e-13 if precision == 0 else 1e-5) * ref_time
    ctx.close()


@pytest.fixture(scope="module")
def lattice(ref_oracle):
    if not has_gpu():
        pytest.skip("no GPU")
    return ref_oracle.cube_run(n=8, steps=STEPS, dump_at=[0, STEPS], extra={"case": "lattice", "nb": "2 2 2"})


@pytest.mark.parametrize("precision,tol", [(0, FP64_TOL), (1, MIXED_TOL)], ids=["fp64", "mixed"])
def test_lattice_matches_reference(lattice, precision, tol):
    """Eight 8^3 blocks tiling the periodic box, stepped 20 times on the GPU
    (one solve of eight blocks) against the reference's multi-block run."""
    import mercury_oracle as mo
    from gpu_helpers import compare, context_from_dump

    ctx = context_from_dump(lattice, 8, precision=precision, lattice=(2, 2, 2))
    ctx.prepare()
    ctx.step(STEPS)
    names = mo.STATE_FIELDS + (mo.DERIVED_FIELDS if precision == 0 else [])
    worst, bad = compare(ctx, lattice, f"step{STEPS}:", names, tol)
    print("lattice precision", precision, "max rel L2:", max(worst.values()))
    assert not bad, {k: v for k, v in worst.items() if v > tol}
    assert ctx.info().step == STEPS
    ctx.close()
