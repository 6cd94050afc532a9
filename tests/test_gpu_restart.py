"""Restart round trips between the GPU solve and the reference, through
MPCNSRST version 1 files (mhd_save_restart / mhd_load_restart and the
reference's own IOModule writer and reader, src/6_io/IOModule_Bin.cpp:168-420),
on the periodic curvilinear Orszag-Tang cube in FP64:

* a checkpoint the GPU writes after A steps is the reference's checkpoint
  after A steps, byte for byte (the time to 1e-13 relative, as the parity
  tests compare it);
* the reference resumed from the GPU's checkpoint, and the GPU resumed from
  the reference's, reach after B more steps the state of the reference's
  uninterrupted A + B steps, bit for bit."""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

N = 12
A = 3
B = 2
TIME_OFF = 16  # byte offset of the time in the header: magic, version, step


@pytest.fixture(scope="module")
def runs(ref_oracle, tmp_path_factory):
    if not has_gpu():
        pytest.skip("no GPU")
    d = tmp_path_factory.mktemp("gpu_restart")
    full = ref_oracle.cube_run(n=N, steps=A + B, dump_at=[0, A, A + B], workdir=str(d / "full"))
    ref_ckpt = str(d / "ref_ckpt.bin")
    job = dict(ref_oracle.CUBE_JOB)
    job.update(n=N, steps=A, dump_at=str(A), write_restart=ref_ckpt, dump_fields="U_H")
    ref_oracle.run_job(job, workdir=str(d / "ckpt"))
    return d, full, ref_ckpt


def _owned(rec):
    g = [-v for v in rec.lo]
    return rec.data[g[0]:rec.hi[0], g[1]:rec.hi[1], g[2]:rec.hi[2]]


def _same_files(a, b):
    ra, rb = open(a, "rb").read(), open(b, "rb").read()
    ta = np.frombuffer(ra[TIME_OFF:TIME_OFF + 8], np.float64)[0]
    tb = np.frombuffer(rb[TIME_OFF:TIME_OFF + 8], np.float64)[0]
    assert abs(ta - tb) <= 1e-13 * abs(tb)
    assert len(ra) == len(rb)
    assert ra[:TIME_OFF] == rb[:TIME_OFF] and ra[TIME_OFF + 8:] == rb[TIME_OFF + 8:]


def test_gpu_checkpoint_is_the_reference_checkpoint(runs):
    import mercury_oracle as mo
    from gpu_helpers import compare, context_from_dump

    d, full, ref_ckpt = runs
    ctx = context_from_dump(full, N)
    ctx.prepare()
    ctx.step(A)
    mine = str(d / "gpu_ckpt.bin")
    ctx.save_restart(mine)
    _same_files(mine, ref_ckpt)
    # saving fills only ghost layers the step does not read: the run goes on unchanged
    ctx.step(B)
    worst, bad = compare(ctx, full, f"step{A + B}:", mo.STATE_FIELDS, 0.0)
    assert not bad, worst
    ctx.close()


def test_reference_resumes_from_gpu_checkpoint(runs, ref_oracle):
    from gpu_helpers import context_from_dump

    d, full, _ = runs
    ctx = context_from_dump(full, N)
    ctx.prepare()
    ctx.step(A)
    mine = str(d / "gpu_ckpt2.bin")
    ctx.save_restart(mine)
    ctx.close()
    job = dict(ref_oracle.CUBE_JOB)
    job.update(n=N, steps=B, dump_at=str(B), read_restart=mine, restart_step0=A,
               dump_fields=" ".join(ref_oracle.STATE_FIELDS))
    resumed = ref_oracle.run_job(job, workdir=str(d / "resume"))
    for name in ref_oracle.STATE_FIELDS:
        assert np.array_equal(_owned(resumed[(f"step{B}:{name}", 0)]), _owned(full[(f"step{A + B}:{name}", 0)])), name


def test_gpu_resumes_from_reference_checkpoint(runs):
    import mercury_oracle as mo
    from gpu_helpers import compare, context_from_dump

    d, full, ref_ckpt = runs
    ctx = context_from_dump(full, N)  # static inputs; the state is replaced by the checkpoint's
    step, time = ctx.load_restart(ref_ckpt)
    assert step == A
    ref_dt, ref_time = full[(f"step{A}:dt_time", -1)].data.ravel()
    assert time == ref_time
    info = ctx.info()
    assert info.step == A and info.time == ref_time
    ctx.step(B)
    worst, bad = compare(ctx, full, f"step{A + B}:", mo.STATE_FIELDS + mo.DERIVED_FIELDS, 0.0)
    assert not bad, worst
    assert ctx.info().step == A + B
    ctx.close()
