"""Batched solves (mhd_batch): every solve's result is the same alone and in
the mix, bit for bit, including solves that join, finish and leave while
others are running on the same CUDA graph.

The single-solve path (mhd_ctx) is itself pinned against the reference in
test_gpu_parity.py; here each batched solve is compared with a single-solve
run of the same inputs, at tolerance 0 (same kernels, same operation order)."""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

SIZES = {0: (8, 8, 8), 1: (10, 8, 12), 2: (12, 12, 12), 3: (8, 12, 10)}


@pytest.fixture(scope="module")
def cases():
    if not has_gpu():
        pytest.skip("no GPU")
    from mpcns_mercury_b200 import workloads as W

    return {sid: W.case_fields(n, solve_id=sid) for sid, n in SIZES.items()}


def _single(fields, n, steps):
    from mpcns_mercury_b200 import Context, reference_constants
    from mpcns_mercury_b200 import workloads as W

    ctx = Context([n], W.NGHOST, reference_constants(cfl=0.4))
    W.upload_case(lambda f, a, lo, hi, b: ctx.upload(f, a, lo, hi, block=b), fields)
    ctx.sync("UCELL")
    ctx.sync("BFACE")
    ctx.prepare()
    if steps:
        ctx.step(steps)
    out = {name: ctx.download(W.capi_field(name), fields[name].lo, fields[name].hi) for name in W.STATE_FIELDS}
    info = ctx.info()
    ctx.close()
    return out, info


def _add(batch, fields, n):
    from mpcns_mercury_b200 import reference_constants
    from mpcns_mercury_b200 import workloads as W
    from mpcns_mercury_b200.capi import SolveDesc

    d = SolveDesc([n], W.NGHOST, reference_constants(cfl=0.4))
    slot = batch.add(d)
    W.upload_case(lambda f, a, lo, hi, b: batch.upload(slot, f, a, lo, hi, block=b), fields)
    batch.sync(slot, "UCELL")
    batch.sync(slot, "BFACE")
    batch.prepare(slot)
    return slot, d


def _state(batch, slot, fields):
    from mpcns_mercury_b200 import workloads as W

    return {name: batch.download(slot, W.capi_field(name), fields[name].lo, fields[name].hi)
            for name in W.STATE_FIELDS}


def _same(a, b):
    return all(np.array_equal(a[k], b[k]) for k in a)


def test_batch_equals_single(cases):
    from mpcns_mercury_b200.capi import Batch

    ref = {sid: _single(cases[sid], SIZES[sid], 4) for sid in (0, 1, 2)}
    b = Batch(4)
    slots = {sid: _add(b, cases[sid], SIZES[sid]) for sid in (0, 1, 2)}
    for sid, (slot, _) in slots.items():
        b.request(slot, 4)
    b.run(4)
    infos = b.poll()
    for sid, (slot, _) in slots.items():
        got = _state(b, slot, cases[sid])
        assert _same(got, ref[sid][0]), f"solve {sid} differs from its single run"
        assert infos[slot].step == 4 and infos[slot].remaining == 0 and infos[slot].status == 0
        assert infos[slot].dt == ref[sid][1].dt and infos[slot].time == ref[sid][1].time
    b.close()


def test_batch_membership_changes(cases):
    """Solves with different step counts; one leaves and a new one joins its
    slot between graph launches; the survivors continue unaffected."""
    from mpcns_mercury_b200.capi import Batch

    b = Batch(3)
    s0, d0 = _add(b, cases[0], SIZES[0])
    s1, d1 = _add(b, cases[1], SIZES[1])
    b.request(s0, 3)
    b.request(s1, 5)
    b.run(5)  # s0 idles for the last two launches
    infos = b.poll()
    assert infos[s0].step == 3 and infos[s1].step == 5
    assert _same(_state(b, s0, cases[0]), _single(cases[0], SIZES[0], 3)[0])
    assert _same(_state(b, s1, cases[1]), _single(cases[1], SIZES[1], 5)[0])
    b.remove(s1)
    s3, d3 = _add(b, cases[3], SIZES[3])
    assert s3 == s1  # the freed slot is reused
    b.request(s0, 2)
    b.request(s3, 2)
    b.run(2)
    assert _same(_state(b, s0, cases[0]), _single(cases[0], SIZES[0], 5)[0])
    assert _same(_state(b, s3, cases[3]), _single(cases[3], SIZES[3], 2)[0])
    b.close()


def test_batch_request_before_prepare_is_refused(cases):
    from mpcns_mercury_b200 import reference_constants
    from mpcns_mercury_b200 import workloads as W
    from mpcns_mercury_b200.capi import Batch, MhdError, SolveDesc

    b = Batch(1)
    d = SolveDesc([SIZES[0]], W.NGHOST, reference_constants(cfl=0.4))
    slot = b.add(d)
    with pytest.raises(MhdError):
        b.request(slot, 1)
    with pytest.raises(MhdError):
        b.add(d)  # capacity 1 is full
    b.close()


def test_reserved_pool_equals_single(cases):
    """Solves added after mhd_batch_reserve take their memory from the grown
    pool; a solve removed and another added in its place reuse it.  Results
    stay bitwise equal to the single-solve path."""
    from mpcns_mercury_b200 import reference_constants
    from mpcns_mercury_b200 import workloads as W
    from mpcns_mercury_b200.capi import Batch, MhdError, SolveDesc

    ref = {sid: _single(cases[sid], SIZES[sid], 3) for sid in (0, 3)}
    b = Batch(2)
    need = 0
    for sid in (0, 3):
        d = SolveDesc([SIZES[sid]], W.NGHOST, reference_constants(cfl=0.4))
        need += d.device_bytes()
        d.close()
    b.reserve(need)
    with pytest.raises(MhdError):
        b.reserve(-1)
    slot, d = _add(b, cases[3], SIZES[3])
    b.request(slot, 1)
    b.run(1)
    b.remove(slot)  # its memory goes back to the pool
    d.close()
    for sid in (0, 3):
        slot, d = _add(b, cases[sid], SIZES[sid])
        b.request(slot, 3)
        b.run(3)
        assert b.poll()[slot].step == 3
        assert _same(_state(b, slot, cases[sid]), ref[sid][0])
        b.remove(slot)
        d.close()
    b.close()


def test_add_periodic_equals_explicit_tables(cases):
    """A solve added with mhd_batch_add_periodic (tables compiled straight from
    the periodic connectivity) steps bit for bit like the same solve added
    from the explicit copy lists of mhd_topology_periodic_block, in both
    precisions."""
    from mpcns_mercury_b200 import reference_constants
    from mpcns_mercury_b200 import workloads as W
    from mpcns_mercury_b200.capi import Batch, SolveDesc

    k0 = reference_constants(cfl=0.4)
    n, fields = SIZES[1], cases[1]
    for precision in (0, 1):
        b = Batch(2, precision)
        d = SolveDesc([n], W.NGHOST, k0, precision=precision)
        slots = [b.add(d), b.add_periodic(n, W.NGHOST, k0)]
        for slot in slots:
            W.upload_case(lambda f, a, lo, hi, blk: b.upload(slot, f, a, lo, hi, block=blk), fields)
            b.sync(slot, "UCELL")
            b.sync(slot, "BFACE")
            b.prepare(slot)
            b.request(slot, 5)
        b.run(5)
        assert _same(_state(b, slots[1], fields), _state(b, slots[0], fields)), precision
        b.close()
        d.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_nonfinite_solve_retires_alone(cases, precision):
    """A NaN planted in one owned cell of one solve's uploaded state: that
    solve retires with MHD_ERR_NONFINITE at its next step, its state is left
    as it was, and the other solves of the batch finish every requested step
    with the same result as when run without it."""
    from mpcns_mercury_b200 import reference_constants
    from mpcns_mercury_b200 import workloads as W
    from mpcns_mercury_b200.capi import Batch, SolveDesc

    steps = 4
    bad_sid, good = 1, (0, 2)

    def add(b, fields, n):
        d = SolveDesc([n], W.NGHOST, reference_constants(cfl=0.4), precision=precision)
        slot = b.add(d)
        W.upload_case(lambda f, a, lo, hi, blk: b.upload(slot, f, a, lo, hi, block=blk), fields)
        b.sync(slot, "UCELL")
        b.sync(slot, "BFACE")
        b.prepare(slot)
        b.request(slot, steps)
        return slot, d

    clean = Batch(4, precision)
    ref = {sid: add(clean, cases[sid], SIZES[sid]) for sid in good}
    clean.run(steps)
    ref_state = {sid: _state(clean, ref[sid][0], cases[sid]) for sid in good}

    poisoned = {k: v for k, v in cases[bad_sid].items()}
    u = poisoned["U_Na"]
    data = u.data.copy()
    g = [-v for v in u.lo]
    data[g[0] + 3, g[1] + 2, g[2] + 5, 4] = np.nan  # energy of one owned cell
    poisoned["U_Na"] = type(u)(u.lo, u.hi, data)

    b = Batch(4, precision)
    slots = {sid: add(b, cases[sid] if sid != bad_sid else poisoned, SIZES[sid]) for sid in (0, 1, 2)}
    b.run(steps)
    infos = b.poll()
    from mpcns_mercury_b200.capi import STATUS

    assert STATUS[infos[slots[bad_sid][0]].status] == "ERR_NONFINITE"
    assert infos[slots[bad_sid][0]].step == 0
    for sid in good:
        slot = slots[sid][0]
        assert infos[slot].status == 0 and infos[slot].step == steps
        assert _same(_state(b, slot, cases[sid]), ref_state[sid]), sid
    for bb, ss in ((clean, ref), (b, slots)):
        for _, d in ss.values():
            d.close()
        bb.close()
