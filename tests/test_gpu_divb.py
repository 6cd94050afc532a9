"""div B on the device (mhd_div_b) against the reference's own calc_divB
after 20 steps of the 16^3 periodic curvilinear Orszag-Tang cube: the field
bit for bit on the owned cells and its maximum; constrained transport keeps
it at roundoff."""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu


def test_div_b_matches_reference(ref_oracle):
    if not has_gpu():
        pytest.skip("no GPU")
    from gpu_helpers import context_from_dump

    dump = ref_oracle.cube_run(n=16, steps=20, dump_at=[0, 20], extra={"calc_divb": 1, "dump_fields": "U_H U_Na B_xi B_eta B_zeta divB"})
    ctx = context_from_dump(dump, 16)
    ctx.prepare()
    ctx.step(20)
    m = ctx.div_b()
    r = dump[("step20:divB", 0)]
    dev = ctx.download("DIVB", r.lo, r.hi)
    g = [-v for v in r.lo]
    sl = (slice(g[0], g[0] + 16), slice(g[1], g[1] + 16), slice(g[2], g[2] + 16))
    assert np.array_equal(dev[sl], r.data[sl])
    assert m == float(np.abs(r.data[sl]).max())
    assert m < 1e-10
