"""The fluid kernel's tile variants and their autotuner: every variant gives
the same steps bit for bit (FP64 and mixed), and timing the variants on a
batch leaves its solves unchanged."""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu


def _state(get, case):
    n = (case.na, case.na, case.nr)
    out = []
    for name, st in (("U_H", (0, 0, 0)), ("U_NA", (0, 0, 0)), ("B_XI", (1, 0, 0)), ("B_ETA", (0, 1, 0)),
                     ("B_ZETA", (0, 0, 1))):
        hi = tuple(n[a] + st[a] for a in range(3))
        out += [get(name, (0, 0, 0), hi, b) for b in range(6)]
    return out


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_every_fluid_tile_gives_the_same_steps(precision):
    if not has_gpu():
        pytest.skip("no GPU")
    from mpcns_mercury_b200 import capi
    from mpcns_mercury_b200 import magnetosphere as M

    case = M.ShellCase(na=10, nr=14)  # extents that no tile divides evenly
    ref = None
    for v in range(capi.NUM_FLUID_TILES):
        ctx = M.context(case, precision=precision)
        ctx.fluid_tile(v)
        ctx.step(4)
        st = _state(lambda f, lo, hi, b: ctx.download(f, lo, hi, block=b), case)
        ctx.close()
        if ref is None:
            ref = st
        else:
            assert all(np.array_equal(a, b) for a, b in zip(st, ref)), v


def test_timing_the_tiles_leaves_the_solves_unchanged():
    if not has_gpu():
        pytest.skip("no GPU")
    from mpcns_mercury_b200 import autotune, capi
    from mpcns_mercury_b200 import magnetosphere as M
    from mpcns_mercury_b200.capi import Batch, SolveDesc

    cases = [M.ShellCase(na=10, nr=14), M.ShellCase(na=12, nr=9, upstream=M.ensemble(1)[0].upstream)]
    results = []
    for tune in (False, True):
        b = Batch(2, 1)
        slots = []
        for c in cases:
            k = M.constants(c)
            d = SolveDesc(c.cells, 4, k, precision=1, topology=M.topology(c))
            s = b.add(d)
            d.close()
            M.set_up(b, c, slot=s, k=k)
            b.prepare(s)
            b.request(s, 5)
            slots.append(s)
        if tune:
            t = autotune.tune(b, 1, [n for c in cases for n in c.cells], reps=2, cache=None)
            assert len(t["ms"]) == capi.NUM_FLUID_TILES and all(v > 0 for v in t["ms"])
            assert t["ms"][t["variant"]] == min(t["ms"])
        b.run(5)
        info = b.poll()
        assert all(info[s].status == 0 and info[s].step == 5 for s in slots)
        results.append([_state(lambda f, lo, hi, blk: b.download(s, f, lo, hi, block=blk), c)
                        for s, c in zip(slots, cases)])
        b.close()
    for a, c in zip(results[0], results[1]):
        assert all(np.array_equal(x, y) for x, y in zip(a, c))
