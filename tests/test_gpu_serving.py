"""Request loop (mpcns_mercury_b200.serving): requests that arrive while
others run are admitted as slots and device memory free up, and every
result is the same as the request run alone — bitwise for the FP64 server,
within 1e-5 relative L2 per field for the mixed-precision server."""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu


def _requests(keep=True):
    from mpcns_mercury_b200 import serving as SV
    from mpcns_mercury_b200 import workloads as W

    shapes = [(8, 8, 8), (10, 8, 12), (12, 10, 8)]
    cases = [W.case_fields(c, solve_id=i) for i, c in enumerate(shapes)]
    steps = [3, 7, 5, 4, 6, 2]
    return [SV.Request(rid=q, arrival_s=0.01 * q, cells=shapes[q % 3], steps=steps[q], fields=cases[q % 3],
                       keep_result=keep) for q in range(len(steps))]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("precision", [0, 1])
def test_serving_results_match_solo_runs(precision):
    if not has_gpu():
        pytest.skip("no GPU")
    from mpcns_mercury_b200 import serving as SV

    solo = _requests()
    SV.serve_one_by_one(solo, precision=0)
    reqs = _requests()
    one = max(SV.Server._bytes(r, precision) for r in reqs)
    # two slots and, beside the three grid templates, room for about two
    # solves: later requests queue for admission
    srv = SV.Server(capacity=2, precision=precision, hbm_budget=5.5 * one, chunk_steps=2)
    stats = srv.serve(reqs)
    srv.close()
    assert stats["requests"] == len(reqs) and stats["latency_p99_s"] >= stats["latency_p50_s"] > 0
    for r, s in zip(reqs, solo):
        assert r.done_s >= r.admitted_s >= r.arrival_s
        for name in s.result:
            if precision == 0:
                assert np.array_equal(r.result[name], s.result[name]), (r.rid, name)
            else:
                assert _rel(r.result[name], s.result[name]) <= 1e-5, (r.rid, name)


def test_requests_with_nodes_set_up_on_the_device():
    """Requests that carry their nodes instead of the static fields: the
    server computes the statics on the device (mhd_batch_setup_geometry) when
    a grid first arrives; results agree with the same requests run alone on
    host-computed statics to 1e-12 relative L2 (the reconstruction weights
    may differ in the last bits)."""
    if not has_gpu():
        pytest.skip("no GPU")
    from mpcns_mercury_b200 import serving as SV
    from mpcns_mercury_b200 import workloads as W

    solo = _requests()
    SV.serve_one_by_one(solo, precision=0)
    shapes = [(8, 8, 8), (10, 8, 12), (12, 10, 8)]
    pool = W.state_cases([(c, i) for i, c in enumerate(shapes)])
    steps = [3, 7, 5, 4, 6, 2]
    reqs = [SV.Request(rid=q, arrival_s=0.01 * q, cells=shapes[q % 3], steps=steps[q], fields=pool[q % 3],
                       keep_result=True) for q in range(len(steps))]
    srv = SV.Server(capacity=2, precision=0, hbm_budget=1e12, chunk_steps=2)
    srv.serve(reqs)
    srv.close()
    for r, s in zip(reqs, solo):
        for name in s.result:
            assert _rel(r.result[name], s.result[name]) <= 1e-12, (r.rid, name)
