"""Serving loop, host side (no GPU): a request whose device footprint exceeds the whole
HBM budget is refused with UEGCCD_ERR_ALLOC as soon as it is set up, and never reaches a
batch; uegccd_footprint is host-only."""
from uegccd_b200 import _capi, serve


def test_request_over_budget_is_refused_without_a_gpu():
    reqs = serve.poisson_stream(3, rate=1e9, seed=5, nelectrons=(54,), ratios=(8,), weights=(0.0, 0.0, 1.0))
    one = _capi.footprint(serve.build_system(reqs[0]), 6)[0]
    srv = serve.Server(hbm_budget=one // 2, max_batch=4)
    srv.run(reqs, realtime=False)
    assert srv.batches_started == 0
    assert all(r.status == _capi.UEGCCD_ERR_ALLOC for r in reqs)
    assert all(r.t_done >= r.t_arrival for r in reqs)
