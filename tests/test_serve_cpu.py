"""Serving workload on the host: the seeded request stream and the summary."""
import numpy as np

from m3lb_b200 import capi
from m3lb_b200 import serve as SV


def test_request_stream_is_seeded_and_in_range():
    a = SV.request_stream(count=500, seed=0)
    b = SV.request_stream(count=500, seed=0)
    assert [(r.arrival, r.n, r.op, r.steps, r.u0) for r in a] == \
           [(r.arrival, r.n, r.op, r.steps, r.u0) for r in b]
    assert a[0].arrival == 0.0
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) >= 0)
    # Poisson arrivals at 50/s: mean gap 20 ms within sampling error
    assert abs(np.mean(np.diff(arr)) - 0.02) < 0.003
    assert {r.n for r in a} == set(SV.SIZES)
    assert {r.op for r in a} == {capi.OP_BGK, capi.OP_TRT, capi.OP_CM}
    assert all(0.02 <= r.u0 <= 0.08 and 200 <= r.steps <= 2000 for r in a)
    c = SV.request_stream(count=500, seed=1)
    assert [r.n for r in c] != [r.n for r in a]


def test_offered_load_exceeds_one_gpu():
    """The stated mix offers ~76 GLUPS on average, above what one B200 can
    serve at the HBM roofline, so the stream is run as a finite batch."""
    reqs = SV.request_stream(count=500, seed=0)
    assert 50e9 < SV.offered_lups(reqs) < 110e9


def test_rates():
    w, w2 = SV.rates(capi.OP_TRT, 0.6)
    assert abs(w - 1 / 0.6) < 1e-15
    # magic parameter (1/w - 1/2)(1/w2 - 1/2) = 3/16
    assert abs((1 / w - 0.5) * (1 / w2 - 0.5) - 3 / 16) < 1e-12
    assert SV.rates(capi.OP_CM)[1] < 0 and SV.rates(capi.OP_BGK)[1] < 0


class _R:
    def __init__(self, arrival, finished, node_steps):
        self.arrival, self.finished, self.node_steps = arrival, finished, node_steps


def test_summary_percentiles():
    res = [_R(0.0, 1.0 + i, 10 ** 6) for i in range(100)]
    s = SV.summary(res)
    assert s["requests"] == 100
    assert abs(s["latency_p50_s"] - 50.5) < 1e-9
    assert s["latency_p99_s"] > 99 and s["latency_max_s"] == 100.0
    assert abs(s["aggregate_mlups"] - 100 / 100.0) < 1e-9


def test_serve_config_is_checked_before_any_device_work():
    import ctypes as C
    lib = capi.lib()
    h = C.c_void_p()
    bad_mapping = capi.ServeConfig(1 << 30, 8, 50, capi.STORE_F16, 0, 5)
    assert lib.m3lb_serve_create(C.byref(bad_mapping), C.byref(h)) == capi.ERR_INVALID
    assert b"mapping" in lib.m3lb_last_error()
    rows_f32 = capi.ServeConfig(1 << 30, 8, 50, capi.STORE_F32, 0, capi.MAP_ROWS)
    assert lib.m3lb_serve_create(C.byref(rows_f32), C.byref(h)) == capi.ERR_UNSUPPORTED
    assert b"16-bit" in lib.m3lb_last_error()
    bad_round = capi.ServeConfig(1 << 30, 8, 0, capi.STORE_F16, 0, capi.MAP_DENSE)
    assert lib.m3lb_serve_create(C.byref(bad_round), C.byref(h)) == capi.ERR_INVALID
    f64 = capi.ServeConfig(1 << 30, 8, 50, capi.STORE_F64, 0, capi.MAP_AUTO)
    assert lib.m3lb_serve_create(C.byref(f64), C.byref(h)) == capi.ERR_UNSUPPORTED
    assert not h.value
