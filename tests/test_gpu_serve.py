"""Serving loop on the GPU (m3lb_serve_*).

A request's result must not depend on what else is resident: the batched
kernels run the paired kernel's per-node arithmetic for every lattice (the
chunk and dense mappings its per-unit code, the row mapping the row kernel,
bit-identical to it), so results are bit-identical alone, in a mix, under a
one-lattice admission limit, with every mapping (chunks, dense strips, whole
rows), and through the single-lattice C ABI with the paired kernel.
"""
import ctypes as C

import numpy as np
import pytest

from m3lb_b200 import capi
from m3lb_b200 import serve as SV
from m3lb_b200 import solver as S

pytestmark = pytest.mark.gpu

MIX = [SV.Request(0, 0.0, 32, capi.OP_CM, 23, 0.05),
       SV.Request(1, 0.0, 48, capi.OP_BGK, 17, 0.03),
       SV.Request(2, 0.0, 64, capi.OP_TRT, 30, 0.07),
       SV.Request(3, 0.0, 80, capi.OP_CM, 12, 0.04),
       SV.Request(4, 0.0, 32, capi.OP_MRT, 9, 0.02),
       SV.Request(5, 0.0, 64, capi.OP_CM, 0, 0.06)]


def _serve(reqs, storage="f16", **kw):
    srv = SV.Server(storage=storage, keep_fields=True, **kw)
    for r in reqs:
        srv.submit(r)
    srv.run(time_limit=120)
    res = {r.id: r for r in srv.results()}
    fields = {i: srv.fields(i) for i in res}
    st = srv.stats()
    srv.close()
    return res, fields, st


def _same(a, b):
    ra, fa = a
    rb, fb = b
    assert ra.mass == rb.mass and ra.energy == rb.energy
    assert list(ra.momentum) == list(rb.momentum)
    for x, y in zip(fa, fb):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("storage", ["f16", "f32"])
def test_alone_equals_mix(cuda_device, storage):
    mix, mix_f, st = _serve(MIX, storage)
    assert len(mix) == len(MIX) and all(r.status == 0 for r in mix.values())
    assert st.rounds >= 1 and st.finished == len(MIX)
    for r in MIX:
        alone, alone_f, _ = _serve([r], storage)
        _same((mix[r.id], mix_f[r.id]), (alone[r.id], alone_f[r.id]))


# Small and ragged boxes: N = 6 and 10 put several rows in one 64-node unit
# and leave the last unit partly empty (N^3 not a multiple of 64); 48 and 80
# split rows across units.
RAGGED = [SV.Request(10, 0.0, 6, capi.OP_CM, 11, 0.05),
          SV.Request(11, 0.0, 10, capi.OP_BGK, 8, 0.04),
          SV.Request(12, 0.0, 48, capi.OP_TRT, 13, 0.06),
          SV.Request(13, 0.0, 80, capi.OP_MRT, 7, 0.03),
          SV.Request(14, 0.0, 64, capi.OP_CM, 9, 0.05)]


@pytest.mark.parametrize("storage", ["f16", "f16c", "bf16", "f32"])
def test_dense_mapping_equals_chunks(cuda_device, storage):
    reqs = MIX + RAGGED
    ch, ch_f, st_c = _serve(reqs, storage, mapping="chunks")
    de, de_f, st_d = _serve(reqs, storage, mapping="dense")
    assert st_c.dense_launches == 0 and st_d.dense_launches == st_d.launches > 0
    for r in reqs:
        assert ch[r.id].status == 0 and de[r.id].status == 0
        _same((ch[r.id], ch_f[r.id]), (de[r.id], de_f[r.id]))
        assert np.isfinite(de[r.id].mass)


def test_auto_mapping_rule(cuda_device):
    # 16-bit storage: whole rows, one launch per (operator, row width) group
    # and step; FP32: every N a multiple of 64 takes chunks, one ragged
    # lattice dense strips for its operator
    _, _, st = _serve([SV.Request(0, 0.0, 64, capi.OP_CM, 5, 0.05),
                       SV.Request(1, 0.0, 128, capi.OP_BGK, 5, 0.05)])
    assert st.rows_launches == st.launches == 10 and st.dense_launches == 0
    _, _, st = _serve([SV.Request(0, 0.0, 64, capi.OP_CM, 5, 0.05),
                       SV.Request(1, 0.0, 128, capi.OP_BGK, 5, 0.05)], "f32")
    assert st.dense_launches == 0 and st.rows_launches == 0
    _, _, st = _serve([SV.Request(0, 0.0, 64, capi.OP_CM, 5, 0.05),
                       SV.Request(1, 0.0, 96, capi.OP_BGK, 5, 0.05)], "f32")
    assert st.dense_launches == 5 and st.launches == 10


@pytest.mark.parametrize("storage", ["f16", "f16c", "bf16"])
def test_rows_mapping_equals_chunks(cuda_device, storage):
    """Whole-row launches (one per operator and row width, lattices finishing
    inside a round) give the chunk mapping's bits, ragged boxes included:
    rows of 1-2 chunks (moved by the update warps themselves), 3 chunks (a
    3-chunk stage and a copy warp, N = 144 with a partial last chunk, two
    lattices in one launch) and 5 chunks (an 8-chunk stage)."""
    reqs = MIX + RAGGED + [SV.Request(20, 0.0, 144, capi.OP_CM, 9, 0.05),
                           SV.Request(21, 0.0, 144, capi.OP_CM, 5, 0.03),
                           SV.Request(22, 0.0, 144, capi.OP_BGK, 6, 0.04),
                           SV.Request(23, 0.0, 272, capi.OP_TRT, 3, 0.05)]
    ch, ch_f, _ = _serve(reqs, storage, mapping="chunks")
    ro, ro_f, st = _serve(reqs, storage, mapping="rows", round_steps=8)
    assert st.rows_launches == st.launches > 0
    for r in reqs:
        assert ro[r.id].status == 0
        _same((ch[r.id], ch_f[r.id]), (ro[r.id], ro_f[r.id]))


def test_rows_rounds_replay_captured_graphs(cuda_device):
    """Lattices arriving and finishing at different times: row rounds keep
    their length, so after the first two rounds of a group set every round
    replays a captured graph, and the results equal the chunk mapping's."""
    reqs = [SV.Request(i, 0.02 * i, n, op, steps, 0.05)
            for i, (n, op, steps) in enumerate([(48, capi.OP_CM, 130), (80, capi.OP_BGK, 70),
                                                (32, capi.OP_TRT, 210), (64, capi.OP_CM, 95),
                                                (96, capi.OP_CM, 160), (48, capi.OP_BGK, 40)])]
    ro, ro_f, st = _serve(reqs, mapping="rows", round_steps=10)
    ch, ch_f, _ = _serve(reqs, mapping="chunks", round_steps=10)
    assert st.graph_launches >= 0.5 * st.rounds, (st.graph_launches, st.rounds)
    for r in reqs:
        _same((ro[r.id], ro_f[r.id]), (ch[r.id], ch_f[r.id]))


def test_tuned_mapping_measures_all_and_keeps_results(cuda_device):
    # 300 steps in rounds of 10: 30 rounds, the first 18 alternate the three
    # mappings (whole rows, chunks, dense strips), 6 timed rounds each
    reqs = [SV.Request(i, 0.0, n, op, 300, 0.05)
            for i, (n, op) in enumerate([(48, capi.OP_CM), (80, capi.OP_BGK), (32, capi.OP_TRT)])]
    tu, tu_f, st = _serve(reqs, round_steps=10, mapping="tune")
    ch, ch_f, _ = _serve(reqs, round_steps=10, mapping="chunks")
    rates = {capi.MAP_CHUNKS: st.tuned_chunks_mlups, capi.MAP_DENSE: st.tuned_dense_mlups,
             capi.MAP_ROWS: st.tuned_rows_mlups}
    assert all(v > 0 for v in rates.values()), rates
    assert st.tuned_mapping == max(rates, key=rates.get)
    assert 0 < st.dense_launches < st.launches and 0 < st.rows_launches < st.launches
    for r in reqs:
        _same((tu[r.id], tu_f[r.id]), (ch[r.id], ch_f[r.id]))


def test_one_resident_at_a_time_equals_mix(cuda_device):
    mix, mix_f, _ = _serve(MIX)
    seq, seq_f, _ = _serve(MIX, max_resident=1, round_steps=7)
    order = sorted(seq.values(), key=lambda r: r.finished)
    assert [r.id for r in order] == [r.id for r in MIX]  # FIFO under the limit
    for r in MIX:
        _same((mix[r.id], mix_f[r.id]), (seq[r.id], seq_f[r.id]))


def _single(r, storage="f16"):
    """The same request through FluidSolver (paired kernel), seeded from the
    serving loop's field generator."""
    import torch
    n = r.n
    w, w2 = SV.rates(r.op)
    if r.op == capi.OP_BGK:
        coll = S.BGK(lattice=S.D3Q27, storage=S.ShiftedPopulations, omega=w)
    elif r.op == capi.OP_TRT:
        coll = S.TRT(lattice=S.D3Q27, storage=S.ShiftedPopulations, omega_p=w, omega_m=w2)
    elif r.op == capi.OP_MRT:
        coll = S.MRT(S.D3Q27, S.NoForcing(), S.ShiftedPopulations, omega=w)
    else:
        coll = S.CentralMoments(S.D3Q27, S.NoForcing(), S.ShiftedPopulations, omega=w)
    s = S.FluidSolver(S.Domain(n, n, n), coll, storage=storage)
    s.set_option(capi.OPT_KERNEL, capi.KERNEL_PAIRS)
    f = [torch.empty((n, n, n), dtype=torch.float32, device="cuda") for _ in range(4)]
    torch.cuda.synchronize()
    capi.check(capi.lib().m3lb_tgv_field(n, r.u0, *[C.c_void_p(t.data_ptr()) for t in f], None))
    torch.cuda.synchronize()
    s.initialize_field_device(*f)
    s.steps(r.steps)
    out = [np.empty((n, n, n), np.float32) for _ in range(4)]
    s.compute_macroscopic_f32(*out)
    red = s.reduce()
    s.close()
    return red, out


def test_serving_equals_single_lattice_api(cuda_device):
    mix, mix_f, _ = _serve(MIX)
    for r in MIX[:4]:
        red, fields = _single(r)
        res = mix[r.id]
        assert res.mass == red[0] and list(res.momentum) == list(red[1:4])
        assert res.energy == red[4]
        for x, y in zip(mix_f[r.id], fields):
            np.testing.assert_array_equal(x, y)


def test_taylor_green_field_matches_formula(cuda_device):
    import torch
    n, u0 = 16, 0.05
    f = [torch.empty((n, n, n), dtype=torch.float32, device="cuda") for _ in range(4)]
    capi.check(capi.lib().m3lb_tgv_field(n, u0, *[C.c_void_p(t.data_ptr()) for t in f], None))
    torch.cuda.synchronize()
    k = 2 * np.pi / n
    i = np.arange(n) * k
    z, y, x = np.meshgrid(i, i, i, indexing="ij")
    rho = 1 + 3 * u0 * u0 / 16 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2)
    ux = u0 * np.sin(x) * np.cos(y) * np.cos(z)
    uy = -u0 * np.cos(x) * np.sin(y) * np.cos(z)
    for got, want in zip(f, (rho, ux, uy, np.zeros_like(ux))):
        np.testing.assert_allclose(got.cpu().numpy(), want, rtol=0, atol=2e-7)


def test_invalid_requests_are_rejected(cuda_device):
    srv = SV.Server(hbm_budget=64 << 20)
    with pytest.raises(capi.M3lbError):
        srv.submit(SV.Request(0, 0.0, 33, capi.OP_CM, 10, 0.05))   # odd N
    with pytest.raises(capi.M3lbError):
        srv.submit(SV.Request(1, 0.0, 160, capi.OP_CM, 10, 0.05))  # above the budget
    with pytest.raises(capi.M3lbError):
        srv.submit(SV.Request(2, 0.0, 32, capi.OP_NONE, 10, 0.05))  # no operator
    srv.close()
    cfg = capi.ServeConfig(1 << 30, 8, 50, capi.STORE_F64, 0)
    h = C.c_void_p()
    assert capi.lib().m3lb_serve_create(C.byref(cfg), C.byref(h)) == capi.ERR_UNSUPPORTED


def test_stream_served_with_latencies(cuda_device):
    """A short seeded stream: every request finishes, latency includes the
    queueing, and the loop's own counters agree with the results."""
    reqs = SV.request_stream(count=24, rate=200.0, seed=3, steps=(20, 120))
    srv = SV.Server(hbm_budget=1 << 30, max_resident=6, round_steps=25)
    for r in reqs:
        srv.submit(r)
    srv.run(time_limit=120)
    res = srv.results()
    st = srv.stats()
    srv.close()
    assert len(res) == len(reqs) and st.finished == len(reqs)
    assert all(r.status == 0 and r.finished >= r.admitted >= r.arrival for r in res)
    assert st.node_steps == sum(q.nodes() * q.steps for q in reqs)
    s = SV.summary(res, reqs)
    assert 0 < s["latency_p50_s"] <= s["latency_p99_s"] <= s["latency_max_s"]
    for r in res:
        assert np.isfinite(r.mass)
