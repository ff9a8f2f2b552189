"""Batched solve server (lbf_server_* of the C ABI) on the GPU.

The claim under test: a solve's result is the same whether it runs alone or
in a mix with other solves of other sizes, classes, step counts and arrival
times -- bit for bit, since every solve runs the single-box kernel's
arithmetic -- and the same as the single-box entry point lbf_step; admission
respects the memory budget; cancelling a resident solve leaves the others
untouched.
"""
import numpy as np
import pytest

from cases import make_case, rel_l2, run_oracle
import lbfast_b200 as L

pytestmark = pytest.mark.gpu

# (case, storage, nsteps): three kernel classes, ragged boxes, wetting on
# obstacles, open faces, bounce-back, the repulsive-flux kernel class, step
# counts that are not multiples of the chunk
MIX = [("q27_2c_dr", "f16", 23), ("q27ho_2c_dr", "f32", 17), ("tg_q19", "f32", 30), ("obs_q27ho_2c_dr", "f32", 12),
       ("q27ho_2c_dr_corr", "f32", 15), ("q19_2c_dr", "f16", 9), ("q27_2c_dr", "f32", 40),
       ("open_q27ho_2c_dr_corr", "f32", 14), ("open_q19_1c", "f16", 11), ("rep_q27ho_2c_dr", "f32", 10),
       ("obs_q19_1c_bb", "f16", 13)]


def _alone(case, storage, n, **kw):
    p, isf, m, phi = make_case(case, storage)
    with L.Server(**kw) as s:
        sid = s.submit(p, m, phi, n, isf if p.obstacles else None)
        s.drain()
        assert s.poll(sid)["state"] == "done"
        return s.fetch(sid)


def _same(a, b):
    return all((x is None and y is None) or np.array_equal(x, y, equal_nan=True) for x, y in zip(a, b))


@pytest.fixture(scope="module")
def alone():
    return {i: _alone(c, st, n, chunk=4) for i, (c, st, n) in enumerate(MIX)}


def test_mix_equals_alone_bitwise(alone):
    """Staggered arrivals into a running server (chunk 4, graphs on): every
    solve's fields equal its solo run exactly."""
    with L.Server(chunk=4) as s:
        ids = {}
        for i, (c, st, n) in enumerate(MIX):
            p, isf, m, phi = make_case(c, st)
            ids[i] = s.submit(p, m, phi, n, isf if p.obstacles else None)
            s.run(1)  # later solves arrive while earlier ones are resident
        s.drain()
        for i, sid in ids.items():
            info = s.poll(sid)
            assert info["state"] == "done" and info["steps_done"] == MIX[i][2]
            assert info["t_submit"] <= info["t_admit"] <= info["t_done"]
            assert _same(s.fetch(sid), alone[i]), MIX[i]


def test_graph_and_direct_launches_agree(alone):
    i = 1
    c, st, n = MIX[i]
    assert _same(_alone(c, st, n, chunk=4, use_graph=False), alone[i])
    assert _same(_alone(c, st, n, chunk=8, use_graph=True), alone[i])


@pytest.mark.parametrize("i", [0, 1, 2, 3, 4, 7, 8, 9, 10])
def test_server_equals_single_box_entry_point(alone, i):
    """The server's result equals lbf_step's on the same inputs."""
    c, st, n = MIX[i]
    p, isf, m, phi = make_case(c, st)
    s = L.Solver(p)
    if p.obstacles:
        s.set_isfluid(isf)
    s.set_fields(m, phi)
    s.step(n)
    mg, pg, _ = s.get_fields()
    s.close()
    ms, ps = alone[i]
    # the batched kernel is a separate compilation of the same step: equal
    # within rounding (alone and in a mix it is the same kernel: equal bits)
    fl = np.abs(isf) == 1
    bar = 1e-6 if st == "f32" else 1e-3
    assert rel_l2(ms, mg, fl) < bar
    if p.twocomponent:
        assert rel_l2(ps, pg, fl) < bar


def test_server_fp32_matches_oracle():
    """FP32 storage through the server within 1e-5 rel-L2 of the FP64 oracle."""
    c, n = "q27ho_2c_dr", 20
    ms, ps = _alone(c, "f32", n)
    mo, po, _ = run_oracle(c, n, "f64").get_fields()
    assert rel_l2(ms, mo) < 1e-5 and rel_l2(ps, po) < 1e-5


def test_admission_respects_budget(alone):
    """A budget of two solves' bytes admits two, queues the rest first in first
    out, and admits them as the resident ones finish."""
    c, st, n = MIX[0]
    p, _, m, phi = make_case(c, st)
    b = L.Server.solve_bytes(p)
    with L.Server(mem_budget=2 * b + b // 2, chunk=4) as s:
        ids = [s.submit(p, m, phi, n) for _ in range(5)]
        assert s.run(0) == (2, 3)
        states = [s.poll(i)["state"] for i in ids]
        assert states == ["active", "active", "queued", "queued", "queued"]
        s.drain()
        t_admit = [s.poll(i)["t_admit"] for i in ids]
        assert t_admit == sorted(t_admit)
        for i in ids:
            assert _same(s.fetch(i), alone[0])


def test_oversize_solve_rejected():
    p, _, m, phi = make_case("q27_2c_dr", "f32")
    with L.Server(mem_budget=L.Server.solve_bytes(p) - 1) as s:
        with pytest.raises(L.LbfError) as e:
            s.submit(p, m, phi, 4)
        assert e.value.code == -3


def test_cancel_resident_solve_leaves_others(alone):
    with L.Server(chunk=4) as s:
        ids = []
        for c, st, n in MIX[:3]:
            p, isf, m, phi = make_case(c, st)
            ids.append(s.submit(p, m, phi, n, isf if p.obstacles else None))
        s.run(2)
        assert s.poll(ids[1])["state"] == "active"
        s.cancel(ids[1])
        s.drain()
        assert _same(s.fetch(ids[0]), alone[0])
        assert _same(s.fetch(ids[2]), alone[2])
        with pytest.raises(L.LbfError):
            s.poll(ids[1])
