"""Many instances on one GPU (eg_batch_*, eg_server_*): every instance keeps
its own kernels and reductions, so its final state must be bitwise the one it
reaches alone; the request loop must respect its device-memory budget and run
requests concurrently when the budget allows."""
import numpy as np
import pytest

from mfem_euler2d_cpp_b200 import capi

pytestmark = pytest.mark.gpu

SHAPES = [(12, 12, 1, 40.0), (12, 10, 2, 45.0), (16, 16, 3, 50.0), (10, 14, 4, 35.0), (8, 12, 6, 60.0),
          (20, 8, 2, 70.0)]


def _alone(nx, ny, k, alpha, steps=1, newton=2, form=capi.FORM_HDG):
    d = capi.simple_wave_desc(nx, ny, k, alpha)
    with capi.Context(d, capi.default_opts(form=form)) as ctx:
        ro, keep = capi.run_options(integrator="ssp-dirk3", steps=steps, newton_steps=newton, cfl=1.0,
                                    form_name="hdg" if form == capi.FORM_HDG else "dg")
        st = capi.Stepper(ctx, ro, keep)
        while st.next() is not None:
            pass
        st.close()
        return ctx.download("U")


def test_batch_states_equal_single_runs():
    descs = [capi.simple_wave_desc(nx, ny, k, a) for nx, ny, k, a in SHAPES]
    opts = [capi.default_opts(form=capi.FORM_HDG) for _ in SHAPES]
    ro, keep = capi.run_options(integrator="ssp-dirk3", steps=1, newton_steps=2, cfl=1.0, form_name="hdg")
    with capi.Batch(descs, opts) as b:
        st = b.run(ro, threads=4)
        assert st.failed == 0
        assert st.updates == len(SHAPES) * 8
        for i, (nx, ny, k, a) in enumerate(SHAPES):
            status, res = b.result(i)
            assert status == capi.OK and res.updates == 8
            nu = nx * ny * 4 * (k + 1) ** 2
            np.testing.assert_array_equal(b.state(i, nu), _alone(nx, ny, k, a))


def test_server_result_same_alone_and_in_the_mix():
    probe = (16, 16, 3, 50.0)
    nu = 16 * 16 * 4 * 16
    with capi.Server(workers=1, keep_states=True) as s:
        rid = s.submit(*probe, steps=1, newton_steps=2)
        s.drain()
        alone = s.state(rid, nu)
        assert s.poll(rid).status == capi.OK
    with capi.Server(workers=6, keep_states=True) as s:
        ids = []
        for i in range(12):
            nx, ny, k, a = SHAPES[i % len(SHAPES)]
            ids.append(s.submit(nx, ny, k, a, steps=1, newton_steps=2))
            if i == 5:
                mine = s.submit(*probe, steps=1, newton_steps=2)
        st = s.drain()
        assert st.failed == 0 and st.completed == 13
        assert st.peak_running > 1  # requests overlapped on the GPU
        np.testing.assert_array_equal(s.state(mine, nu), alone)
        for rid in ids:
            r = s.poll(rid)
            assert r.status == capi.OK and r.finish_s >= r.start_s >= r.submit_s


def test_pooled_context_takes_the_new_request_geometry():
    """A finished context is reused for a request of the same size but another
    angle: the result must be the one a fresh context gives."""
    nu = 16 * 16 * 4 * 9
    with capi.Server(workers=1, keep_states=True) as s:
        first = s.submit(16, 16, 2, 25.0, steps=1, newton_steps=2)
        second = s.submit(16, 16, 2, 65.0, steps=1, newton_steps=2)
        s.drain()
        assert s.poll(first).status == capi.OK and s.poll(second).status == capi.OK
        np.testing.assert_array_equal(s.state(second, nu), _alone(16, 16, 2, 65.0))


def test_server_admission_respects_the_memory_budget():
    with capi.Server(workers=1, keep_contexts=False) as s:
        rid = s.submit(24, 24, 3, 40.0, steps=1, newton_steps=1)
        s.drain()
        need = s.poll(rid).bytes
    assert need > 0
    budget = int(need * 1.5)  # room for one such request at a time
    with capi.Server(workers=4, budget_bytes=budget, keep_contexts=False) as s:
        for _ in range(4):
            s.submit(24, 24, 3, 40.0, steps=1, newton_steps=1)
        st = s.drain()
        assert st.completed == 4
        assert st.peak_running == 1
        assert st.peak_bytes <= budget
