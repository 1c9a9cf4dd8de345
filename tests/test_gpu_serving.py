"""Batching and serving: jobs of uneven size and mode run concurrently on several lanes, each with
its own stream and device arena, and every result equals the same job partitioned alone."""
import numpy as np
import pytest

import axoncuda_b200 as ax

pytestmark = pytest.mark.gpu


def mixed_jobs(count, seed0=200):
    """Circuit and SNN hypergraphs of uneven size, k-way (k in 2, 8, 32) and INCC."""
    jobs = []
    rng = np.random.default_rng(seed0)
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(1500), np.log(20000))))
        if i % 2 == 0:
            g = ax.gen_circuit(n, int(n * 1.1), 2, 32, 2.5, 0.9, 0.02, seed0 + i)
        else:
            g = ax.gen_snn(6, max(n // 6, 64), 24, 0.0, 0, 1.0, seed0 + i)
        if i % 3 == 2:
            p = ax.params_incc(128, 1024, 1048576, cnc=4, rfr=8)
        else:
            p = ax.params_kway([2, 8, 32][i % 3], 0.03, cnc=4, rfr=8)
        jobs.append((g, p))
    return jobs


def test_lanes_match_solo(ctx):
    jobs = mixed_jobs(12)
    solo = [ctx.partition(g, p)[0] for g, p in jobs]
    with ax.Context(0, 256 << 20) as srv:
        srv.serve_configure(6, 8 << 30)
        ids = [srv.submit(g, p) for g, p in jobs]
        for (g, _), jid, s in zip(jobs, ids, solo):
            part, st = srv.poll(jid, g.n)
            np.testing.assert_array_equal(part, s)
            assert st.valid == 1
            assert st.ms_run > 0 and st.ms_queued >= 0
            assert 0 < st.device_bytes_peak


def test_batch_call_matches_solo(ctx):
    jobs = mixed_jobs(8, seed0=300)
    solo = [ctx.partition(g, p)[0] for g, p in jobs]
    with ax.Context(0, 256 << 20) as srv:
        srv.serve_configure(4, 8 << 30)
        res = srv.partition_batch(jobs)
    for (part, st), s in zip(res, solo):
        np.testing.assert_array_equal(part, s)
        assert st.valid == 1


def test_budget_smaller_than_a_job_runs_it_alone(ctx):
    """A job whose estimate exceeds the budget still runs (alone); results are unchanged."""
    jobs = mixed_jobs(4, seed0=400)
    solo = [ctx.partition(g, p)[0] for g, p in jobs]
    with ax.Context(0, 256 << 20) as srv:
        srv.serve_configure(3, 1 << 20)  # 1 MiB: nothing fits beside another job
        ids = [srv.submit(g, p) for g, p in jobs]
        for (g, _), jid, s in zip(jobs, ids, solo):
            part, _ = srv.poll(jid, g.n)
            np.testing.assert_array_equal(part, s)


def test_configure_after_start_is_refused():
    with ax.Context(0, 256 << 20) as srv:
        srv.serve_configure(2, 1 << 30)
        g, p = mixed_jobs(1)[0]
        jid = srv.submit(g, p)
        srv.poll(jid, g.n)
        with pytest.raises(ax.AxcError) as e:
            srv.serve_configure(4, 1 << 30)
        assert e.value.code == 9  # AXC_EBUSY


def test_destroy_answers_waiting_pollers():
    """Destroying a serving context while jobs are queued: the running job finishes, every queued
    job is answered with AXC_ECANCELED, and pollers already waiting (timeout -1) return instead of
    waiting for good."""
    import ctypes as C
    import threading
    import time
    g = ax.gen_snn(10, 4000, 64, 0.0, 0, 1.0, 77)  # 2.3M pins: each job runs alone on the device
    p = ax.params_kway(8, 0.03, cnc=4, rfr=8)
    srv = ax.Context(0, 256 << 20)
    srv.serve_configure(1, 8 << 30)
    ids = [srv.submit(g, p) for _ in range(12)]
    rcs, entered = {}, [threading.Event() for _ in range(3)]
    bufs = [np.zeros(g.n, np.uint32) for _ in range(3)]

    def wait(i):
        h = srv._h  # NULL once the context is closed: axc_poll would then say AXC_EINVAL
        entered[i].set()
        rcs[i] = ax.lib().axc_poll(h, ids[9 + i], bufs[i].ctypes.data_as(C.POINTER(C.c_uint32)), None, -1)

    threads = [threading.Thread(target=wait, args=(i,)) for i in range(3)]
    for t in threads:
        t.start()
    for e in entered:
        assert e.wait(30)
    time.sleep(0.05)  # the pollers are inside axc_poll, waiting
    srv.close()  # axc_destroy: shuts the executor down
    for t in threads:
        t.join(timeout=120)
        assert not t.is_alive()
    assert all(rc in (0, 12) for rc in rcs.values()), rcs  # AXC_OK or AXC_ECANCELED
    assert 12 in rcs.values()  # the last jobs were still queued behind the running one


def test_tuning_changes_speed_not_results(ctx):
    """axc_tune_set: every tile and table size gives the same partitions; bad values and unknown
    keys are refused; executor settings are refused once the executor has started."""
    jobs = mixed_jobs(6, seed0=500)
    solo = [ctx.partition(g, p)[0] for g, p in jobs]
    with ax.Context(0, 1 << 30) as c2:
        for key, value in (("rate.try_slots", 256), ("rate.mid_slots", 1024), ("cascade.block_movers", 128)):
            c2.tune(key, value)
        for (g, p), s in zip(jobs, solo):
            np.testing.assert_array_equal(c2.partition(g, p)[0], s)
        for key, value, code in (("rate.try_slots", 3000, 1), ("cascade.block_movers", 64, 1), ("no.such", 1, 8)):
            with pytest.raises(ax.AxcError) as e:
                c2.tune(key, value)
            assert e.value.code == code
    with ax.Context(0, 256 << 20) as srv:
        srv.serve_configure(3, 8 << 30)
        srv.tune("class.0.min_pins", 0)
        srv.tune("class.0.rate.try_slots", 512)
        srv.tune("class.1.min_pins", 50000)
        srv.tune("class.1.cascade.block_movers", 256)
        srv.tune("serve.exclusive_pins", 0)
        res = srv.partition_batch(jobs)
        for (part, st), s in zip(res, solo):
            np.testing.assert_array_equal(part, s)
        with pytest.raises(ax.AxcError) as e:
            srv.tune("class.2.min_pins", 1)
        assert e.value.code == 9  # AXC_EBUSY
