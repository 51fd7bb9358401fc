"""Batched and served forms: every job's result is the same alone and in the
mix (bit for bit: a job's arithmetic does not depend on its neighbours in the
shared launches), admission respects the HBM budget, and errors are reported."""
import time

import numpy as np
import pytest
from conftest import golden_links

from msc_project_b200 import FP32MIXED, FP64, Job, LGFError, Server
from msc_project_b200 import _capi as C

pytestmark = pytest.mark.gpu


def alone(ctx, job: Job):
    with ctx.lattice(job.shape, job.precision) as lat:
        if job.links is not None:
            lat.upload(job.links)
        else:
            lat.generate(job.seed, job.gen_scale)
        r = lat.flow(job.eps, job.nsteps, job.meas_every, job.t0, job.measure_at_t0, job.reunit_every)
        return r, lat.download()


def mixed_jobs():
    return [
        Job((8, 8, 8, 8), FP64, links=golden_links("hb8_seed1.bin"), nsteps=12, meas_every=4, want_links=True),
        Job((4, 4, 6, 6), FP64, seed=101, nsteps=7, meas_every=2, want_links=True),
        Job((6, 6, 6, 12), FP64, seed=102, nsteps=10, meas_every=5, want_links=True),
        Job((8, 8, 8, 8), FP32MIXED, seed=103, nsteps=12, meas_every=3, reunit_every=5, want_links=True),
        Job((4, 8, 8, 8), FP32MIXED, seed=104, nsteps=5, meas_every=5, want_links=True),
        Job((6, 6, 6, 6), FP64, seed=105, nsteps=6, meas_every=3, want_links=True),  # V = 1296: not a whole number of 32-site blocks
        Job((6, 6, 6, 6), FP32MIXED, seed=106, nsteps=6, meas_every=3, reunit_every=3, want_links=True),
    ]


def test_batch_equals_alone(ctx):
    jobs = mixed_jobs()
    st = ctx.batch_run(jobs)
    assert st.site_steps == sum(np.prod(j.shape) * j.nsteps for j in jobs)
    assert st.seconds > 0 and st.launches > 0 and st.block_threads in (128, 256, 384)
    for j in jobs:
        r, links = alone(ctx, Job(**{k: getattr(j, k) for k in ("shape", "precision", "links", "seed", "nsteps",
                                                                     "meas_every", "reunit_every")}))
        assert np.array_equal(j.result.t, r.t)
        assert np.array_equal(j.result.E, r.E), j.shape
        assert np.array_equal(j.result.Q, r.Q), j.shape
        assert np.array_equal(j.links_out, links)


def test_autotune_picks_a_candidate(ctx):
    assert ctx.autotune(FP64, (8, 8, 8, 16)) in (128, 256, 384)


def test_server_alone_vs_mix_and_latency(ctx):
    jobs = mixed_jobs()
    refs = [alone(ctx, Job(**{k: getattr(j, k) for k in ("shape", "precision", "links", "seed", "nsteps",
                                                            "meas_every", "reunit_every")})) for j in jobs]
    # budget for about two resident jobs: the rest queue and are admitted as memory frees up
    budget = 2 * ctx.lib.lgf_lattice_footprint((C.ctypes.c_int * 4)(8, 8, 8, 8), FP64) + (1 << 20)
    with Server(ctx, budget, max_active=4, steps_per_tick=1) as srv:
        ids = []
        for j in jobs:
            ids.append(srv.submit(j))
            time.sleep(0.005)
        sts = [srv.wait(i, 120.0) for i in ids]
    for j, st, (r, links) in zip(jobs, sts, refs):
        assert st.state == C.LGF_JOB_DONE and st.error == 0
        assert st.submit_s <= st.start_s <= st.end_s
        assert np.array_equal(j.result.E, r.E) and np.array_equal(j.result.Q, r.Q)
        assert np.array_equal(j.links_out, links)
    lat = np.array([s.end_s - s.submit_s for s in sts])
    assert np.percentile(lat, 99) >= np.percentile(lat, 50) > 0


def test_server_launch_segments_alone_vs_mix(ctx):
    """Resident jobs large enough for launch segments of their own (each
    kernel launched once per job, small jobs sharing one) give the same bits
    as each job flowed alone."""
    def jobs():
        return [Job((16, 16, 24, 24), FP64, seed=201, nsteps=6, meas_every=2, want_links=True),
                Job((8, 8, 8, 8), FP64, seed=202, nsteps=6, meas_every=3, want_links=True),
                Job((4, 4, 6, 6), FP64, seed=205, nsteps=5, meas_every=1, want_links=True),
                Job((16, 16, 24, 24), FP64, seed=203, nsteps=4, meas_every=2, want_links=True),
                Job((24, 16, 16, 16), FP32MIXED, seed=204, nsteps=6, meas_every=2, reunit_every=3, want_links=True)]
    refs = [alone(ctx, j) for j in jobs()]
    mix = jobs()
    with Server(ctx, 1 << 33, max_active=5, steps_per_tick=2) as srv:
        ids = [srv.submit(j) for j in mix]
        sts = [srv.wait(i, 120.0) for i in ids]
    for j, st, (r, links) in zip(mix, sts, refs):
        assert st.state == C.LGF_JOB_DONE and st.error == 0
        assert np.array_equal(j.result.E, r.E) and np.array_equal(j.result.Q, r.Q)
        assert np.array_equal(j.links_out, links)


def test_server_rejects_jobs_that_never_fit(ctx):
    with Server(ctx, 1 << 20, max_active=2) as srv:
        with pytest.raises(LGFError) as e:
            srv.submit(Job((8, 8, 8, 8), FP64, seed=1, nsteps=1))
        assert e.value.code == C.LGF_ENOMEM
        with pytest.raises(LGFError) as e:
            srv.submit(Job((8, 8, 7, 8), FP64, seed=1, nsteps=1))
        assert e.value.code == C.LGF_EINVAL
        rc, _ = srv.poll(12345)
        assert rc == C.LGF_ENOTFOUND


def test_server_stop_while_threads_wait(ctx):
    """lgf_serve_stop while other threads block in lgf_serve_wait (one on the
    running job, one on a queued job): both waits return with the job ended
    by LGF_ESHUTDOWN, and the server is freed only after they have left."""
    import ctypes
    import threading
    srv = Server(ctx, 1 << 34, max_active=1, steps_per_tick=1)
    ids = [srv.submit(Job((16, 16, 16, 16), FP64, seed=2, nsteps=50000, measure_at_t0=False)),
           srv.submit(Job((8, 8, 8, 8), FP64, seed=3, nsteps=10, measure_at_t0=False))]
    results = {}

    def waiter(jid):
        st = C.lgf_job_status()
        rc = ctx.lib.lgf_serve_wait(srv.h, ctypes.c_uint64(jid), 120.0, ctypes.byref(st))
        results[jid] = (rc, st.state, st.error)

    threads = [threading.Thread(target=waiter, args=(i,)) for i in ids]
    for t in threads:
        t.start()
    time.sleep(1.0)  # both waiters are blocked inside lgf_serve_wait
    assert not results
    srv.stop()
    for t in threads:
        t.join(30.0)
        assert not t.is_alive()
    for jid in ids:
        assert results[jid] == (C.LGF_OK, C.LGF_JOB_FAILED, C.LGF_ESHUTDOWN)


def test_server_snapshots_at_measurements_and_resume(ctx, tmp_path):
    """A served job with a snapshot prefix writes its links after every
    measured step in the reference's flowed-file layout and naming; each file
    equals the links lgf_flow reaches after that many steps, and a job resumed
    from a snapshot (links = file, t0 = its flow time) ends on the same links
    and E, Q as the uninterrupted job."""
    U = golden_links("hb8_seed1.bin")
    shape = (8, 8, 8, 8)
    prefix = str(tmp_path / "torus_extdof4_0")
    job = Job(shape, FP64, links=U, nsteps=30, meas_every=10, want_links=True, snapshot_prefix=prefix)
    with Server(ctx, 1 << 30, max_active=2, steps_per_tick=4) as srv:
        st = srv.wait(srv.submit(job), 120.0)
        time.sleep(0.2)
        stats = srv.stats()
    assert st.state == C.LGF_JOB_DONE and st.error == 0
    assert stats["snapshots"] == 3 and stats["jobs_done"] == 1 and stats["steps"] == 30
    assert stats["measurements"] == 4 and stats["ticks"] >= 8
    assert 0 < stats["device_busy_s"] <= stats["wall_s"]
    for k, t in ((1, "0.100000"), (2, "0.200000"), (3, "0.300000")):
        f = tmp_path / f"torus_extdof4_0_Flowtime{t}.bin"
        _, ref = alone(ctx, Job(shape, FP64, links=U, nsteps=10 * k, meas_every=10))
        assert np.array_equal(np.fromfile(f), ref), t
    assert not (tmp_path / "torus_extdof4_0_Flowtime0.000000.bin").exists()  # the input itself is not written
    snap = np.fromfile(tmp_path / "torus_extdof4_0_Flowtime0.200000.bin")
    resumed = Job(shape, FP64, links=snap, t0=0.2, nsteps=10, meas_every=10, measure_at_t0=False, want_links=True)
    with Server(ctx, 1 << 30, max_active=2) as srv:
        st = srv.wait(srv.submit(resumed), 120.0)
    assert st.state == C.LGF_JOB_DONE
    assert np.array_equal(resumed.links_out, np.fromfile(tmp_path / "torus_extdof4_0_Flowtime0.300000.bin"))
    assert abs(resumed.result.t[-1] - job.result.t[-1]) < 1e-12
    assert resumed.result.E[-1] == job.result.E[-1] and resumed.result.Q[-1] == job.result.Q[-1]


def test_server_snapshot_write_failure_fails_the_job(ctx, tmp_path):
    job = Job((4, 4, 6, 6), FP64, seed=7, nsteps=4, meas_every=2,
              snapshot_prefix=str(tmp_path / "no_such_dir" / "cfg"))
    with Server(ctx, 1 << 28, max_active=1) as srv:
        st = srv.wait(srv.submit(job), 60.0)
    assert st.state == C.LGF_JOB_FAILED and st.error == C.LGF_EIO
