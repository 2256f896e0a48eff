"""Failure handling of the reconstruction server, with every failure made on
the host (nothing faults, traps or hangs the GPU): malformed jobs are
rejected at submission, cancelled and timed-out jobs leave without a result,
a lane whose allocation fails (simulated out-of-memory from the fault
injector) keeps its jobs queued and serves them after the retry, a lane whose
step raises fails its own jobs while the others finish, and an evicted SQS job
resumes from its snapshot to the same result.  The jobs that finish match the
same jobs served alone."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

MIX_TOL = 1e-6


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _setup(n_iter=6):
    from test_gpu_serving import _jobs, _protocols

    return _protocols(n_iter=n_iter), _jobs


def _alone(protos, jobs_fn, name, nz, seed0):
    from ctprojector_b200.serving import Engine

    job = jobs_fn(protos, [(name, nz, 0.0)], seed0=seed0)[0]
    eng = Engine()
    eng.run([job], realtime=False)
    eng.close()
    return job.result.numpy()


def test_malformed_jobs_are_rejected_and_the_rest_served():
    from ctprojector_b200.serving import Engine, Job

    protos, jobs_fn = _setup()
    good = jobs_fn(protos, [("fan_sqs", 2, 0.0), ("par_fbp", 1, 0.0)])
    p = protos["fan_sqs"]
    bad = [Job(10, p, torch.zeros(2, p.nview, 1, 7), nz=2),                      # wrong detector width
           Job(11, p, torch.zeros(0, p.nview, 1, int(p.scan.nu)), nz=0),        # no slices
           Job(12, p, torch.zeros(2, p.nview, 1, int(p.scan.nu), dtype=torch.int32), nz=2),  # not floating
           Job(0, p, good[0].sinogram, nz=2)]                                     # duplicate id
    eng = Engine()
    summary = eng.run(good + bad, realtime=False)
    assert summary["jobs"] == 2
    assert [j.status for j in bad] == ["rejected"] * 4 and all(j.error for j in bad)
    assert all(j.status == "done" for j in good)
    assert rel_l2(good[0].result.numpy(), _alone(protos, jobs_fn, "fan_sqs", 2, 0)) <= MIX_TOL
    eng.close()


def test_cancel_queued_and_running_jobs():
    from ctprojector_b200.serving import Engine

    protos, jobs_fn = _setup(n_iter=10)
    a, b, c = jobs_fn(protos, [("fan_sqs", 2, 0.0), ("fan_sqs", 3, 0.0), ("par_sqs", 1, 0.0)])
    eng = Engine()
    for j in (a, b, c):
        eng.submit(j)
    eng._admit(0.0)
    for _ in range(3):
        torch.cuda.synchronize()
        eng._step()
    assert b.status == "running"
    assert eng.cancel(b.job_id)  # running: its slots are freed, the others packed
    assert not eng.cancel(b.job_id)
    while eng.busy():
        eng.pass_once(0.0)
        torch.cuda.synchronize()
    assert b.status == "cancelled" and b.result is None
    assert a.status == "done" and c.status == "done"
    assert rel_l2(a.result.numpy(), _alone(protos, jobs_fn, "fan_sqs", 2, 0)) <= MIX_TOL
    assert rel_l2(c.result.numpy(), _alone(protos, jobs_fn, "par_sqs", 1, 2)) <= MIX_TOL
    # a queued job cancelled before admission
    d = jobs_fn(protos, [("par_fbp", 1, 0.0)], seed0=9)[0]
    eng.submit(d)
    assert eng.cancel(d.job_id) and d.status == "cancelled" and not eng.busy()
    eng.close()


def test_deadline_times_out_a_slow_job():
    from ctprojector_b200.serving import Engine

    protos, jobs_fn = _setup(n_iter=40)
    a, b = jobs_fn(protos, [("fan_sqs", 1, 0.0), ("par_fbp", 1, 0.0)])
    a.deadline = 0.0  # the client stops waiting at once
    eng = Engine()
    eng.run([a, b], realtime=True)
    assert a.status == "timeout" and a.result is None and "after arrival" in a.error
    assert b.status == "done"
    eng.close()


def test_allocation_failure_keeps_jobs_queued_then_serves_them():
    from ctprojector_b200.serving import Engine

    protos, jobs_fn = _setup()
    calls = {"n": 0}

    def faults(event, protocol):
        if event == "lane_alloc" and protocol.name == "fan_sqs" and calls["n"] < 2:
            calls["n"] += 1
            raise torch.cuda.OutOfMemoryError("simulated: no device memory for the lane")

    jobs = jobs_fn(protos, [("fan_sqs", 2, 0.0), ("par_fbp", 2, 0.0)])
    eng = Engine(faults=faults, max_alloc_retries=3)
    eng.run(jobs, realtime=False)
    assert calls["n"] == 2 and eng.alloc_failures["fan_sqs"] == 2
    assert all(j.status == "done" for j in jobs)
    assert rel_l2(jobs[0].result.numpy(), _alone(protos, jobs_fn, "fan_sqs", 2, 0)) <= MIX_TOL
    eng.close()

    # a lane that never gets its memory: its jobs fail, the others are served
    def never(event, protocol):
        if event == "lane_alloc" and protocol.name == "fan_sqs":
            raise torch.cuda.OutOfMemoryError("simulated: no device memory for the lane")

    jobs = jobs_fn(protos, [("fan_sqs", 2, 0.0), ("par_fbp", 2, 0.0)])
    eng = Engine(faults=never, max_alloc_retries=2)
    eng.run(jobs, realtime=False)
    assert jobs[0].status == "failed" and "OutOfMemoryError" in jobs[0].error
    assert jobs[1].status == "done"
    eng.close()


def test_failing_lane_step_fails_only_its_jobs():
    from ctprojector_b200.serving import Engine

    protos, jobs_fn = _setup()

    def faults(event, protocol):
        if event == "lane_step" and protocol.name == "par_sqs":
            raise RuntimeError("simulated projector error")

    jobs = jobs_fn(protos, [("par_sqs", 2, 0.0), ("fan_sqs", 1, 0.0), ("cone_sqs", 1, 0.0)])
    eng = Engine(faults=faults)
    eng.run(jobs, realtime=False)
    assert jobs[0].status == "failed" and "simulated projector error" in jobs[0].error
    assert "par_sqs" not in eng.lanes
    assert jobs[1].status == "done" and jobs[2].status == "done"
    assert rel_l2(jobs[1].result.numpy(), _alone(protos, jobs_fn, "fan_sqs", 1, 1)) <= MIX_TOL
    eng.close()


@pytest.mark.parametrize("name,nz", [("fan_sqs", 3), ("cone_sqs", 1)])
def test_evicted_job_resumes_to_the_same_result(name, nz):
    from ctprojector_b200.serving import Engine

    protos, jobs_fn = _setup(n_iter=10)
    job, other = jobs_fn(protos, [(name, nz, 0.0), ("par_sqs", 2, 0.0)])
    eng = Engine()
    eng.submit(job)
    eng.submit(other)
    eng._admit(0.0)
    for _ in range(4):
        torch.cuda.synchronize()
        eng._step()
    snap = eng.evict(job.job_id)
    assert job.status == "evicted" and snap.done == 4
    while eng.busy():  # the other job goes on while the evicted one is off the device
        eng.pass_once(0.0)
        torch.cuda.synchronize()
    torch.cuda.synchronize()
    assert snap.ready()
    resumed = snap.job()
    eng.run([resumed], realtime=False)
    assert resumed.status == "done"
    ref = _alone(protos, jobs_fn, name, nz, 0)
    assert rel_l2(resumed.result.numpy(), ref) <= MIX_TOL
    assert rel_l2(other.result.numpy(), _alone(protos, jobs_fn, "par_sqs", 2, 1)) <= MIX_TOL
    eng.close()
