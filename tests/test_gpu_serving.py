"""The continuous-batching reconstruction server on the GPU: fused SQS-TV
update against the FP64 oracle, served results against FP64 reconstructions
(tolerance 1e-4 relative L2), each result the same alone and in the mix,
jobs joining a running lane, admission by HBM budget, low-precision storage.

The oracle always reconstructs from the FP32 sinogram a job was made from,
before any storage rounding, so a low-precision storage format's rounding
counts as error."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SERVE_TOL = 1e-4  # served result vs FP64 oracle reconstruction, relative L2
MIX_TOL = 1e-6  # the same job alone vs in the mix


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _protocols(n_iter=6, storage="float32"):
    from ctprojector_b200 import synthetic as S
    from ctprojector_b200.serving import Protocol

    fan = S.Scan(64, 64, 1, 1.0, 1.0, 1.0, 96, 1, 1.2858, 1.0, 90)
    par = S.Scan(64, 64, 1, 1.0, 1.0, 1.0, 96, 1, 1.0, 1.0, 90)
    cone = S.Scan(48, 48, 8, 1.0, 1.0, 1.0, 72, 12, 1.2858, 1.0, 24)
    cgeo = S.helical(24, 1.0, cone.dso, cone.dsd, 8 * cone.dso / cone.dsd)
    kw = dict(n_iter=n_iter, beta=2e-3, tv_weights=(0.5, 1.0, 1.0), eps=1e-6, storage=storage)
    return {
        "fan_sqs": Protocol("fan_sqs", "fan", "sqs", fan, angles=S.angles(90, 2 * np.pi), **kw),
        "par_sqs": Protocol("par_sqs", "parallel", "sqs", par, angles=S.angles(90, np.pi), **kw),
        "cone_sqs": Protocol("cone_sqs", "cone", "sqs", cone, cone=cgeo, **kw),
        "fan_fbp": Protocol("fan_fbp", "fan", "fbp", fan, angles=S.angles(90, 2 * np.pi), storage=storage),
        "par_fbp": Protocol("par_fbp", "parallel", "fbp", par, angles=S.angles(90, np.pi), storage=storage),
    }


def _sinogram(proto, nz, seed):
    """Seeded phantom projected by the FP32 projector, with noise, on the host:
    (the sinogram in the protocol's storage, the FP32 sinogram)."""
    from ctprojector_b200 import synthetic as S
    from ctprojector_b200.projector import _device as D
    from ctprojector_b200.serving import DTYPES

    rng = np.random.default_rng(seed)
    s = proto.scan
    if proto.kind == "cone":
        img = S.ellipsoid_phantom(rng, int(s.nz), int(s.ny), int(s.nx), s.dz, s.dy, s.dx, supersample=1)[None]
        geo = [torch.tensor(a, device="cuda") for a in proto.cone]
        y = D.siddon_fp(s, torch.tensor(img, device="cuda"), *geo)
    else:
        img = np.stack([S.ellipse_phantom(rng, int(s.nx), int(s.ny), s.dx, s.dy)[None] for _ in range(nz)])
        geom = 0 if proto.kind == "fan" else 1
        y = D.dd_fp(s, torch.tensor(img, device="cuda"), torch.tensor(proto.angles, device="cuda"), geom)
    y = y.cpu()
    y = y + 0.01 * y.abs().max() * torch.tensor(rng.standard_normal(y.shape), dtype=torch.float32)
    if proto.storage == "q16":
        from ctprojector_b200 import quant

        return quant.quantize(y.cuda()).cpu().pin_memory(), y
    return y.to(DTYPES[proto.storage]).pin_memory(), y


def _jobs(protos, spec, seed0=0):
    from ctprojector_b200.serving import Job

    jobs = []
    for i, (name, nz, t) in enumerate(spec):
        p = protos[name]
        nz = 1 if p.kind == "cone" else nz
        stored, y32 = _sinogram(p, nz, seed0 + i)
        jobs.append(Job(i, p, stored, arrival=t, nz=nz, tag=y32))
    return jobs


def _oracle_result(job, y32=None):
    """FP64 reconstruction of the job's FP32 sinogram (``y32``, or the job's
    tag), before storage rounding."""
    from oracle import recon as R

    p = job.protocol
    y = (job.tag if y32 is None else y32).float().numpy().astype(np.float64)
    if p.algo == "fbp":
        return R.fbp(p.scan, p.kind, y, p.angles, p.filter)
    geo = p.cone if p.kind == "cone" else p.angles
    return R.sqs_tv(p.scan, p.kind, y, geo, p.n_iter, p.beta, p.tv_weights, p.eps)


MIX = [("fan_sqs", 2, 0.0), ("par_sqs", 1, 0.0), ("cone_sqs", 1, 0.0), ("fan_fbp", 3, 0.0), ("fan_sqs", 1, 0.0),
       ("par_fbp", 2, 0.0), ("par_sqs", 3, 0.0), ("cone_sqs", 1, 0.0), ("fan_sqs", 3, 0.0)]


def test_sqs_tv_update_matches_oracle(oracle):
    from ctprojector_b200.recon import sqs_tv_update

    rng = np.random.default_rng(4)
    depths = [3, 1, 4]
    ns, ny, nx = sum(depths), 21, 19
    x = rng.uniform(0, 1, (ns, ny, nx)).astype(np.float32)
    bp = rng.standard_normal((ns, ny, nx)).astype(np.float32)
    norm = rng.uniform(1, 2, (2, ny, nx)).astype(np.float32)
    zl = np.concatenate([[0] if d == 1 else [2] + [3] * (d - 2) + [1] for d in depths]).astype(np.uint8)
    w, beta = (0.25, 1.0, 2.0), 0.5
    t = lambda a: torch.tensor(a, device="cuda")  # noqa: E731
    xlp = torch.empty(ns, ny, nx, dtype=torch.bfloat16, device="cuda")
    out = sqs_tv_update(t(x), t(bp), t(norm), beta, w, 2.0 ** -20, zlink=t(zl), x_lp=xlp)
    ref = oracle.sqs_tv_update(x, bp, norm, zl, w, beta, 2.0 ** -20)
    assert rel_l2(out.cpu().numpy(), ref) <= 1e-5
    assert torch.equal(xlp, out.to(torch.bfloat16))
    # no z links: every slice on its own
    out = sqs_tv_update(t(x), t(bp), t(norm), beta, w, 2.0 ** -20)
    assert rel_l2(out.cpu().numpy(), oracle.sqs_tv_update(x, bp, norm, None, w, beta, 2.0 ** -20)) <= 1e-5


def test_served_results_match_fp64_oracle():
    from ctprojector_b200.serving import Engine

    jobs = _jobs(_protocols(), MIX)
    eng = Engine()
    summary = eng.run(jobs, realtime=False)
    assert summary["jobs"] == len(jobs)
    for job in jobs:
        err = rel_l2(job.result.numpy(), _oracle_result(job))
        assert err <= SERVE_TOL, (job.protocol.name, err)
    eng.close()


@pytest.mark.parametrize("graphs", [True, False])
def test_result_same_alone_and_in_the_mix(graphs):
    from ctprojector_b200.serving import Engine

    protos = _protocols()
    mixed = _jobs(protos, MIX)
    eng = Engine(use_graphs=graphs)
    eng.run(mixed, realtime=False)
    for job in _jobs(protos, MIX):
        alone = Engine(use_graphs=graphs)
        alone.run([job], realtime=False)
        ref = mixed[job.job_id].result.numpy()
        assert rel_l2(job.result.numpy(), ref) <= MIX_TOL, job.protocol.name
        alone.close()
    eng.close()


def test_job_joins_a_running_lane():
    """A job admitted while another is mid-way through its iterations runs in
    the same lane from the next iteration and still gets its own result."""
    from ctprojector_b200.serving import Engine

    protos = _protocols(n_iter=10)
    a, b = _jobs(protos, [("fan_sqs", 2, 0.0), ("fan_sqs", 3, 0.0)])
    eng = Engine()
    eng.submit(a)
    eng._admit(0.0)
    lane = eng.lanes["fan_sqs"]
    for _ in range(4):
        torch.cuda.synchronize()  # a lane with two steps in flight is not stepped
        eng._step()
    eng.submit(b)
    eng._admit(0.0)
    assert set(lane.jobs) == {a.job_id, b.job_id}
    assert lane.jobs[a.job_id][1] == 6 and lane.jobs[b.job_id][1] == 10
    while eng.busy():
        eng._step()
        torch.cuda.synchronize()
        eng._poll(lambda: 0.0)
    for job in (a, b):
        ref = Engine()
        alone = _jobs(protos, [("fan_sqs", job.nz, 0.0)], seed0=job.job_id)[0]
        ref.run([alone], realtime=False)
        assert rel_l2(job.result.numpy(), alone.result.numpy()) <= MIX_TOL
    eng.close()


def test_admission_waits_for_memory():
    """With a budget too small for every lane at once, jobs of other
    protocols wait until an idle lane is torn down; all of them finish and the
    reservations never exceed the budget."""
    from ctprojector_b200.serving import Engine, FBPLane, SQSLane

    protos = _protocols()
    need = max(SQSLane.bytes_per_unit(protos["fan_sqs"]) * 8, SQSLane.bytes_per_unit(protos["cone_sqs"]) * 1,
               FBPLane.bytes_per_unit(protos["par_fbp"]) * 8)
    eng = Engine(hbm_bytes=int(need * 1.2), slices_per_lane=8, capacity={"cone_sqs": 1})
    jobs = _jobs(protos, [("fan_sqs", 2, 0.0), ("cone_sqs", 1, 0.0), ("par_fbp", 3, 0.0), ("fan_sqs", 1, 0.0)])
    summary = eng.run(jobs, realtime=False)
    assert summary["jobs"] == 4
    assert eng.evictions >= 1 and eng.peak_reserved <= eng.budget.total
    for job in jobs:
        assert rel_l2(job.result.numpy(), _oracle_result(job)) <= SERVE_TOL
    eng.close()


# Rounding of 16-bit sinogram storage against the FP32-input FP64 oracle: the
# affine codes (q16) meet SERVE_TOL; BF16 and FP16 (relative rounding 2^-9 and
# 2^-12, magnified by the ramp filter of the FBP jobs) do not, and are held to
# these measured ceilings instead.
LOWP_CEILING = {"q16": SERVE_TOL, "float16": 3e-3, "bfloat16": 3e-2}


@pytest.mark.parametrize("storage", ["q16", "float16", "bfloat16"])
def test_low_precision_sinogram_storage(storage):
    """Sinograms held in 16 bits on the device, iterate and sums in FP32,
    against the FP64 reconstruction of the FP32 sinogram."""
    from ctprojector_b200.serving import Engine

    protos = _protocols(storage=storage)
    jobs = _jobs(protos, [("fan_sqs", 2, 0.0), ("par_fbp", 2, 0.0), ("cone_sqs", 1, 0.0), ("fan_fbp", 1, 0.0)])
    eng = Engine()
    eng.run(jobs, realtime=False)
    errs = {}
    for job in jobs:
        dt = job.sinogram.code.dtype if storage == "q16" else job.sinogram.dtype
        assert dt != torch.float32
        errs[job.protocol.name] = rel_l2(job.result.numpy(), _oracle_result(job))
    print(storage, {k: f"{v:.3g}" for k, v in errs.items()})
    assert all(e <= LOWP_CEILING[storage] for e in errs.values()), errs
    eng.close()


def test_per_call_path_matches_server():
    from ctprojector_b200.serving import Engine
    from ctprojector_b200.serving.per_call import run_per_call

    protos = _protocols()
    a = _jobs(protos, MIX[:4])
    b = _jobs(protos, MIX[:4])
    Engine().run(a, realtime=False)
    run_per_call(b, realtime=False)
    for x, y in zip(a, b):
        assert rel_l2(x.result.numpy(), y.result.numpy()) <= 1e-5


def test_full_size_protocols_match_fp64_oracle():
    """The served stream's own protocols at full size, with the sinograms in
    the served storage (q16): the results of the jobs the FP64 oracle
    reconstructs in seconds are within 1e-4 of its reconstruction of the FP32
    sinograms (relative L2)."""
    from ctprojector_b200 import quant
    from ctprojector_b200.serving import Engine
    from ctprojector_b200.serving import workload as W

    p32 = W.catalog(storage="float32")
    protos = W.catalog(storage="q16")
    stream = [(0.0, "fan256_sqs", 1), (0.0, "fan256_fbp", 2), (0.0, "par512_fbp", 1), (0.0, "fan512_fbp", 1)]
    pools32 = {n: W.sinogram_pool(p32[n], 1, 2, seed=i) for i, (_, n, _) in enumerate(stream)}
    pools = {n: [quant.quantize(t.cuda()).cpu().pin_memory() for t in v] for n, v in pools32.items()}
    jobs = W.make_jobs(protos, stream, pools)
    eng = Engine()
    eng.run(jobs, realtime=False)
    for job in jobs:
        name, k = job.tag
        err = rel_l2(job.result.numpy(), _oracle_result(job, pools32[name][k][:job.nz]))
        assert err <= SERVE_TOL, (job.protocol.name, err)
    eng.close()
