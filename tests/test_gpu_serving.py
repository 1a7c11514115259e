"""Serving loop (csipm_server_*): requests of uneven sizes admitted by device
footprint, solved concurrently on per-slot streams.  Each result must equal the
same request solved alone (beta within 1e-12 relative: the kernels and their
reductions are deterministic, so concurrency changes nothing)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

MIX = [("1d", (2048,), "fp64", 1e-8), ("1d", (4096,), "mixed", 1e-2), ("2d", (64, 64), "fp64", 1e-2),
       ("2d", (96, 128), "mixed", 1e-5), ("3d", (32, 32, 32), "fp64", 1e-8), ("3d", (32, 64, 24), "mixed", 1e-2),
       ("3d", (48, 48, 48), "fp64", 1e-3), ("2d", (120, 64), "mixed", 1e-8), ("3d", (16, 16, 16), "mixed", 1e-4),
       ("1d", (6000,), "fp64", 1e-3)]


def _problem(kind, dims, seed):
    import csipm.problems as P
    spec = P.make_spec(kind, dims=dims, seed=seed)
    op0 = O.Operator(spec.size)
    return P.finalize(spec, op0.A, op0.At)


@pytest.fixture(scope="module")
def problems():
    return [_problem(kind, dims, seed=10 + k) for k, (kind, dims, _, _) in enumerate(MIX)]


def _alone(torch, prob, precision, rtol):
    import csipm
    size = prob.size
    params = csipm.FFTParameters(len(size), size, torch.tensor(prob.z0, device="cuda"), prob.lam, prob.missing)
    nlp = csipm.FFTNLPModel(params, rdft=True, precision=precision, tol=1e-10, ipm_cg_rtol=rtol)
    res = csipm.ipm_solve(nlp)
    nlp.op_fft.close()
    return res


@pytest.mark.parametrize("graphs", [False, True])
def test_results_same_alone_and_in_the_mix(cuda, problems, graphs):
    """Served with plain launches or with each request's iterations as one
    graph launch, every result equals the request solved alone."""
    from csipm.serving import Server
    torch = cuda
    with Server(slots=4, cuda_graphs=graphs) as srv:
        for k, (prob, (_, _, prec, rtol)) in enumerate(zip(problems, MIX)):
            srv.submit(prob.size, prob.z0, prob.lam, prob.missing, tag=k, precision=prec, tol=1e-10,
                       ipm_cg_rtol=rtol)
        got = {r.tag: r for r in srv.drain()}
    assert sorted(got) == list(range(len(MIX)))
    for k, (prob, (_, _, prec, rtol)) in enumerate(zip(problems, MIX)):
        r = got[k]
        assert r.status == 0, (k, r.stats)
        alone = _alone(torch, prob, prec, rtol)
        b = alone.beta.cpu().numpy()
        assert np.linalg.norm(r.beta - b) <= 1e-12 * np.linalg.norm(b), k
        assert r.stats["ipm_iter"] == alone.stats["ipm_iter"]
        assert r.latency_ms >= r.queue_ms >= 0.0


def test_admission_by_footprint(cuda, problems):
    """A budget that holds about one large request at a time still completes
    every request (smaller ones go first while a large one waits)."""
    from csipm.serving import Server, footprint
    fps = [footprint(p.size, prec, p.missing.size if p.missing is not None else 0)
           for p, (_, _, prec, _) in zip(problems, MIX)]
    budget = int(1.2 * max(fps))
    with Server(slots=4, hbm_budget=budget) as srv:
        for k, (prob, (_, _, prec, rtol)) in enumerate(zip(problems, MIX)):
            srv.submit(prob.size, prob.z0, prob.lam, prob.missing, tag=k, precision=prec, tol=1e-10,
                       ipm_cg_rtol=rtol)
        res = srv.drain()
    assert len(res) == len(MIX)
    assert all(r.status == 0 for r in res)
    assert all(r.footprint == fps[r.tag] for r in res)


def test_requests_arriving_while_others_run(cuda, problems):
    """Continuous admission: requests submitted after earlier ones are already
    on the GPU join them; every result arrives."""
    from csipm.serving import Server
    with Server(slots=3) as srv:
        half = len(MIX) // 2
        for k in range(half):
            prob = problems[k]
            srv.submit(prob.size, prob.z0, prob.lam, prob.missing, tag=k, precision=MIX[k][2], tol=1e-10,
                       ipm_cg_rtol=MIX[k][3])
        first = srv.poll(timeout_ms=-1)
        assert first
        for k in range(half, len(MIX)):
            prob = problems[k]
            srv.submit(prob.size, prob.z0, prob.lam, prob.missing, tag=k, precision=MIX[k][2], tol=1e-10,
                       ipm_cg_rtol=MIX[k][3])
        rest = srv.drain()
    tags = sorted(r.tag for r in first + rest)
    assert tags == list(range(len(MIX)))
    assert all(r.status == 0 for r in first + rest)


def test_footprint_bounds_the_handle(cuda, problems):
    """csipm_footprint is an upper bound of what a handle holds once it has
    solved (+ the server's z0/beta staging) and not far above it; before its
    first solve a handle holds only the operator, A^T z0 and two scratch
    vectors (the interior-point state is allocated by the first solve)."""
    import csipm
    from csipm.serving import footprint
    torch = cuda
    for prob, (_, _, prec, rtol) in list(zip(problems, MIX))[:6]:
        size = prob.size
        params = csipm.FFTParameters(len(size), size, torch.tensor(prob.z0, device="cuda"), prob.lam, prob.missing)
        nlp = csipm.FFTNLPModel(params, rdft=True, precision=prec, tol=1e-6)
        before = nlp.op_fft.device_bytes()
        csipm.ipm_solve(nlp)
        assert nlp.op_fft.device_bytes() > before + 10 * 8 * int(np.prod(size))
        held = nlp.op_fft.device_bytes() + 16 * int(np.prod(size))
        fp = footprint(size, prec, prob.missing.size if prob.missing is not None else 0)
        nlp.op_fft.close()
        assert held <= fp <= 1.6 * held + (8 << 20), (size, held, fp)


def test_failed_request_reports_its_message(cuda, problems):
    """A request the library rejects comes back with its status and the
    failure's message (the worker's error does not stay on its thread); the
    requests around it still succeed."""
    from csipm import _native
    from csipm.serving import Server
    good = problems[0]
    n = int(np.prod(good.size))
    with Server(slots=2) as srv:
        srv.submit(good.size, good.z0, good.lam, good.missing, tag=0, precision="fp64", tol=1e-8)
        srv.submit(good.size, good.z0, good.lam, np.array([0, n + 5], dtype=np.int64), tag=1, precision="fp64")
        srv.submit(good.size, good.z0, good.lam, good.missing, tag=2, precision="fp64", tol=1e-8)
        got = {r.tag: r for r in srv.drain()}
    assert got[0].status == 0 and got[2].status == 0
    assert got[0].message == ""
    assert got[1].status == _native.CSIPM_ERR_INVALID
    assert "out of range" in got[1].message


def test_batched_serving_matches_alone(cuda, problems):
    """With batching on, each slot solves up to four admitted requests of one
    batch class together (csipm_solve_batch, FP64, reference-order passes);
    every result equals the request solved alone in FP64 up to the order of
    floating-point sums (beta within 1e-6 relative, IPM iterations within 1),
    and mixed-precision requests come back with FP64 iterates."""
    from csipm.serving import Server
    torch = cuda
    with Server(slots=2, batch=4) as srv:
        for k, (prob, (_, _, prec, rtol)) in enumerate(zip(problems, MIX)):
            srv.submit(prob.size, prob.z0, prob.lam, prob.missing, tag=k, precision=prec, tol=1e-10,
                       ipm_cg_rtol=rtol)
        got = {r.tag: r for r in srv.drain()}
    assert sorted(got) == list(range(len(MIX)))
    assert max(r.group for r in got.values()) > 1        # some requests were solved as one batch
    for k, (prob, (_, _, prec, rtol)) in enumerate(zip(problems, MIX)):
        r = got[k]
        assert r.status == 0, (k, r.stats, r.message)
        alone = _alone(torch, prob, "fp64", rtol)
        b = alone.beta.cpu().numpy()
        assert np.linalg.norm(r.beta - b) <= 1e-6 * np.linalg.norm(b), k
        assert abs(r.stats["ipm_iter"] - alone.stats["ipm_iter"]) <= 1
        assert r.latency_ms >= r.queue_ms >= 0.0


def test_batched_serving_member_failures(cuda, problems):
    """In a batch, a request the library rejects (a missing index out of
    range) and one capped at 2 iterations return their own status and
    message; the members beside them converge."""
    from csipm import _native
    from csipm.serving import Server
    good = problems[2]                      # 2D 64 x 64
    other = problems[7]                     # 2D 120 x 64
    big = problems[6]                       # 3D 48^3, another batch class: keeps the one slot busy
    n = int(np.prod(good.size))
    with Server(slots=1, batch=4) as srv:
        srv.submit(big.size, big.z0, big.lam, big.missing, tag=9, tol=1e-10, ipm_cg_rtol=1e-8)
        srv.submit(good.size, good.z0, good.lam, good.missing, tag=0, tol=1e-8)
        srv.submit(good.size, good.z0, good.lam, np.array([0, n + 5], dtype=np.int64), tag=1)
        srv.submit(other.size, other.z0, other.lam, other.missing, tag=2, tol=1e-8, max_iter=2)
        srv.submit(other.size, other.z0, other.lam, other.missing, tag=3, tol=1e-8)
        got = {r.tag: r for r in srv.drain()}
    assert got[9].status == 0
    assert all(got[k].group == 4 for k in range(4))         # the four 2D requests formed one batch
    assert got[0].status == 0 and got[3].status == 0
    assert got[0].message == "" and got[3].message == ""
    assert got[1].status == _native.CSIPM_ERR_INVALID and "out of range" in got[1].message
    assert got[2].status == _native.CSIPM_ERR_IPM_MAXITER and got[2].stats["ipm_iter"] == 2
    assert "max_iter" in got[2].message


def test_batched_serving_size_cap(cuda, problems):
    """batch_max_n: a request above the cap is solved alone (group 1) even
    with requests of its class waiting; those below the cap still batch."""
    from csipm.serving import Server
    blocker = problems[3]                   # 2D 96 x 128: keeps the one slot busy while the rest queue
    big = problems[6]                       # 3D 48^3 = 110592 samples, above the cap
    small = [problems[4], problems[8], problems[5]]   # 3D 32^3, 16^3, 32x64x24
    with Server(slots=1, batch=4, batch_max_n=60000) as srv:
        srv.submit(blocker.size, blocker.z0, blocker.lam, blocker.missing, tag=9, tol=1e-10, ipm_cg_rtol=1e-8)
        srv.submit(big.size, big.z0, big.lam, big.missing, tag=0, tol=1e-8)
        for k, p in enumerate(small):
            srv.submit(p.size, p.z0, p.lam, p.missing, tag=1 + k, tol=1e-8)
        got = {r.tag: r for r in srv.drain()}
    assert all(r.status == 0 for r in got.values()), {t: r.message for t, r in got.items()}
    assert got[0].group == 1
    assert all(got[t].group == 3 for t in (1, 2, 3))
