"""The device interior-point solve against the CPU twin (oracle_ipm) and the
reference's known-answer checks."""
import os

import numpy as np
import pytest

import oracle as O
import oracle_ipm as OI

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "known_answers.npz")


@pytest.mark.parametrize("key", ["100", "200", "500", "16x16", "12x18", "16x24", "32x32", "8x8x8", "6x10x12",
                                 "14x8x4", "8x6x4", "16x16x16"])
@pytest.mark.parametrize("rdft", [True, False])
def test_known_answer(cuda, key, rdft):
    """test/ipm_example_{1,2,3}D.jl with check=true: no noise, no mask, lambda = 0,
    ||beta_true - beta|| <= 1e-6 with beta_true = DFT_to_beta(fft(x)/sqrt(N))."""
    import csipm
    torch = cuda
    g = np.load(GOLD)
    size = tuple(int(s) for s in key.split("x"))
    params = csipm.FFTParameters(len(size), size, torch.tensor(g["x_" + key], device="cuda"), 0.0, None)
    nlp = csipm.FFTNLPModel(params, rdft=rdft)
    res = csipm.ipm_solve(nlp)
    assert res.status == 0, res.stats
    assert np.linalg.norm(g["beta_" + key] - res.beta.cpu().numpy()) <= 1e-6


def _problem(kind, dims, seed):
    import csipm.problems as P
    spec = P.make_spec(kind, dims=dims, seed=seed)
    op0 = O.Operator(spec.size)
    return P.finalize(spec, op0.A, op0.At)


@pytest.mark.parametrize("kind,dims", [("1d", (2048,)), ("1d", (16384,)), ("2d", (64, 64)), ("2d", (128, 96)),
                                       ("2d", (96, 128)), ("3d", (16, 16, 16)), ("3d", (32, 32, 32)),
                                       ("3d", (32, 64, 24)), ("3d", (64, 64, 64)), ("3d", (60, 48, 40)),
                                       ("3d", (72, 90, 54))])
def test_parity_with_cpu_twin(cuda, kind, dims):
    """Same seed, same algorithm: beta within 1e-6 relative, objective within
    1e-8 relative, IPM iteration count within 1."""
    import csipm
    torch = cuda
    prob = _problem(kind, dims, seed=1)
    size = prob.size
    params = csipm.FFTParameters(len(size), size, torch.tensor(prob.z0, device="cuda"), prob.lam, prob.missing)
    nlp = csipm.FFTNLPModel(params, rdft=True, tol=1e-10)
    res = csipm.ipm_solve(nlp)
    assert res.status == 0, res.stats
    op = O.Operator(size, prob.spec.keep)
    b = op.At(prob.z0)
    beta, c, info = OI.ipm(op, b, prob.lam, float(prob.z0 @ prob.z0), tol=1e-10)
    assert info["status"] == "ok"
    bg = res.beta.cpu().numpy()
    assert np.linalg.norm(bg - beta) / np.linalg.norm(beta) <= 1e-6
    Fg = OI.lasso_value(op, bg, prob.z0, prob.lam)
    Fc = OI.lasso_value(op, beta, prob.z0, prob.lam)
    assert abs(Fg - Fc) <= 1e-8 * Fc
    assert abs(res.stats["ipm_iter"] - info["ipm_iter"]) <= 1
    assert abs(res.stats["obj"] - info["obj"]) <= 1e-8 * abs(info["obj"])


@pytest.mark.parametrize("kind,dims", [("2d", (64, 64)), ("2d", (200, 160)), ("3d", (32, 64, 24)),
                                       ("3d", (40, 128, 32)), ("3d", (64, 64, 64))])
def test_solver_order_matches_reference_order(cuda, kind, dims):
    """The solve in the half-spectrum solver order (second dimension with a
    two-level factor pair: 64, 128, 160, 256, 320) and in the reference packing
    take the same iterates up to the order of floating-point sums."""
    import csipm
    torch = cuda
    prob = _problem(kind, dims, seed=3)
    size = prob.size
    out = {}
    for layout in ("solver", "reference"):
        params = csipm.FFTParameters(len(size), size, torch.tensor(prob.z0, device="cuda"), prob.lam, prob.missing)
        nlp = csipm.FFTNLPModel(params, rdft=True, tol=1e-10, layout=layout)
        res = csipm.ipm_solve(nlp)
        assert res.status == 0, res.stats
        out[layout] = res
    bs, br = out["solver"].beta.cpu().numpy(), out["reference"].beta.cpu().numpy()
    assert np.linalg.norm(bs - br) / np.linalg.norm(br) <= 1e-7
    assert abs(out["solver"].stats["ipm_iter"] - out["reference"].stats["ipm_iter"]) <= 1
    assert abs(out["solver"].stats["lasso_obj"] - out["reference"].stats["lasso_obj"]) <= 1e-10 * abs(out["reference"].stats["lasso_obj"])


@pytest.mark.parametrize("kind,dims,precision,rtol", [("3d", (32, 64, 24), "fp64", 1e-8), ("2d", (96, 128), "mixed", 1e-8),
                                                      ("1d", (4096,), "fp64", 1e-8), ("3d", (64, 64, 64), "mixed", 1e-8),
                                                      ("3d", (64, 64, 64), "fp64", 1e-2), ("3d", (48, 40, 36), "mixed", 1e-2),
                                                      ("2d", (128, 96), "mixed", 1e-3), ("1d", (16384,), "fp64", 1e-2)])
def test_cuda_graph_replay_changes_nothing(cuda, kind, dims, precision, rtol):
    """Graph replays run the same kernels with the same arguments as plain
    launches: identical beta and counts.  FP64 solves, and mixed ones with
    FP32 directions (Newton rtol >= 1e-4), replay whole iterations (the stop
    test on the device, one host wait per solve); the rest replay their CG
    loops."""
    import csipm
    torch = cuda
    prob = _problem(kind, dims, seed=4)
    size = prob.size
    out = {}
    for graphs in (True, False):
        params = csipm.FFTParameters(len(size), size, torch.tensor(prob.z0, device="cuda"), prob.lam, prob.missing)
        nlp = csipm.FFTNLPModel(params, rdft=True, precision=precision, tol=1e-10, cuda_graphs=graphs,
                                ipm_cg_rtol=rtol)
        res = csipm.ipm_solve(nlp)
        assert res.status == 0, res.stats
        out[graphs] = res
    assert torch.equal(out[True].beta, out[False].beta)
    for key in ("ipm_iter", "cg_iter", "matvecs"):
        assert out[True].stats[key] == out[False].stats[key]
    whole = precision == "fp64" or rtol >= 1e-4
    assert out[False].stats["graph_iters"] == 0
    if whole:   # every iteration after the first ran inside the graph
        assert out[True].stats["graph_iters"] == out[True].stats["ipm_iter"]
    else:
        assert out[True].stats["graph_iters"] == 0


def test_graph_replay_stops_at_max_iter(cuda):
    """The device stop test honours max_iter: a replayed solve capped at 3
    iterations stops there, like the plain loop."""
    import csipm
    torch = cuda
    prob = _problem("3d", (32, 32, 32), seed=2)
    size = prob.size
    got = {}
    for graphs in (True, False):
        params = csipm.FFTParameters(len(size), size, torch.tensor(prob.z0, device="cuda"), prob.lam, prob.missing)
        nlp = csipm.FFTNLPModel(params, rdft=True, tol=1e-10, max_iter=3, cuda_graphs=graphs, ipm_cg_rtol=1e-2)
        res = csipm.ipm_solve(nlp)
        assert res.status == -8, res.stats
        got[graphs] = res
    assert got[True].stats["ipm_iter"] == got[False].stats["ipm_iter"] == 3
    assert torch.equal(got[True].beta, got[False].beta)


@pytest.mark.parametrize("kind,dims", [("3d", (48, 40, 36)), ("2d", (100, 96)), ("3d", (32, 64, 24))])
def test_autotuned_and_heuristic_configs_agree(cuda, kind, dims):
    """The autotuner only picks among launch configurations of the same
    transforms: both solves reach the same optimum."""
    import csipm
    torch = cuda
    prob = _problem(kind, dims, seed=6)
    size = prob.size
    out = {}
    for tune in (True, False):
        params = csipm.FFTParameters(len(size), size, torch.tensor(prob.z0, device="cuda"), prob.lam, prob.missing)
        nlp = csipm.FFTNLPModel(params, rdft=True, tol=1e-10, autotune=tune)
        res = csipm.ipm_solve(nlp)
        assert res.status == 0, res.stats
        out[tune] = res.beta.cpu().numpy()
    assert np.linalg.norm(out[True] - out[False]) <= 1e-7 * np.linalg.norm(out[False])


def test_tune_cache_persists_across_processes(cuda, tmp_path):
    """CSIPM_TUNE_CACHE names a file: the first process tunes a size and
    appends its choice (one JSON object per line); a second process reads it
    back and tunes nothing, so no second line appears."""
    import json
    import subprocess
    import sys
    from conftest import PKG
    path = tmp_path / "tune.jsonl"
    code = ("import sys; sys.path.insert(0, %r); import numpy as np, torch, csipm\n"
            "size = (48, 40, 36)\n"
            "z = torch.zeros(int(np.prod(size)), dtype=torch.float64, device='cuda')\n"
            "op = csipm.FFTOperator(csipm.FFTParameters(3, size, z, 0.1, None), autotune=True)\n"
            "op.close()\n") % PKG
    env = dict(os.environ, CSIPM_TUNE_CACHE=str(path))
    for _ in range(2):
        subprocess.run([sys.executable, "-c", code], env=env, check=True, timeout=600)
    lines = path.read_text().splitlines()
    assert len(lines) == 1
    entry = json.loads(lines[0])
    assert entry["n"] == [48, 40, 36] and entry["dim"] == 3 and entry["elem"] == 8
