"""The warm-start network: its hand-written BF16 forward and backward kernels against the FP64
restatement (oracle/mlp_oracle.py), its training, and what a trained network gains the IPM on a
parametric LP family (fewer iterations, the same optimum)."""
import numpy as np
import pytest

from oracle import mlp_oracle
from sovereign_b200 import problems as P
from sovereign_b200.ipm import InteriorPointOptions
from sovereign_b200.warmstart import Mlp, Normalizer, WarmStart, solve_many

pytestmark = pytest.mark.gpu


def test_forward_and_gradients_match_fp64_restatement():
    rng = np.random.default_rng(0)
    dims = (96, 64, 3, 80)  # n_in, hidden, layers, n_out: partial 128-tiles on every side
    mlp = Mlp(dims[0], dims[3], dims[1], dims[2], seed=3)
    x = rng.standard_normal((40, dims[0])).astype(np.float32)
    t = rng.standard_normal((40, dims[3])).astype(np.float32)
    loss, g = mlp.loss_grad(x, t)
    ref_loss, ref_g, ref_y = mlp_oracle.loss_and_grad(mlp.params, mlp.dims, x, t)
    y = mlp.forward(x)
    # BF16 operands (8-bit mantissa), FP32 accumulation: ~1e-2 relative agreement
    assert np.linalg.norm(y - ref_y) / np.linalg.norm(ref_y) < 2e-2
    assert abs(loss - ref_loss) / ref_loss < 2e-2
    cos = float(g @ ref_g / (np.linalg.norm(g) * np.linalg.norm(ref_g)))
    assert cos > 0.999
    assert abs(np.linalg.norm(g) / np.linalg.norm(ref_g) - 1.0) < 3e-2
    # per layer, against the restatement with the kernels' BF16 operand rounding: only the
    # accumulation order differs
    _, bf_g, bf_y = mlp_oracle.loss_and_grad(mlp.params, mlp.dims, x, t, bf16_operands=True)
    assert np.linalg.norm(y - bf_y) <= 1e-3 * np.linalg.norm(bf_y)
    off = 0
    for l in range(len(mlp.dims) - 1):
        for size in (mlp.dims[l + 1] * mlp.dims[l], mlp.dims[l + 1]):
            a, b = g[off:off + size], bf_g[off:off + size]
            assert np.linalg.norm(a - b) <= 5e-3 * np.linalg.norm(b) + 1e-7, (l, size)
            off += size


def test_production_shape_gradients_match_restatement():
    # the multicommodity network's own shape (4040 -> 512 x 3 -> 11800): many K chunks and N tiles per
    # product, and a weight-gradient reduction over the batch, through the pipelined GEMM
    rng = np.random.default_rng(7)
    dims = (4040, 512, 3, 11800)
    mlp = Mlp(dims[0], dims[3], dims[1], dims[2], seed=5)
    x = rng.standard_normal((128, dims[0])).astype(np.float32)
    t = rng.standard_normal((128, dims[3])).astype(np.float32)
    loss, g = mlp.loss_grad(x, t)
    bf_loss, bf_g, bf_y = mlp_oracle.loss_and_grad(mlp.params, mlp.dims, x, t, bf16_operands=True)
    y = mlp.forward(x)
    assert np.linalg.norm(y - bf_y) <= 1e-3 * np.linalg.norm(bf_y)
    assert abs(loss - bf_loss) <= 1e-3 * bf_loss
    # per layer against the BF16-faithful restatement: the backward pass crosses four products whose
    # BF16 operand roundings flip where FP32 accumulation orders differ, so the deepest layer's
    # gradient agrees to about 1 % in norm (measured 0.74 %) and its direction to cosine > 0.9999
    off = 0
    for l in range(len(mlp.dims) - 1):
        for size in (mlp.dims[l + 1] * mlp.dims[l], mlp.dims[l + 1]):
            a, b = g[off:off + size].astype(np.float64), bf_g[off:off + size]
            assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-7, (l, size)
            assert a @ b / (np.linalg.norm(a) * np.linalg.norm(b)) > 0.9999, (l, size)
            off += size


def test_pipelined_gemm_equals_single_stage_kernel(monkeypatch):
    # the same products through the single-stage kernel (SOVEREIGN_MLP_GEMM=single, read when the
    # library first runs a product in a process) and through the pipelined one agree to accumulation
    # order; run in a child process so the switch takes effect
    import subprocess
    import sys
    code = ("import numpy as np, sys; sys.path.insert(0, '.');"
            "from sovereign_b200.warmstart import Mlp;"
            "r = np.random.default_rng(2); m = Mlp(300, 200, 160, 2, seed=1);"
            "x = r.standard_normal((70, 300)).astype(np.float32); t = r.standard_normal((70, 200)).astype(np.float32);"
            "l, g = m.loss_grad(x, t); np.save(sys.argv[1], np.concatenate([[l], g, m.forward(x).ravel()]))")
    import os
    import tempfile
    out = {}
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for mode in ("single", "pipelined"):
        env = dict(os.environ)
        if mode == "single":
            env["SOVEREIGN_MLP_GEMM"] = "single"
        else:
            env.pop("SOVEREIGN_MLP_GEMM", None)
        f = os.path.join(tempfile.mkdtemp(), f"{mode}.npy")
        subprocess.run([sys.executable, "-c", code, f], check=True, cwd=root, env=env, timeout=300)
        out[mode] = np.load(f)
    a, b = out["single"], out["pipelined"]
    assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(a)


def test_training_reduces_loss():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((512, 32)).astype(np.float32)
    w = rng.standard_normal((32, 16)).astype(np.float32) / 6
    t = np.tanh(x @ w).astype(np.float32)
    mlp = Mlp(32, 16, 64, 2, seed=0)
    before, _ = mlp.loss_grad(x, t)
    after = mlp.train(x, t, epochs=60, batch=64, lr=3e-3)
    assert after < 0.2 * before


def test_warm_start_saves_iterations_on_a_parametric_family():
    fam = P.MulticommodityFamily(nodes=30, arcs=100, commodities=2, sinks=3, seed=11)
    train = [fam.instance_from_seed(1000 + k) for k in range(192)]
    test = [fam.instance_from_seed(5000 + k) for k in range(24)]
    opts = InteriorPointOptions()
    # targets: the iterate at the start of iteration 5, an early, well-centred point of the path
    cold_train, _ = solve_many([m for m, _ in train], InteriorPointOptions(ipm_iterate_at=5))
    ws = WarmStart(fam.param_dim, cold_train[0].n_ipm, cold_train[0].m_ipm, hidden=128, layers=3, seed=0)
    ws.fit(np.stack([p for _, p in train]), cold_train, epochs=150, batch=64, lr=2e-3)
    cold, _ = solve_many([m for m, _ in test], opts)
    warm, _ = solve_many([m for m, _ in test], opts, warm=ws.predict(np.stack([p for _, p in test])))
    for c, w in zip(cold, warm):
        assert c.status_name == "OPTIMAL" and w.status_name == "OPTIMAL"
        assert abs(c.objective_value - w.objective_value) <= 1e-8 * max(1.0, abs(c.objective_value))
    used = sum(w.diagnostics["warm_start_used"] for w in warm)
    gain = np.mean([c.iterations for c in cold]) - np.mean([w.iterations for w in warm])
    info = (gain, used, [c.iterations for c in cold], [w.iterations for w in warm])
    assert gain > 0.5, info
    assert used >= len(test) // 2, info


def test_predict_start_matches_host_decoding():
    # sov_mlp_predict_start (normalization, network, decoding on the GPU) against the network's
    # plain forward pass decoded on the host with the same formulas
    rng = np.random.default_rng(3)
    n_param, n, m = 24, 30, 11
    ws = WarmStart(n_param, n, m, hidden=64, layers=2, seed=1)
    ws.fin = Normalizer(rng.normal(size=n_param), rng.uniform(0.5, 2.0, size=n_param))
    ws.fout = Normalizer(rng.normal(size=2 * n + m), rng.uniform(0.5, 2.0, size=2 * n + m))
    params = rng.normal(size=(37, n_param))
    got = ws.predict(params)
    out = ws.fout.invert(ws.mlp.forward(ws.fin.apply(params)).astype(np.float64))
    xs = np.maximum(np.exp(np.clip(out[:, :n], -40, 40)), 1e-6)
    ss = np.maximum(np.exp(np.clip(out[:, n + m:], -40, 40)), 1e-6)
    for k in range(len(params)):
        np.testing.assert_allclose(got[k][0], xs[k], rtol=1e-12)
        np.testing.assert_allclose(got[k][1], out[k, n:n + m], rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(got[k][2], ss[k], rtol=1e-12)


def test_batch_from_device_starts_equals_host_starts(monkeypatch):
    # sov_lp_solve_batch_predicted keeps the predicted starts on the device; given the same network
    # and parameters it must give exactly what the batch gives with the same starts from host arrays.
    # The call is split into three parts, so each part gathers its starts from an offset other than 0.
    from sovereign_b200.ipm import solve_batch
    fam = P.TransportFamily()
    train = [fam.instance_from_seed(300 + k) for k in range(64)]
    test = [fam.instance_from_seed(900 + k) for k in range(48)]
    early, _ = solve_many([m for m, _ in train], InteriorPointOptions(ipm_iterate_at=5))
    ws = WarmStart(fam.param_dim, early[0].n_ipm, early[0].m_ipm, hidden=64, layers=2, seed=0)
    ws.fit(np.stack([p for _, p in train]), early, epochs=30, batch=32, lr=2e-3)
    models, params = [m for m, _ in test], np.stack([p for _, p in test])
    host = solve_batch(models, warm_starts=ws.predict(params), with_diag=True)
    monkeypatch.setenv("SOVEREIGN_BATCH_PARTS", "3")
    dev = ws.solve_batch(models, params, with_diag=True)
    for h, d in zip(host, dev):
        assert d.status_name == "OPTIMAL" and h.status == d.status and h.iterations == d.iterations
        assert h.objective_value == d.objective_value
        np.testing.assert_array_equal(h.primal, d.primal)
        assert h.diagnostics["warm_start_used"] == d.diagnostics["warm_start_used"]
    assert sum(d.diagnostics["warm_start_used"] for d in dev) > 0
    # an LP whose IPM form does not match the network's output is refused
    with pytest.raises(Exception):
        ws.solve_batch([P.transport(5, 6, 1)], params[:1])
