"""The surrogate's tensor-core kernels: the tcgen05 GEMM against an FP32
matrix product of the same BF16 inputs, and its epilogues."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


# N not a multiple of 32 takes the one-tile-per-CTA kernels; the others the
# persistent kernel: resident B (K <= 256), streamed B (K = 512), more row
# tiles than SMs (both accumulators of a CTA in use), split K (few row
# tiles, long K).
@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (256, 16, 64), (512, 128, 256), (256, 64, 4096),
                                   (128, 48, 128), (384, 256, 256), (40960, 256, 64), (40960, 128, 256),
                                   (20480, 256, 512), (256, 256, 4096), (128, 32, 8192), (1024, 64, 1024)])
def test_umma_gemm_matches_fp32_product(M, N, K):
    import torch
    from dense_b200.surrogate import Kernels
    k = Kernels()
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    D = torch.full((M, N), float("nan"), device="cuda")
    k.gemm(A, B, D)
    k.check()
    ref = A.float() @ B.float().T
    err = (D - ref).abs().max().item() / ref.abs().max().item()
    assert err < 1e-5, err


@pytest.mark.parametrize("M,N,K", [(40960, 256, 256), (256, 128, 2048), (2048, 256, 256), (512, 128, 64)])
def test_persistent_gemm_epilogues(M, N, K):
    """Bias and bias+GELU through the persistent kernel's TMA-store
    epilogue (first shape), the split-K reduction (second) and column
    blocks of 64 columns (third and fourth: few row tiles, short K), into
    matrices whose leading dimension exceeds N."""
    import torch
    from dense_b200.surrogate import EPI_BIAS, EPI_BIAS_GELU, Kernels
    k = Kernels()
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    Zw = torch.full((M, N + 64), float("nan"), device="cuda")
    Hw = torch.zeros((M, N + 32), device="cuda", dtype=torch.bfloat16)
    Z, H = Zw[:, :N], Hw[:, :N]
    k.gemm(A, B, Z, EPI_BIAS_GELU, bias, H)
    Y = torch.empty(M, N, device="cuda")
    k.gemm(A, B, Y, EPI_BIAS, bias)
    k.check()
    ref = A.float() @ B.float().T + bias
    scale = ref.abs().max().item()
    assert (Z - ref).abs().max().item() < 1e-5 * scale
    assert (Y - ref).abs().max().item() < 1e-5 * scale
    assert torch.isnan(Zw[:, N:]).all(), "columns past N were written"
    gelu = torch.nn.functional.gelu(ref)
    assert (H.float() - gelu).abs().max().item() < 1e-2 * max(1.0, gelu.abs().max().item())
    assert (Hw[:, N:] == 0).all()


def test_split_k_is_deterministic():
    """Split-K sums the partials in split order: repeated products are
    bit-identical."""
    import torch
    from dense_b200.surrogate import Kernels
    k = Kernels()
    g = torch.Generator(device="cuda").manual_seed(11)
    A = torch.randn(256, 4096, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(256, 4096, device="cuda", generator=g).to(torch.bfloat16)
    outs = []
    for _ in range(5):
        D = torch.empty(256, 256, device="cuda")
        k.gemm(A, B, D)
        outs.append(D)
    k.check()
    for D in outs[1:]:
        assert torch.equal(D, outs[0])


@pytest.mark.parametrize("rows,cols", [(4096, 256), (4133, 200), (5, 64), (0, 32)])
def test_column_sums(rows, cols):
    """The bias gradient's column sums (cluster reduction over distributed
    shared memory) against a float64 sum, and bit-identical on repeat."""
    import torch
    from dense_b200.surrogate import Kernels
    k = Kernels()
    g = torch.Generator(device="cuda").manual_seed(rows + cols)
    Z = torch.randn(rows, cols, device="cuda", generator=g)
    db = torch.full((cols,), float("nan"), device="cuda")
    k.colsum(Z, db)
    db2 = torch.empty_like(db)
    k.colsum(Z, db2)
    torch.cuda.synchronize()
    ref = Z.double().sum(0)
    assert (db.double() - ref).abs().max().item() <= 1e-5 * max(1.0, Z.abs().sum(0).max().item())
    assert torch.equal(db, db2)


def test_batch_gather_matches_numpy():
    import torch
    from dense_b200.surrogate import IN_PAD, Kernels
    k = Kernels()
    rng = np.random.Generator(np.random.PCG64(4))
    X = rng.normal(size=(1000, 44)).astype(np.float32)
    T = rng.normal(size=(1000, 5)).astype(np.float32)
    M = (rng.uniform(size=(1000, 5)) > 0.3).astype(np.float32)
    idx = rng.permutation(1000)[:300].astype(np.int32)
    dev = torch.device("cuda")
    Xb = torch.full((384, IN_PAD), 7.0, device=dev).to(torch.bfloat16)
    Tb = torch.full((384, 5), 7.0, device=dev)
    Mb = torch.full((384, 5), 7.0, device=dev)
    k.gather(torch.tensor(X, device=dev), torch.tensor(T, device=dev), torch.tensor(M, device=dev),
             torch.tensor(idx, device=dev), Xb, Tb, Mb)
    torch.cuda.synchronize()
    want = np.zeros((384, IN_PAD), np.float32)
    want[:300, :44] = torch.tensor(X[idx]).to(torch.bfloat16).float().numpy()
    assert np.array_equal(Xb.float().cpu().numpy(), want)
    wt = np.zeros((384, 5), np.float32)
    wt[:300] = T[idx]
    wm = np.zeros((384, 5), np.float32)
    wm[:300] = M[idx]
    assert np.array_equal(Tb.cpu().numpy(), wt) and np.array_equal(Mb.cpu().numpy(), wm)


def test_captured_training_follows_the_launched_steps():
    """The graph-captured fit (device-resident data, two graphs per step)
    takes the same batches, schedule and updates as the step-by-step path:
    loss histories and weights agree to rounding."""
    import torch
    from dense_b200.surrogate import MLP
    rng = np.random.Generator(np.random.PCG64(9))
    X = rng.uniform(-1, 1, size=(6000, 10)).astype(np.float32)
    T = np.stack([np.sin(2 * X[:, 0]), X[:, 1] * X[:, 2], np.cos(X[:, 3])], 1).astype(np.float32)
    M = np.ones_like(T)
    M[::7, 1] = 0
    a, b = MLP(10, 3, seed=5), MLP(10, 3, seed=5)
    ha = a.fit(X, T, M, epochs=3, batch=1024, seed=2, captured=True)
    hb = b.fit(X, T, M, epochs=3, batch=1024, seed=2, captured=False)
    assert a.steps == b.steps == 15
    assert np.allclose(ha, hb, rtol=2e-3), (ha, hb)
    for wa, wb in zip(a.W + a.b, b.W + b.b):
        d = (wa - wb).norm().item() / max(wb.norm().item(), 1e-12)
        assert d < 1e-3, d


def test_concurrent_ensemble_training_equals_one_by_one():
    """Networks trained at once on separate streams end with the weights of
    the same networks trained one after the other (every kernel of a step
    is deterministic)."""
    from dense_b200.surrogate import MLP, fit_concurrently
    rng = np.random.Generator(np.random.PCG64(10))
    X = rng.uniform(-1, 1, size=(5000, 12)).astype(np.float32)
    T = np.stack([np.sin(X[:, 0]), X[:, 1] * X[:, 2]], 1).astype(np.float32)
    M = np.ones_like(T)
    seq = [MLP(12, 2, seed=s) for s in (1, 2, 3)]
    for net, s in zip(seq, (11, 12, 13)):
        net.fit(X, T, M, epochs=3, batch=1024, seed=s)
    con = [MLP(12, 2, seed=s) for s in (1, 2, 3)]
    hists = fit_concurrently(con, X, T, M, [11, 12, 13], epochs=3, batch=1024)
    assert len(hists) == 3 and all(len(h) == 3 for h in hists)
    for a, b in zip(seq, con):
        for wa, wb in zip(a.W + a.b, b.W + b.b):
            assert (wa == wb).all()


def test_umma_gemm_bias_gelu_epilogue():
    import torch
    from dense_b200.surrogate import EPI_BIAS, EPI_BIAS_GELU, Kernels
    k = Kernels()
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(256, 128, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(96, 128, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(96, device="cuda", generator=g)
    Z = torch.empty(256, 96, device="cuda")
    H = torch.empty(256, 96, device="cuda", dtype=torch.bfloat16)
    k.gemm(A, B, Z, EPI_BIAS_GELU, bias, H)
    Y = torch.empty(256, 96, device="cuda")
    k.gemm(A, B, Y, EPI_BIAS, bias)
    k.check()
    ref = A.float() @ B.float().T + bias
    assert (Z - ref).abs().max().item() < 1e-3
    assert (Y - ref).abs().max().item() < 1e-3
    gelu = torch.nn.functional.gelu(ref)
    assert (H.float() - gelu).abs().max().item() < 2e-2 * max(1.0, gelu.abs().max().item())


def test_mlp_gradients_match_fp64_oracle():
    """One batch through the tensor-core backward pass against the float64
    chain rule on the same (BF16-rounded) weights and inputs; BF16
    activations bound the agreement, 3e-2 relative in norm per tensor."""
    import torch
    from dense_b200.surrogate import IN_PAD, MLP
    from oracle.mlp_oracle import loss_and_grads
    rng = np.random.Generator(np.random.PCG64(7))
    n_in, n_out, B = 44, 4, 256
    net = MLP(n_in, n_out, seed=1)
    X = rng.uniform(-1, 1, size=(B, n_in)).astype(np.float32)
    T = rng.normal(size=(B, n_out)).astype(np.float32)
    mask = (rng.uniform(size=(B, n_out)) > 0.2).astype(np.float32)
    loss, dW, db = net.gradients(X, T, mask)
    Wb = [w.to(torch.bfloat16).float().cpu().numpy() for w in net.W]
    bb = [b.cpu().numpy() for b in net.b]
    Xp = np.zeros((B, IN_PAD), np.float32)
    Xp[:, :n_in] = torch.tensor(X).to(torch.bfloat16).float().numpy()
    rloss, rdW, rdb = loss_and_grads(Wb, bb, Xp, T, mask)
    assert abs(loss - rloss) / rloss < 1e-2
    for i in range(4):
        g = dW[i].cpu().numpy()
        assert np.linalg.norm(g - rdW[i]) / np.linalg.norm(rdW[i]) < 3e-2, i
        h = db[i].cpu().numpy()
        assert np.linalg.norm(h - rdb[i]) / max(np.linalg.norm(rdb[i]), 1e-12) < 3e-2, i


def test_mlp_learns_a_smooth_map():
    """Training on the tensor-core kernels fits a smooth 3-output function
    of 8 inputs (held-out error falls well below the target spread)."""
    from dense_b200.surrogate import MLP
    rng = np.random.Generator(np.random.PCG64(8))
    X = rng.uniform(-1, 1, size=(24576, 8)).astype(np.float32)
    T = np.stack([np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2], np.cos(X[:, 3] + X[:, 4]), X[:, 5] ** 2 - X[:, 6]], 1)
    T = T.astype(np.float32)
    mask = np.ones_like(T)
    net = MLP(8, 3, seed=2, lr=2e-3)
    hist = net.fit(X[:20480], T[:20480], mask[:20480], epochs=12, batch=2048)
    pred = net.predict(X[20480:])
    rmse = np.sqrt(((pred - T[20480:]) ** 2).mean())
    assert hist[-1] < hist[0] * 0.2
    assert rmse < 0.15 * T.std(), (rmse, T.std())


def test_search_pipeline_small():
    """Features from the FP64 engine, surrogate training, screened search and
    SRES on a small her_model_2014 case (50 cells, 200 minutes)."""
    from dense_b200 import search as S
    sim = dict(minutes=200.0, cells=50, width=5)
    P = S.draw_candidates(4096, 5)
    F = S.simulate_features(P, **sim)
    assert np.isfinite(F["period"]).sum() > 50
    assert F["oscillates"].sum() > 50
    syn = F["synchrony"][np.isfinite(F["synchrony"])]
    assert ((syn >= -1.0001) & (syn <= 1.0001)).all()
    net = S.train_surrogate(P, F, epochs=60, batch=512, ensemble=2)
    err = S.feature_errors(net, P, F)
    assert err["period_median"] < 0.5 and err["oscillation_accuracy"] > 0.6
    res = S.screened_search(net, 20000, 6, keep=0.01, plain_sample=2000, sim_kwargs=sim)
    assert res["kept"] == 200 and res["plain_sample"] == 2000
    # what the network gains: the share of the kept candidates that the FP64
    # re-simulation accepts is above the share of random candidates it accepts
    screened_fraction = res["accepted_screened"] / res["kept"]
    assert screened_fraction > 2.0 * res["plain_accept_fraction"], res
    fit = lambda X: S.search_fitness(S.simulate_features(S.decode(X), **sim))  # noqa: E731
    es = S.SRES(len(S.active_params()), fit, mu=4, lam=32, seed=1)
    assert es.evaluations == 32
    assert np.isfinite(es.step())
    assert es.evaluations == 64


def test_synchrony_known_answers():
    from dense_b200.search import synchrony
    t = np.linspace(0, 20, 400)[:, None]
    same = np.sin(t) * np.ones((1, 8))
    assert abs(synchrony(same) - 1.0) < 1e-12
    anti = np.concatenate([np.sin(t), -np.sin(t)], 1)
    assert abs(synchrony(anti) + 1.0) < 1e-12


def test_synchrony_kernel_matches_numpy():
    """The per-set synchrony kernel against search.synchrony on trajectories
    with different sample counts, a constant cell, an all-constant set, a
    set with a NaN sample and a set with no samples, read through a strided
    view [sets][samples][species 1 of 2][cells]."""
    import torch
    from dense_b200 import search as S
    rng = np.random.Generator(np.random.PCG64(12))
    sets, cap, cells = 7, 90, 37
    X = rng.normal(size=(sets, cap, 2, cells))
    t = np.arange(cap)[:, None]
    X[:, :, 1, :] = np.sin(0.2 * t + rng.uniform(0, 0.5, size=(1, cells))) + 0.1 * X[:, :, 1, :]
    X[1, :, 1, 5] = 3.0            # a constant cell
    X[2, :, 1, :] = 1.5            # every cell constant
    X[3, 17, 1, 4] = np.nan        # a NaN sample
    counts = np.array([90, 60, 90, 90, 1, 0, 33], np.int32)
    got = S.synchrony_batch(torch.tensor(X, device="cuda")[:, :, 1, :], counts)
    for i in range(sets):
        want = S.synchrony(X[i, :counts[i], 1, :]) if counts[i] > 0 else float("nan")
        if np.isnan(want):
            assert np.isnan(got[i]), (i, got[i])
        else:
            assert abs(got[i] - want) < 1e-12, (i, got[i], want)


def test_ensemble_scoring_on_the_gpu_matches_the_host():
    """score_candidates with a two-network Surrogate (standardised outputs)
    against predicted_score(Surrogate.predict(encode(P)))."""
    from dense_b200 import search as S
    from dense_b200.surrogate import MLP
    nets = [MLP(len(S.active_params()), 5, seed=s) for s in (3, 4)]
    sur = S.Surrogate(nets, mu=[3.3, 3.9, 0.2, 0.0, 0.0], sd=[0.4, 0.8, 0.3, 1.0, 1.0])
    P = S.draw_candidates(3000, 8)
    host = S.predicted_score(sur.predict(S.encode(P)))
    dev = S.score_candidates(sur, P, chunk=1024, batch=512)
    assert np.max(np.abs(host - dev)) < 1e-4


def test_sharded_screening_single_rank_matches_direct_resimulation():
    """The multi-GPU screening path on one process: the top k of the scored
    candidate range, re-simulated, gives the accepted count a direct
    simulation of the same candidates gives."""
    from dense_b200 import distributed as D
    from dense_b200 import search as S
    from dense_b200.surrogate import MLP
    net = MLP(len(S.active_params()), 5, seed=3)
    sim = dict(minutes=20.0, cells=40, width=4)
    r = S.screened_search_sharded(net, 3000, seed=11, keep=0.01, sim_kwargs=sim)
    assert r["kept"] == 30 and r["ranks"] == 1
    P = D.candidate_range(0, 3000, 11, S._draw_rows)
    score = S.predicted_score(net.predict(S.encode(P)))
    _, top = D.local_top(score, np.arange(3000), 30)
    F = S.simulate_features(D.candidates_at(top, 11, S._draw_rows), **sim)
    assert r["accepted_screened"] == int(S.accepted(F).sum())


def test_synchrony_batch_matches_per_set():
    """The batched GPU synchrony equals the per-set one (random traces, a
    constant cell, sets with fewer samples than the buffer holds)."""
    import torch
    from dense_b200.search import synchrony, synchrony_batch
    rng = np.random.Generator(np.random.PCG64(4))
    X = rng.normal(size=(6, 50, 9))
    X[1, :, 3] = 2.5
    X[2] = np.sin(np.linspace(0, 9, 50))[:, None] * np.ones((1, 9))
    counts = np.array([50, 50, 50, 31, 2, 1])
    got = synchrony_batch(torch.tensor(X, device="cuda"), counts)
    for i in range(6):
        want = synchrony(X[i, :counts[i]])
        if np.isnan(want):
            assert np.isnan(got[i])
        else:
            assert abs(got[i] - want) < 1e-9, (i, got[i], want)


def test_batched_reads_match_per_set_reads():
    """read_oscillation_all and the device trajectory copy give what the
    per-set readers give."""
    from dense_b200 import engine as E
    from dense_b200 import workloads
    from dense_b200.tissue import default_graph
    P = workloads.log_uniform_params(5, seed=13)
    off, ids = default_graph(40, 4)
    sets = [E.ParameterSet(off, ids, P[i], duration=(12.0 if i != 2 else 3.0)) for i in range(5)]
    mh1 = workloads.her_species("mh1")
    an = [E.Analysis.oscillation(mh1, 0, 40, 0.0, 10.0, 2.0, 0.1), E.Analysis.trajectory(mh1, 0, 40, 0.0, 10.0)]
    b = E.Batch("her_model_2014", sets, 0.01, 0.1, an)
    b.run()
    b.sync()
    amps, pers = b.oscillation_all(0)
    traj, cnt = b.trajectory_device(1)
    traj = traj.cpu().numpy()
    for i in range(5):
        o = b.oscillation(0, i)
        assert np.array_equal(amps[i], o["amps"], equal_nan=True)
        assert np.array_equal(pers[i], o["pers"], equal_nan=True)
        _, vals = b.trajectory(1, i)
        assert cnt[i] == vals.shape[0]
        assert np.array_equal(traj[i, :cnt[i]], vals)
    b.close()


def test_device_scoring_matches_host_scoring():
    """score_candidates (encoding, network and score on the GPU) ranks like
    the host path predicted_score(net.predict(encode(P)))."""
    from dense_b200 import search as S
    from dense_b200.surrogate import MLP
    net = MLP(len(S.active_params()), 5, seed=7)
    P = S.draw_candidates(5000, 3)
    host = S.predicted_score(net.predict(S.encode(P)))
    dev = S.score_candidates(net, P, chunk=2048)
    # float32 encodings computed on two devices: equal to rounding
    assert np.max(np.abs(host - dev)) < 1e-4
    top_h, top_d = set(np.argsort(-host)[:50].tolist()), set(np.argsort(-dev)[:50].tolist())
    assert len(top_h & top_d) >= 45
