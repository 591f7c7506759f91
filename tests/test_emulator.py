"""Learned emulator: CPU reference checks, tensor-core kernels vs the CPU reference, training on
solver trajectories, and what the trained network gains over the method without it."""
from __future__ import annotations

import numpy as np
import pytest


def _rand_params(rng, scale=0.1):
    W = [rng.standard_normal((64, 128)) * scale, rng.standard_normal((128, 128)) * scale,
         rng.standard_normal((128, 128)) * scale, rng.standard_normal((128, 64)) * scale]
    W[0][30:, :] = 0
    W[3][:, 1:] = 0
    b = [rng.standard_normal(128) * 0.05, rng.standard_normal(128) * 0.05, rng.standard_normal(128) * 0.05,
         rng.standard_normal(64) * 0.05]
    return W, b


def test_reference_backward_matches_finite_differences():
    from emu_ref import loss_and_grads

    rng = np.random.default_rng(0)
    W, b = _rand_params(rng, 0.3)
    X = rng.standard_normal((16, 64))
    X[:, 30:] = 0
    t = rng.standard_normal(16)
    _, gW, gb = loss_and_grads(X, t, W, b, bf16=False)
    eps = 1e-6
    for li, (r, c) in [(0, (3, 7)), (1, (10, 20)), (2, (5, 100)), (3, (17, 0))]:
        Wp = [w.copy() for w in W]
        Wm = [w.copy() for w in W]
        Wp[li][r, c] += eps
        Wm[li][r, c] -= eps
        num = (loss_and_grads(X, t, Wp, b, False)[0] - loss_and_grads(X, t, Wm, b, False)[0]) / (2 * eps)
        assert abs(num - gW[li][r, c]) < 1e-5 * max(1.0, abs(num)), (li, num, gW[li][r, c])
    bp = [v.copy() for v in b]
    bp[2][9] += eps
    bm = [v.copy() for v in b]
    bm[2][9] -= eps
    num = (loss_and_grads(X, t, W, bp, False)[0] - loss_and_grads(X, t, W, bm, False)[0]) / (2 * eps)
    assert abs(num - gb[2][9]) < 1e-5 * max(1.0, abs(num))


def test_nse_known_answers():
    from cmf_b200.emulator import nse

    obs = np.array([[1.0, 2.0], [2.0, 4.0], [3.0, 9.0], [4.0, 1.0]])
    assert np.allclose(nse(obs, obs), 1.0)
    assert np.allclose(nse(np.repeat(obs.mean(0, keepdims=True), 4, 0), obs), 0.0)
    sim = obs + np.array([[0.1, 0.0]] * 4)
    assert np.isclose(nse(sim, obs)[0], 1.0 - 4 * 0.01 / 5.0)


@pytest.mark.gpu
@pytest.mark.parametrize("ta,tb,ks,M,N,K", [(0, 0, 1, 128, 64, 256), (1, 0, 1, 128, 64, 256), (0, 1, 1, 128, 64, 256),
                                          (1, 0, 4, 128, 64, 256), (0, 0, 1, 384, 128, 96), (1, 0, 3, 64, 128, 1024),
                                          (0, 1, 1, 192, 128, 128), (1, 1, 2, 64, 64, 160)])
def test_gemm_kernel_matches_numpy(ta, tb, ks, M, N, K):
    """The tcgen05 GEMM (products in tensor memory) against float64 numpy and against the legacy
    mma.sync tiles on the same bf16 operands: every transpose combination, split-K accumulation,
    tiles of 64 and 128 columns, 64-row problems (half a tcgen05 tile) and K chunks of 32."""
    import torch

    from cmf_b200.emulator import _emu_lib, echeck
    from emu_ref import to_bf16

    lib = _emu_lib()
    rng = np.random.default_rng(ta * 2 + tb + ks + M + N + K)
    A = to_bf16(rng.standard_normal((K, M) if ta else (M, K)))
    B = to_bf16(rng.standard_normal((N, K) if tb else (K, N)))
    dev = torch.device("cuda", 0)
    tA = torch.tensor(A, device=dev).to(torch.bfloat16)
    tB = torch.tensor(B, device=dev).to(torch.bfloat16)
    bias = torch.tensor(rng.standard_normal(N).astype(np.float32), device=dev)
    acc = 1 if ks > 1 else 0
    out = {}
    for name, fn in (("tc", lib.cmf_emu_gemm), ("mma", lib.cmf_emu_gemm_mma)):
        C = torch.zeros(M, N, device=dev)
        echeck(fn(M, N, K, tA.data_ptr(), A.shape[1], ta, tB.data_ptr(), B.shape[1], tb, C.data_ptr(), N,
                  None, 0, None, 0, acc, ks, None), name)
        out[name] = C
        if not acc:   # epilogue: bias + ReLU into fp32 and bf16
            Cr = torch.zeros(M, N, device=dev)
            Cb = torch.zeros(M, N, dtype=torch.bfloat16, device=dev)
            echeck(fn(M, N, K, tA.data_ptr(), A.shape[1], ta, tB.data_ptr(), B.shape[1], tb, Cr.data_ptr(), N,
                      Cb.data_ptr(), N, bias.data_ptr(), 1, 0, 1, None), name)
            out[name + "_relu"] = (Cr, Cb)
    torch.cuda.synchronize()
    assert lib.cmf_emu_mlp_tc_status() == 0
    ref = (A.T if ta else A).astype(np.float64) @ (B.T if tb else B).astype(np.float64)
    for name in ("tc", "mma"):
        assert np.allclose(out[name].cpu().numpy(), ref, rtol=1e-5, atol=1e-3), name
    assert np.allclose(out["tc"].cpu().numpy(), out["mma"].cpu().numpy(), rtol=1e-5, atol=1e-4)
    if not acc:
        rr = np.maximum(ref + bias.cpu().numpy()[None, :].astype(np.float64), 0.0)
        Cr, Cb = out["tc_relu"]
        assert np.allclose(Cr.cpu().numpy(), rr, rtol=1e-5, atol=1e-3)
        assert np.allclose(Cb.float().cpu().numpy(), to_bf16(Cr.cpu().numpy()))


@pytest.mark.gpu
@pytest.mark.parametrize("ta,tb,ks,M,N,K", [(1, 0, 4, 128, 128, 16384), (1, 0, 3, 64, 64, 1024), (0, 1, 2, 128, 64, 256)])
def test_splitk_gemm_is_deterministic(ta, tb, ks, M, N, K):
    """Split-K on the tensor cores with the slices summed in slice order: C += op(A) op(B) within
    fp32 accumulation tolerance of float64 numpy, and the same bits on every call."""
    import torch

    from cmf_b200.emulator import _emu_lib, echeck
    from emu_ref import to_bf16

    lib = _emu_lib()
    rng = np.random.default_rng(ks + M + N + K)
    A = to_bf16(rng.standard_normal((K, M) if ta else (M, K)))
    B = to_bf16(rng.standard_normal((N, K) if tb else (K, N)))
    C0 = rng.standard_normal((M, N)).astype(np.float32)
    dev = torch.device("cuda", 0)
    tA = torch.tensor(A, device=dev).to(torch.bfloat16)
    tB = torch.tensor(B, device=dev).to(torch.bfloat16)
    need = int(lib.cmf_emu_gemm_splitk_ws_floats(M, N, K, ks))
    assert need >= M * N * min(ks, K // 64)
    ws = torch.empty(need, dtype=torch.float32, device=dev)
    outs = []
    for _ in range(3):
        C = torch.tensor(C0, device=dev)
        echeck(lib.cmf_emu_gemm_splitk(M, N, K, tA.data_ptr(), A.shape[1], ta, tB.data_ptr(), B.shape[1], tb,
                                       C.data_ptr(), N, ks, ws.data_ptr(), need, None), "gemm_splitk")
        outs.append(C.cpu().numpy())
    torch.cuda.synchronize()
    assert lib.cmf_emu_mlp_tc_status() == 0
    ref = C0.astype(np.float64) + (A.T if ta else A).astype(np.float64) @ (B.T if tb else B).astype(np.float64)
    assert np.allclose(outs[0], ref, rtol=1e-5, atol=1e-3 * np.sqrt(K / 256))
    for o in outs[1:]:
        assert np.array_equal(o.view(np.uint32), outs[0].view(np.uint32))
    # a workspace below the required size is refused, not overrun
    assert lib.cmf_emu_gemm_splitk(M, N, K, tA.data_ptr(), A.shape[1], ta, tB.data_ptr(), B.shape[1], tb,
                                   torch.zeros(M, N, device=dev).data_ptr(), N, ks, ws.data_ptr(), need - 1, None) != 0


@pytest.mark.gpu
def test_training_is_deterministic():
    """Two trainings from the same seed on the same rows end with the same weights, bit for bit
    (row sampling is seeded and every reduction, split-K included, runs in a fixed order)."""
    import torch

    from cmf_b200 import emulator as E

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(7)
    Xh = rng.standard_normal((40000, E.NFEAT)).astype(np.float32)
    th = (0.3 * Xh[:, 0] - 0.2 * Xh[:, 5] + 0.1 * Xh[:, 9] * Xh[:, 2]).astype(np.float32)
    X = torch.zeros(Xh.shape[0], E.IN, dtype=torch.bfloat16, device=dev)
    X[:, :E.NFEAT] = torch.tensor(Xh, device=dev).to(torch.bfloat16)
    t = torch.tensor(th, device=dev)
    Ws = []
    for _ in range(2):
        mlp = E.MLP(dev, seed=0, lr=2e-3)
        E.train(mlp, X, t, iters=12, batch=16384, seed=0)
        torch.cuda.synchronize()
        Ws.append([w.detach().cpu().numpy().copy() for w in mlp.W] + [v.detach().cpu().numpy().copy() for v in mlp.b])
    for a, b in zip(*Ws):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.gpu
def test_training_kernels_gradients_match_cpu_reference():
    import torch

    from cmf_b200.emulator import MLP
    from emu_ref import loss_and_grads, to_bf16

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(3)
    mlp = MLP(dev, seed=1)
    W, b = _rand_params(rng, 0.15)
    mlp.load({"W": W, "b": b})
    R = 512
    X = to_bf16(rng.standard_normal((R, 64)))
    X[:, 30:] = 0
    t = rng.standard_normal(R).astype(np.float32)
    loss = mlp.loss_and_grad(torch.tensor(X, device=dev).to(torch.bfloat16), torch.tensor(t, device=dev), R)
    torch.cuda.synchronize()
    # reference with the GPU chain's rounding points (bf16 inputs, weights, activations and dZ) and
    # float64 accumulation: the remaining differences are the fp32 accumulation order of the tensor
    # cores and the rare bf16 roundings such a difference flips
    rloss, gW, gb = loss_and_grads(X, t, [w.astype(np.float32) for w in W], [v.astype(np.float32) for v in b], bf16=True,
                                   acc64=True)
    assert abs(float(loss) - rloss) <= 1e-4 * abs(rloss)
    for li in range(4):
        g = mlp.gW[li].cpu().numpy()
        err = np.linalg.norm(g - gW[li]) / max(np.linalg.norm(gW[li]), 1e-30)
        e2 = np.linalg.norm(mlp.gb[li].cpu().numpy() - gb[li]) / max(np.linalg.norm(gb[li]), 1e-30)
        print(f"layer {li}: relative gradient error W {err:.2e}, b {e2:.2e}")
        assert err < 1e-4, (li, err)
        assert e2 < 1e-4, (li, e2)


@pytest.mark.gpu
@pytest.mark.parametrize("R", [16, 1040, 70000])
def test_fused_inference_equals_layerwise_forward(R):
    """The fused 4-layer kernel (activations in registers) against the layer-by-layer GEMM chain:
    identical bits; and against the CPU bf16 reference within fp32 accumulation-order tolerance."""
    import torch

    from cmf_b200.emulator import MLP
    from emu_ref import forward, to_bf16

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(R)
    mlp = MLP(dev, seed=2)
    W, b = _rand_params(rng, 0.2)
    mlp.load({"W": W, "b": b})
    X = to_bf16(rng.standard_normal((R, 64)) * 2.0)
    X[:, 30:] = 0
    tX = torch.tensor(X, device=dev).to(torch.bfloat16)
    y = mlp.infer(tX)
    Rp = (R + 63) // 64 * 64
    Xp = torch.zeros(Rp, 64, dtype=torch.bfloat16, device=dev)
    Xp[:R] = tX
    Y, _ = mlp.forward(Xp, keep=False)
    torch.cuda.synchronize()
    assert torch.equal(y, Y[:R, 0].contiguous())
    ref, _ = forward(X[:2048], [w.astype(np.float32) for w in W], [v.astype(np.float32) for v in b], bf16=True)
    got = y[:2048].cpu().numpy()
    assert np.allclose(got, ref[:, 0], rtol=2e-2, atol=2e-2 * float(np.abs(ref[:, 0]).max()))


@pytest.mark.gpu
@pytest.mark.parametrize("R", [16, 1040, 70000])
def test_tcgen05_inference_matches_mma_sync_and_reference(R):
    """The tcgen05 (tensor-memory) fused kernel against the mma.sync fused kernel and the CPU bf16
    reference: same rounding points, so differences come only from the fp32 accumulation order
    inside an MMA (and the bf16 roundings that such a difference may flip)."""
    import torch

    from cmf_b200.emulator import MLP, _emu_lib
    from emu_ref import forward, to_bf16

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(R + 1)
    mlp = MLP(dev, seed=2)
    W, b = _rand_params(rng, 0.2)
    mlp.load({"W": W, "b": b})
    X = to_bf16(rng.standard_normal((R, 64)) * 2.0)
    X[:, 30:] = 0
    tX = torch.tensor(X, device=dev).to(torch.bfloat16)
    y_tc = mlp.infer_tc(tX)
    y_ms = mlp.infer(tX)
    torch.cuda.synchronize()
    assert _emu_lib().cmf_emu_mlp_tc_status() == 0
    a, m = y_tc.cpu().numpy(), y_ms.cpu().numpy()
    scale = float(np.abs(m).max())
    assert np.all(np.isfinite(a))
    assert np.abs(a - m).max() <= 2e-2 * scale, np.abs(a - m).max() / scale
    assert np.median(np.abs(a - m)) <= 1e-3 * scale
    ref, _ = forward(X[:2048], [w.astype(np.float32) for w in W], [v.astype(np.float32) for v in b], bf16=True)
    assert np.allclose(a[:2048], ref[:, 0], rtol=2e-2, atol=2e-2 * float(np.abs(ref[:, 0]).max()))


@pytest.mark.gpu
def test_tcgen05_bounded_wait_reports_and_recovers():
    """With the MMA completion bound set to 0 every tcgen05 launch gives up at its first wait: the
    kernel still drains its MMA in flight and frees its tensor memory, returns, and the status
    reports CMF_E_CUDA once (cleared on read).  With the default bound restored the next launch is
    correct again."""
    import torch

    from cmf_b200.emulator import MLP, _emu_lib

    lib = _emu_lib()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(5)
    mlp = MLP(dev, seed=3)
    W, b = _rand_params(rng, 0.2)
    mlp.load({"W": W, "b": b})
    X = torch.tensor(rng.standard_normal((4096, 64)) * 2.0, device=dev).to(torch.bfloat16)
    X[:, 30:] = 0
    ref = mlp.infer(X)
    torch.cuda.synchronize()
    assert lib.cmf_emu_mlp_tc_status() == 0
    try:
        assert lib.cmf_emu_mlp_tc_set_wait_limit(0) == 0
        mlp.infer_tc(X)
        torch.cuda.synchronize()
        assert lib.cmf_emu_mlp_tc_status() == 1          # CMF_E_CUDA: a wait ran out
        assert lib.cmf_emu_mlp_tc_status() == 0          # cleared on read
    finally:
        lib.cmf_emu_mlp_tc_set_wait_limit(-1)
    y = mlp.infer_tc(X)
    torch.cuda.synchronize()
    assert lib.cmf_emu_mlp_tc_status() == 0
    scale = float(ref.abs().max())
    assert float((y - ref).abs().max()) <= 2e-2 * scale


def _raw_i32(ptr, n, dev):
    import torch

    class _CAI:
        def __init__(self):
            self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False), "version": 3}

    return torch.as_tensor(_CAI(), device=dev)


@pytest.mark.gpu
@pytest.mark.parametrize("hops", [1, 2, 5, 8])
def test_message_planes_equal_upstream_sums(case_dirs, hops):
    """E2: hop h of the message passing is the fp32 sum, in the upstream-matrix order, of hop h-1 over
    each cell's upstream cells (hop 0 = last-step outflow and runoff rounded to fp32) -- bit for bit,
    whether the kernels take the hops one or two at a time; unused hop columns of X stay zero."""
    import ctypes as C

    import torch

    from cmf_b200 import HostModel, PhysicsGPU
    from cmf_b200 import emulator as E

    h = HostModel(case_dirs["cfg1s"])
    M, N = 3, h.dims.nseqall
    p = PhysicsGPU(h, nmembers=M)
    gr = h.map("grarea")
    gens = E.runoff_generators(N, M, 3)
    for _ in range(3):
        p.put_runoff(E.runoff_step(gens, gr))
        p.advance()
    fe = E.Features(p, E.qref_from_host(h))
    dev = fe.dev
    planes = torch.full((2 * (hops + 1) * M * N,), float("nan"), dtype=torch.float32, device=dev)
    X = torch.zeros(M * fe.Np, E.IN, dtype=torch.bfloat16, device=dev)
    p.synchronize()
    E.echeck(fe.lib.cmf_emu_features(C.byref(fe.net), C.byref(fe.mb), M, X.data_ptr(), E.IN, fe.Np, hops,
                                     planes.data_ptr(), torch.cuda.current_stream(dev).cuda_stream), "features")
    torch.cuda.synchronize()
    up_ptr = _raw_i32(fe.net.up_ptr, N + 1, dev).cpu().numpy()
    up_idx = _raw_i32(fe.net.up_idx, int(up_ptr[-1]), dev).cpu().numpy()
    rows = np.repeat(np.arange(N), np.diff(up_ptr))
    got = planes.cpu().numpy().reshape(2 * (hops + 1), M, N)
    cur = [fe.qprev().cpu().numpy().astype(np.float32), fe.runoff_view().cpu().numpy().astype(np.float32)]
    assert np.any(cur[0]) and np.any(cur[1])
    for k in range(hops):
        nxt = []
        for v in cur:
            out = np.zeros_like(v)
            for m in range(M):
                np.add.at(out[m], rows, v[m, up_idx])      # in order: ascending cell, then matrix order
            nxt.append(out)
        cur = nxt
        for c in (0, 1):
            assert np.array_equal(got[2 * k + 2 + c].view(np.int32), cur[c].view(np.int32)), (k, c)
    x = X.float().cpu().numpy().reshape(M, fe.Np, E.IN)[:, :N]
    assert not np.any(x[:, :, 14 + 2 * hops:30])
    assert np.all(np.isfinite(x[:, :, :32]))
    p.close()


@pytest.mark.gpu
def test_trained_emulator_beats_untrained_and_persistence(case_dirs):
    """E1-E5 on the config-1 laws: train on solver trajectories, then roll out 24 h from a plain
    state and compare the gauge discharge with the plain solver: the trained network must be far
    closer than the untrained one and than persistence (last-step outflow held for the day)."""
    import torch

    from cmf_b200 import HostModel, PhysicsGPU
    from cmf_b200 import emulator as E

    h = HostModel(case_dirs["cfg1s"])
    dev = torch.device("cuda", 0)
    X, t = E.generate_trajectories(h, members=6, hours=72, spinup=12, seed=10)
    mlp = E.MLP(dev, seed=0, lr=2e-3)
    hist = E.train(mlp, X, t, iters=3000, batch=4096, seed=0)
    print("training loss", hist[0], hist[-1])
    assert hist[-1][1] < 0.5 * hist[0][1]
    # evaluation: 24 h rollout from a spun-up plain state with unseen forcing
    M = 2
    gr = h.map("grarea")
    gens = E.runoff_generators(h.dims.nseqall, M, 999)
    plain = PhysicsGPU(h, nmembers=M)
    for _ in range(24):
        plain.put_runoff(E.runoff_step(gens, gr))
        plain.advance()
    qref = E.qref_from_host(h)
    gauges = np.argsort(-qref)[:20]
    runs = {}
    for name, net in (("trained", mlp), ("untrained", E.MLP(dev, seed=5))):
        ens = E.SurrogateEnsemble(h, net, members=M, judge_slots=1, gauges=gauges, resync_hours=10 ** 6)
        ens.set_state_from(plain)
        runs[name] = ens
    q0 = runs["trained"].fe.qprev().cpu().numpy()[:, gauges]
    truth = []
    est = {k: [] for k in runs}
    for hh in range(24):
        r = E.runoff_step(gens, gr)
        plain.put_runoff(r)
        plain.advance()
        truth.append(plain.get_diag_fields({"outflw_aavg": np.zeros(M * h.dims.nseqall)})["outflw_aavg"].reshape(M, -1)[:, gauges])
        for k, ens in runs.items():
            ens.emu.put_runoff(r)
            ens.emu_step()
            ens.emu.stage()
            est[k].append(ens.fe.qprev().cpu().numpy()[:, gauges])
    truth = np.stack(truth)
    err = {k: float(np.mean(np.abs(np.stack(v) - truth) / np.maximum(np.abs(truth), 1e-3))) for k, v in est.items()}
    err["persistence"] = float(np.mean(np.abs(q0[None] - truth) / np.maximum(np.abs(truth), 1e-3)))
    print("mean relative gauge-discharge error over 24 h:", err)
    assert err["trained"] < 0.5 * err["untrained"]
    assert err["trained"] < err["persistence"]


@pytest.mark.gpu
def test_surrogate_controller_judges_resyncs_and_hands_back(case_dirs):
    """Controller mechanics: a rotating subset is judged every 24 h and re-synced to the plain state;
    with a tolerance nobody can meet, every judged member is handed back to the plain solver and from
    then on reports the plain solver's discharge."""
    import torch

    from cmf_b200 import HostModel, PhysicsGPU
    from cmf_b200 import emulator as E

    h = HostModel(case_dirs["cfg0"])
    dev = torch.device("cuda", 0)
    M = 4
    gr = h.map("grarea")
    gens = E.runoff_generators(h.dims.nseqall, M, 5)
    plain = PhysicsGPU(h, nmembers=M)
    for _ in range(6):
        plain.put_runoff(E.runoff_step(gens, gr))
        plain.advance()
    runoff = np.stack([E.runoff_step(gens, gr) for _ in range(48)])
    G = np.argsort(-E.qref_from_host(h))[:10]
    ens = E.SurrogateEnsemble(h, E.MLP(dev, seed=3), members=M, judge_slots=2, gauges=G, tol_rel=-1.0)
    ens.set_state_from(plain)
    out = ens.run(E.ArrayForcing(runoff, dev), runoff.shape[0])
    # day 1 judges members 0 and 1, both fail and are handed back; on day 2 they fill both judge slots
    assert ens.stats["judged"] == 2 and ens.stats["fallback"] == 2 and sorted(ens.plain) == [0, 1]
    # members handed back after day 1 report the plain solver: compare with the truth on day 2
    truth = []
    for hh in range(48):
        plain.put_runoff(runoff[hh])
        plain.advance()
        truth.append(plain.get_diag_fields({"outflw_aavg": np.zeros(M * h.dims.nseqall)})["outflw_aavg"].reshape(M, -1)[:, G])
    truth = np.stack(truth)
    for m in sorted(ens.plain)[:2]:
        assert np.allclose(out[24:, m], truth[24:, m], rtol=1e-9, atol=1e-9)


def test_snapshot_cells_uniform_and_weighted():
    """Uniform snapshots are the plain draw without replacement (same generator calls as before the
    helper); weighted snapshots are distinct, of the requested size, include the heavy cells, never
    pick weight-0 cells while enough others remain, and follow the weights in frequency."""
    from cmf_b200.emulator import snapshot_cells

    N, k = 5000, 300
    a = snapshot_cells(np.random.default_rng(3), N, k)
    b = np.random.default_rng(3).choice(N, size=k, replace=False)
    assert np.array_equal(a, b)
    assert snapshot_cells(np.random.default_rng(0), 10, 50).size == 10
    w = np.ones(N)
    w[:20] = 1e6                        # 20 very heavy cells
    w[100:200] = 0.0                    # never needed
    hits = np.zeros(N)
    rng = np.random.default_rng(1)
    for _ in range(200):
        idx = snapshot_cells(rng, N, k, w)
        assert idx.size == k and np.unique(idx).size == k
        assert not np.any((idx >= 100) & (idx < 200))
        assert np.all(np.isin(np.arange(20), idx))
        hits[idx] += 1
    light = hits[np.r_[20:100, 200:N]] / 200.0
    assert abs(light.mean() - (k - 20) / (N - 120)) < 0.005
