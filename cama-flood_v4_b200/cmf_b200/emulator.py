"""Learned per-cell emulator of the coupling step (no counterpart in the reference).

E1  trajectories: the GPU solver advances ensemble members; before each coupling step the features
    of every cell are taken from the state, after it the target is the cell's mean outflow over the
    step (D2OUTFLW_aAVG of the physics).
E2  graph messages: 8 hops of upstream sums (CSR gather along I1NEXT) of the last-step outflow and
    of the runoff, normalised by the receiving cell's discharge scale.
E3  MLP 64 (32 used) -> 128 -> 128 -> 128 -> 1 with ReLU, BF16 weights and activations, FP32
    accumulation on the tensor cores, FP32 master weights and Adam -- kernels in csrc/cmf_emu.cu
    (training on mma.sync tiles; inference fused on tcgen05 with tensor-memory accumulators).
E4  rollout: predicted outflows update storage through the same upstream gather (mass conserved
    exactly), the stage scheme recomputes depths.  Every `resync_hours` the plain solver, started
    from the same state, judges a rotating subset of members: their daily-mean discharge error at
    the gauges is measured, they are re-synced to the plain state, and a member whose error is
    above the tolerance is handed back to the plain solver for good.
E5  daily-discharge Nash-Sutcliffe efficiency, 1 - sum((s-o)^2) / sum((o - mean(o))^2)
    (the NS formula of etc/validation/src/discharge_validation.py:39-53).
Torch only allocates device buffers and holds pointers; the arithmetic runs in the library's kernels.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi
from ._abi import check

IN, HID, OUT = 64, 128, 64      # padded widths (32 input features, 1 output)
NFEAT, HOPS = 32, 8


class EmuNet(C.Structure):
    _fields_ = [("nseqall", C.c_int32), ("nseqriv", C.c_int32)] + [(n, C.c_void_p) for n in (
        "next", "up_ptr", "up_idx", "rivelv", "elevtn", "nxtdst", "rivwth", "rivhgt", "rivlen", "rivstomax", "qref",
        "rivman")] + [("pmanfld", C.c_double)]


class EmuMember(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("rivsto", "fldsto", "levsto", "rivdph", "flddph", "fldfrc", "qprev", "runoff",
                                          "rivout_pre", "fldout_pre")]


def _emu_lib():
    lib = _abi.load()
    if not getattr(lib, "_emu_ready", False):
        vp, i, f, d = C.c_void_p, C.c_int, C.c_float, C.c_double
        lib.cmf_emu_gemm.argtypes = [i, i, i, vp, i, i, vp, i, i, vp, i, vp, i, vp, i, i, i, vp]
        lib.cmf_emu_gemm_mma.argtypes = [i, i, i, vp, i, i, vp, i, i, vp, i, vp, i, vp, i, i, i, vp]
        lib.cmf_emu_gemm_splitk_ws_floats.restype = C.c_size_t
        lib.cmf_emu_gemm_splitk_ws_floats.argtypes = [i, i, i, i]
        lib.cmf_emu_gemm_splitk.argtypes = [i, i, i, vp, i, i, vp, i, i, vp, i, i, vp, C.c_size_t, vp]
        lib.cmf_emu_relu_bwd.argtypes = [i, vp, vp, vp, vp, vp]
        lib.cmf_emu_colsum.argtypes = [i, i, vp, vp, vp]
        lib.cmf_emu_mse_grad.argtypes = [i, i, i, vp, vp, vp, vp, vp, vp]
        lib.cmf_emu_adam.argtypes = [i, vp, vp, vp, vp, vp, f, f, f, f, i, f, vp]
        lib.cmf_emu_features.argtypes = [C.POINTER(EmuNet), C.POINTER(EmuMember), i, vp, i, i, i, vp, vp]
        lib.cmf_emu_rollout.argtypes = [C.POINTER(EmuNet), C.POINTER(EmuMember), i, vp, vp, i, i, d, i, vp, vp]
        lib.cmf_emu_mlp_pack_bytes.restype = C.c_size_t
        lib.cmf_emu_mlp_pack.argtypes = [vp, vp, vp, vp, i, vp, vp]
        lib.cmf_emu_mlp_fused.argtypes = [vp, i, i, vp, vp, vp, vp, vp, vp, vp]
        lib.cmf_emu_mlp_tc_pack_bytes.restype = C.c_size_t
        lib.cmf_emu_mlp_tc_pack.argtypes = [vp, vp, vp, vp, i, vp, vp]
        lib.cmf_emu_mlp_tc.argtypes = [vp, i, i, vp, vp, vp, vp, vp, vp, vp]
        lib.cmf_emu_mlp_tc_set_wait_limit.argtypes = [C.c_int32]
        lib.cmf_emu_last_error.restype = C.c_char_p
        lib.cmf_gpu_ctx_emu_views.argtypes = [vp, C.c_int32, C.POINTER(EmuNet), C.POINTER(EmuMember)]
        lib.cmf_gpu_ctx_copy_member.argtypes = [vp, C.c_int32, vp, C.c_int32]
        lib._emu_ready = True
    return lib


def echeck(rc, what):
    if rc != 0:
        lib = _emu_lib()
        raise RuntimeError(f"{what}: status {rc}: {lib.cmf_emu_last_error().decode()} {lib.cmf_gpu_last_error().decode()}")


def qref_from_host(host) -> np.ndarray:
    """Discharge scale per cell: upstream area x 2 mm/day (m3/s), accumulated along I1NEXT."""
    gr = host.map("grarea")
    nxt = host.map("i1next")
    up = gr.copy()
    for i in range(host.dims.nseqriv):
        up[nxt[i] - 1] += up[i]
    return np.maximum(up * 2.0e-3 / 86400.0, 1e-3)


def pad64(n: int) -> int:
    return (n + 63) // 64 * 64


def nse(sim: np.ndarray, obs: np.ndarray) -> np.ndarray:
    """Nash-Sutcliffe efficiency along axis 0 (time) for every column."""
    o = obs - obs.mean(axis=0, keepdims=True)
    den = np.sum(o * o, axis=0)
    num = np.sum((sim - obs) ** 2, axis=0)
    return 1.0 - num / np.maximum(den, 1e-300)


def _raw_f64(ptr: int, n: int, dev):
    """float64 device tensor aliasing library memory (valid while the context lives)."""
    import torch

    class _CAI:
        def __init__(self, p, size):
            self.__cuda_array_interface__ = {"shape": (size,), "typestr": "<f8", "data": (p, False), "version": 3}

    return torch.as_tensor(_CAI(ptr, n), device=dev)


class MLP:
    """Parameters and the forward/backward/Adam chain on the GPU."""

    def __init__(self, device, seed: int = 0, lr: float = 1e-3):
        import torch

        self.torch = torch
        self.dev = device
        self.lib = _emu_lib()
        g = torch.Generator().manual_seed(seed)
        shapes = [(IN, HID), (HID, HID), (HID, HID), (HID, OUT)]
        self.W, self.Wb, self.b, self.mW, self.vW, self.mb, self.vb, self.gW, self.gb = ([] for _ in range(9))
        for li, (k, n) in enumerate(shapes):
            w = torch.randn(k, n, generator=g) * math.sqrt(2.0 / (NFEAT if li == 0 else k))
            if li == 0:
                w[NFEAT:, :] = 0.0          # padded input columns
            if li == 3:
                w[:, 1:] = 0.0              # only output column 0 is real
                w *= 0.1
            w = w.to(device)
            self.W.append(w)
            self.Wb.append(w.to(torch.bfloat16))
            self.b.append(torch.zeros(n, device=device))
            for lst in (self.mW, self.vW, self.gW):
                lst.append(torch.zeros_like(w))
            for lst in (self.mb, self.vb, self.gb):
                lst.append(torch.zeros(n, device=device))
        self.step = 0
        self.lr = lr
        self.stream = torch.cuda.current_stream(device).cuda_stream

    def state_dict(self):
        return {"W": [w.cpu().numpy() for w in self.W], "b": [b.cpu().numpy() for b in self.b]}

    def load(self, sd):
        for k in range(4):
            self.W[k].copy_(self.torch.from_numpy(np.asarray(sd["W"][k], dtype=np.float32)))
            self.Wb[k].copy_(self.W[k].to(self.torch.bfloat16))
            self.b[k].copy_(self.torch.from_numpy(np.asarray(sd["b"][k], dtype=np.float32)))
        self._packed_step = None
        self._tc_step = None

    def _gemm(self, M, N, K, A, lda, ta, B, ldb, tb, C=None, Cb=None, bias=None, relu=0, acc=0, ksplit=1):
        p = lambda t: (t.data_ptr() if t is not None else None)  # noqa: E731
        echeck(self.lib.cmf_emu_gemm(M, N, K, p(A), lda, ta, p(B), ldb, tb, p(C), N if C is not None else 0, p(Cb),
                                     N if Cb is not None else 0, p(bias), relu, acc, ksplit, self.stream), "gemm")

    def forward(self, X, keep: bool = True):
        """X: [R, 64] bf16 (R % 64 == 0) -> (Y fp32 [R, 64], activations for the backward pass)."""
        torch = self.torch
        R = X.shape[0]
        acts = [X]
        a = X
        for li in range(3):
            out = torch.empty(R, HID, dtype=torch.bfloat16, device=self.dev)
            self._gemm(R, HID, a.shape[1], a, a.shape[1], 0, self.Wb[li], HID, 0, Cb=out, bias=self.b[li], relu=1)
            acts.append(out)
            a = out
        Y = torch.empty(R, OUT, dtype=torch.float32, device=self.dev)
        self._gemm(R, OUT, HID, a, HID, 0, self.Wb[3], OUT, 0, C=Y, bias=self.b[3])
        return Y, (acts if keep else None)

    def infer(self, X, y=None):
        """Fused inference: X [R, 64] bf16 (R % 16 == 0) -> y [R] fp32, equal to forward()'s column 0."""
        torch = self.torch
        if getattr(self, "_packed_step", None) != self.step or getattr(self, "_pack", None) is None:
            if getattr(self, "_pack", None) is None:
                self._pack = torch.empty(self.lib.cmf_emu_mlp_pack_bytes(), dtype=torch.uint8, device=self.dev)
            echeck(self.lib.cmf_emu_mlp_pack(self.Wb[0].data_ptr(), self.Wb[1].data_ptr(), self.Wb[2].data_ptr(),
                                             self.Wb[3].data_ptr(), OUT, self._pack.data_ptr(), self.stream), "mlp_pack")
            self._packed_step = self.step
        R = X.shape[0]
        if y is None:
            y = torch.empty(R, dtype=torch.float32, device=self.dev)
        echeck(self.lib.cmf_emu_mlp_fused(X.data_ptr(), X.shape[1], R, self._pack.data_ptr(), self.b[0].data_ptr(),
                                          self.b[1].data_ptr(), self.b[2].data_ptr(), self.b[3].data_ptr(), y.data_ptr(),
                                          self.stream), "mlp_fused")
        return y

    def infer_tc(self, X, y=None):
        """Fused inference on the tcgen05 tensor cores: X [R, 64] bf16 -> y [R] fp32."""
        torch = self.torch
        if getattr(self, "_tc_step", None) != self.step or getattr(self, "_tc_pack", None) is None:
            if getattr(self, "_tc_pack", None) is None:
                self._tc_pack = torch.empty(self.lib.cmf_emu_mlp_tc_pack_bytes(), dtype=torch.uint8, device=self.dev)
            echeck(self.lib.cmf_emu_mlp_tc_pack(self.Wb[0].data_ptr(), self.Wb[1].data_ptr(), self.Wb[2].data_ptr(),
                                                self.Wb[3].data_ptr(), OUT, self._tc_pack.data_ptr(), self.stream),
                   "mlp_tc_pack")
            self._tc_step = self.step
        R = X.shape[0]
        if y is None:
            y = torch.empty(R, dtype=torch.float32, device=self.dev)
        echeck(self.lib.cmf_emu_mlp_tc(X.data_ptr(), X.shape[1], R, self._tc_pack.data_ptr(), self.b[0].data_ptr(),
                                       self.b[1].data_ptr(), self.b[2].data_ptr(), self.b[3].data_ptr(), y.data_ptr(),
                                       self.stream), "mlp_tc")
        return y

    def backward(self, acts, dY, dYb):
        """Parameter gradients into gW/gb from dY = dLoss/dY ([R, 64], fp32 and bf16)."""
        torch = self.torch
        R = dY.shape[0]
        ks = max(1, R // 4096)
        for g in self.gW:
            g.zero_()
        dZf, dZb = dY, dYb
        for li in (3, 2, 1, 0):
            a = acts[li]
            K_in = a.shape[1]
            n_out = self.W[li].shape[1]
            # a^T dZ, split over the rows with the slices summed in a fixed order (deterministic)
            need = int(self.lib.cmf_emu_gemm_splitk_ws_floats(K_in, n_out, R, ks))
            if getattr(self, "_ws", None) is None or self._ws.numel() < need:
                self._ws = torch.empty(need, dtype=torch.float32, device=self.dev)
            echeck(self.lib.cmf_emu_gemm_splitk(K_in, n_out, R, a.data_ptr(), K_in, 1, dZb.data_ptr(), n_out, 0,
                                                self.gW[li].data_ptr(), n_out, ks, self._ws.data_ptr(),
                                                self._ws.numel(), self.stream), "gemm_splitk")
            echeck(self.lib.cmf_emu_colsum(R, n_out, dZf.data_ptr(), self.gb[li].data_ptr(), self.stream), "colsum")
            if li == 0:
                break
            dA = torch.empty(R, K_in, dtype=torch.float32, device=self.dev)
            self._gemm(R, K_in, n_out, dZb, n_out, 0, self.Wb[li], n_out, 1, C=dA)                        # dZ W^T
            nz = torch.empty(R, K_in, dtype=torch.bfloat16, device=self.dev)
            nzf = torch.empty(R, K_in, dtype=torch.float32, device=self.dev)
            echeck(self.lib.cmf_emu_relu_bwd(R * K_in, dA.data_ptr(), a.data_ptr(), nz.data_ptr(), nzf.data_ptr(),
                                             self.stream), "relu_bwd")
            dZf, dZb = nzf, nz

    def adam(self, wd: float = 0.0):
        self.step += 1
        for k in range(4):
            echeck(self.lib.cmf_emu_adam(self.W[k].numel(), self.W[k].data_ptr(), self.Wb[k].data_ptr(), self.gW[k].data_ptr(),
                                         self.mW[k].data_ptr(), self.vW[k].data_ptr(), self.lr, 0.9, 0.999, 1e-8, self.step,
                                         wd, self.stream), "adam")
            echeck(self.lib.cmf_emu_adam(self.b[k].numel(), self.b[k].data_ptr(), None, self.gb[k].data_ptr(),
                                         self.mb[k].data_ptr(), self.vb[k].data_ptr(), self.lr, 0.9, 0.999, 1e-8, self.step,
                                         0.0, self.stream), "adam")

    def loss_and_grad(self, X, t, valid: int):
        torch = self.torch
        Y, acts = self.forward(X)
        R = X.shape[0]
        dY = torch.empty(R, OUT, dtype=torch.float32, device=self.dev)
        dYb = torch.empty(R, OUT, dtype=torch.bfloat16, device=self.dev)
        parts = torch.empty((R + 255) // 256, dtype=torch.float32, device=self.dev)
        echeck(self.lib.cmf_emu_mse_grad(R, valid, OUT, Y.data_ptr(), t.data_ptr(), dY.data_ptr(), dYb.data_ptr(),
                                         parts.data_ptr(), self.stream), "mse_grad")
        self.backward(acts, dY, dYb)
        return parts.sum() / valid


class Features:
    """E1/E2 for every member of a PhysicsGPU context: X [M * Np, 64] bf16 (member m at rows m*Np)."""

    def __init__(self, phys, qref: np.ndarray):
        import torch

        self.torch = torch
        self.phys = phys
        self.lib = _emu_lib()
        self.dev = torch.device("cuda", phys.opts.device)
        self.M, self.N = phys.M, phys.N
        self.Np = pad64(self.N)
        self.qref = torch.tensor(qref, dtype=torch.float64, device=self.dev)
        self.net = EmuNet()
        check(self.lib.cmf_gpu_ctx_emu_views(phys.h, 0, C.byref(self.net), None), "emu_views")
        self.net.qref = self.qref.data_ptr()
        self.mb = EmuMember()
        check(self.lib.cmf_gpu_ctx_emu_views(phys.h, 0, None, C.byref(self.mb)), "emu_views")
        self.scratch = self.X = self.qout = None     # allocated on first use (views-only users need none)

    # The library works on its own non-blocking stream, the emulator on torch's current stream:
    # every boundary drains the side that wrote last, so neither reads the other's arrays mid-update.
    def build(self):
        torch = self.torch
        if self.X is None:
            self.scratch = torch.empty(2 * (HOPS + 1) * self.M * self.N, dtype=torch.float32, device=self.dev)
            self.X = torch.zeros(self.M * self.Np, IN, dtype=torch.bfloat16, device=self.dev)
        self.phys.synchronize()
        echeck(self.lib.cmf_emu_features(C.byref(self.net), C.byref(self.mb), self.M, self.X.data_ptr(), IN, self.Np, HOPS,
                                         self.scratch.data_ptr(), self.torch.cuda.current_stream(self.dev).cuda_stream),
               "features")
        return self.X

    def qprev(self):
        """[M, N] copy of the last-step mean outflow."""
        self.phys.synchronize()
        out = _raw_f64(self.mb.qprev, self.M * self.N, self.dev).clone().view(self.M, self.N)
        self.torch.cuda.current_stream(self.dev).synchronize()
        return out

    def at(self, cells):
        """[M, len(cells)] last-step mean outflow at the given cells (device gather, host array)."""
        self.phys.synchronize()
        v = _raw_f64(self.mb.qprev, self.M * self.N, self.dev).view(self.M, self.N)
        return v.index_select(1, cells).cpu().numpy()

    def runoff_view(self):
        """[M, N] device view of the context's runoff input (written by the caller before a step)."""
        return _raw_f64(self.mb.runoff, self.M * self.N, self.dev).view(self.M, self.N)

    def rollout(self, Y, active, ldy: int = OUT, residual: bool = True):
        if self.qout is None:
            self.qout = self.torch.empty(self.M * self.N, dtype=self.torch.float64, device=self.dev)
        echeck(self.lib.cmf_emu_rollout(C.byref(self.net), C.byref(self.mb), self.M, active.data_ptr(), Y.data_ptr(), ldy,
                                        self.Np, float(self.phys.host.dt), int(residual), self.qout.data_ptr(),
                                        self.torch.cuda.current_stream(self.dev).cuda_stream), "rollout")
        self.torch.cuda.current_stream(self.dev).synchronize()


def target_transform(torch, q, qref):
    return torch.log1p(torch.clamp(q, min=0.0) / qref)


def residual_target(torch, q_new, q_prev, qref):
    """Training target: change of log1p(Q/qref) over the step (the rollout adds it back)."""
    return target_transform(torch, q_new, qref) - target_transform(torch, q_prev, qref)


def runoff_generators(N: int, members: int, seed: int):
    from . import synth

    return [synth.AR1GammaRunoff(N, seed + 7919 * m) for m in range(members)]


def runoff_step(gens, gr, scale: float = 1.0) -> np.ndarray:
    return np.stack([np.maximum((g.next().astype(np.float64) * scale * gr) / 86400000.0, 0.0) for g in gens])


def snapshot_cells(rng: np.random.Generator, N: int, k: int, weights: np.ndarray | None = None) -> np.ndarray:
    """min(k, N) distinct cells of N: uniformly (one `rng.choice` without replacement), or, with
    `weights`, a weighted draw without replacement by Efraimidis-Spirakis keys (the k largest
    log(u)/w; cells of weight 0 only when fewer than k cells weigh more)."""
    k = min(k, N)
    if weights is None:
        return rng.choice(N, size=k, replace=False)
    w = np.asarray(weights, dtype=np.float64)
    with np.errstate(divide="ignore"):
        keys = np.log(rng.random(N)) / w
    return np.argpartition(-keys, k - 1)[:k]


def generate_trajectories(host, members: int, hours: int, spinup: int, seed: int, cells_per_snapshot: int | None = None,
                          residual: bool = True, cell_weights: np.ndarray | None = None,
                          device_forcing: int | None = None):
    """E1: the plain GPU solver advances `members` members (different runoff seeds); returns feature
    rows X [S, 64] (bf16) and targets t [S] (fp32).  With `cells_per_snapshot`, each (hour, member)
    snapshot keeps that many cells, drawn uniformly or in proportion to `cell_weights` [N].
    Forcing: an independent host-generated AR(1)-gamma field per member (default), or, with
    `device_forcing` = K, a `DeviceForcing` of K distinct fields built in HBM straight into the
    context's runoff input (for large domains, where host generation dominates)."""
    import torch

    from .model import PhysicsGPU

    phys = PhysicsGPU(host, nmembers=members)
    N = phys.N
    gr = host.map("grarea")
    if device_forcing:
        fe = Features(phys, qref_from_host(host))
        fo = DeviceForcing(host, members, spinup + hours, seed, fe.dev, distinct=device_forcing)
        runv = fe.runoff_view()

        def put(h):
            fo.fill(h, runv)
            torch.cuda.current_stream(fe.dev).synchronize()

        def advance():
            phys.advance_device(1, None, 0)            # runoff already in the context's input array
            phys.synchronize()
    else:
        gens = runoff_generators(N, members, seed)

        def put(h):
            phys.put_runoff(runoff_step(gens, gr))

        def advance():
            phys.advance()
    for h in range(spinup):
        put(h)
        advance()
    if not device_forcing:
        fe = Features(phys, qref_from_host(host))
    rng = np.random.default_rng(seed)
    Xs, ts = [], []
    for h in range(hours):
        put(spinup + h)
        X = fe.build().clone()                        # state at the start of the step + its runoff
        q0 = fe.qprev()
        torch.cuda.current_stream(fe.dev).synchronize()
        advance()
        q1 = fe.qprev()                                                          # mean outflow over the step
        t = (residual_target(torch, q1, q0, fe.qref[None, :]) if residual else target_transform(torch, q1, fe.qref[None, :])).float()
        for m in range(members):
            idx = np.arange(N) if cells_per_snapshot is None else snapshot_cells(rng, N, cells_per_snapshot, cell_weights)
            it = torch.as_tensor(idx, device=fe.dev)
            Xs.append(X[m * fe.Np + it])
            ts.append(t[m][it])
    phys.close()
    return torch.cat(Xs), torch.cat(ts)


def dagger_trajectories(host, mlp: "MLP", members: int, hours: int, spinup: int, seed: int,
                        cells_per_snapshot: int | None = None):
    """Rows from the emulator's own rollout (states it actually visits), labelled by the plain
    solver: every hour each member's emulated state is copied into a plain context, the plain
    solver advances it one step and its mean outflow is the target; the emulator then advances
    itself.  Corrects the drift a network trained on solver states only accumulates."""
    import torch

    from .model import PhysicsGPU

    residual = getattr(mlp, "residual", True)
    ens = SurrogateEnsemble(host, mlp, members=members, judge_slots=1, gauges=np.zeros(1, dtype=np.int64),
                            resync_hours=10 ** 9)
    teach = PhysicsGPU(host, nmembers=members)
    tf = Features(teach, qref_from_host(host))
    N = teach.N
    fo = DeviceForcing(host, members, spinup + hours, seed, tf.dev)
    st = torch.cuda.current_stream(tf.dev)
    for h in range(spinup):
        r = fo.hour(h)
        st.synchronize()
        teach.advance_device(1, r.data_ptr(), 0)
    teach.synchronize()
    ens.set_state_from(teach)
    rng = np.random.default_rng(seed)
    Xs, ts = [], []
    fe = ens.fe
    for h in range(hours):
        for m in range(members):
            check(ens.lib.cmf_gpu_ctx_copy_member(teach.h, m, ens.emu.h, m), "copy_member")
        r = fo.hour(spinup + h)
        fe.runoff_view().copy_(r)
        X = fe.build().clone()
        q0 = fe.qprev()
        st.synchronize()
        teach.advance_device(1, r.data_ptr(), 0)
        q1 = tf.qprev()
        t = (residual_target(torch, q1, q0, fe.qref[None, :]) if residual else target_transform(torch, q1, fe.qref[None, :])).float()
        for m in range(members):
            idx = np.arange(N) if cells_per_snapshot is None else rng.choice(N, size=min(cells_per_snapshot, N), replace=False)
            it = torch.as_tensor(idx, device=fe.dev)
            Xs.append(X[m * fe.Np + it])
            ts.append(t[m][it])
        ens.emu_step()
        ens.emu.stage()
    teach.close()
    ens.emu.close()
    ens.judge.close()
    return torch.cat(Xs), torch.cat(ts)


def discharge_weights(X):
    """Row weights sqrt(qref): feature column 11 holds log(qref) - 3 (bf16)."""
    import torch

    return torch.exp(0.5 * (X[:, 11].float() + 3.0))


def train(mlp: MLP, X, t, iters: int, batch: int, seed: int = 0, lr_max: float | None = None, weights=None,
          noise: float = 0.0):
    """Adam with cosine-decayed learning rate on random mini-batches of the trajectory rows (drawn
    uniformly, or with probability proportional to `weights`); `noise` > 0 adds Gaussian noise of
    that standard deviation to the used feature columns of every batch (robustness to the
    emulator's own drift during rollouts)."""
    import torch

    g = torch.Generator(device=X.device).manual_seed(seed)
    S = X.shape[0]
    hist = []
    lr0 = lr_max if lr_max is not None else mlp.lr
    cdf = None
    if weights is not None:                   # inverse-CDF draws (any number of rows)
        cdf = torch.cumsum(weights.double(), 0)
    for it in range(iters):
        mlp.lr = lr0 * (0.05 + 0.95 * 0.5 * (1.0 + math.cos(math.pi * it / max(iters, 1))))
        if weights is None:
            idx = torch.randint(0, S, (batch,), device=X.device, generator=g)
        else:
            u = torch.rand(batch, device=X.device, dtype=torch.float64, generator=g) * cdf[-1]
            idx = torch.clamp(torch.searchsorted(cdf, u), max=S - 1)
        xb = X[idx].contiguous()
        if noise > 0.0:
            xb[:, :NFEAT] = (xb[:, :NFEAT].float() + noise * torch.randn(batch, NFEAT, device=X.device, generator=g)
                             ).to(torch.bfloat16)
        loss = mlp.loss_and_grad(xb, t[idx].contiguous(), batch)
        mlp.adam()
        if it % 50 == 0 or it == iters - 1:
            hist.append((it, float(loss)))
    return hist


class DeviceForcing:
    """Hourly runoff of an M-member ensemble held in HBM.  `distinct` AR(1)-gamma fields per hour
    (the config-1 forcing law, generated once on the host) are uploaded; member m uses field
    m % distinct times its own lognormal(0, 0.3) factor, so members differ in timing and volume."""

    def __init__(self, host, members: int, hours: int, seed: int, device, distinct: int = 8):
        import torch

        N = host.dims.nseqall
        gr = host.map("grarea")
        K = min(distinct, members)
        gens = runoff_generators(N, K, seed)
        self.fields = torch.empty(hours, K, N, dtype=torch.float64, device=device)
        for h in range(hours):
            self.fields[h].copy_(torch.from_numpy(runoff_step(gens, gr)))
        rng = np.random.default_rng(seed + 1)
        self.factor = torch.tensor(np.exp(0.3 * rng.standard_normal(members) - 0.045), device=device)[:, None]
        self.idx = torch.arange(members, device=device) % K
        self.buf = torch.empty(members, N, dtype=torch.float64, device=device)
        self.torch = torch

    def fill(self, h: int, out) -> None:
        """Runoff of hour h into `out` ([M, N] device tensor, e.g. a context's runoff view) in one
        pass: members m = j*K + k take field k, so the product broadcasts over j.  `out` may hold
        the first M members of the ensemble only (M <= members)."""
        M, N = out.shape
        K = self.fields.shape[1]
        if M == self.factor.shape[0] and M % K == 0:
            self.torch.mul(self.fields[h].unsqueeze(0), self.factor.view(M // K, K, 1), out=out.view(M // K, K, N))
        else:
            self.torch.mul(self.fields[h].index_select(0, self.idx[:M]), self.factor[:M], out=out)

    def hour(self, h: int):
        """[M, N] runoff of hour h (device; valid until the next call)."""
        self.fill(h, self.buf)
        return self.buf


class ArrayForcing:
    """Forcing from a host array [hours, M, N], uploaded once."""

    def __init__(self, runoff: np.ndarray, device):
        import torch

        self.t = torch.tensor(np.ascontiguousarray(runoff, dtype=np.float64), device=device)

    def hour(self, h: int):
        return self.t[h]

    def fill(self, h: int, out) -> None:
        out.copy_(self.t[h])


class SurrogateEnsemble:
    """E4: ensemble advanced by the emulator with plain-solver judging and hand-back."""

    def __init__(self, host, mlp: MLP, members: int, judge_slots: int, gauges: np.ndarray, tol_rel: float = 0.05,
                 resync_hours: int = 24, schedule: dict | None = None):
        """schedule: launch schedule for the judging plain solver (PhysicsGPU.set_schedule keys), e.g. the
        one the plain ensemble tuned; without it the judging solver runs phase kernels at 128 threads."""
        import torch

        from .model import PhysicsGPU

        self.torch = torch
        self.host = host
        self.mlp = mlp
        self.M = members
        self.emu = PhysicsGPU(host, nmembers=members, block_size=128)     # stage scheme only: no tuning
        self.judge = PhysicsGPU(host, nmembers=judge_slots, block_size=128)
        if schedule:
            self.judge.set_schedule(**{k: schedule[k] for k in ("mode", "flux_block", "rate_block", "store_block",
                                                                 "profile")})
        self.fe = Features(self.emu, qref_from_host(host))
        self.jfe = Features(self.judge, qref_from_host(host))
        self.lib = _emu_lib()
        self.gauges = np.asarray(gauges)
        self.tol = tol_rel
        self.resync = resync_hours
        self.slots = judge_slots
        self.plain = set()
        self.active = torch.ones(members, dtype=torch.int32, device=self.fe.dev)
        self.stats = {"judged": 0, "fallback": 0, "emu_member_hours": 0, "plain_member_hours": 0, "errors": []}

    def set_state_from(self, phys):
        for m in range(self.M):
            check(self.lib.cmf_gpu_ctx_copy_member(self.emu.h, m, phys.h, m), "copy_member")

    def emu_step(self):
        X = self.fe.build()
        self._y = self.mlp.infer_tc(X, getattr(self, "_y", None))     # tcgen05 tensor cores
        self.fe.rollout(self._y, self.active, ldy=1, residual=getattr(self.mlp, "residual", True))

    def run(self, forcing, hours: int, h0: int = 0):
        """Advances `hours` coupling steps with the runoff forcing.fill(h0 + h, ...) writes; returns the
        hourly mean discharge at the gauges [hours, M, G] (the judged plain value for members
        handed back to the plain solver)."""
        torch = self.torch
        G = torch.as_tensor(self.gauges, device=self.fe.dev)
        out = np.zeros((hours, self.M, len(self.gauges)))
        slots = []
        buf_e, buf_j = [], []
        day = 0
        emu_runoff = self.fe.runoff_view()
        jfe = self.jfe
        cur_plain = None
        for h in range(hours):
            if h % self.resync == 0:
                plain = sorted(self.plain)[: self.slots]
                free = self.slots - len(plain)
                cand = [m for m in range(self.M) if m not in self.plain]
                judged = [cand[(day * free + k) % len(cand)] for k in range(min(free, len(cand)))] if cand else []
                slots = plain + judged
                for k, m in enumerate(slots):
                    check(self.lib.cmf_gpu_ctx_copy_member(self.judge.h, k, self.emu.h, m), "copy_member")
                slot_idx = torch.as_tensor(slots + [slots[0]] * (self.slots - len(slots)) if slots else [0] * self.slots,
                                           device=self.fe.dev)
                buf_e, buf_j = [], []
                day += 1
            if cur_plain != self.plain:
                self.active.copy_(torch.tensor([0 if m in self.plain else 1 for m in range(self.M)], dtype=torch.int32))
                cur_plain = set(self.plain)
            forcing.fill(h0 + h, emu_runoff)                   # straight into the emulator's runoff input
            jr = emu_runoff.index_select(0, slot_idx)
            torch.cuda.current_stream(self.fe.dev).synchronize()
            self.judge.advance_device(1, jr.data_ptr(), 0)
            self.emu_step()
            self.emu.stage()
            self.stats["emu_member_hours"] += self.M - len(self.plain)
            self.stats["plain_member_hours"] += len(slots)
            qe = self.fe.at(G)
            qjudge = jfe.at(G)
            out[h] = qe
            for k, m in enumerate(slots):
                if m in self.plain:
                    out[h, m] = qjudge[k]
            buf_e.append(qe)
            buf_j.append(qjudge)
            if (h + 1) % self.resync == 0:
                we = np.stack(buf_e).mean(0)
                wj = np.stack(buf_j).mean(0)
                for k, m in enumerate(slots):
                    if m not in self.plain:
                        err = float(np.median(np.abs(we[m] - wj[k]) / np.maximum(np.abs(wj[k]), 1e-6)))
                        self.stats["errors"].append(err)
                        self.stats["judged"] += 1
                        if err > self.tol:
                            self.plain.add(m)
                            self.stats["fallback"] += 1
                    check(self.lib.cmf_gpu_ctx_copy_member(self.emu.h, m, self.judge.h, k), "copy_member")
        return out


def time_inference(rows: int, reps: int = 5, device: int = 0) -> dict:
    """CUDA-event timing of the fused inference kernels on `rows` random feature rows (seeded
    weights): the tcgen05 kernel and the mma.sync kernel, ms per call and TFLOP/s."""
    import torch

    dev = torch.device("cuda", device)
    mlp = MLP(dev, seed=2)
    g = torch.Generator(device=dev).manual_seed(1)
    X = (torch.randn(rows, IN, device=dev, generator=g) * 2).to(torch.bfloat16)
    X[:, NFEAT:] = 0
    out = {"rows": rows}
    flops = 2.0 * rows * (32 * HID + HID * HID * 2 + HID * 8)
    for name, fn in (("tcgen05", mlp.infer_tc), ("mma_sync", mlp.infer)):
        y = fn(X)
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        for _ in range(reps):
            fn(X, y)
        ev[1].record()
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1]) / reps
        out[name] = {"ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}
    out["tcgen05_status"] = _emu_lib().cmf_emu_mlp_tc_status()
    return out


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser(description="time the fused emulator inference kernels")
    ap.add_argument("--time-mlp", type=int, default=2 * 1024 * 1024, metavar="ROWS")
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    print(json.dumps(time_inference(a.time_mlp, a.reps)))
