"""Learned interpolation of the fluid velocity at droplets (no counterpart in the reference).

``LearnedInterp`` owns the MLP parameters (FP32) and their packed BF16 copy on the device and
drives the kernels of csrc/ld_mlp.cu:

* ``make_samples``: training pairs from a DNS state.  For a random sub-grid shift s, the spectrum
  is phase-shifted by exp(i k.s dx) and inverse-transformed: the result at grid point j is the
  exact spectral velocity at x_j + s dx.  Random grid points j of that field give exact targets at
  uniformly distributed points; features come from the unshifted grid.  Each sample carries the
  weight scale^2, so that the weighted loss on normalised targets is the mean squared velocity
  error the judge measures.
* ``calibrate``: fixes the feature and output scales from samples (before training).
* ``train``: Adam on mini-batches with the project's forward/backward kernels.
* ``infer``: fused stencil gather + tricubic + MLP correction at droplet positions.
* ``judge``: relative L2 error against the exact direct Fourier sum (``Plan.exact_sum``) on a
  sample of droplets, with tricubic as the comparison; with the default rule ("tolerance")
  ``enabled`` turns off when the learned error exceeds the tolerance, and back on when a later
  judgement meets it.  The rule "tolerance_or_better" keeps the network while it still beats
  tricubic (off only when it misses the tolerance and loses to tricubic).
"""
import ctypes
import time

import numpy as np

from . import _lib
from ._lib import check, ptr, stream_ptr

TWO_PI = 2.0 * np.pi


def _torch():
    import torch
    return torch


def sizes():
    a, b = ctypes.c_int64(), ctypes.c_int64()
    k, t = ctypes.c_int32(), ctypes.c_int32()
    check(_lib.lib().ld_mlp_sizes(ctypes.byref(a), ctypes.byref(b), ctypes.byref(k), ctypes.byref(t)))
    return a.value, b.value, k.value, t.value


D_IN, H, D_OUT, K1, N3 = 195, 128, 3, 208, 8
# algorithmic FLOPs of one training sample: forward 2 (195*128 + 128*128 + 128*3), backward the
# weight gradients and the two activation gradients 2 (128*3 + 3*128 + 128*128 + 128*128 + 195*128)
TRAIN_FLOP_PER_SAMPLE = 2 * (D_IN * H + H * H + H * D_OUT) + 2 * (2 * H * D_OUT + 2 * H * H + D_IN * H)
OFF_W1 = 0
OFF_B1 = OFF_W1 + K1 * H
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H * N3
OFF_FS = OFF_B3 + N3       # 64 feature scales (per polynomial coefficient, shared by components)
OFF_OS = OFF_FS + 64       # output scale, then the scale mode (0: all coefficients, 1: order >= 3)
N_PARAMS = OFF_OS + 8


def flat_from_mats(W1, b1, W2, b2, W3, b3, fs=None, os=1.0, scale_mode=1):
    """(195,128),(128),(128,128),(128),(128,3),(3) [+ feature scales (64), output scale] -> the
    flat padded parameter vector."""
    p = np.zeros(N_PARAMS, np.float32)
    p[OFF_FS:OFF_FS + 64] = 1.0 if fs is None else fs
    p[OFF_OS] = os
    p[OFF_OS + 1] = scale_mode
    p[OFF_W1:OFF_B1].reshape(K1, H)[:D_IN] = W1
    p[OFF_B1:OFF_W2] = b1
    p[OFF_W2:OFF_B2] = np.asarray(W2).reshape(-1)
    p[OFF_B2:OFF_W3] = b2
    p[OFF_W3:OFF_B3].reshape(H, N3)[:, :D_OUT] = W3
    p[OFF_B3:OFF_B3 + D_OUT] = b3
    return p


def mats_from_flat(p):
    p = np.asarray(p, np.float32)
    return dict(W1=p[OFF_W1:OFF_B1].reshape(K1, H)[:D_IN].copy(), b1=p[OFF_B1:OFF_W2].copy(),
                W2=p[OFF_W2:OFF_B2].reshape(H, H).copy(), b2=p[OFF_B2:OFF_W3].copy(),
                W3=p[OFF_W3:OFF_B3].reshape(H, N3)[:, :D_OUT].copy(), b3=p[OFF_B3:OFF_B3 + D_OUT].copy(),
                fs=p[OFF_FS:OFF_FS + 64].copy(), os=float(p[OFF_OS]), scale_mode=int(p[OFF_OS + 1]))


def init_flat(seed=0, scale_mode=1):
    """He-uniform initial weights, zero biases, a small last layer."""
    rng = np.random.default_rng(seed)

    def lin(i, o):
        lim = np.sqrt(6.0 / i)
        return rng.uniform(-lim, lim, (i, o)).astype(np.float32), np.zeros(o, np.float32)

    W1, b1 = lin(D_IN, H)
    W2, b2 = lin(H, H)
    W3, b3 = lin(H, D_OUT)
    return flat_from_mats(W1, b1, W2, b2, 0.1 * W3, b3, scale_mode=scale_mode)


class LearnedInterp:
    """MLP parameters, optimiser state and packed weights on one device."""

    RULES = ("tolerance", "tolerance_or_better")

    def __init__(self, plan, seed=0, params=None, tol=1e-4, scale_mode=1, rule="tolerance"):
        torch = _torch()
        n_params, n_packed, k_in, tile = sizes()
        assert n_params == N_PARAMS and k_in == K1
        self.plan = plan
        dev = plan.device
        flat = init_flat(seed, scale_mode) if params is None else np.asarray(params, np.float32)
        self.params = torch.as_tensor(flat).to(dev).contiguous()
        self.packed = torch.empty(n_packed, dtype=torch.bfloat16, device=dev)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)
        self.step_count = 0
        if rule not in self.RULES:
            raise ValueError(f"rule must be one of {self.RULES}")
        self.tol = tol
        self.rule = rule
        self.enabled = True
        self.history = []
        check(_lib.lib().ld_mlp_pack(ptr(self.params), ptr(self.packed), stream_ptr()))

    def set_params(self, flat):
        self.params.copy_(_torch().as_tensor(np.asarray(flat, np.float32)))
        check(_lib.lib().ld_mlp_pack(ptr(self.params), ptr(self.packed), stream_ptr()))

    # ---- inference ------------------------------------------------------------------------------
    def infer(self, u4, pos, out=None, stream=None, work=None):
        """Velocity (n, 3) at pos: tricubic + learned correction.  work (uint8 device tensor, see
        workspace()) holds the feature tiles; without it the plan's transform workspace does, so the
        call must not overlap the plan's transforms."""
        torch = _torch()
        n = int(pos.shape[0])
        if out is None:
            out = torch.empty((n, 3), dtype=self.plan.rdtype, device=self.plan.device)
        check(_lib.lib().ld_mlp_infer_ws(self.plan.handle, ptr(u4), ptr(pos), n, ptr(self.packed), ptr(self.params),
                                         ptr(out), ptr(work), int(work.numel()) if work is not None else 0,
                                         stream_ptr(stream)))
        return out

    def workspace(self, n):
        """A feature-tile workspace for inference of n droplets in one batch."""
        torch = _torch()
        return torch.empty(int(_lib.lib().ld_mlp_infer_workspace_bytes(int(n))), dtype=torch.uint8,
                           device=self.plan.device)

    # ---- data -------------------------------------------------------------------------------------
    def interleaved(self, uk):
        """Interleaved (N,N,N,4) physical velocity of a cube-layout spectrum."""
        torch = _torch()
        p = self.plan
        u = p.irfft_cube(uk)
        u4 = torch.empty((p.N, p.N, p.N, 4), dtype=p.rdtype, device=p.device)
        check(_lib.lib().ld_interleave3(p.handle, ptr(u), ptr(u4), stream_ptr()))
        return u4

    def make_samples(self, uk, n_shifts, per_shift, seed=0, X=None, T=None, W=None, offset=0):
        """Training pairs from a cube-layout spectrum: n_shifts random sub-grid shifts, per_shift
        random grid points each, written at rows offset.. of X, T, W (allocated when X is None).
        Returns (X bf16 (ns, 208), T (ns,3), W (ns) = scale^2, aux (ns,4) of this call)."""
        torch = _torch()
        p = self.plan
        ns = n_shifts * per_shift
        rng = np.random.default_rng(seed)
        if X is None:
            X = torch.empty((ns, K1), dtype=torch.bfloat16, device=p.device)
            T = torch.empty((ns, 3), dtype=torch.float32, device=p.device)
            W = torch.empty(ns, dtype=torch.float32, device=p.device)
            offset = 0
        aux = torch.empty((ns, 4), dtype=torch.float32, device=p.device)
        u4 = self.interleaved(uk)
        shifted = p.empty_cube(3)
        L = _lib.lib()
        for i in range(n_shifts):
            s = rng.uniform(0.0, 1.0, 3)
            check(L.ld_phase_shift(p.handle, ptr(uk), ptr(shifted), float(s[0]), float(s[1]), float(s[2]),
                                   stream_ptr()))
            ue = p.irfft_cube(shifted)
            idx = torch.as_tensor(rng.integers(0, p.N ** 3, per_shift, dtype=np.int64)).to(p.device)
            a = offset + i * per_shift
            check(L.ld_mlp_samples(p.handle, ptr(u4), ptr(ue), ptr(idx), per_shift, float(s[0]), float(s[1]),
                                   float(s[2]), ptr(self.params), ptr(X[a:a + per_shift]), ptr(T[a:a + per_shift]),
                                   ptr(aux[i * per_shift:(i + 1) * per_shift]), stream_ptr()))
        if W is not None:
            W[offset:offset + ns] = aux[:, 3].square()
        return X, T, W, aux

    def calibrate(self, uk, n_shifts=16, per_shift=8192, seed=12345):
        """Set the feature scales (each polynomial coefficient to unit RMS) and the output scale
        (targets to unit RMS) from samples of a cube-layout spectrum.  Call before generating the
        training set; the scales are then fixed."""
        torch = _torch()
        X, T, W, _ = self.make_samples(uk, n_shifts, per_shift, seed=seed)
        f = X[:, :192].float().view(-1, 3, 64)
        rms = f.pow(2).mean(dim=(0, 1)).sqrt().clamp_min(1e-30)
        # output scale: RMS of the targets with the training weights
        t_rms = float(((T.square().sum(1) * W).sum() / (3 * W.sum())).sqrt().clamp_min(1e-30))
        self.params[OFF_FS:OFF_FS + 64].div_(rms)
        self.params[OFF_OS] *= t_rms
        check(_lib.lib().ld_mlp_pack(ptr(self.params), ptr(self.packed), stream_ptr()))
        del X, T, W, f
        torch.cuda.synchronize(self.plan.device)
        return rms.cpu().numpy(), t_rms

    def normalise_targets(self, T, W):
        """Rescale a generated training set so that its weighted target RMS is 1, moving the
        factor into the output scale (targets drift while a flow develops)."""
        r = float(((T.square().sum(1) * W).sum() / (3 * W.sum())).sqrt().clamp_min(1e-30))
        T.div_(r)
        self.params[OFF_OS] *= r
        check(_lib.lib().ld_mlp_pack(ptr(self.params), ptr(self.packed), stream_ptr()))
        return r

    # ---- training ---------------------------------------------------------------------------------
    def loss_and_grad(self, X, T, W=None, work=None):
        """Exact batch loss and gradient (device tensors); deterministic.  W: per-sample weights
        (None: unit weights)."""
        torch = _torch()
        nb = int(X.shape[0])
        L = _lib.lib()
        if work is None:
            work = torch.empty(int(L.ld_mlp_partial_floats(nb)), dtype=torch.float32, device=self.plan.device)
        check(L.ld_mlp_grad(ptr(X), ptr(T), ptr(W) if W is not None else None, nb, ptr(self.params),
                            ptr(self.packed), ptr(work), ptr(self.grad), ptr(self.loss), stream_ptr()))
        return self.loss, self.grad

    def train(self, X, T, W=None, epochs=1, batch=4096, lr=1e-3, lr_final=None, seed=0, log_every=0):
        """Adam over shuffled mini-batches; returns the per-epoch mean loss (host floats).  W: sample
        weights, used normalised to mean 1.  Each epoch is one native call (ld_mlp_train_epoch: per
        batch, the tensor-core forward/backward kernel on the permuted rows, then the fixed-order
        gradient sum fused with Adam and the BF16 re-pack)."""
        torch = _torch()
        n = int(X.shape[0])
        if n < 1:
            raise ValueError("MLP training: no samples")
        L = _lib.lib()
        dev = self.plan.device
        wn = (W / W.mean()).contiguous() if W is not None else None
        g = torch.Generator(device=dev).manual_seed(seed)  # the permutations are drawn on the device
        batch = min(batch, n)  # fewer samples than a batch: one batch of all of them
        nbatch = n // batch
        total = epochs * nbatch
        work = torch.empty(int(L.ld_mlp_partial_floats(batch)), dtype=torch.float32, device=dev)
        out = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g, device=dev).to(torch.int32)
            acc = torch.zeros(1, dtype=torch.float32, device=dev)
            check(L.ld_mlp_train_epoch(ptr(X), ptr(T), ptr(wn) if wn is not None else None, ptr(perm), nbatch, batch,
                                       ptr(self.params), ptr(self.packed), ptr(self.m), ptr(self.v), self.step_count,
                                       float(lr), float(lr_final) if lr_final is not None else 0.0, max(total, 1),
                                       ptr(work), ptr(acc), stream_ptr()))
            self.step_count += nbatch
            loss = float(acc.item()) / max(nbatch, 1)
            if not np.isfinite(loss):
                raise RuntimeError("MLP training: non-finite epoch loss (diverged, or a kernel gave up a "
                                   "bounded wait)")
            out.append(loss)
            if log_every and (ep + 1) % log_every == 0:
                print(f"epoch {ep + 1}: loss {out[-1]:.4e}")
        return out

    def fit(self, snapshots, n_pairs=20_000_000, per_shift=40_000, epochs=16, batch=4096, lr=2e-3, decay=0.8,
            seed=0, log=None):
        """Train on DNS snapshots (cube-layout spectra, e.g. every 100 steps of a run): feature
        scales from the latest snapshot, n_pairs exact-target pairs spread over the snapshots,
        targets normalised, then ``epochs`` passes of Adam with the learning rate lr * decay^epoch.
        Returns a summary dict (pairs, per-epoch losses)."""
        torch = _torch()
        p = self.plan
        ns = len(snapshots)
        n_shifts = max(1, int(n_pairs) // (ns * per_shift))
        total = ns * n_shifts * per_shift
        torch.cuda.synchronize(p.device)
        t0 = time.perf_counter()
        self.calibrate(snapshots[-1], seed=seed + 7)
        X = torch.empty((total, K1), dtype=torch.bfloat16, device=p.device)
        T = torch.empty((total, 3), dtype=torch.float32, device=p.device)
        W = torch.empty(total, dtype=torch.float32, device=p.device)
        for k, uk in enumerate(snapshots):
            self.make_samples(uk, n_shifts, per_shift, seed=seed * 1009 + k, X=X, T=T, W=W,
                              offset=k * n_shifts * per_shift)
        self.normalise_targets(T, W)
        torch.cuda.synchronize(p.device)
        t1 = time.perf_counter()
        losses = []
        for ep in range(epochs):
            losses += self.train(X, T, W, epochs=1, batch=batch, lr=lr * decay ** ep, seed=seed * 1009 + ep)
            if log:
                log(f"epoch {ep}: weighted loss {losses[-1]:.4e}")
        t2 = time.perf_counter()  # train() read the last epoch's loss: the device is idle
        del X, T, W
        trained = epochs * (total // min(batch, total)) * min(batch, total)
        return {"pairs": total, "snapshots": ns, "epochs": epochs, "batch": batch, "losses": losses,
                "samples_s": t1 - t0, "epochs_s": t2 - t1, "train_flop_per_sample": TRAIN_FLOP_PER_SAMPLE,
                "train_tflops": trained * TRAIN_FLOP_PER_SAMPLE / (t2 - t1) / 1e12}

    # ---- judge ------------------------------------------------------------------------------------
    def judge(self, uk, u4, pos, n_sample=None, seed=0):
        """Relative L2 errors (learned, tricubic) against the exact Fourier sum on a sample of
        positions; sets ``enabled`` by the judge's rule (default: off when the learned error
        exceeds the tolerance)."""
        torch = _torch()
        p = self.plan
        n = int(pos.shape[0])
        if n_sample is not None and n_sample < n:
            g = torch.Generator(device="cpu").manual_seed(seed)
            sel = torch.randperm(n, generator=g)[:n_sample].to(p.device)
            pos = pos[sel].contiguous()
        exact = p.exact_sum(uk, pos)
        learned = self.infer(u4, pos).to(torch.float64)
        tric = torch.empty((pos.shape[0], 3), dtype=p.rdtype, device=p.device)
        check(_lib.lib().ld_gather4(p.handle, ptr(u4), ptr(pos), int(pos.shape[0]), _lib.LD_INTERP["tricubic"],
                                    ptr(tric), stream_ptr()))
        den = torch.linalg.norm(exact)
        e_l = float(torch.linalg.norm(learned - exact) / den)
        e_t = float(torch.linalg.norm(tric.to(torch.float64) - exact) / den)
        if self.rule == "tolerance":
            self.enabled = e_l <= self.tol
        else:
            self.enabled = (e_l <= self.tol) or (e_l < e_t)
        self.history.append((e_l, e_t, self.enabled))
        return e_l, e_t

