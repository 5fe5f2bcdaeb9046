"""Learned block preconditioner for the implicit solves.

A small network (FP32, hand-written CUDA kernels in csrc/mlp.cu) maps a cell's state to a
correction of the Maxwellian-linearised blocks,

    P_q(f, dt) = P_eq,q(dt) + scale * Delta_q(features(f), log10(dt nu)),

and GMRES applies the per-cell P.  It is trained on probe pairs the exact operator generates: for
a training state f and random probes v_p, a_p = (I - dt J(f)) v_p comes from the library's J.v, and
the loss asks each block P_q to map a_{p,q} back to v_{p,q} (the block-Jacobi inverse that fits A(f)
best on the probes).  The Maxwellian blocks stay the fallback and the initial point (Delta = 0 at
initialisation); GMRES's true FP64 residual decides convergence in every case.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import _lib, implicit, workloads


def _dp(t) -> int:
    return int(t.data_ptr())


def _s(stream=None) -> int:
    import torch

    return int((stream or torch.cuda.current_stream()).cuda_stream)


class MLP:
    """Handle on the library's network (cf_mlp_*)."""

    def __init__(self, n_in: int, n_hidden: int, n_out: int, max_batch: int, seed: int = 0, device: int = 0):
        self.n_in, self.n_hid, self.n_out, self.max_batch = n_in, n_hidden, n_out, max_batch
        h = C.c_void_p()
        _lib.check(_lib.load().cf_mlp_create(C.byref(h), n_in, n_hidden, n_out, max_batch, seed, device))
        self._h = h
        n = C.c_int64()
        _lib.check(_lib.load().cf_mlp_num_params(h, C.byref(n)))
        self.n_params = int(n.value)

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().cf_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, dtype=np.float32)
        _lib.check(_lib.load().cf_mlp_copy(self._h, out.ctypes.data_as(C.c_void_p), 0))
        return out

    def set_params(self, flat: np.ndarray):
        flat = np.ascontiguousarray(flat, dtype=np.float32)
        _lib.check(_lib.load().cf_mlp_copy(self._h, flat.ctypes.data_as(C.c_void_p), 1))

    def grads(self) -> np.ndarray:
        out = np.zeros(self.n_params, dtype=np.float32)
        _lib.check(_lib.load().cf_mlp_copy(self._h, out.ctypes.data_as(C.c_void_p), 2))
        return out

    def forward(self, x, y, train: bool = False, stream=None):
        _lib.check(_lib.load().cf_mlp_forward(self._h, _dp(x), _dp(y), x.shape[0], int(train), _s(stream)))
        return y

    def backward(self, x, dy, stream=None):
        _lib.check(_lib.load().cf_mlp_backward(self._h, _dp(x), _dp(dy), x.shape[0], _s(stream)))

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, wd=0.0, stream=None):
        _lib.check(_lib.load().cf_mlp_adam_step(self._h, lr, b1, b2, eps, wd, _s(stream)))


class LearnedPreconditioner:
    """Per-cell block preconditioner predicted by the network, on top of the Maxwellian blocks."""

    def __init__(self, op, hidden: int = 512, max_batch: int = 2048, scale: float = 0.1, seed: int = 0):
        self.op = op
        self.K, self.NQ = op.K, op.N_Q
        self.M = self.K * self.NQ
        self.n_in = self.M + 1
        self.n_out = self.NQ * self.K * self.K
        self.scale = float(scale)
        self.net = MLP(self.n_in, hidden, self.n_out, max_batch, seed=seed, device=op.device)
        self.mu = np.zeros(self.n_in, dtype=np.float32)
        self.sd = np.ones(self.n_in, dtype=np.float32)
        self.nu = abs(implicit.equilibrium_jacobian_blocks(op)[min(6, self.NQ - 1)][0, 0])
        self.gain = {}  # log10(dt nu) (rounded) -> multiplier of the correction, from calibrate()
        self.benefit = {}  # log10(dt nu) (rounded) -> fraction of the Maxwellian blocks' probe loss it removes
        # below this calibrated benefit predict() returns the Maxwellian blocks and skips the network
        # (a correction that removes less than a tenth of the probe loss cannot pay for its inference)
        self.min_benefit = 0.1

    def _key(self, dt) -> float:
        return round(math.log10(max(dt * self.nu, 1e-12)), 6)

    def _gain(self, dt) -> float:
        return self.gain.get(self._key(dt), 1.0)

    def uses_network(self, dt) -> bool:
        """Whether predict() runs the network at this time step (calibrated benefit >= min_benefit;
        uncalibrated time steps use it)."""
        return self._gain(dt) > 0.0 and self.benefit.get(self._key(dt), 1.0) >= self.min_benefit

    def features(self, f, dt):
        """[B, M + 1] float32: the coefficients (standardised) and log10(dt nu)."""
        import torch

        B = f.shape[0]
        x = torch.empty((B, self.n_in), dtype=torch.float32, device=f.device)
        x[:, : self.M] = f.reshape(B, -1).to(torch.float32)
        x[:, self.M] = math.log10(max(dt * self.nu, 1e-12))
        mu = torch.as_tensor(self.mu, device=f.device)
        sd = torch.as_tensor(self.sd, device=f.device)
        return (x - mu) / sd

    def predict(self, f, dt, peq=None):
        """Per-cell blocks [B, N_Q, K, K] float64 on the device, or -- where calibrate() found that the
        correction removes less than min_benefit of the Maxwellian blocks' probe loss at this time step,
        so that it cannot pay for its inference -- the shared Maxwellian blocks [N_Q, K, K] themselves
        (no network call, no per-cell assembly)."""
        import torch

        B = f.shape[0]
        peq = torch.as_tensor(implicit.block_preconditioner(self.op, dt) if peq is None else peq,
                              dtype=torch.float64, device=f.device).contiguous()
        if not self.uses_network(dt):
            return peq
        P = torch.empty((B, self.NQ, self.K, self.K), dtype=torch.float64, device=f.device)
        for b0 in range(0, B, self.net.max_batch):
            b1 = min(B, b0 + self.net.max_batch)
            x = self.features(f[b0:b1], dt)
            d = torch.empty((b1 - b0, self.n_out), dtype=torch.float32, device=f.device)
            self.net.forward(x, d)
            _lib.check(_lib.load().cf_precond_assemble(_dp(d), _dp(peq), _dp(P[b0:b1]), self.scale * self._gain(dt),
                                                       b1 - b0, self.NQ, self.K, _s()))
        return P

    # ------------------------------------------------------------------ training
    def make_samples(self, n_states: int, dt_nu_values=(1.0, 10.0, 100.0), n_probes: int = 8, seed: int = 0,
                     amp_range=(0.0, 0.3)):
        """States f, dt per state, probes v and a = (I - dt J(f)) v from the exact operator's J.v."""
        import torch

        rng = np.random.default_rng(seed)
        K, L = self.K, int(round(math.sqrt(self.NQ))) - 1
        amps = rng.uniform(*amp_range, size=n_states)
        cells = workloads.stress_cells(K, L, n_states, seed=seed, amplitude=1.0)
        cells[:, 0, 4:9] *= amps[:, None]
        cells += workloads.perturbation(K, L, n_states, rng, 2e-3, 0.6)
        cells[:, 0, 0] = 1.0
        dts = rng.choice(np.asarray(dt_nu_values), size=n_states) / self.nu
        f = torch.from_numpy(cells).cuda(self.op.device)
        gen = torch.Generator(device=f.device)
        gen.manual_seed(int(seed) + 12345)
        v = torch.randn((n_states, n_probes, K, self.NQ), dtype=torch.float64, device=f.device, generator=gen)
        a = torch.empty_like(v)
        chunk = max(1, 65536 // n_probes)
        for s0 in range(0, n_states, chunk):
            s1 = min(n_states, s0 + chunk)
            fs = f[s0:s1].unsqueeze(1).expand(-1, n_probes, -1, -1).reshape(-1, K, self.NQ).contiguous()
            vs = v[s0:s1].reshape(-1, K, self.NQ).contiguous()
            jv = self.op.jv(fs, vs).reshape(s1 - s0, n_probes, K, self.NQ)
            dtt = torch.as_tensor(dts[s0:s1], device=f.device).view(-1, 1, 1, 1)
            a[s0:s1] = v[s0:s1] - dtt * jv
        # probe blocks [n, np, nq*K] with block q at q*K: transpose [K, NQ] -> [NQ, K]
        vb = v.transpose(2, 3).reshape(n_states, n_probes, -1).to(torch.float32).contiguous()
        ab = a.transpose(2, 3).reshape(n_states, n_probes, -1).to(torch.float32).contiguous()
        return {"f": f, "dt": dts, "v": vb, "av": ab, "vn2": (vb.double() ** 2).sum(-1).float().contiguous()}

    def fit_normalisation(self, samples):
        import torch

        f = samples["f"]
        B = f.shape[0]
        x = torch.empty((B, self.n_in), dtype=torch.float64, device=f.device)
        x[:, : self.M] = f.reshape(B, -1)
        x[:, self.M] = torch.as_tensor(np.log10(samples["dt"] * self.nu), device=f.device)
        self.mu = x.mean(0).float().cpu().numpy()
        self.sd = np.maximum(x.std(0).float().cpu().numpy(), 1e-6).astype(np.float32)

    def train(self, samples, epochs: int = 10, batch: int = 512, lr: float = 1e-3, seed: int = 0, log=None):
        import torch

        dev = samples["f"].device
        n = samples["f"].shape[0]
        peq_cache = {}
        rng = np.random.default_rng(seed)
        loss_dev = torch.zeros(1, dtype=torch.float64, device=dev)
        d = torch.empty((batch, self.n_out), dtype=torch.float32, device=dev)
        g = torch.empty_like(d)
        history = []
        t0 = time.perf_counter()
        groups = {float(dt): np.flatnonzero(samples["dt"] == dt) for dt in np.unique(samples["dt"])}
        for ep in range(epochs):
            # batches never mix time steps, so P_eq is uniform inside the loss kernel
            batches = []
            for dt, members in groups.items():
                perm = rng.permutation(members)
                batches += [(dt, perm[b0:b0 + batch]) for b0 in range(0, len(perm) - batch + 1, batch)]
            order = rng.permutation(len(batches))
            tot, nb = 0.0, 0
            for bi in order:
                dt, idx = batches[bi]
                it = torch.as_tensor(idx, device=dev)
                f = samples["f"][it]
                if dt not in peq_cache:
                    peq_cache[dt] = torch.as_tensor(implicit.block_preconditioner(self.op, dt), device=dev).contiguous()
                x = self.features(f, dt)
                m = x.shape[0]
                self.net.forward(x, d[:m], train=True)
                loss_dev.zero_()
                # the gathered probe batches are held in names for the duration of the call: a pointer
                # into a temporary would be released to the allocator (and reused) before the kernel runs
                av_b = samples["av"][it].contiguous()
                v_b = samples["v"][it].contiguous()
                vn2_b = samples["vn2"][it].contiguous()
                _lib.check(_lib.load().cf_precond_probe_loss(
                    _dp(d), _dp(peq_cache[dt]), _dp(av_b), _dp(v_b), _dp(vn2_b), self.scale, m, samples["v"].shape[1],
                    self.NQ, self.K, _dp(g), _dp(loss_dev), _s()))
                self.net.backward(x, g[:m])
                self.net.adam(lr=lr)
                tot += float(loss_dev.item())
                nb += 1
            history.append(tot / max(nb, 1))
            if log:
                log(f"epoch {ep}: loss {history[-1]:.4e} ({time.perf_counter() - t0:.1f} s)")
        return history

    def probe_loss(self, samples, dt_value, use_net: bool = True):
        """Mean probe loss on the samples with the given dt (network vs Maxwellian blocks alone)."""
        import torch

        dev = samples["f"].device
        idx = np.flatnonzero(samples["dt"] == dt_value)
        it = torch.as_tensor(idx, device=dev)
        f = samples["f"][it]
        m = f.shape[0]
        peq = torch.as_tensor(implicit.block_preconditioner(self.op, dt_value), device=dev).contiguous()
        d = torch.zeros((m, self.n_out), dtype=torch.float32, device=dev)
        if use_net:
            for b0 in range(0, m, self.net.max_batch):
                b1 = min(m, b0 + self.net.max_batch)
                self.net.forward(self.features(f[b0:b1], dt_value), d[b0:b1])
        g = torch.empty_like(d)
        loss = torch.zeros(1, dtype=torch.float64, device=dev)
        av_b = samples["av"][it].contiguous()
        v_b = samples["v"][it].contiguous()
        vn2_b = samples["vn2"][it].contiguous()
        _lib.check(_lib.load().cf_precond_probe_loss(
            _dp(d), _dp(peq), _dp(av_b), _dp(v_b), _dp(vn2_b), self.scale * self._gain(dt_value), m,
            samples["v"].shape[1], self.NQ, self.K, _dp(g), _dp(loss), _s()))
        return float(loss.item())

    def calibrate(self, samples, max_gain: float = 2.0) -> dict:
        """Least-squares multiplier of the network's correction, per time step, on held-out probes.

        The probe loss of P_eq + s * scale * Delta is quadratic in s; its minimiser over the samples,
        s* = -sum w <r0, D a> / sum w |D a|^2 (r0 = P_eq a - v, D = scale * Delta), clipped to
        [0, max_gain], is kept for that time step.  s* = 0 (the Maxwellian blocks alone) is chosen
        whenever the network does not lower the loss on these samples.
        """
        import torch

        dev = samples["f"].device
        out = {}
        n_p = samples["v"].shape[1]
        for dt_value in np.unique(samples["dt"]):
            idx = np.flatnonzero(samples["dt"] == dt_value)
            it = torch.as_tensor(idx, device=dev)
            f = samples["f"][it]
            m = f.shape[0]
            d = torch.zeros((m, self.n_out), dtype=torch.float32, device=dev)
            for b0 in range(0, m, self.net.max_batch):
                b1 = min(m, b0 + self.net.max_batch)
                self.net.forward(self.features(f[b0:b1], float(dt_value)), d[b0:b1])
            D = d.double().view(m, self.NQ, self.K, self.K) * self.scale
            peq = torch.as_tensor(implicit.block_preconditioner(self.op, float(dt_value)), device=dev)
            a = samples["av"][it].double().view(m, n_p, self.NQ, self.K)
            v = samples["v"][it].double().view(m, n_p, self.NQ, self.K)
            w = (1.0 / samples["vn2"][it].double()).view(m, n_p, 1, 1)
            r0 = torch.einsum("qij,npqj->npqi", peq, a) - v
            da = torch.einsum("nqij,npqj->npqi", D, a)
            num = float((w * r0 * da).sum())
            den = float((w * da * da).sum())
            loss0 = float((w * r0 * r0).sum())
            s_opt = min(max(-num / den, 0.0), max_gain) if den > 0 else 0.0
            key = self._key(float(dt_value))
            self.gain[key] = s_opt
            # probe loss at s_opt: loss0 + 2 s num + s^2 den; the fraction of loss0 it removes
            self.benefit[key] = (-(2.0 * s_opt * num + s_opt * s_opt * den) / loss0) if loss0 > 0 else 0.0
            out[float(dt_value) * self.nu] = s_opt
        return out
