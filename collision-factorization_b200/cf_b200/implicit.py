"""Implicit relaxation with the GPU operator: block preconditioners, batched GMRES, backward Euler.

The reference steps the homogeneous Boltzmann equation only explicitly, with its dense assembled
tensor (tutorial_stress_relaxation.m:77-91, tutorial_collisions_bwu_solution.m:77-92).  Stiff
collision rates (dt * nu >> 1) need implicit steps; here each cell's Newton system
(I - dt J(f)) x = r is solved by the library's batched GMRES (cf_gmres_solve_tiled) with J(f).v
from the contraction kernels.

The Maxwellian-linearised block preconditioner uses the equilibrium Jacobian, which is
block-diagonal over the angular modes because Y_00 is constant (Gaunt(q1, q2, 1) vanishes unless
q1 = q2): one K x K block per q, the block the reference extracts for its Chapman-Enskog check
(tutorial_chapman_enscog_decay_rates.m:42-48).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def _tiled_len(B: int, M: int) -> int:
    return ((B + 31) // 32) * 32 * M


class Tiled:
    """Device buffers in the tiled cell layout, with pack/unpack through the plan."""

    def __init__(self, op, B: int):
        import torch

        self.op, self.B = op, B
        self.M = op.N_Q * op.K
        self.n = _tiled_len(B, self.M)
        self.dev = torch.device("cuda", op.device)

    def empty(self):
        import torch

        return torch.zeros(self.n, dtype=torch.float64, device=self.dev)

    def pack(self, cells, out=None, stream=None):
        out = self.empty() if out is None else out
        sh = _stream(stream)
        _lib.check(_lib.load().cf_pack_cells(self.op._h, int(out.data_ptr()), int(cells.data_ptr()), self.B, sh))
        return out

    def unpack(self, tiled, out=None, stream=None):
        import torch

        out = torch.empty((self.B, self.op.K, self.op.N_Q), dtype=torch.float64, device=self.dev) if out is None else out
        _lib.check(_lib.load().cf_unpack_cells(self.op._h, int(out.data_ptr()), int(tiled.data_ptr()), self.B,
                                               _stream(stream)))
        return out


def _stream(stream):
    import torch

    return int((stream or torch.cuda.current_stream()).cuda_stream)


def equilibrium_jacobian_blocks(op, rho: float = 1.0) -> np.ndarray:
    """K x K blocks J_q of the Jacobian at the absolute Maxwellian c = rho e_(k=0, q=1).

    Returned as [N_Q, K, K] with J_q[a, b] = dQ[(q, a)] / dc[(q, b)].  Probing with v_b = sum_q e_(b, q)
    recovers every block at once because the equilibrium Jacobian couples no two angular modes.
    """
    import torch

    K, NQ = op.K, op.N_Q
    f = torch.zeros((K, K, NQ), dtype=torch.float64, device=f"cuda:{op.device}")
    f[:, 0, 0] = rho
    v = torch.zeros_like(f)
    for b in range(K):
        v[b, b, :] = 1.0
    out = op.jv(f, v).cpu().numpy()  # [probe b, k, q]
    return np.ascontiguousarray(out.transpose(2, 1, 0))  # [q, a, b]


def block_preconditioner(op, dt: float, rho: float = 1.0) -> np.ndarray:
    """Inverses of I - dt J_q for every angular mode q: [N_Q, K, K]."""
    J = equilibrium_jacobian_blocks(op, rho)
    A = np.eye(op.K)[None] - dt * J
    return np.ascontiguousarray(np.linalg.inv(A))


def exact_block_jacobi(op, f, dt: float, probes_per_launch: int = 131072):
    """The exact block-Jacobi preconditioner of each cell's (I - dt J(f)): [B, N_Q, K, K] float64 on the
    device, the inverses of the K x K diagonal blocks of A(f) over the angular modes.

    Column (b, q) of J(f) is J(f) e_(b,q), one J.v with a unit probe: K N_Q probes per state, batched
    over states and probes through the library's J.v.  This is the best any block-diagonal
    preconditioner over the angular modes can be for A(f) itself, the ceiling of the learned blocks.
    """
    import torch

    B, K, NQ = f.shape[0], op.K, op.N_Q
    M = K * NQ
    dev = f.device
    blocks = torch.empty((B, NQ, K, K), dtype=torch.float64, device=dev)  # [s, q, a, b]: J[(a,q),(b,q)]
    per = max(1, probes_per_launch // M)  # states per launch
    eye = torch.eye(M, dtype=torch.float64, device=dev).view(M, K, NQ)  # probe p = b * NQ + q: e_(b,q)
    qs = torch.arange(NQ, device=dev)
    for s0 in range(0, B, per):
        s1 = min(B, s0 + per)
        n = s1 - s0
        fs = f[s0:s1].unsqueeze(1).expand(-1, M, -1, -1).reshape(-1, K, NQ).contiguous()
        vs = eye.unsqueeze(0).expand(n, -1, -1, -1).reshape(-1, K, NQ).contiguous()
        out = op.jv(fs, vs).view(n, K, NQ, K, NQ)  # [s, b, q (probe), a, q' (output)]
        # diagonal blocks: q' = q
        d = out[:, :, qs, :, qs]  # [q, s, b, a]
        blocks[s0:s1] = d.permute(1, 0, 3, 2)
        del fs, vs, out
    A = torch.eye(K, dtype=torch.float64, device=dev).view(1, 1, K, K) - dt * blocks
    return torch.linalg.inv(A).contiguous()


def gmres_solve(op, f, b, dt: float, x0=None, restart: int = 30, tol: float = 1e-10, max_iters: int = 3000,
                precond=None, stream=None, raise_on_timeout: bool = True):
    """Solve (I - dt J(f)) x = b for every cell with GMRES(restart).

    f, b (and x0) are [B, K, N_Q] float64 CUDA tensors.  precond: None, a [N_Q, K, K] array shared
    by all cells, or a [B, N_Q, K, K] array per cell (numpy or torch).  Returns (x, iters, relres).
    """
    import torch

    B = f.shape[0]
    t = Tiled(op, B)
    ft, bt = t.pack(f, stream=stream), t.pack(b, stream=stream)
    xt = t.pack(x0, stream=stream) if x0 is not None else t.empty()
    per_cell = 0
    pdev = None
    if precond is not None:
        P = torch.as_tensor(np.ascontiguousarray(precond) if isinstance(precond, np.ndarray) else precond,
                            dtype=torch.float64).to(t.dev).contiguous()
        per_cell = 1 if P.dim() == 4 else 0
        pdev = P
    lib = _lib.load()
    need = C.c_size_t()
    _lib.check(lib.cf_gmres_workspace_size(op._h, B, restart, C.byref(need)))
    ws = torch.empty(need.value // 8 + 1, dtype=torch.float64, device=t.dev)
    iters = np.zeros(B, dtype=np.int32)
    rel = np.zeros(B, dtype=np.float64)
    st = lib.cf_gmres_solve_tiled(op._h, int(ft.data_ptr()), float(dt), int(bt.data_ptr()), int(xt.data_ptr()), B,
                                  restart, max_iters, tol, int(pdev.data_ptr()) if pdev is not None else None,
                                  per_cell, iters.ctypes.data_as(C.c_void_p), rel.ctypes.data_as(C.c_void_p),
                                  int(ws.data_ptr()), ws.numel() * 8, _stream(stream))
    if st != 0 and (st != 9 or raise_on_timeout):
        _lib.check(st)
    return t.unpack(xt, stream=stream), iters, rel


def backward_euler_step(op, f, dt: float, newton_tol: float = 1e-10, max_newton: int = 8, **gmres_kw):
    """One backward-Euler step f_new = f + dt Q(f_new), solved by Newton with GMRES inner solves.

    Each Newton correction solves (I - dt J(x)) d = -(x - f - dt Q(x)) for all cells at once.
    Returns (f_new, stats) with the GMRES iteration counts of every Newton step.
    """
    import torch

    x = f.clone()
    stats = []
    for _ in range(max_newton):
        q = op.q(x)
        res = -(x - f - dt * q)
        nres = float(res.abs().amax())
        scale = float(x.abs().amax())
        if nres <= newton_tol * scale:
            break
        d, iters, rel = gmres_solve(op, x, res, dt, **gmres_kw)
        stats.append({"gmres_iters_mean": float(np.mean(iters)), "gmres_iters_max": int(np.max(iters)),
                      "relres_max": float(np.max(rel)), "newton_residual": nres})
        x = x + d
        del d
    torch.cuda.synchronize()
    return x, stats
