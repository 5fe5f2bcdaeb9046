"""Batched explicit time stepping df/dt = Q(f) (Heun's method) on the GPU.

The reference advances one cell with its dense tensor (tutorial_stress_relaxation.m:77-91,
tutorial_collisions_bwu_solution.m:77-92).  ``RK2Stepper`` advances a whole batch with the
factorised operator: the state is packed once into the library's tiled layout, each call of
``step`` runs n steps of the library (cf_rk2_steps_tiled: two contraction launches and two vector
passes per step), and ``step_graph`` replays n steps recorded once into a CUDA graph.
"""
from __future__ import annotations

import ctypes as C

from . import _lib


class RK2Stepper:
    def __init__(self, op, f, form: str = "af"):
        """op: CollisionOperator; f: [B, K, N_Q] float64 CUDA tensor (the initial cells)."""
        import torch

        from .implicit import Tiled

        self.op, self.form = op, form
        self.B = int(f.shape[0])
        self.tiled = Tiled(op, self.B)
        self.state = self.tiled.pack(f.contiguous())
        need = C.c_size_t()
        _lib.check(_lib.load().cf_rk2_workspace_size(op._h, self.B, C.byref(need)))
        self.ws = torch.empty(need.value // 8 + 1, dtype=torch.float64, device=self.state.device)
        self._graphs = {}

    def _launch(self, dt: float, n: int, stream):
        _lib.check(_lib.load().cf_rk2_steps_tiled(self.op._h, int(self.state.data_ptr()), self.B, float(dt), int(n),
                                                  _lib.FORMS[self.form], int(self.ws.data_ptr()),
                                                  self.ws.numel() * 8, int(stream.cuda_stream)))

    def step(self, dt: float, n: int = 1, stream=None):
        import torch

        self._launch(dt, n, stream or torch.cuda.current_stream())

    def step_graph(self, dt: float, n: int):
        """n steps from a CUDA graph recorded on first use for (dt, n)."""
        import torch

        key = (float(dt), int(n))
        g = self._graphs.get(key)
        if g is None:
            # one eager step on a saved state builds what the library creates lazily (kernel
            # attributes, the folded operator) outside the recording; the state is then restored
            saved = self.state.clone()
            self.step(dt, 1)
            self.state.copy_(saved)
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream()
            with torch.cuda.graph(g, stream=s, capture_error_mode="thread_local"):
                self._launch(dt, n, s)
            self._graphs[key] = g
        g.replay()

    def cells(self):
        """The current state as [B, K, N_Q]."""
        return self.tiled.unpack(self.state)
