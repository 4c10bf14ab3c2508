"""Full-waveform inversion outer loop over the adjoint gradient (no counterpart in the reference,
which stops at the data misfit, forward.cpp:414-445).

One iteration: every rank computes the misfit and the gradient of its own shots with
tw_adjoint_gradient (shots are dealt to ranks round-robin), the gradients of rho, vp and vs and
the misfits are summed over ranks with one all-reduce each (NCCL across GPUs, gloo on CPU), and
the model takes a steepest-descent step along the summed gradient with a backtracking line search
on the summed misfit (every rank evaluates the same trial models, so all ranks keep identical
models without exchanging them). Which parameters move is configurable; the others stay fixed.

The per-shot work is a callable `shot_fn(model, shot, want_gradient) -> (J, {name: gradient})`;
the default runs the library on the current GPU (`elastic_shot_fn`), and a test may pass its own.
"""
from __future__ import annotations

import dataclasses
from typing import Callable, Sequence

import numpy as np

PARAMS = ("rho", "vp", "vs")


@dataclasses.dataclass
class Shot:
    """One source and its receivers: the source on grid `src_grid` at (ix, iy); receivers as
    (grid, ix array, iy array) groups; the observed traces [n_rcv, 2, nt]."""
    src_grid: int
    src_ix: int
    src_iy: int
    receivers: list
    obs: np.ndarray


def elastic_shot_fn(tw, Mx: int, My: int, num_dx: int, den_dx: int, dt: float, nt: int, *,
                    central_f: float, time_delay: float, precision: str = "f32", ckpt_every: int = 50,
                    device: int = 0) -> Callable:
    """The library's forward / adjoint solve of one elastic shot (module `tw` = the ctypes front end)."""
    def run(model: dict, shot: Shot, want_gradient: bool):
        s = tw.Solver(Mx, My, num_dx, den_dx, dt, precision=precision, central_f=central_f,
                      time_delay=time_delay, max_steps=nt, energy=False, device=device)
        try:
            s.set_material_model(model["rho"], model["vp"], model["vs"])
            s.set_source(shot.src_grid, shot.src_ix, shot.src_iy)
            for grid, ix, iy in shot.receivers:
                s.add_receivers(grid, ix, iy)
            if want_gradient:
                out = s.adjoint_gradient(nt, shot.obs, ckpt_every=ckpt_every)
                return out["misfit"], {k: out[k] for k in PARAMS}
            s.run(nt)
            return 0.5 * float(np.sum((s.read_receivers() - shot.obs) ** 2)), {}
        finally:
            s.close()
    return run


class FWI:
    """Steepest descent with backtracking over shots dealt to `world` ranks; `allreduce(array)`
    sums a float64 numpy array over ranks in place (identity on one rank)."""

    def __init__(self, shots: Sequence[Shot], shot_fn: Callable, *, params: Sequence[str] = ("vp",),
                 rank: int = 0, world: int = 1, allreduce: Callable | None = None,
                 bounds: dict | None = None):
        self.shots = list(shots)
        self.shot_fn = shot_fn
        self.params = tuple(params)
        self.rank, self.world = rank, world
        self.allreduce = allreduce or (lambda a: a)
        self.bounds = bounds or {}
        self.history: list = []

    def my_shots(self):
        return self.shots[self.rank::self.world]

    def misfit(self, model: dict) -> float:
        J = np.array([sum(self.shot_fn(model, sh, False)[0] for sh in self.my_shots())], np.float64)
        self.allreduce(J)
        return float(J[0])

    def gradient(self, model: dict):
        """Summed misfit and gradients over all shots of all ranks."""
        J = np.zeros(1)
        g = {k: np.zeros_like(model[k], dtype=np.float64) for k in self.params}
        for sh in self.my_shots():
            j, gs = self.shot_fn(model, sh, True)
            J[0] += j
            for k in self.params:
                g[k] += gs[k]
        self.allreduce(J)
        for k in self.params:   # one reduction per parameter array
            self.allreduce(g[k])
        return float(J[0]), g

    def _apply(self, model: dict, g: dict, alpha: float, scale: dict) -> dict:
        new = dict(model)
        for k in self.params:
            v = model[k] - alpha * scale[k] * g[k]
            lo, hi = self.bounds.get(k, (None, None))
            if lo is not None or hi is not None:
                v = np.clip(v, lo, hi)
            new[k] = v
        return new

    def iterate(self, model: dict, step: float = 0.02, max_halvings: int = 8):
        """One iteration; `step` is the largest relative change of any parameter at alpha = 1.
        Returns (new model, misfit before, misfit after)."""
        J0, g = self.gradient(model)
        # normalise each parameter's step by its gradient's largest magnitude and its own scale
        scale = {}
        for k in self.params:
            gm = float(np.abs(g[k]).max())
            scale[k] = step * float(np.abs(model[k]).max()) / gm if gm > 0 else 0.
        alpha = 1.0
        for _ in range(max_halvings + 1):
            trial = self._apply(model, g, alpha, scale)
            J1 = self.misfit(trial)
            if J1 < J0:
                self.history.append((J0, J1, alpha))
                return trial, J0, J1
            alpha *= 0.5
        self.history.append((J0, J0, 0.0))
        return model, J0, J0


def torch_allreduce(device=None):
    """An `allreduce` over the default torch.distributed process group: in place on a float64
    numpy array, through a tensor on `device` (a CUDA device for NCCL, None for gloo on the CPU)."""
    import torch
    import torch.distributed as dist

    def reduce(a: np.ndarray):
        t = torch.from_numpy(a) if device is None else torch.from_numpy(a).to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        a[...] = t.cpu().numpy() if device is not None else t.numpy()
        return a
    return reduce
