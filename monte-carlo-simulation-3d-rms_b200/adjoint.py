"""PyTorch binding of the adjoint (rms_adjoint_run in include/rms.h).

``waveform_signal`` is the normalised waveform-mode signal -- mean over walkers
of s0 (cos phase_j, sin phase_j) per waveform j, shape [nwave, 2] -- as a
differentiable function of the waveforms, the diffusivity D (shared by every
labelled compartment), the membrane permeability kappa and the per-compartment
T2.  The forward pass is the split walk (rms_sim_run); the backward pass
(rms_adjoint_run) walks the same walkers again from their counter-based random
streams, keeping per-bin displacement sums and a few checkpoints per walker in
device memory, and walks each walker that made a permeation draw once more
from a checkpoint.  Gradients: exact pathwise
for the waveforms, analytic for T2, time rescaling (minus the kappa term) for
D, forced permeation draws (the weak derivative of the Bernoulli draws) for
kappa.  torch is the plumbing here; all arithmetic runs in librms.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import engine


@dataclass
class WalkSetup:
    """The fixed part of the simulation: lattice (labels 0..nc-1, label 0 is
    never entered), time step, steps, walkers, voxel size, walls, seed."""
    labels: np.ndarray
    dt: float
    tn: int
    npar: int
    res: float
    seed: int = 0
    boundary: str = "mirror"
    timepoints: int = 0
    device: int = 0
    nc: int = field(init=False)

    def __post_init__(self):
        self.nc = int(self.labels.max()) + 1

    def sim(self, wave: np.ndarray, D: float, kappa: float, t2: np.ndarray) -> engine.Sim:
        diff = [0.0] + [float(D)] * (self.nc - 1)
        return engine.Sim(self.labels, dt=self.dt, tn=self.tn, npar=self.npar, res=self.res, diffusivity=diff,
                          t2=[float(x) for x in t2], wave=wave, boundary=self.boundary,
                          timepoints=self.timepoints or min(self.tn, 1000), permeation="kappa", kappa=float(kappa))


class _WaveformSignal(torch.autograd.Function):
    @staticmethod
    def forward(ctx, wave, D, kappa, t2, setup: WalkSetup):
        w = wave.detach().cpu().double().numpy()
        sim = setup.sim(w, D.item(), kappa.item(), t2.detach().cpu().double().numpy())
        sim.run(seed=setup.seed, precision="split", device=setup.device)
        sig = torch.from_numpy(sim.get("sigw").reshape(-1, 2) / setup.npar)
        sim.close()
        ctx.save_for_backward(wave, D, kappa, t2)
        ctx.setup = setup
        return sig.to(wave.dtype)

    @staticmethod
    def backward(ctx, grad):
        wave, D, kappa, t2 = ctx.saved_tensors
        setup: WalkSetup = ctx.setup
        sim = setup.sim(wave.detach().cpu().double().numpy(), D.item(), kappa.item(),
                        t2.detach().cpu().double().numpy())
        g = grad.detach().cpu().double().numpy().reshape(-1) / setup.npar
        r = sim.adjoint(g, seed=setup.seed, device=setup.device)
        sim.close()
        d_wave = torch.from_numpy(r["d_wave"]).to(wave.dtype)
        return (d_wave, torch.tensor(r["d_diffusivity"], dtype=D.dtype), torch.tensor(r["d_kappa"], dtype=kappa.dtype),
                torch.from_numpy(r["d_t2"][: t2.numel()]).to(t2.dtype), None)


def waveform_signal(wave: torch.Tensor, D: torch.Tensor, kappa: torch.Tensor, t2: torch.Tensor,
                    setup: WalkSetup) -> torch.Tensor:
    """Normalised signal [nwave, 2] of waveforms ``wave`` [nwave, nbins, 3]
    (phase per um per ms, i.e. gamma g), differentiable in all four inputs."""
    return _WaveformSignal.apply(wave, D, kappa, t2, setup)


def signal_jacobian(wave: torch.Tensor, D: float, kappa: float, t2, setup: WalkSetup) -> dict:
    """d(normalised signal)/d(D, kappa, T2) for every waveform in one reverse
    pass (rms_adjoint_jacobian) instead of one backward pass per signal:
    tensors "D", "kappa", "kappa_score" [nwave, 2] (cos and sin parts) and "T2"
    [nwave, 2, nc], and the signal itself, "signal" [nwave, 2], for the walk
    ``waveform_signal`` evaluates with the same setup."""
    t2a = torch.as_tensor(t2, dtype=torch.float64).cpu().numpy()
    sim = setup.sim(wave.detach().cpu().double().numpy(), float(D), float(kappa), t2a)
    J = sim.jacobian(seed=setup.seed, device=setup.device)
    sim.close()
    out = {k: torch.from_numpy(J[k] / setup.npar) for k in ("D", "kappa", "kappa_score", "T2")}
    out["signal"] = torch.from_numpy(J["sigw"] / setup.npar)
    return out
