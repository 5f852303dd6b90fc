"""FIRE relaxation of one density on the device pipeline.

Restates Fire (cmmdft/solver.py:606-698): the log-density moves with a
velocity field V driven by the force F = -beta dOmega/drho, with the FIRE
time-step and mixing control (N_pos / N_neg counters, dt growth after
N_delay positive-power steps, reset on negative power) and, for
'abc-fire', the bias-corrected velocity.  The update acts on the points of
``mask`` only, a boolean field the caller sets (the reference reads
``self.mask`` without assigning it); it must select points with rho > 0
(the reference takes ln(rho) there only).  Every C1 is one pass of the
functional pipeline; the field algebra runs as torch operations on the
device.  The counters N_pos and N_neg persist across solves of one solver
object, dt and alpha are reset per solve, as in the reference.
"""
import numpy as np
import torch

from .quasinewton import QuasiNewtonSolve

__all__ = ['FireSolve']


class FireSolve(QuasiNewtonSolve):
    """One density, one chemical potential: Fire.solve on the GPU."""

    def __init__(self, fn, mask, nsteps=500, method='abc-fire', alpha=0.2, dt=0.02, threshold=1e-6,
                 criterion='riue', a_tol=1e-6, r_tol=1e-4):
        super().__init__(fn, nsteps=nsteps, threshold=threshold, criterion=criterion, a_tol=a_tol, r_tol=r_tol)
        self.fire_method = method
        self.alpha0 = self.alpha = alpha
        self.dt0 = self.dt = dt
        self.alpha_max = 0.5
        self.Ndelay = 20
        self.Nnegmax = 2000
        self.dtmax = 5 * self.dt0
        self.dtmin = 0.01 * self.dt0
        self.Npos = 1
        self.Nneg = 0
        self.finc, self.fdec, self.fa = 1.1, 0.5, 0.99
        self.set_mask(mask)

    def set_mask(self, mask):
        m = torch.as_tensor(np.asarray(mask, dtype=bool).reshape(-1), device="cuda")
        if m.numel() != self.npts:
            raise ValueError("mask must have one entry per grid point")
        self.mask = m
        # the masked points as indices (ascending, as boolean indexing takes
        # them): gathers and scatters by index need no device read-back
        self.midx = torch.nonzero(m).squeeze(1)

    def _solve(self, rho):
        self.vel = torch.zeros(self.npts, dtype=torch.float64, device="cuda")   # _initiate_solving (V there)
        self.dt, self.alpha = self.dt0, self.alpha0
        return super()._solve(rho)

    def update(self, rho, C1):   # Fire.update_rho (solver.py:660-698)
        m = self.midx   # the mask's points, in the order boolean indexing gives them
        beta = self.fn.beta
        lnrho = torch.where(rho > 0, torch.log(torch.where(rho > 0, rho, torch.ones_like(rho))), torch.zeros_like(rho))
        F = -beta * self.domega(rho, C1)
        Fm = F[m]
        V = self.vel   # the reference's self.V (this class's self.V is the external potential)
        V[m] += Fm * 0.5 * self.dt          # curr_step >= 1 inside the loop
        P = float(torch.sum(Fm * V[m]))
        rho_new = rho.clone()
        if P > 0:
            self.Npos += 1
            if self.Npos > self.Ndelay:
                self.dt = min(self.dt * self.finc, self.dtmax)
                self.alpha = max(1.0e-10, self.alpha * self.fa)
        else:
            self.Npos = 1
            self.Nneg += 1
            if self.Nneg > self.Nnegmax:
                raise Exception('The system cannot relax further!')
            if self.steps - 1 > self.Ndelay:
                self.dt = max(self.dt * self.fdec, self.dtmin)
                self.alpha = self.alpha0
            lnrho[m] -= V[m] * 0.5 * self.dt
            V[m] = 0.0
        V[m] += Fm * 0.5 * self.dt
        Vm = V[m]
        V[m] = (1 - self.alpha) * Vm + self.alpha * Fm * torch.linalg.vector_norm(Vm) / torch.linalg.vector_norm(Fm)
        if self.fire_method == 'abc-fire':
            V[m] *= 1 / (1 - (1 - self.alpha) ** self.Npos)
        lnrho[m] += self.dt * V[m]
        rho_new[m] = torch.exp(lnrho[m])
        rho_new = self._clip(rho_new)
        return rho_new, self.C1(rho_new)
