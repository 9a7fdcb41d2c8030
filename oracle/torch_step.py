"""Float64 PyTorch restatement of the resident step, differentiable (TEST INFRASTRUCTURE ONLY).

The checker of the adjoint, never the product: only ``tests/`` and
``bench.py`` may use it. It restates the discrete step of the reference's
resident kernels -- edge flux (``inundation/vulkan/shaders/flux.py:63-182``),
gather and update (``inundation/vulkan/shaders/resident.py:187-513``),
film drag (``flux.py:43-54``), sources (``resident.py:665-733``) -- in float64
over all cells and edges, with every step's dt and clock given (frozen), and
with the inflow hydrographs evaluated as the product evaluates them
(piecewise linear in the knots at each step's start time). The bed enters
through the face steps dzL = max(zL, zR) - zL, dzR = max(zL, zR) - zR
(``inundation/mesh/geometry.py:241-254``).

Non-smooth points take the same one-sided derivatives as the CUDA adjoint:
square roots at zero and the momentum magnitude at rest have derivative 0,
clamps pass the derivative of the branch taken. ``torch.autograd`` gives the
gradient of ``misfit`` with respect to n, z and the knot discharges;
evaluated without gradients, the same function is the float64 forward of
the finite-difference checks.
"""

from __future__ import annotations

from collections.abc import Sequence

import numpy as np
import torch

FILM_DEPTHS = 4.0


def _sqrt0(x: torch.Tensor) -> torch.Tensor:
    pos = x > 0
    return torch.where(pos, torch.sqrt(torch.where(pos, x, torch.ones_like(x))), torch.zeros_like(x))


def _div0(num: torch.Tensor, den: torch.Tensor, ok: torch.Tensor) -> torch.Tensor:
    return torch.where(ok, num / torch.where(ok, den, torch.ones_like(den)), torch.zeros_like(num))


class TorchStep:
    """The discrete step over one mesh, float64, on ``device``."""

    def __init__(self, geom, g: float = 9.81, dry_tol: float = 1e-4, device: str = "cpu", cut_depth: float = 0.0) -> None:
        t = lambda a, dt=torch.float64: torch.as_tensor(np.asarray(a), dtype=dt, device=device)  # noqa: E731
        self.N, self.E = int(geom.N), int(geom.E)
        self.g, self.dry = float(g), float(dry_tol)
        self.cut = float(cut_depth)  # no derivative through depths below this (0: the exact derivative)
        self.device = device
        self.cl = t(geom.edge_cellL, torch.int64)
        cr = np.asarray(geom.edge_cellR, np.int64)
        self.wall = t(cr < 0, torch.bool)
        self.cr = t(np.where(cr >= 0, cr, 0), torch.int64)  # walls read their left cell, then mirror
        self.wall_cl = self.cl
        self.nx, self.ny, self.len = t(geom.edge_nx), t(geom.edge_ny), t(geom.edge_len)
        self.area = t(geom.area)

    # -- edge flux -------------------------------------------------------------------------------
    def _sv(self, h, q):
        e2 = (FILM_DEPTHS * self.dry) ** 2
        h2 = h * h
        return torch.where(h > self.dry, 2.0 * h * q / (h2 + torch.maximum(h2, torch.full_like(h2, e2))),
                           torch.zeros_like(h))

    def _cut(self, h, *vals):
        if self.cut <= 0.0:
            return vals
        thin = h < self.cut
        return tuple(torch.where(thin, v.detach(), v) for v in vals)

    def edge_words(self, h, hu, hv, dzL, dzR):
        g, dry = self.g, self.dry
        nx, ny, ln = self.nx, self.ny, self.len
        hL, huL, hvL = h[self.cl], hu[self.cl], hv[self.cl]
        hL, huL, hvL = self._cut(hL, hL, huL, hvL)
        hR = torch.where(self.wall, hL, h[self.cr])
        dot = huL * nx + hvL * ny
        huR = torch.where(self.wall, huL - 2.0 * dot * nx, hu[self.cr])
        hvR = torch.where(self.wall, hvL - 2.0 * dot * ny, hv[self.cr])
        hR, huR, hvR = self._cut(hR, hR, huR, hvR)
        zero = torch.zeros_like(hL)
        hLs = torch.clamp(hL - dzL, min=0.0)
        hRs = torch.clamp(hR - dzR, min=0.0)
        (hLs,) = self._cut(hLs, hLs)
        (hRs,) = self._cut(hRs, hRs)
        uL, vL, uR, vR = self._sv(hL, huL), self._sv(hL, hvL), self._sv(hR, huR), self._sv(hR, hvR)
        huLs, hvLs, huRs, hvRs = hLs * uL, hLs * vL, hRs * uR, hRs * vR
        hqnL, hqtL = huLs * nx + hvLs * ny, -huLs * ny + hvLs * nx
        hqnR, hqtR = huRs * nx + hvRs * ny, -huRs * ny + hvRs * nx
        unL, utL, unR, utR = self._sv(hLs, hqnL), self._sv(hLs, hqtL), self._sv(hRs, hqnR), self._sv(hRs, hqtR)
        cL, cR = _sqrt0(g * hLs), _sqrt0(g * hRs)
        sqL, sqR = _sqrt0(hLs), _sqrt0(hRs)
        den = sqL + sqR
        u_roe = _div0(sqL * unL + sqR * unR, den, den > 1e-12)
        c_roe = _sqrt0(g * 0.5 * (hLs + hRs))
        aL, bL = unL - cL, u_roe - c_roe
        SL0 = torch.where(bL < aL, bL, aL)
        aR, bR = unR + cR, u_roe + c_roe
        SR0 = torch.where(aR < bR, bR, aR)
        wetL = torch.clamp(hLs / dry - 1.0, 0.0, 1.0)
        wetR = torch.clamp(hRs / dry - 1.0, 0.0, 1.0)
        dryLeft = (1.0 - wetL) * wetR
        dryRight = (1.0 - wetR) * wetL
        roe = 1.0 - dryLeft - dryRight
        SL = roe * SL0 + dryLeft * (unR - 2.0 * cR) + dryRight * (unL - cL)
        SR = roe * SR0 + dryLeft * (unR + cR) + dryRight * (unL + 2.0 * cL)
        num = SL * hRs * (unR - SR) - SR * hLs * (unL - SL)
        dsm = hRs * (unR - SR) - hLs * (unL - SL)
        SM = _div0(num, dsm, dsm.abs() > 1e-12)
        # the four HLLC regions
        fLh, fLn, fLt = hLs * unL, hLs * unL * unL + 0.5 * g * hLs * hLs, hLs * unL * utL
        fRh, fRn, fRt = hRs * unR, hRs * unR * unR + 0.5 * g * hRs * hRs, hRs * unR * utR
        dSL = SL - SM
        dSL = torch.where(dSL.abs() > 1e-14, dSL, torch.full_like(dSL, 1e-14))
        kL = hLs * (SL - unL) / dSL
        sLh = fLh + SL * (kL - hLs)
        sLn = fLn + SL * (kL * SM - hLs * unL)
        sLt = fLt + SL * (kL * utL - hLs * utL)
        dSR = SR - SM
        dSR = torch.where(dSR.abs() > 1e-14, dSR, torch.full_like(dSR, 1e-14))
        kR = hRs * (SR - unR) / dSR
        sRh = fRh + SR * (kR - hRs)
        sRn = fRn + SR * (kR * SM - hRs * unR)
        sRt = fRt + SR * (kR * utR - hRs * utR)
        b0, b1, b2 = SL >= 0, SM >= 0, SR >= 0

        def pick(a, b, c, d):
            return torch.where(b0, a, torch.where(b1, b, torch.where(b2, c, d)))

        Fh = torch.where(self.wall, zero, pick(fLh, sLh, sRh, fRh))
        Fhn = pick(fLn, sLn, sRn, fRn)
        Fht = pick(fLt, sLt, sRt, fRt)
        Fhu = Fhn * nx - Fht * ny
        Fhv = Fhn * ny + Fht * nx
        SLg = 0.5 * g * (hL * hL - hLs * hLs)
        SRg = 0.5 * g * (hR * hR - hRs * hRs)
        live = ~((hL < dry) & (hR < dry))
        m = live.to(hL.dtype)
        w0 = Fh * ln * m
        w1 = (Fhu * ln + SLg * nx * ln) * m
        w2 = (Fhv * ln + SLg * ny * ln) * m
        w3 = (Fhu * ln + SRg * nx * ln) * m
        w4 = (Fhv * ln + SRg * ny * ln) * m
        return w0, w1, w2, w3, w4

    def bed_steps(self, z):
        zL = z[self.cl]
        zR = torch.where(self.wall, zL, z[self.cr])
        face = torch.maximum(zL, zR)
        return face - zL, torch.where(self.wall, torch.zeros_like(zL), face - zR)

    # -- stages ------------------------------------------------------------------------------------
    def sums(self, h, hu, hv, dzL, dzR):
        w0, w1, w2, w3, w4 = self.edge_words(h, hu, hv, dzL, dzR)
        inner = ~self.wall
        sh = torch.zeros(self.N, dtype=h.dtype, device=h.device).index_add(0, self.cl, w0)
        sh = sh.index_add(0, self.cr[inner], -w0[inner])
        su = torch.zeros_like(sh).index_add(0, self.cl, w1).index_add(0, self.cr[inner], -w3[inner])
        sv = torch.zeros_like(sh).index_add(0, self.cl, w2).index_add(0, self.cr[inner], -w4[inner])
        return sh, su, sv

    def update(self, h, hu, hv, sh, su, sv, n, dt):
        g, dry = self.g, self.dry
        e = FILM_DEPTHS * dry
        dti = dt / self.area
        h, hu, hv = self._cut(h, h, hu, hv)
        h_new = torch.clamp(h - dti * sh, min=0.0)
        hu_a = hu - dti * su
        hv_a = hv - dti * sv
        wet = h_new >= dry
        hs = torch.where(wet, h_new, torch.ones_like(h_new))
        rate = (e * e - hs * hs) / (2.0 * hs * hs) * np.sqrt(g / e)
        drag = torch.where(hs < e, 1.0 / (1.0 + dt * rate), torch.ones_like(hs))
        (drag,) = self._cut(hs, drag)
        hu_b, hv_b = hu_a * drag, hv_a * drag
        (hf,) = self._cut(hs, hs)  # the friction's depth
        u, v = hu_b / hf, hv_b / hf
        spd = _sqrt0(u * u + v * v)
        Sf = g * n * n * spd / torch.pow(hf, 4.0 / 3.0)
        den = 1.0 + dt * Sf
        hu_new = torch.where(wet, hu_b / den, torch.zeros_like(hu_b))
        hv_new = torch.where(wet, hv_b / den, torch.zeros_like(hv_b))
        return h_new, hu_new, hv_new

    def step(self, h, hu, hv, n, dzL, dzR, dt, src_cells=None, src_inc=None):
        h1, hu1, hv1 = self.update(h, hu, hv, *self.sums(h, hu, hv, dzL, dzR), n, dt)
        h2, hu2, hv2 = self.update(h1, hu1, hv1, *self.sums(h1, hu1, hv1, dzL, dzR), n, dt)
        hf = 0.5 * (h + h2)
        wet = hf >= self.dry
        huf = torch.where(wet, 0.5 * (hu + hu2), torch.zeros_like(hf))
        hvf = torch.where(wet, 0.5 * (hv + hv2), torch.zeros_like(hf))
        if src_cells is not None:
            hf = hf.index_add(0, src_cells, dt * src_inc)
        return hf, huf, hvf


def hydrograph_value(knot_t: torch.Tensor, knot_q: torch.Tensor, t: float) -> torch.Tensor:
    """Piecewise linear in the knots, end values outside them (as the product evaluates it)."""
    tt = knot_t.detach().cpu().numpy()
    if not t > tt[0]:
        return knot_q[0]
    if not t < tt[-1]:
        return knot_q[-1]
    i = int(np.searchsorted(tt, t, side="right")) - 1
    i = min(max(i, 0), tt.size - 2)
    f = (t - float(tt[i])) / (float(tt[i + 1]) - float(tt[i]))
    return knot_q[i] + (knot_q[i + 1] - knot_q[i]) * f


def misfit(
    model: TorchStep,
    h0, hu0, hv0,
    n: torch.Tensor,
    z: torch.Tensor,
    knots_q: torch.Tensor | None,
    dts: Sequence[float],
    times: Sequence[float],
    gauges: torch.Tensor,
    obs: torch.Tensor,
    hydro: Sequence[tuple] = (),
    rate=None,
    checkpoint: bool = True,
) -> torch.Tensor:
    """Sum over steps and gauges of (h after the step - obs)^2, float64.

    ``hydro``: (cells, hscale, knot_t, knot slice) per hydrograph; ``rate``:
    constant per-cell source rates in m/s (or None).
    """
    dzL, dzR = model.bed_steps(z)
    h, hu, hv = h0, hu0, hv0
    loss = torch.zeros((), dtype=torch.float64, device=h0.device)
    for k, (dt, t) in enumerate(zip(dts, times, strict=True)):
        cells, inc = None, None
        if hydro or rate is not None:
            incs, cl = [], []
            if rate is not None:
                nz = torch.nonzero(rate).flatten()
                cl.append(nz)
                incs.append(rate[nz])
            for hcells, hscale, kt, ks in hydro:
                q = hydrograph_value(kt, knots_q[ks], t)
                cl.append(hcells)
                incs.append(hscale * q)
            cells, inc = torch.cat(cl), torch.cat(incs)

        def one(h, hu, hv, n, dzL, dzR, inc, dt=dt, cells=cells):
            return model.step(h, hu, hv, n, dzL, dzR, dt, cells, inc)

        if checkpoint and torch.is_grad_enabled():
            h, hu, hv = torch.utils.checkpoint.checkpoint(one, h, hu, hv, n, dzL, dzR, inc, use_reentrant=False)
        else:
            h, hu, hv = one(h, hu, hv, n, dzL, dzR, inc)
        d = h[gauges] - obs[k]
        loss = loss + (d * d).sum()
    return loss


__all__ = ["TorchStep", "hydrograph_value", "misfit"]
