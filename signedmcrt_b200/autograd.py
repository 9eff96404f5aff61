"""Differentiable transport for PyTorch: per-packet fluence and detector counts
as functions of the optical properties (mu_a, mu_s, g) of region groups.

    phi, det = transport(params, scene_fn, settings, region_group, nphotons, seed)

`params` is a (ngroups, 3) tensor of (mu_a, mu_s, g); `scene_fn(optics)` builds
the sdf array from a (ngroups, 3) numpy array (for example a preset with its
regions tied to the groups); `region_group[r]` gives the group of region r (-1:
fixed).  The forward pass runs the FP32 transport (smcrt_run_device) and returns
phi = jmean / nphotons as an (nxg, nyg, nzg) tensor and det = bins / nphotons.
The backward pass calls smcrt_adjoint on the SAME packets (same seed): the path-
replay score-function gradient of <grad_phi, phi> + <grad_det, det>.  Refractive
indices are not differentiated (Fresnel events do not depend on mu_a, mu_s, g).
"""
from __future__ import annotations

import numpy as np
import torch

from .transport import Transport


class _Transport(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, scene_fn, settings, region_group, nphotons, seed):
        optics = params.detach().cpu().numpy().astype(np.float64)
        dev = torch.device("cuda")
        # the transport runs on torch's current stream, so it follows the zero-fills
        # below and precedes the ops that read the tallies
        stream = torch.cuda.current_stream(dev)
        tr = Transport(scene_fn(optics), settings, kernel="pathlength", precision="fp32",
                       stream=stream.cuda_stream)
        jm = torch.zeros(tr.ncell, dtype=torch.float64, device=dev)
        bins = torch.zeros(max(tr.nbins, 1), dtype=torch.float64, device=dev)
        tr.run_device(0, int(nphotons), int(seed), jm.data_ptr(), bins.data_ptr() if tr.nbins else None)
        nx, ny, nz = tr.shape
        phi = (jm / nphotons).reshape(nz, ny, nx).permute(2, 1, 0)
        det = bins[: tr.nbins] / nphotons
        ctx.tr, ctx.region_group, ctx.n, ctx.seed = tr, list(region_group), int(nphotons), int(seed)
        ctx.ngroups = params.shape[0]
        ctx.param_dtype, ctx.param_device = params.dtype, params.device
        return phi, det

    @staticmethod
    def backward(ctx, grad_phi, grad_det):
        tr = ctx.tr
        nx, ny, nz = tr.shape
        if grad_phi is None:
            grad_phi = torch.zeros((nx, ny, nz), dtype=torch.float64, device="cuda")
        # voxel weights in the tally's column-major order
        w = grad_phi.permute(2, 1, 0).contiguous().reshape(-1).to(torch.float32)
        gb = None
        if grad_det is not None and tr.nbins:
            gb = grad_det.to(torch.float64).contiguous()
        # the adjoint launches on the forward's stream: the weights made on the
        # backward's current stream must be complete first
        torch.cuda.current_stream(w.device).synchronize()
        grad, _ = tr.adjoint(ctx.n, ctx.seed, w.data_ptr(), gb.data_ptr() if gb is not None else None,
                             ctx.region_group, ctx.ngroups)
        tr.close()
        g = torch.as_tensor(grad.T / ctx.n, dtype=ctx.param_dtype, device=ctx.param_device)
        return g, None, None, None, None, None


def transport(params: torch.Tensor, scene_fn, settings, region_group, nphotons: int, seed: int):
    """(phi (nxg, nyg, nzg), det (nbins,)) per packet, differentiable in params."""
    return _Transport.apply(params, scene_fn, settings, region_group, nphotons, seed)


def layered_groups():
    """(scene_fn, region_group) for the layered_vessels scene with 5 parameter
    groups -- vessels (all 4 capsules), layer 1, layer 2, layer 3, ambient -- the
    refractive indices staying those of the preset."""
    from . import presets as P

    def scene_fn(optics):
        # preset order per group: (mus, mua, g, n)
        full = []
        for k in range(5):
            mua, mus, g = optics[k]
            n = 1.0 if k == 4 else (P.LAYER_OPT[k - 1][3] if k > 0 else 0.0)
            full.append((mus, mua, g, n))
        return P.layered_vessels(optics=full)

    return scene_fn, [0, 0, 0, 0, 1, 2, 3, 4]
