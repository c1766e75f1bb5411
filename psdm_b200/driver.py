"""Shot loop of the RTM driver over torch.distributed.

Host orchestration of calculate_PSDM_RTM (src/calculate_PSDM_RTM.f90:151-497)
around the engine: shots are dealt to ranks round-robin, each rank migrates
its shot of the round inside its migration window, the window images and
their fold are embedded into the full grid and summed over the ranks once per
round, and the running sums are normalised by the fold at the end.

One process drives one GPU.  The per-round sum is the reference's
MPI_ALLREDUCE (:493-494), here a torch.distributed all-reduce (NCCL between
GPUs, gloo between CPU processes).  Shots are independent, so no other
communication is needed.
"""
from __future__ import annotations

import math
from typing import Callable, Optional, Tuple

import numpy as np


def n_rounds(nsamples: int, numtasks: int) -> int:
    """Number of rounds of the shot loop (ntimes, calculate_PSDM_RTM.f90:151-159)."""
    if numtasks > 1:
        return math.ceil(nsamples / numtasks) if nsamples > numtasks else 1
    return nsamples


def shot_of(itimes: int, numtasks: int, rank: int, line_i: int) -> int:
    """Shot line handled by `rank` in round `itimes` (1-based; icount, :166)."""
    return (itimes - 1) * numtasks + rank + line_i


class ImageStack:
    """Running image and fold sums over the full model grid (PSDM_sum, Cov_sum).

    Arrays are (nx, ny) in C order, i.e. the reference's (ny, nx) column-major
    layout.  Every rank must call add_round once per round, with or without a
    shot, because the per-round sum is a collective.
    """

    def __init__(self, ny: int, nx: int, device=None, dtype=None, group=None):
        """dtype: float32 (default) sums as the reference does
        (calculate_PSDM_RTM.f90:493-497); float64 keeps the cross-shot stack
        in double precision (window images are widened once)."""
        import torch
        self.torch = torch
        self.ny, self.nx = ny, nx
        dtype = dtype or torch.float32
        self.psdm_sum = torch.zeros((nx, ny), dtype=dtype, device=device)
        self.cov_sum = torch.zeros((nx, ny), dtype=dtype, device=device)
        self._img = torch.zeros_like(self.psdm_sum)
        self._cov = torch.zeros_like(self.cov_sum)
        self.group = group

    def _world(self) -> int:
        dist = self.torch.distributed
        if dist.is_available() and dist.is_initialized():
            return dist.get_world_size(self.group)
        return 1

    def add_round(self, window_image=None, x_i: int = 1, x_f: int = 0) -> None:
        """Embed this rank's window image (nx_w, ny) at model columns x_i..x_f
        (1-based, inclusive; Cov_w = 1 there, :471-483), sum over ranks and
        add to the running sums (:493-497).  window_image=None: no shot on
        this rank this round."""
        self._img.zero_()
        self._cov.zero_()
        if window_image is not None:
            nx_w = x_f - x_i + 1
            if nx_w < 1 or x_i < 1 or x_f > self.nx:
                raise ValueError(f"window {x_i}..{x_f} outside the model (nx={self.nx})")
            self._img[x_i - 1:x_f] = window_image[:nx_w]
            self._cov[x_i - 1:x_f] = 1.0
        if self._world() > 1:
            dist = self.torch.distributed
            dist.all_reduce(self._img, group=self.group)
            dist.all_reduce(self._cov, group=self.group)
        self.psdm_sum.add_(self._img)
        self.cov_sum.add_(self._cov)

    def normalized(self) -> np.ndarray:
        """PSDM = PSDM_sum / Cov_sum where the fold is positive
        (normalize_psdm, src/auxiliar_PSDM.f90:1-20), on the host.  A stack
        kept in float64 is divided in float64 and rounded once to float32."""
        from psdm_b200 import rtm
        if self.psdm_sum.dtype == self.torch.float64:
            s = self.psdm_sum.detach().cpu().numpy()
            c = self.cov_sum.detach().cpu().numpy()
            out = np.zeros(s.shape, np.float64)
            np.divide(s, c, out=out, where=c > 0)
            return out.astype(np.float32)
        s = self.psdm_sum.detach().to("cpu", self.torch.float32).numpy()
        c = self.cov_sum.detach().to("cpu", self.torch.float32).numpy()
        return rtm.normalize_psdm(s, c)


ShotFn = Callable[[int], Optional[Tuple[object, int, int]]]


def migrate_lines(migrate_shot: ShotFn, line_i: int, line_f: int, stack: ImageStack, rank: int = 0,
                  numtasks: int = 1, on_round: Optional[Callable[[int], None]] = None) -> ImageStack:
    """Run the shot loop (calculate_PSDM_RTM.f90:164-497) on this rank.

    migrate_shot(icount) migrates shot line `icount` and returns
    (window_image, x_i, x_f), or None when the shot is skipped (the
    reference's `nxSou < 0` case, :377).  Lines line_i..line_f inclusive.
    """
    nsamples = line_f - line_i + 1
    for itimes in range(1, n_rounds(nsamples, numtasks) + 1):
        icount = shot_of(itimes, numtasks, rank, line_i)
        res = migrate_shot(icount) if line_i <= icount <= line_f else None
        if res is None:
            stack.add_round(None)
        else:
            img, x_i, x_f = res
            stack.add_round(img, x_i, x_f)
        if on_round is not None:
            on_round(itimes)
    return stack
