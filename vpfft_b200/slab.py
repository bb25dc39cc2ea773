"""Decomposition of ONE RVE over several GPUs: the slab layout of the
reference's FFTW-MPI build (MaterialGrid.cpp:344-376: fftw_mpi_local_size_3d
gives each rank a block of ceil(Nx / P) planes along x; the transforms are
collective; the reference medium and the error norms are all-reduced,
MaterialGrid.cpp:257-271, 1009-1045).

This module holds the host-side plan of that decomposition, for one process
per GPU over torch.distributed (NCCL between GPUs, gloo on CPU):

  real-space fields        rank r owns voxels x in [x0_r, x1_r), all y, z
  z and y line passes      local: their lines lie inside an x plane
  spectral x lines         need every x of a (kz, ky) line: an all-to-all
                           moves the half spectrum from x slabs to kz slabs
                           (rank r owns kz in [k0_r, k1_r)), the x pass and
                           the Green operator run locally, and the inverse
                           all-to-all brings it back
  per-voxel NR sweep       local
  sums (L0, <sigma>, norms) one all-reduce of the per-rank partial sums

The line transforms themselves are the device passes of the single-GPU path,
applied to each rank's local block; this module moves the blocks between
ranks and never transforms anything.  Layouts follow the device passes:
after the y pass a rank holds B[c][kz][ky][x in its slab] (x fastest), and
the x pass wants B[c][kz in its kz slab][ky][x] with complete x lines.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch
import torch.distributed as dist


def block_split(n: int, parts: int) -> list[tuple[int, int]]:
    """FFTW's default block distribution: blocks of ceil(n / parts) in rank
    order, the last ones possibly short or empty."""
    b = -(-n // parts)
    return [(min(n, r * b), min(n, (r + 1) * b)) for r in range(parts)]


@dataclass(frozen=True)
class SlabPlan:
    """Ownership of one nx x ny x nz RVE across `world` ranks."""

    nx: int
    ny: int
    nz: int
    world: int

    @property
    def nh(self) -> int:
        return self.nz // 2 + 1

    @property
    def x_slabs(self) -> list[tuple[int, int]]:
        return block_split(self.nx, self.world)

    @property
    def kz_slabs(self) -> list[tuple[int, int]]:
        return block_split(self.nh, self.world)

    def local_voxels(self, rank: int) -> int:
        x0, x1 = self.x_slabs[rank]
        return (x1 - x0) * self.ny * self.nz

    def exchange_elements(self, src: int, dst: int, ncomp: int = 5) -> int:
        """Complex values rank src sends rank dst in one transpose: its x slab
        of dst's kz slab, every ky and component."""
        x0, x1 = self.x_slabs[src]
        k0, k1 = self.kz_slabs[dst]
        return ncomp * (k1 - k0) * self.ny * (x1 - x0)


def _pack_for_x(plan: SlabPlan, rank: int, b_local: torch.Tensor) -> list[torch.Tensor]:
    """Split a rank's B[c][kz][ky][x-slab] into the per-destination blocks."""
    return [b_local[:, k0:k1].contiguous() for (k0, k1) in plan.kz_slabs]


def to_x_lines(plan: SlabPlan, rank: int, b_local: torch.Tensor,
               group=None) -> torch.Tensor:
    """All-to-all from x slabs to kz slabs.  b_local: (ncomp, nh, ny, nx_r)
    complex (this rank's x slab after the y pass).  Returns (ncomp, nk_r, ny,
    nx): this rank's kz slab with complete x lines."""
    ncomp = b_local.shape[0]
    x_slabs, (k0, k1) = plan.x_slabs, plan.kz_slabs[rank]
    assert b_local.shape[1:] == (plan.nh, plan.ny, x_slabs[rank][1] - x_slabs[rank][0])
    send = _pack_for_x(plan, rank, b_local)
    recv = [torch.empty((ncomp, k1 - k0, plan.ny, x1 - x0), dtype=b_local.dtype,
                        device=b_local.device) for (x0, x1) in x_slabs]
    _all_to_all(recv, send, group)
    return torch.cat(recv, dim=3) if recv else b_local.new_empty((ncomp, 0, plan.ny, 0))


def from_x_lines(plan: SlabPlan, rank: int, b_kz: torch.Tensor, group=None) -> torch.Tensor:
    """The inverse all-to-all: (ncomp, nk_r, ny, nx) back to this rank's x
    slab (ncomp, nh, ny, nx_r)."""
    ncomp = b_kz.shape[0]
    x_slabs, kz_slabs = plan.x_slabs, plan.kz_slabs
    x0, x1 = x_slabs[rank]
    send = [b_kz[..., a:b].contiguous() for (a, b) in x_slabs]
    recv = [torch.empty((ncomp, k1 - k0, plan.ny, x1 - x0), dtype=b_kz.dtype,
                        device=b_kz.device) for (k0, k1) in kz_slabs]
    _all_to_all(recv, send, group)
    return torch.cat(recv, dim=1)


def _all_to_all(recv: list, send: list, group) -> None:
    """All-to-all of complex blocks as one flat exchange (all_to_all_single,
    which NCCL and gloo both provide) with per-rank split sizes; empty blocks
    take part with size 0, so every rank makes the same collective call."""
    real = [torch.view_as_real(t).reshape(-1) for t in send]
    sbuf = torch.cat(real) if real else torch.empty(0)
    rsizes = [2 * t.numel() for t in recv]
    rbuf = torch.empty(sum(rsizes), dtype=sbuf.dtype, device=sbuf.device)
    dist.all_to_all_single(rbuf, sbuf, output_split_sizes=rsizes,
                           input_split_sizes=[r.numel() for r in real], group=group)
    off = 0
    for t, n in zip(recv, rsizes):
        torch.view_as_real(t).reshape(-1).copy_(rbuf[off:off + n])
        off += n


def all_reduce_sums(partial: torch.Tensor, group=None) -> torch.Tensor:
    """The reductions of one iteration (the 12 sums of <sigma>, <edot> and the
    two error norms, or the 25 of L0) over all ranks, in FP64."""
    out = partial.to(torch.float64).clone()
    dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
    return out
