"""k-point parallelism across processes: one process per GPU, the k-points of an SCF run dealt out
to the ranks, and the two exchanges the SCF iteration needs.

The reference runs its k-points on worker threads that share one density buffer
(kpoint/workers.zig:133-180, kpoint/density.zig): each worker solves its k-points and adds its
bands into the density.  Across GPUs the same work splits by k-point with no communication during
the eigensolves.  After them every rank holds a partial density (its own k-points' bands) and the
eigenvalues of its own k-points; one sum-reduction of each gives every rank the full density and
the full eigenvalue table, from which the occupations (fermi_level.zig), the energy and the mixing
step are computed redundantly and identically on every rank.  The wave functions stay on the rank
that owns their k-point, where they warm-start the next iteration's solve.

The collectives go through ``torch.distributed``: NCCL (device tensors) on GPU ranks, gloo (host
tensors) on CPU ranks.  Both reductions are small next to the solves (the density is N doubles,
the eigenvalue table nk x nbands doubles)."""
from __future__ import annotations

import numpy as np


def deal_kpoints(nk: int, size: int, costs=None) -> list:
    """Owner rank of each of ``nk`` k-points.  With ``costs`` (e.g. plane waves per k-point) the
    k-points go largest first to the least-loaded rank; without, in contiguous equal blocks."""
    if size <= 1:
        return [0] * nk
    if costs is None:
        return [k * size // nk for k in range(nk)]
    load = [0.0] * size
    owner = [0] * nk
    for k in sorted(range(nk), key=lambda i: (-float(costs[i]), i)):
        r = min(range(size), key=lambda j: (load[j], j))
        owner[k] = r
        load[r] += float(costs[k])
    return owner


class KpointComm:
    """The process group an SCF run's k-points are dealt over.

    ``group`` is a ``torch.distributed`` process group (None = the default group).  Reductions move
    numpy arrays through a float64 tensor on ``device`` (the rank's GPU for NCCL, the host for
    gloo); every rank receives the same bits, so the replicated SCF state stays identical."""

    def __init__(self, group=None, device=None):
        import torch
        import torch.distributed as dist

        self._dist = dist
        self._torch = torch
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        backend = dist.get_backend(group)
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
        self.device = torch.device(device)

    def sum(self, a):
        """Element-wise sum over the ranks (all-reduce), returned to every rank: numpy arrays come
        back as numpy, tensors as tensors on their own device (reduced in place on the group's
        device when they are already there: NCCL on GPU ranks)."""
        torch = self._torch
        if isinstance(a, torch.Tensor):
            t = a.to(self.device, dtype=torch.float64).contiguous()
            if t.data_ptr() == a.data_ptr():
                t = t.clone()
            self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM, group=self.group)
            return t.to(a.device)
        a = np.ascontiguousarray(a, dtype=np.float64)
        t = torch.from_numpy(a.copy()).to(self.device)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM, group=self.group)
        return t.cpu().numpy().reshape(a.shape)

    def barrier(self):
        self._dist.barrier(group=self.group)


class SerialComm:
    """A one-rank stand-in with the KpointComm interface (every k-point local, sums are copies)."""

    rank = 0
    size = 1

    def sum(self, a):
        if hasattr(a, "clone"):
            return a.clone()
        return np.array(a, dtype=np.float64, copy=True)

    def barrier(self):
        pass
