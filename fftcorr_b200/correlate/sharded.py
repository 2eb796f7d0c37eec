"""A survey correlation with its (ell, m) terms split over processes.

Each rank of a torch.distributed process group computes the terms
i % world == rank of the loop over (ell, m) (ell ascending, then m; the loop
of Correlator::correlate_internal, cc/correlate/correlator.h:421-489) on its
own GPU, histograms its share, and one all-reduce (sum) of the FP64
histograms and zero lag gives every rank the full result: the histograms are
linear in the terms.  Bin counts depend only on the geometry and are the same
on every rank, so they are not reduced.  Works on any backend (NCCL with the
tensors on the rank's GPU, gloo on the CPU).
"""
import numpy as np

__all__ = ["owned_terms", "reduce_results", "ShardedCorrelator"]


def owned_terms(maxell, rank, world):
    """Indices (into the (ell, m) loop order) of the terms a rank computes,
    with the (ell, m) of each: [(i, ell, m), ...]."""
    if not (world >= 1 and 0 <= rank < world):
        raise ValueError("term shard needs 0 <= rank < world")
    out, i = [], 0
    for ell in range(0, maxell + 1, 2):
        for m in range(-ell, ell + 1):
            if i % world == rank:
                out.append((i, ell, m))
            i += 1
    return out


def _flat(res):
    return np.concatenate([np.ravel(res["rhist"]), np.ravel(res["khist"]),
                           [res["zerolag"] or 0.0]]).astype(np.float64)


def reduce_results(res, group=None, device=None):
    """Sums the rhist, khist and zerolag of a results() dict over the ranks
    of `group` (one all-reduce); returns a new dict.  `device` is where the
    reduction buffer lives (the rank's GPU for NCCL; None picks cuda for
    NCCL and cpu otherwise)."""
    import torch
    import torch.distributed as dist
    if device is None:
        nccl = dist.get_backend(group) == "nccl"
        device = (torch.device("cuda", torch.cuda.current_device()) if nccl
                  else torch.device("cpu"))
    buf = torch.from_numpy(_flat(res)).to(device)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    flat = buf.cpu().numpy()
    out = dict(res)
    nr, nk = np.size(res["rhist"]), np.size(res["khist"])
    out["rhist"] = flat[:nr].reshape(np.shape(res["rhist"]))
    out["khist"] = flat[nr:nr + nk].reshape(np.shape(res["khist"]))
    out["zerolag"] = float(flat[nr + nk])
    return out


class ShardedCorrelator:
    """Wraps a survey Correlator so that autocorrelate / cross_correlate run
    this rank's share of the (ell, m) terms and return the full tables."""

    def __init__(self, correlator, group=None):
        import torch.distributed as dist
        self.correlator = correlator
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        correlator.set_term_shard(self.rank, self.world)

    def _tables(self, squeeze):
        c = self.correlator
        res = reduce_results(c.results(), self.group)
        return c._power_spectrum(res, squeeze), c._correlation(res, squeeze)

    def results(self):
        return reduce_results(self.correlator.results(), self.group)

    def autocorrelate(self, grid, squeeze=True):
        self.correlator.autocorrelate(grid, squeeze)
        return self._tables(squeeze)

    def cross_correlate(self, grid1, grid2=None, squeeze=True):
        self.correlator.cross_correlate(grid1, grid2, squeeze)
        return self._tables(squeeze)
