"""Term-sharded survey correlation on CPU: two gloo ranks each take their
share of the (ell, m) terms (here computed by the oracle, standing in for
the GPU), and fftcorr_b200.correlate.sharded.reduce_results sums the shares
in one all-reduce.  The sum must equal the unsharded correlation."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _field(shape, seed):
    return np.random.default_rng(seed).standard_normal(shape)


ARGS = (12.0, np.array([-100.0, 250.0, -300.0]), 2, 70.0, 10.0, 0.12, 0.02, 4)


def _rank(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from oracle import fc_oracle as O
    from fftcorr_b200.correlate.sharded import owned_terms, reduce_results
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}",
                            rank=rank, world_size=world)
    try:
        grid = _field((16, 16, 16), 5)
        terms = {i for i, _, _ in owned_terms(4, rank, world)}
        part = O.survey_correlate(grid, *ARGS, terms=terms)
        q.put((rank, reduce_results(part)))
    finally:
        dist.destroy_process_group()


class _OracleShare:
    """Stands in for a survey Correlator on CPU: the oracle computes the
    terms this rank owns."""

    def __init__(self):
        from fftcorr_b200.correlate.correlator import BaseCorrelator
        self._power_spectrum = BaseCorrelator._power_spectrum.__get__(self)
        self._correlation = BaseCorrelator._correlation.__get__(self)
        self.rank, self.world = 0, 1

    def set_term_shard(self, rank, world):
        self.rank, self.world = rank, world

    def autocorrelate(self, grid, squeeze=True):
        from oracle import fc_oracle as O
        from fftcorr_b200.correlate.sharded import owned_terms
        terms = {i for i, _, _ in owned_terms(4, self.rank, self.world)}
        self.res = O.survey_correlate(grid, *ARGS, terms=terms)

    def results(self):
        return self.res


def _rank_tables(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from fftcorr_b200.correlate.sharded import ShardedCorrelator
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}",
                            rank=rank, world_size=world)
    try:
        sc = ShardedCorrelator(_OracleShare())
        ps, xi = sc.autocorrelate(_field((16, 16, 16), 5))
        q.put((rank, np.asarray(xi["xi"]), np.asarray(ps["ps"])))
    finally:
        dist.destroy_process_group()


def test_sharded_correlator_tables_on_two_gloo_ranks():
    import sys
    sys.path.insert(0, ROOT)
    from oracle import fc_oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_tables, args=(r, 2, port, q))
             for r in range(2)]
    for p in procs:
        p.start()
    res = {r: (xi, ps) for r, xi, ps in (q.get(timeout=300) for _ in procs)}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = O.survey_correlate(_field((16, 16, 16), 5), *ARGS)
    with np.errstate(divide="ignore", invalid="ignore"):
        xi_ref = np.transpose(full["rhist"] / full["rcounts"])
        ps_ref = np.transpose(full["khist"] / full["kcounts"])
    for rank in (0, 1):
        xi, ps = res[rank]
        np.testing.assert_allclose(xi, xi_ref, rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(ps, ps_ref, rtol=1e-12, atol=1e-300)


def test_owned_terms_partition_the_loop():
    import sys
    sys.path.insert(0, ROOT)
    from fftcorr_b200.correlate.sharded import owned_terms
    for world in (1, 2, 3, 8):
        got = sorted(t for r in range(world) for t in owned_terms(4, r, world))
        assert [i for i, _, _ in got] == list(range(15))
        assert [(ell, m) for _, ell, m in got][:6] == [
            (0, 0), (2, -2), (2, -1), (2, 0), (2, 1), (2, 2)]
    with pytest.raises(ValueError):
        owned_terms(4, 2, 2)


def test_two_gloo_ranks_reduce_to_the_full_correlation():
    import sys
    sys.path.insert(0, ROOT)
    from oracle import fc_oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = O.survey_correlate(_field((16, 16, 16), 5), *ARGS)
    for rank in (0, 1):
        got = res[rank]
        np.testing.assert_array_equal(got["rcounts"], full["rcounts"])
        np.testing.assert_array_equal(got["kcounts"], full["kcounts"])
        for k in ("rhist", "khist"):
            scale = np.max(np.abs(full[k]))
            assert np.max(np.abs(got[k] - full[k])) <= 1e-12 * scale
        assert got["zerolag"] == pytest.approx(full["zerolag"], rel=1e-12)
