"""The profiling cases in raptr_b200/profile_case.py: the column-slab case
orders its rows as the library orders a matrix it built, and runs."""
import pytest

from raptr_b200 import config as cfg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def test_channel_order_matches_the_library(rlib, torch):
    from raptr_b200 import profile_case as pc

    g = cfg.SMALL
    ctx = rlib.Context(g, 0)
    lst = torch.arange(g.n_channels, dtype=torch.int32, device="cuda")
    A = ctx.build(lst, 20, 7)
    A.transpose()
    assert A.row_order is not None
    order, rank = pc.channel_order(torch, g, g.n_channels)
    assert torch.equal(order, A.row_order)
    assert torch.equal(rank, A.row_rank)


def test_column_slab_case_runs(rlib, torch, capsys):
    from raptr_b200 import profile_case as pc

    w = cfg.WORKLOADS["small"]
    ctx = rlib.Context(w["geom"], 0)
    pc.column_slab_case(rlib, torch, ctx, w["geom"], w, 18, 22, 40000)
    out = capsys.readouterr().out
    assert "column-slab case" in out
    assert abs(float(out.rsplit("x sum", 1)[1]) - 1.0) < 1e-4
