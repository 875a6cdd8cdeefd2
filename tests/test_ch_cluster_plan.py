"""Which grids the cluster-resident integrator takes (host logic only, no
GPU work): the cluster's CTA count for a grid, storage type, order and
integrator, 0 where the state does not fit one cluster's shared memory."""
import gridcalc_b200 as gc
import torch


def test_capacity_query():
    f64, f32 = torch.float64, torch.float32
    assert gc.ch_cluster_ctas(gc.Grid(128, 128, 1), f64, 2) == 8
    assert gc.ch_cluster_ctas(gc.Grid(240, 240, 1), f64, 2) == 16
    assert gc.ch_cluster_ctas(gc.Grid(256, 256, 1), f64, 2) == 0
    assert gc.ch_cluster_ctas(gc.Grid(256, 256, 1), f32, 2) > 0
    assert gc.ch_cluster_ctas(gc.Grid(1024, 1024, 1), f64, 2) == 0
    assert gc.ch_cluster_ctas(gc.Grid(64, 64, 64), f64, 2) == 0       # 3-D: per-stage kernels
    assert gc.ch_cluster_ctas(gc.Grid(5, 3, 1), f64, 2) == 3           # fewer rows than 8: one row per CTA
    assert gc.ch_cluster_ctas(gc.Grid(128, 128, 1), f64, 2, gc.ExplicitEuler) == 8
    assert gc.ch_cluster_ctas(gc.Grid(128, 128, 1), f64, 3) == 0       # not an order
