"""critmc_run_items inside a captured CUDA graph: one block per item and
thread-block-cluster teams, the descriptors copied from pinned staging, the
launch groups forked to the library's streams and joined back.  Replaying the
graph once gives, bit for bit, what the same call gives run directly."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from critmc_b200.items import CritmcItem, ItemRun, launch_items

from test_gpu_items import MIX, _assert_same, _pair

pytestmark = pytest.mark.gpu


def test_items_call_replays_from_a_cuda_graph(cuda):
    sel = [0, 3, 8, 11, 12, 15]
    teams = [1, 4, 1, 8, 2, 1]
    # warm-up call: library streams, kernel attributes and team capacities exist before capture
    # (the runs own the items' output buffers: they must outlive the launch)
    warm = [_pair(100 + i, MIX[i][0], MIX[i][1], cuda) for i in sel]
    warm_runs = [ItemRun(m, c[0], r[0], MIX[i][3], np.array(MIX[i][2]), 2, team=t)
                 for (m, c, r), i, t in zip(warm, sel, teams)]
    buf = launch_items([w.item for w in warm_runs], cuda, None)
    torch.cuda.synchronize()
    del warm_runs

    pairs = [_pair(i, MIX[i][0], MIX[i][1], cuda) for i in sel]
    direct = [ItemRun(m, c[0], r[0], MIX[i][3], np.array(MIX[i][2]), 5, team=t)
              for (m, c, r), i, t in zip(pairs, sel, teams)]
    graphed = [ItemRun(m, c[1], r[1], MIX[i][3], np.array(MIX[i][2]), 5, team=t)
               for (m, c, r), i, t in zip(pairs, sel, teams)]
    staging = torch.empty(len(sel) * ctypes.sizeof(CritmcItem), dtype=torch.uint8, pin_memory=True)
    gbuf = torch.empty_like(buf)
    arr = (CritmcItem * len(graphed))(*[g.item for g in graphed])

    s = torch.cuda.Stream(cuda)
    s.wait_stream(torch.cuda.current_stream(cuda))
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        launch_items(arr, cuda, gbuf, staging=staging, stream=s.cuda_stream)
    graph.replay()
    launch_items([d.item for d in direct], cuda, buf)
    torch.cuda.synchronize()
    for (model, chains, _), d, g in zip(pairs, direct, graphed):
        _assert_same(d.finish(), g.finish())
        np.testing.assert_array_equal(chains[0].fetch(), chains[1].fetch())
