"""Bounded runs of the persistent kernels: a time budget and a host cancel word.

The EA campaign kernel and the work-item kernels poll a ``RunControl``
between PT steps or measurements.  These tests make the budget run out (a
tiny budget) and set the cancel word from the host while a long launch is in
flight; in both cases the kernel must return by itself, early, with the
matching status, and the device must stay usable.  Nothing faults or hangs:
the kernels only stop doing work.  A generous budget must change nothing.
"""

from __future__ import annotations

import time

import numpy as np
import pytest
import torch

from critmc_b200 import Ising, cubic, square
from critmc_b200.control import CANCELLED, OK, TIMEOUT, RunControl, RunStopped
from critmc_b200.glass import EdwardsAnderson, MultiSizeCampaign, SpinGlassCampaign, geometric_temperatures
from critmc_b200.items import ItemRun, run_items

pytestmark = pytest.mark.gpu


def _campaign(cuda, sizes, n_samples, seed=0):
    temps = geometric_temperatures(0.5, 2.0, 32)
    camps = [SpinGlassCampaign([EdwardsAnderson(cubic(L), disorder="bimodal", seed=seed + 1000 * L + i)
                                for i in range(n_samples)], temps,
                               seeds=[seed + 7000 * L + i for i in range(n_samples)], device=cuda)
             for L in sizes]
    return MultiSizeCampaign(camps)


def _device_seconds(fn) -> float:
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) * 1e-3


def test_generous_budget_changes_nothing(cuda):
    a = _campaign(cuda, (4, 6, 8), 4)
    b = _campaign(cuda, (4, 6, 8), 4)
    ctl = RunControl(cuda).arm(60.0)
    ra = a.run(6)
    rb = b.run(6, control=ctl)
    assert ctl.status() == OK
    for runs_a, runs_b in zip(ra, rb):
        for x, y in zip(runs_a, runs_b):
            np.testing.assert_array_equal(x.acc, y.acc)
            np.testing.assert_array_equal(x.trips, y.trips)
    for ca, cb in zip(a.campaigns, b.campaigns):
        np.testing.assert_array_equal(ca.spins(), cb.spins())


def test_campaign_returns_on_its_own_when_the_budget_runs_out(cuda):
    mc = _campaign(cuda, (16,), 148)  # 2^16 - 1 steps of 148 L=16 samples: over a second unbounded
    ctl = RunControl(cuda).arm(2e-3)
    secs = _device_seconds(lambda: mc.launch(16, control=ctl))
    assert ctl.wait() == TIMEOUT
    assert secs < 0.25, f"the bounded launch took {secs:.3f} s"
    with pytest.raises(RunStopped):
        _campaign(cuda, (16,), 8).run(16, control=ctl.arm(1e-3))
    # the device is still usable: a bounded run with room to finish gives the unbounded result
    a, b = _campaign(cuda, (4, 8), 3, seed=5), _campaign(cuda, (4, 8), 3, seed=5)
    ra, rb = a.run(4), b.run(4, control=ctl.arm(30.0))
    assert ctl.status() == OK
    np.testing.assert_array_equal(ra[1][2].acc, rb[1][2].acc)


def test_host_cancel_stops_a_launch_in_flight(cuda):
    mc = _campaign(cuda, (16,), 148, seed=3)
    ctl = RunControl(cuda).arm(None)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    mc.launch(16, control=ctl)
    e1.record()
    time.sleep(0.05)
    assert ctl.status() == OK  # still running, nothing stopped yet
    ctl.cancel()
    assert ctl.wait() == CANCELLED
    secs = e0.elapsed_time(e1) * 1e-3
    assert secs < 0.5, f"the cancelled launch took {secs:.3f} s"


def test_work_items_stop_on_budget_and_on_cancel(cuda):
    model = Ising(square(1024, 64))
    rng = np.random.default_rng(4)

    def items():
        out = []
        for i in range(64):
            s0 = model.initial_state("random", rng)
            ch = model.to_device(s0, np.random.default_rng(100 + i), cuda)
            # 10,000 measurements of 20 sweeps: several tenths of a second unbounded
            out.append(ItemRun(model, ch, model.begin(s0), 0.44, np.array([[0, 20]]), 10000))
        return out

    ctl = RunControl(cuda).arm(2e-3)
    runs = items()
    secs = _device_seconds(lambda: run_items(runs, cuda, control=ctl))
    assert ctl.wait() == TIMEOUT
    assert secs < 0.15, f"the bounded item launch took {secs:.3f} s"
    runs = items()
    ctl.arm(None)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run_items(runs, cuda, control=ctl)
    e1.record()
    time.sleep(0.05)
    ctl.cancel()
    assert ctl.wait() == CANCELLED
    secs = e0.elapsed_time(e1) * 1e-3
    assert secs < 0.2, f"the cancelled item launch took {secs:.3f} s"
