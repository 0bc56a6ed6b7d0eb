"""Host watchdog: a wait for a call's results with a timeout polls the call's
CUDA event (cudaEventQuery) and raises PrrtcTimeout instead of blocking for
good.  The CPU test drives the wait with fake events -- one that completes
after a few polls, one that never completes -- so no GPU is stopped to test it;
the GPU test times out a plan that is still running, then collects it."""
from __future__ import annotations

import time

import numpy as np
import pytest


class FakeEvent:
    def __init__(self, polls_until_done: int | None):
        self.left, self.polls, self.synced = polls_until_done, 0, False

    def query(self) -> bool:
        self.polls += 1
        return self.left is not None and self.polls > self.left

    def synchronize(self) -> None:
        self.synced = True


def test_wait_returns_when_the_event_completes():
    from prrtc_b200 import _lib

    ev = FakeEvent(5)
    _lib.wait_event(ev, 10.0, "test")
    assert ev.polls == 6 and not ev.synced


def test_wait_without_timeout_blocks_on_the_event():
    from prrtc_b200 import _lib

    ev = FakeEvent(None)
    _lib.wait_event(ev, None, "test")
    assert ev.synced and ev.polls == 0


def test_wait_that_never_completes_raises_after_the_timeout():
    from prrtc_b200 import PrrtcError, PrrtcTimeout, _lib

    ev = FakeEvent(None)
    t0 = time.monotonic()
    with pytest.raises(PrrtcTimeout, match="not complete after 0.05 s"):
        _lib.wait_event(ev, 0.05, "planner results")
    dt = time.monotonic() - t0
    assert 0.05 <= dt < 1.0 and ev.polls >= 2
    assert issubclass(PrrtcTimeout, PrrtcError)


@pytest.mark.gpu
def test_batch_results_time_out_then_complete(cuda, orc):
    """A batch of unsolvable problems (start configuration more than 2 cm deep
    in an obstacle, so no edge leaves it) runs to its iteration limit;
    results(timeout_s=0) raises PrrtcTimeout while it runs, and the same pending
    batch then returns its results -- every problem unsolved -- with no timeout."""
    import torch

    from conftest import make_problem
    from prrtc_b200 import PrrtcTimeout, prrtc_plan_batch_async

    pr = make_problem("spheres16", 31)
    sc = orc.Scene(pr.context, pr.dim)
    rng = np.random.default_rng(31)
    while True:
        bad = rng.uniform(pr.lower, pr.upper).astype(np.float32)
        if sc.in_collision(bad) and sc.min_distance(bad) < -0.02:
            break
    B = 64
    p = prrtc_plan_batch_async(np.repeat(bad[None], B, 0), np.repeat(pr.goals[:1][None], B, 0),
                               max_iterations=5000, num_new_samples=2, max_nodes=65536, min_vals=pr.lower,
                               max_vals=pr.upper, collision_context=pr.context, device=cuda)
    with pytest.raises(PrrtcTimeout):
        p.results(timeout_s=0.0)
    out = p.results()
    torch.cuda.synchronize()
    assert len(out) == B and not any(r.solved for r in out) and all(r.path is None for r in out)
