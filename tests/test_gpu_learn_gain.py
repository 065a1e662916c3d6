"""What the trained proposal network gains over the plain uniform sampler.

The shipped network (kino-pax-fork_b200/weights/quad_proposal.npz, trained on the GPU by the
library's own FP32 kernels from plain-planner trees of 512 training scenes) against the plain
planner, on held-out scenes of the learned family (building scenes with 200-2000 boxes, start and
goal 25-45 m apart).  Plans are deterministic (Philox streams, fixed seeds), so these are
regression checks of the measured gain, not statistical trials: with epsilon = 0.2 the learned
planner solves more of the 256 held-out scenes and gets closer to the goal (median over scenes of
the tree's closest approach)."""
import pytest

import kpax_learn as L

pytestmark = pytest.mark.gpu


def test_learned_planner_beats_plain_on_held_out_scenes(cuda):
    cfg = L.quad_config()
    net = L.load_network()
    seeds = [L.EVAL_SEED0 + i for i in range(256)]
    plain = L.summarize(L.evaluate(seeds, cfg, progress=True))
    learned = L.summarize(L.evaluate(seeds, cfg, net, 0.2, progress=True))
    print({"plain": plain, "learned": learned})
    assert learned["success"] > plain["success"]
    assert learned["closest_median"] < plain["closest_median"]
