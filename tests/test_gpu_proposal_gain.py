"""What the learned proposal gains (GPU, end to end).

A network is trained from scratch on the GPU with the library's own kernels
on (state features, u*) pairs that plain MPPI at K = 16384, H = 64
produces on the batched unicycle problem, then judged by plain MPPI's
closed-loop cost on held-out agents (other seeds: other starts, goals,
obstacles and sigmas):

  proposal-MPPI at K = 256 (half of the samples around the prediction)
    - beats plain MPPI at the same K = 256 by at least 3 %, and
    - stays within 2 % of plain MPPI at K = 4096 (16x the rollouts).
The executed cost is the model's stage cost along the driven trajectory plus
its terminal cost (models.unicycle_executed_cost).  A smaller training set
than the configuration's 1.2e6 pairs keeps the test short.
"""
from __future__ import annotations

import numpy as np
import pytest

from mppi_metal_b200 import models

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    from mppi_metal_b200 import proposal as P
    net, hist, pairs = P.train_unicycle_proposal(seeds=(300, 301), agents=512, epochs=15,
                                                 batch=8192)
    assert pairs == 2 * 512 * 300
    assert hist[-1] < hist[0]  # the loss went down
    return net


def test_proposal_gains_over_plain_mppi(trained):
    from mppi_metal_b200 import proposal as P
    w = models.unicycle_batch(seed=310, N=128, K=4096, H=64, T=300)
    plain_4096 = P.closed_loop(w)["cost"].mean()
    plain_256 = P.closed_loop(w, sample_count=256)["cost"].mean()
    prop_256 = P.closed_loop(w, trained, 128, sample_count=256)["cost"].mean()
    assert prop_256 <= 0.97 * plain_256, (prop_256, plain_256)
    assert prop_256 <= 1.02 * plain_4096, (prop_256, plain_4096)


@pytest.fixture(scope="module")
def trained_quadrotor():
    from mppi_metal_b200 import proposal as P
    net, hist, pairs = P.train_quadrotor_proposal(seeds=(510, 511), agents=128,
                                                  sample_count=16384, epochs=30)
    assert pairs == 2 * 128 * 100
    return net


def test_quadrotor_proposal_gains_over_plain_mppi(trained_quadrotor):
    """The large-rollout quadrotor problem: K = 4096 with 1024 samples around
    a 60-step prediction, against plain MPPI at the same K on held-out
    quadrotors (other waypoints and obstacle fields)."""
    from mppi_metal_b200 import proposal as P
    w = models.quadrotor_batch(seed=610, N=32, K=65536, H=100, T=100)
    plain_4096 = P.closed_loop(w, sample_count=4096)["cost"].mean()
    prop_4096 = P.closed_loop(w, trained_quadrotor, 1024, sample_count=4096)["cost"].mean()
    assert prop_4096 <= 0.985 * plain_4096, (prop_4096, plain_4096)
