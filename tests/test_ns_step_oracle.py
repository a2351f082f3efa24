"""The full-step oracle (the reference's stable quick-start pipeline composed
from this repository's operator oracles) against six steps of the
reference itself (tests/golden/c1_golden.npz, written by
tests/golden/make_golden.py): psi, u, v and p bit for bit."""

import os

import numpy as np

from oracle import step as ostep
from oracle.ns_step import QuickStartStep

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "c1_golden.npz"))


def test_quickstart_steps_match_reference():
    s = QuickStartStep((64, 64), (1.0, 1.0), G["psi0"])
    for k in range(6):
        dt = float(G[f"s{k}/dt"])
        if k > 0:   # the reference's CFL time step from the previous state (convective + capillary bounds)
            assert ostep.cfl_dt(s.vel, s.mu, s.rho, (1.0, 1.0), (64, 64), 0.3, We=10.0, rho_ratio=0.1) == dt
        s.step(dt)
        np.testing.assert_array_equal(s.psi, G[f"s{k}/psi"])
        np.testing.assert_array_equal(s.vel[0], G[f"s{k}/u"])
        np.testing.assert_array_equal(s.vel[1], G[f"s{k}/v"])
        np.testing.assert_array_equal(s.p, G[f"s{k}/p"])
