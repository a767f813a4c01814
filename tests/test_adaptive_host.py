"""Host logic of turbchannel_b200.run_adaptive (no GPU): a fake solver whose CFL number is
proportional to tau records the calls, so the driver's decisions can be checked against
the reference's rule (staggered/main.cpp:361-370): above cfl_max halve tau until the
estimate is below it, below cfl_min enlarge it by 1.5, and restart the BDF order at 1
after every change."""
import numpy as np

import turbchannel_b200 as tb


class FakeSolver:
    def __init__(self, speed):
        self.speed = speed  # CFL = speed * tau
        self.calls = []

    def Step(self, t, tau, cur, order):
        self.calls.append(("step", round(t, 12), tau, cur, order))

    def run_graph(self, tau, cur, nsteps, check_every, cfl_mode, cfl_min, cfl_max):
        cfl = self.speed * tau
        done = check_every if not (cfl_min <= cfl <= cfl_max) else nsteps
        self.calls.append(("graph", tau, cur, nsteps, done))
        return done, cfl


def test_halves_tau_above_cfl_max_and_restarts_order():
    S = FakeSolver(speed=100.0)  # CFL 2.0 at tau 0.02
    t, tau, cur = tb.run_adaptive(S, 0.0, 0.02, 1, 40, 0.1, 0.5, check_every=4)
    # two ramp steps, a graph that stops at its first check (CFL 2 > 0.5), tau / 4 (CFL 0.5)
    assert S.calls[0] == ("step", 0.0, 0.02, 1, 1) and S.calls[1][4] == 2
    g = S.calls[2]
    assert g[0] == "graph" and g[1] == 0.02 and g[2] == 3 and g[4] == 4
    assert tau == 0.005
    # order restart after the change: orders 1, 2 by tc_step, then a graph at the new tau
    assert [c[4] for c in S.calls[3:5]] == [1, 2] and S.calls[3][2] == 0.005
    assert S.calls[5][0] == "graph" and S.calls[5][1] == 0.005
    steps = sum(1 for c in S.calls if c[0] == "step") + sum(c[4] for c in S.calls if c[0] == "graph")
    assert steps == 40
    assert np.isclose(t, 2 * 0.02 + 4 * 0.02 + 34 * 0.005)
    assert cur == (1 + 40) % 4


def test_enlarges_tau_below_cfl_min():
    S = FakeSolver(speed=1.0)  # CFL 0.02 at tau 0.02, below cfl_min 0.1
    t, tau, cur = tb.run_adaptive(S, 0.0, 0.02, 0, 24, 0.1, 0.5, check_every=4)
    assert tau > 0.02
    taus = [c[2] if c[0] == "step" else c[1] for c in S.calls]
    assert all(b >= a for a, b in zip(taus, taus[1:]))  # tau only grows here
    assert sum(1 for c in S.calls if c[0] == "step") + sum(c[4] for c in S.calls if c[0] == "graph") == 24


def test_tail_steps_below_check_every_use_tc_step():
    S = FakeSolver(speed=10.0)  # CFL 0.2, inside [0.1, 0.5]: one graph, then the tail
    tb.run_adaptive(S, 0.0, 0.02, 0, 2 + 8 + 3, 0.1, 0.5, check_every=4)
    kinds = [c[0] for c in S.calls]
    assert kinds == ["step", "step", "graph", "step", "step", "step"]
    assert S.calls[2][3] == 8 and [c[4] for c in S.calls[3:]] == [3, 3, 3]
