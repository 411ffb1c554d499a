"""Many independent cases in one context (the batched launch), bitwise against the
oracle run of each case alone; and against the same cases run one at a time."""
import numpy as np
import pytest

import helpers as H
from multiblockmomentsfv_b200 import solver as sv

pytestmark = pytest.mark.gpu


def test_batch_equals_each_case_alone(oracle_mod):
    cases = sv.batch_workload(seed=5, ncases=10, nmin=8, nmax=40)
    steps = 25
    with sv.BatchSolver(cases) as bs:
        bs.initialise()
        t, ns, nr = bs.steps(0.0, 1.0, max_steps=steps)
        got = [[bs.download(0, k, b) for b in range(len(d.blocks))] for k, (d, _) in enumerate(cases)]
    for k, (d, scn) in enumerate(cases):
        o = oracle_mod.Oracle(d, scn)
        o.initialise()
        t_o, n_o, r_o, _ = o.steps(0.0, 1.0, max_steps=steps)
        assert (t_o, n_o, r_o) == (t[k], ns[k], nr[k]), k
        for b in range(len(d.blocks)):
            H.assert_bitwise(got[k][b], o.get_layer(0, b), f"case {k} block {b}")


def test_batch_cases_finish_independently(oracle_mod):
    """Per-case end times: cases stop at their own tend, the others go on."""
    cases = sv.batch_workload(seed=8, ncases=4, nmin=8, nmax=24)
    tend = np.array([0.01, 0.02, 0.005, 0.03])
    with sv.BatchSolver(cases) as bs:
        bs.initialise()
        t, ns, nr = bs.steps(0.0, tend)
        got = [bs.download(0, k, 0) for k in range(len(cases))]
    for k, (d, scn) in enumerate(cases):
        o = oracle_mod.Oracle(d, scn)
        o.initialise()
        t_o, n_o, r_o, _ = o.steps(0.0, float(tend[k]))
        assert (t_o, n_o) == (t[k], ns[k])
        H.assert_bitwise(got[k], o.get_layer(0, 0), f"case {k}")
