"""The autotuner (scout_b200/autotune.py): every knob configuration leaves the same solution,
and the configuration it picks is no slower than the defaults when measured again."""
import numpy as np
import pytest

import scout_b200 as sb
from gpu_util import stream
from scout_b200 import autotune as at

pytestmark = pytest.mark.gpu


def _batches(off, adj):
    small = stream(off, adj, sb.STREAM_PREFERENTIAL, 2000, 3, seed=131)
    large = stream(off, adj, sb.STREAM_PREFERENTIAL, 40000, 3, seed=132)
    return [small[0], large[0], small[1], large[1], small[2], large[2]]


@pytest.mark.parametrize("problem", ["bfs", "cc"])
def test_autotuner_choice_is_exact_and_no_slower(rmat16, problem):
    g, (off, adj) = rmat16
    init = g.init_state(problem, 0)
    batches = _batches(off, adj)
    r = at.tune_single(problem, off, adj, init, batches, blocks=(1, 4), chunks=(8, 10), lanes=(0, 32, 1024))
    crcs = {row["solution_crc"] for row in r["table"]}
    assert len(crcs) == 1   # tune_single raises otherwise; the table says so too
    assert any({k: row[k] for k in at.DEFAULT} == at.DEFAULT for row in r["table"])
    best = r["best"]
    # measured again, best of three: the choice within noise of the defaults or faster
    t_best = min(at.run_config(problem, off, adj, init, batches, best)[0] for _ in range(3))
    t_def = min(at.run_config(problem, off, adj, init, batches, at.DEFAULT)[0] for _ in range(3))
    assert t_best <= 1.25 * t_def + 0.3, (best, t_best, t_def)


def test_lanes_per_vertex_values(rmat16):
    g, (off, adj) = rmat16
    init = g.init_state("bfs", 0)
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        ctx.upload("bfs", init)
        with pytest.raises(sb.ScoutError):
            ctx.repair("bfs", np.zeros((0, 2), np.int32), sched={"lanes_per_vertex": 48})
        with pytest.raises(sb.ScoutError):
            ctx.repair("bfs", np.zeros((0, 2), np.int32), sched={"frontier": 7})
