"""Round formation of the batched multi-stream engine (host logic, no GPU)."""
import numpy as np

import scout_b200 as sb


def test_rounds_keep_stream_order_and_cap():
    r = np.random.default_rng(3)
    arrivals = [(int(r.integers(0, 7)), np.zeros((int(r.integers(1, 50)), 2), np.int32)) for _ in range(300)]
    for i, (s, b) in enumerate(arrivals):
        b[:, 0] = i   # tag each batch with its arrival index
    rounds = sb.form_rounds(arrivals, 100)
    seen = {}
    for k, rd in enumerate(rounds):
        sids = [s for s, _ in rd]
        assert len(sids) == len(set(sids)), "a stream appears twice in a round"
        tot = sum(len(b) for _, b in rd)
        assert tot <= 100 or len(rd) == 1
        for s, b in rd:
            seen.setdefault(s, []).append((k, int(b[0, 0])))
    assert sum(len(v) for v in seen.values()) == len(arrivals)
    for s, lst in seen.items():
        ks = [k for k, _ in lst]
        idx = [i for _, i in lst]
        assert ks == sorted(ks) and len(set(ks)) == len(ks)
        assert idx == sorted(idx), "a stream's batches left arrival order"


def test_oversized_batch_forms_its_own_round():
    rounds = sb.form_rounds([(0, np.zeros((5, 2))), (1, np.zeros((500, 2))), (2, np.zeros((3, 2)))], 100)
    assert [[s for s, _ in rd] for rd in rounds] == [[0, 2], [1]]
