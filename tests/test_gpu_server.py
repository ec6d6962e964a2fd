"""Request loop with continuous batching (qs_server_*)."""
import numpy as np
import pytest

from oracle.pyoracle import OracleState
from qpanda_b200 import FusionPlan, Server, StateVector, circuits
from qpanda_b200.capi import QSError

pytestmark = pytest.mark.gpu


def requests(seed, count=12):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        q = int(rng.choice([6, 9, 11, 12, 13, 15, 16]))
        g = circuits.random_layers(q, int(rng.integers(2, 7)), 100 * seed + k, iswap_frac=0.1)
        kind = "shots" if k % 2 == 0 else "probs"
        u = rng.uniform(size=(64, q)) if kind == "shots" else None
        out.append((q, g, kind, u))
    return out


def collect(srv, ids, reqs):
    res = []
    for rid, (q, g, kind, u) in zip(ids, reqs):
        srv.wait(rid)
        res.append(srv.shots(rid).copy() if kind == "shots" else srv.fetch_probs(rid))
        srv.release(rid)
    return res


def test_result_same_alone_and_in_the_mix(need_gpu):
    reqs = requests(1)
    alone = []
    s1 = Server(slots=1)
    for q, g, kind, u in reqs:
        rid = s1.submit(q, g, kind, u)
        alone += collect(s1, [rid], [(q, g, kind, u)])
    s1.close()
    s4 = Server(slots=4)
    ids = [s4.submit(q, g, kind, u) for q, g, kind, u in reqs]     # all in flight together
    mix = collect(s4, ids, reqs)
    assert s4.stats()["max_concurrent"] >= 2
    s4.close()
    for (q, g, kind, u), a, m in zip(reqs, alone, mix):
        assert np.array_equal(a, m), (q, kind)                     # bitwise, not just within tolerance
        if kind == "probs":
            o = OracleState(q)
            o.apply(g)
            assert np.abs(a - o.probs()).max() < 1e-5
        else:
            sv = StateVector(q, "c64")
            if q >= 12:
                FusionPlan(q, g).apply(sv)
            else:
                sv.apply(g)
            assert np.array_equal(a, sv.sample(np.arange(q, dtype=np.int32), u))


def test_admission_by_footprint_and_error_isolation(need_gpu):
    # room for one 20-qubit request at a time (8 MB state + 64 MB scratch + 8 MB probs)
    srv = Server(budget_bytes=100 << 20, slots=4)
    with pytest.raises(QSError) as e:
        srv.submit(24, circuits.random_layers(24, 1, 0), "probs")
    assert e.value.code == -3
    bad = circuits.make_gates([("CNOT", (3, 3))])
    good = [circuits.random_layers(20, 2, k) for k in range(3)]
    ids = [srv.submit(20, good[0], "probs"), srv.submit(20, bad, "probs"), srv.submit(20, good[1], "probs"),
           srv.submit(20, good[2], "probs")]
    srv.wait(ids[0])
    with pytest.raises(QSError):
        srv.wait(ids[1])
    for k in (2, 3):
        srv.wait(ids[k])
        o = OracleState(20)
        o.apply(good[k - 1])
        assert np.abs(srv.fetch_probs(ids[k]) - o.probs()).max() < 1e-5
        srv.release(ids[k])
    srv.release(ids[0])
    srv.release(ids[1])
    assert srv.stats()["max_concurrent"] == 1                       # the budget serialised them
    srv.close()


def test_destroy_with_queued_requests(need_gpu):
    srv = Server(slots=1)
    for k in range(6):
        srv.submit(22, circuits.random_layers(22, 8, k), "probs")
    srv.close()                                                       # queued ones end, running one finishes
