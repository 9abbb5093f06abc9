"""Batched and served forms (dl_session_*, dl_run_batch) on the GPU.

Every instance of a union session must give exactly what the plain engine
gives on the same edges: rows in the reference's file order, iteration count,
per-iteration delta sizes, and for WCC the labels and the largest component.
The same instance must give the same result alone and in any mix, whatever
iteration it was admitted at."""
import numpy as np
import pytest

from mnmgdatalog_b200 import graphs

pytestmark = pytest.mark.gpu


def _instances(prog: str, seed: int = 0):
    """Instances of uneven sizes, including the edge cases of the plain tests."""
    rng = np.random.default_rng(seed)
    out = [
        np.array([[1, 2]], np.int32),
        np.array([[5, 5]], np.int32),
        np.array([[1, 2], [2, 1]], np.int32),
        np.array([[1, 2], [1, 2], [2, 3], [2, 3], [3, 1]], np.int32),
        np.array([[-2**31, 2**31 - 1], [2**31 - 1, 0], [0, -2**31]], np.int32),
        np.zeros((0, 2), np.int32),
        rng.integers(0, 300, (900, 2)).astype(np.int32),
        np.stack([np.arange(0, 400), np.arange(1, 401)], 1).astype(np.int32),
    ]
    if prog == "tc":
        out += [graphs.dag(n=n, extra=n // 3, seed=seed + i) for i, n in enumerate((300, 1200, 4000, 700))]
    elif prog == "sg":
        out += [graphs.lattice3d(side=s, seed=seed + s) for s in (6, 11, 15)]
    else:
        out += [graphs.chung_lu(n=n, m=3 * n, gamma=2.3, seed=seed + i) for i, n in enumerate((500, 3000, 9000))]
        out += [np.concatenate([graphs.dag(n=800, seed=seed), graphs.dag(n=800, seed=seed + 1) + 1000])]
    return out


def _same(a, b, prog, tag=""):
    assert a.iterations == b.iterations, tag
    assert a.deltas.tolist() == b.deltas.tolist(), tag
    assert a.output_tuples == b.output_tuples, tag
    assert np.array_equal(a.rows, b.rows), tag
    if prog == "wcc":
        assert a.largest_component == b.largest_component, tag
        if a.labels is not None and b.labels is not None:
            assert np.array_equal(a.node_ids, b.node_ids), tag
            assert np.array_equal(a.labels, b.labels), tag


CASES = [("tc", "reference"), ("sg", "reference"), ("wcc", "reference"), ("wcc", "fixpoint")]


@pytest.mark.parametrize("prog,stop", CASES)
def test_session_all_at_once(engine, prog, stop):
    inst = _instances(prog)
    labels = prog == "wcc"
    plain = [engine.run(prog, e, wcc_stop=stop, labels=labels) for e in inst]
    with engine.session(prog, wcc_stop=stop) as s:
        ids = [s.admit(e) for e in inst]
        assert ids == list(range(len(inst)))
        finished = s.poll()
        steps = 0
        while s.step():
            steps += 1
            finished += s.poll()
        finished += s.poll()
        assert sorted(finished) == ids
        assert steps + 1 == max(p.iterations for p in plain)
        for i, p in zip(ids, plain):
            _same(s.result(i, labels=labels), p, prog, f"instance {i}")


@pytest.mark.parametrize("prog,stop", CASES)
def test_session_staggered_admission(engine, prog, stop):
    """Continuous batching: instances join while others are mid-fixpoint."""
    inst = _instances(prog, seed=7)
    labels = prog == "wcc"
    plain = [engine.run(prog, e, wcc_stop=stop, labels=labels) for e in inst]
    order = np.random.default_rng(3).permutation(len(inst))
    got = {}
    with engine.session(prog, wcc_stop=stop) as s:
        pending = list(order)
        id_of = {}
        while pending or s.memory()[1]:
            for _ in range(2):  # two arrivals per step
                if pending:
                    k = pending.pop()
                    id_of[s.admit(inst[k])] = k
            s.step()
            for i in s.poll():
                got[id_of[i]] = s.result(i, labels=labels)
                s.release(i)
        for i in s.poll():
            got[id_of[i]] = s.result(i, labels=labels)
    assert sorted(got) == list(range(len(inst)))
    for k, p in enumerate(plain):
        _same(got[k], p, prog, f"input {k}")


@pytest.mark.parametrize("prog", ["tc", "sg", "wcc"])
def test_alone_equals_mixed(engine, prog):
    inst = _instances(prog, seed=11)
    big = max(range(len(inst)), key=lambda k: len(inst[k]))
    with engine.session(prog) as s:
        i = s.admit(inst[big])
        s.run()
        alone = s.result(i, labels=True)
    with engine.session(prog) as s:
        ids = [s.admit(e) for e in inst]
        s.run()
        mixed = s.result(ids[big], labels=True)
    _same(alone, mixed, prog)


@pytest.mark.parametrize("prog", ["tc", "sg", "wcc"])
def test_run_batch(engine, prog):
    inst = _instances(prog, seed=5)
    res = engine.run_batch(prog, inst, labels=True)
    for k, e in enumerate(inst):
        _same(res[k], engine.run(prog, e, labels=True), prog, f"input {k}")


def test_run_batch_device_inputs(engine):
    import torch
    inst = _instances("tc", seed=2)
    dev = [torch.from_numpy(e).cuda() for e in inst]
    res = engine.run_batch("tc", dev, output="device")
    for k, e in enumerate(inst):
        assert np.array_equal(res[k].rows.cpu().numpy(), engine.tc(e).rows)


def test_session_max_iterations(engine):
    inst = _instances("tc", seed=4)
    with engine.session("tc", max_iterations=3) as s:
        ids = [s.admit(e) for e in inst]
        s.run()
        for i, e in zip(ids, inst):
            _same(s.result(i), engine.tc(e, max_iterations=3), "tc", f"instance {i}")


def test_session_reuse_after_idle(engine):
    """The union state restarts once every instance has finished."""
    inst = _instances("tc", seed=9)
    with engine.session("tc") as s:
        a = s.admit(inst[-1])
        s.run()
        b = s.admit(inst[-2])
        c = s.admit(inst[-1])
        s.run()
        _same(s.result(a), s.result(c), "tc")
        _same(s.result(b), engine.tc(inst[-2]), "tc")
        before, active = s.memory()
        assert active == 0 and before > 0
        for i in (a, b, c):
            s.release(i)
        with pytest.raises(Exception):
            s.result(a)


def test_session_errors(engine):
    from mnmgdatalog_b200 import DatalogError
    with pytest.raises(DatalogError):
        engine.session("single_join")
    with engine.session("tc") as s:
        i = s.admit(np.array([[1, 2], [2, 3]], np.int32))
        with pytest.raises(DatalogError):
            s.result(i)  # not finished yet
        with pytest.raises(DatalogError):
            s.release(i)
        s.run()
        assert len(s.result(i).rows) == 3
        with pytest.raises(DatalogError):
            s.result(99)
    with engine.session("tc", max_nodes=4) as s:
        s.admit(np.array([[1, 2], [2, 3]], np.int32))
        with pytest.raises(DatalogError):
            s.admit(np.array([[7, 8], [8, 9]], np.int32))  # 6 nodes > 4


@pytest.mark.parametrize("prog", ["tc", "sg", "wcc"])
def test_admit_many_while_running(engine, prog):
    """Groups of instances (with empty ones among them) admitted in one call,
    between steps of the running ones."""
    inst = _instances(prog, seed=13)
    plain = [engine.run(prog, e, labels=True) for e in inst]
    got = {}
    with engine.session(prog) as s:
        first = s.admit_many(inst[:5])
        assert first == list(range(5))
        s.step()
        second = s.admit_many(inst[5:])
        assert second == list(range(5, len(inst)))
        assert s.admit_many([]) == []
        s.run()
        for i in range(len(inst)):
            got[i] = s.result(i, labels=True)
    for k, p in enumerate(plain):
        _same(got[k], p, prog, f"input {k}")
