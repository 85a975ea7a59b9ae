"""Host logic of the autotuner's table (no GPU)."""
from traceon_b200 import autotune


def test_size_buckets():
    assert [autotune._bucket(x) for x in (0, 1, 2, 3, 1000, 1024, 1025)] == [0, 1, 2, 4, 1024, 1024, 2048]


def test_table_is_copied_and_cleared():
    autotune.clear()
    with autotune._lock:
        autotune._table[('k',)] = 4
    t = autotune.table()
    t[('k',)] = 8
    assert autotune.table() == {('k',): 4}
    autotune.clear()
    assert autotune.table() == {}


def test_lookahead_tuner_picks_the_fastest_width(monkeypatch):
    """tune_solve_lookahead with a fake backend: every candidate width is
    timed once, the fastest is left set, the setting in force before the
    tuning is restored around it, and a second call of the same size bucket
    reuses the table entry without timing again."""
    import types
    from traceon_b200 import backend as B
    state = {'reserve': 29, 'calls': []}

    def set_la(r):
        prev = state['reserve']
        state['reserve'] = 29 if r < 0 else r
        state['calls'].append(r)
        return prev

    cost = {0: 48.0, 15: 44.0, 30: 39.5, 44: 40.8}
    timed = []

    def fake_time(fn, reps=2):
        timed.append(state['reserve'])
        return cost[state['reserve']]

    class FakeCuda:
        @staticmethod
        def get_device_name(dev):
            return 'fake B200'

    monkeypatch.setattr(B, 'num_sms', lambda: 148)
    monkeypatch.setattr(B, 'set_solve_lookahead', set_la)
    monkeypatch.setattr(B, 'dev_solve_mixed', lambda A, F: None)
    monkeypatch.setattr(B, '_torch', lambda: types.SimpleNamespace(cuda=FakeCuda))
    monkeypatch.setattr(autotune, '_time_ms', fake_time)
    A = types.SimpleNamespace(shape=(16384, 16384), device='cuda:0')
    autotune.clear()
    try:
        hit = autotune.tune_solve_lookahead(A, None)
        assert sorted(timed) == [0, 15, 30, 44]
        assert hit == {'reserve_sms': 30, 'times_ms': cost}
        assert state['reserve'] == 30
        assert state['calls'][0] == -1 and state['calls'][-2:] == [29, 30]  # restored, then the choice set
        n = len(timed)
        state['reserve'] = 29
        assert autotune.tune_solve_lookahead(A, None)['reserve_sms'] == 30
        assert len(timed) == n and state['reserve'] == 30
    finally:
        autotune.clear()
