"""The autotuner's search (erebus_b200.autotune.tune), on the CPU with a
synthetic timing function in place of device timesteps: coordinate descent
over the candidate values from the defaults, one parameter at a time, each
parameter left at its fastest value before the next is tried."""


def test_coordinate_descent_finds_the_separable_minimum(pkg, monkeypatch):
    from erebus_b200 import autotune
    best_of = {"mf_leaf_vector": 48, "mf_leaf_scalar": 128, "mf_local_factor_ops": 4,
               "mf_local_solve_tiles": 24}
    calls = []

    def fake_time(make_state, opts, steps, warmup):
        calls.append(dict(opts))
        assert opts["krylov"] == 1          # the base options reach every trial
        return 10.0 + sum(abs(opts[k] - v) / max(v, 1) for k, v in best_of.items())

    monkeypatch.setattr(autotune, "time_config", fake_time)
    best, trials = autotune.tune(lambda: None, {"krylov": 1}, steps=1, warmup=0,
                                 log=lambda m: None)
    assert best == best_of
    assert len(trials) == len(calls)
    # every candidate value of every parameter is tried once, except the
    # value in force when that parameter's turn comes
    n = 1 + sum(len(v) - 1 for v in autotune.CANDIDATES.values())
    assert len(calls) == n
    assert min(ms for _, ms in trials) == 10.0


def test_defaults_are_candidates(pkg):
    from erebus_b200 import autotune
    assert set(autotune.DEFAULTS) == set(autotune.CANDIDATES)
    for k, v in autotune.DEFAULTS.items():
        assert v in autotune.CANDIDATES[k], k
