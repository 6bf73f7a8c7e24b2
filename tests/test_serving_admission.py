"""Admission of serving-loop simulations by device footprint (host logic, no
GPU): the budget is never exceeded, busy simulations are never evicted, idle
ones are evicted least recently used first, and a simulation larger than the
budget is refused."""
from maos_b200.serving import Admission, draw_sim_cfg, poisson_arrivals


def _adm(budget, sizes):
    log = []
    resident = set()

    def load(i):
        resident.add(i)
        log.append(("load", i))
        return sizes[i]

    def unload(i):
        resident.discard(i)
        log.append(("unload", i))

    return Admission(budget, load, unload, lambda i: sizes[i]), log, resident


def test_budget_and_lru_eviction():
    sizes = {0: 40, 1: 30, 2: 20, 3: 50}
    a, log, resident = _adm(100, sizes)
    assert a.try_admit(0, busy=set()) and a.try_admit(1, busy=set()) and a.try_admit(2, busy=set())
    assert a.used == 90
    a.touch(0)  # 1 is now the least recently used
    assert a.try_admit(3, busy={0})  # needs 50: evicts 1 (idle, LRU) then 2
    assert ("unload", 1) in log and ("unload", 2) in log and a.used == 90
    assert resident == {0, 3} and a.evictions == 2


def test_busy_sims_are_not_evicted_and_oversize_refused():
    sizes = {0: 60, 1: 50, 2: 200}
    a, log, _ = _adm(100, sizes)
    assert a.try_admit(0, busy=set())
    assert not a.try_admit(1, busy={0})  # would need to evict a busy sim
    assert a.used == 60 and a.evictions == 0
    assert not a.try_admit(2, busy=set())  # larger than the budget


def test_sim_draws_and_arrivals_are_seeded():
    a, b = draw_sim_cfg(7), draw_sim_cfg(7)
    assert a == b and draw_sim_cfg(8) != a
    assert a["D"] in (8.0, 10.0, 30.0) and a["order"] in (16, 32, 60) and a["notf"] in (32, 64)
    assert 1 <= a["nwfs"] <= 6 and 2 <= len(a["atm"]["ht"]) <= 7
    arr = poisson_arrivals(5000.0, 4000, 32, seed=3)
    gaps = [t1 - t0 for (t0, _), (t1, _) in zip(arr, arr[1:])]
    assert abs(sum(gaps) / len(gaps) - 1 / 5000.0) < 0.1 / 5000.0
    assert {i for _, i in arr} <= set(range(32))
