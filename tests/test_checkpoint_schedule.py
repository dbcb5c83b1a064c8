"""The binomial checkpoint cost that fm_adjoint_breakthrough's reverse sweep
attains (it splits each reversal at the j minimising j + t(l-j, c-1) + t(j, c))
equals the optimal-split recurrence, so the recomputation counts the GPU test
expects are the optimum."""
from functools import lru_cache

from tests.helpers import revolve_cost


@lru_cache(None)
def _best(l, c):
    if l <= 1:
        return 0
    if l - 1 <= c:
        return l - 1
    if c == 1:
        return l * (l - 1) // 2
    return min(j + _best(l - j, c - 1) + _best(j, c) for j in range(1, l))


def test_revolve_cost_is_the_optimal_split_recurrence():
    for l in range(1, 70):
        for c in range(1, 10):
            assert revolve_cost(l, c) == _best(l, c), (l, c)


def test_revolve_cost_store_all_and_single_buffer():
    assert revolve_cost(200, 199) == 199
    assert revolve_cost(30, 1) == 435
    assert revolve_cost(150, 6) == 480
