"""Batch admission of the serving loop (host logic, no GPU): `serve.take_batch` keeps arrival order,
honours the batch limit and the HBM budget, carries the request that did not fit to the head of the
next batch, and leaves the shutdown sentinel on the queue."""
import queue

from dynlplus_b200.serve import take_batch


def fill(items):
    q = queue.Queue()
    for x in items:
        q.put(x)
    return q


def rest(q):
    out = []
    while True:
        try:
            out.append(q.get_nowait())
        except queue.Empty:
            return out


def test_drains_everything_without_limit_or_budget():
    q = fill([2, 3, 4])
    items, carry = take_batch(q, 1)
    assert items == [1, 2, 3, 4] and carry is None and rest(q) == []


def test_limit_leaves_the_rest_queued_in_order():
    q = fill([2, 3, 4, 5])
    items, carry = take_batch(q, 1, limit=3)
    assert items == [1, 2, 3] and carry is None and rest(q) == [4, 5]
    q = fill([2])
    assert take_batch(q, 1, limit=1) == ([1], None) and rest(q) == [2]  # one at a time


def test_budget_carries_the_first_misfit_and_keeps_arrival_order():
    # costs are the values themselves; budget 10
    q = fill([3, 5, 2, 1])
    items, carry = take_batch(q, 4, limit=8, cost=lambda x: x, budget=10)
    assert items == [4, 3] and carry == 5  # 4+3+5 > 10: 5 waits, and 2 and 1 do not overtake it
    assert rest(q) == [2, 1]
    q = fill([2, 1])
    items, carry = take_batch(q, carry, limit=8, cost=lambda x: x, budget=10)
    assert items == [5, 2, 1] and carry is None


def test_first_request_is_taken_even_above_the_budget():
    q = fill([1])
    items, carry = take_batch(q, 50, limit=8, cost=lambda x: x, budget=10)
    assert items == [50] and carry == 1 and rest(q) == []


def test_sentinel_ends_the_batch_and_stays_queued():
    q = fill([2, None, 3])
    items, carry = take_batch(q, 1)
    assert items == [1, 2] and carry is None
    assert rest(q) == [3, None]  # put back behind what was queued after it; the worker stops on it
    q = fill([None])
    items, carry = take_batch(q, 1, cost=lambda x: x, budget=10)
    assert items == [1] and carry is None and rest(q) == [None]
