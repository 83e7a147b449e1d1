"""Host logic of the continuous-batching server: HBM admission and batch
formation (no GPU)."""
from dataclasses import dataclass

import pytest

from differentiable_gaussian_mixture_renderer_b200.serving import HbmBudget, form_batch


@dataclass
class Req:
    scene_id: str
    backward: bool = False
    nbytes: int = 10


def cost(batch):
    return sum(r.nbytes for r in batch)


def test_budget_reserve_release():
    b = HbmBudget(100)
    assert b.fits(100) and not b.fits(101)
    b.reserve(60)
    assert b.fits(40) and not b.fits(41)
    with pytest.raises(RuntimeError):
        b.reserve(41)
    b.release(60)
    assert b.in_use == 0


def test_batch_keeps_arrival_order_and_view_limit():
    q = [Req("a"), Req("b"), Req("a"), Req("c"), Req("a")]
    ids = [id(r) for r in q]
    batch, nbytes = form_batch(q, 3, 16, cost, HbmBudget(1000))
    assert [id(r) for r in batch] == ids[:3]
    assert nbytes == 30
    assert [id(r) for r in q] == ids[3:]


def test_gradient_requests_take_their_own_scene_entry():
    # render requests of one scene share an entry; each gradient request has its own
    q = [Req("a"), Req("a"), Req("a", True), Req("a", True), Req("b")]
    batch, _ = form_batch(q, 8, 3, cost, HbmBudget(1000))
    assert len(batch) == 4  # entries: a, a(grad), a(grad) -> the 'b' request would need a 4th
    assert len(q) == 1 and q[0].scene_id == "b"


def test_budget_cuts_the_batch_and_head_that_does_not_fit_waits():
    q = [Req("a", nbytes=40), Req("b", nbytes=40), Req("c", nbytes=40)]
    budget = HbmBudget(100)
    batch, nbytes = form_batch(q, 8, 16, cost, budget)
    assert len(batch) == 2 and nbytes == 80
    budget.reserve(nbytes)
    batch2, _ = form_batch(q, 8, 16, cost, budget)
    assert batch2 == [] and len(q) == 1  # waits for memory to free up
    budget.release(nbytes)
    batch3, _ = form_batch(q, 8, 16, cost, budget)
    assert len(batch3) == 1 and q == []
