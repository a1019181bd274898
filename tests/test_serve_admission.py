"""The serving loop's admission by free device memory (``jaxrans_b200.serve.Admission``),
on the host: slot counts of new pools, and the release of idle pools to sizes that wait."""

from __future__ import annotations

from dataclasses import dataclass

from jaxrans_b200.serve import Admission

GB = 1 << 30


@dataclass
class FakePool:
    key: tuple
    live: bool


def test_a_new_pool_keeps_room_for_the_sizes_not_seen_yet():
    adm = Admission(max_slots=64, memory_fraction=0.8, n_classes=4)
    # first pool of four sizes: 0.8 of 100 GB shared with the three unseen sizes, 1 GB slots
    assert adm.new_pool_slots(100 * GB, GB, (385, 97), set()) == 20
    # the last size to be seen takes its whole share
    seen = {(193, 49), (385, 97), (513, 129)}
    assert adm.new_pool_slots(100 * GB, GB, (769, 193), seen) == 64
    assert adm.new_pool_slots(40 * GB, GB, (769, 193), seen) == 32
    # another pool of a size already pooled: only the unseen sizes are kept room for
    assert adm.new_pool_slots(40 * GB, GB, (385, 97), {(385, 97)}) == 8


def test_no_pool_when_not_one_slot_fits():
    adm = Admission(max_slots=64, memory_fraction=0.8, n_classes=1)
    assert adm.new_pool_slots(GB, 2 * GB, (385, 97), set()) == 0
    assert adm.new_pool_slots(3 * GB, 2 * GB, (385, 97), set()) == 1


def test_idle_pools_are_released_only_for_a_waiting_size():
    pools = [FakePool((193, 49), live=False), FakePool((385, 97), live=True), FakePool((513, 129), live=False),
             FakePool((769, 193), live=False)]
    # nobody starved: nothing is released
    assert Admission.releasable(pools, starved=set(), waiting={(769, 193)}) == []
    # a 513 request waits for memory: the idle pools of sizes with no request waiting go
    out = Admission.releasable(pools, starved={(513, 129)}, waiting={(513, 129), (769, 193)})
    assert [p.key for p in out] == [(193, 49)]
