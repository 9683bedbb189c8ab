"""The GPU feeder's ordering (GpuScorer.score_batches, the CLI's
score_batches, crates/eschalign-cli/src/align.rs:2801-2917), on the CPU with a
stand-in device: each batch is prepared and submitted before the one ahead
of it is finished, results come back in order, and an abandoned feed still
finishes what it queued."""
from eschalign_b200.scorer import GpuScorer


class FakeDevice:
    def __init__(self):
        self.log = []

    def submit(self, b):
        self.log.append(("submit", b))


def feed(batches, dev, timing=None):
    def prepare(r):
        dev.log.append(("prepare", r))
        return r

    def finish(b):
        dev.log.append(("finish", b))
        return b * 10
    return GpuScorer._feed(dev, batches, prepare, finish, timing)


def test_two_batches_in_flight_results_in_order():
    dev = FakeDevice()
    t = {}
    assert list(feed(iter([1, 2, 3]), dev, t)) == [10, 20, 30]
    assert dev.log == [("prepare", 1), ("submit", 1), ("prepare", 2), ("submit", 2),
                       ("finish", 1), ("prepare", 3), ("submit", 3), ("finish", 2),
                       ("finish", 3)]
    assert set(t) == {"prepare_s", "submit_s", "finish_s"}


def test_empty_and_single():
    dev = FakeDevice()
    assert list(feed([], dev)) == []
    assert list(feed([7], dev)) == [70]


def test_abandoned_feed_finishes_what_it_queued():
    dev = FakeDevice()
    g = feed(iter([1, 2, 3]), dev)
    assert next(g) == 10
    g.close()
    assert ("finish", 2) in dev.log and ("submit", 3) not in dev.log
