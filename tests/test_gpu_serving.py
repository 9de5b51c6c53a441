"""Serving (continuous batching over the resident waveform): every request's answers are
bit-identical to the same request searched alone and to the oracle, however the
requests were grouped into batches; admission respects max_batch and the memory budget;
state errors while serving."""
import threading
import time

import numpy as np
import pytest

import tremor_b200 as tb
from tests.test_gpu_batching import _check, _requests, _waveform

pytestmark = pytest.mark.gpu


def _collect(server, count, timeout_s=120.0):
    got, t0 = {}, time.time()
    while len(got) < count and time.time() - t0 < timeout_s:
        for c in server.poll(64, timeout_ms=200):
            got[c.ticket] = c
    return got


def _same(a, b):
    return np.array_equal(a[0], b[0]) and np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


def test_served_results_equal_alone_and_oracle():
    x = _waveform(1 << 17, 21)
    rng = np.random.default_rng(22)
    lengths = [int(v) for v in rng.choice([40, 64, 100, 128, 200, 333, 512, 1000, 2048], size=36)]
    reqs = _requests(x, rng, lengths)
    with tb.Context(x) as ctx:
        alone = [ctx.scan_batch([r])[0] for r in reqs]
        tickets = {}
        with ctx.serve(workers=2, max_batch=16) as server:
            # a burst (batched together) and a trickle from a second thread (arrives while
            # earlier batches are on the GPU)
            def trickle():
                for i in range(18, 36):
                    time.sleep(float(rng.uniform(0.0, 0.01)))
                    tickets[server.submit(reqs[i])] = i
            th = threading.Thread(target=trickle)
            th.start()
            for i in range(18):
                tickets[server.submit(reqs[i])] = i
            th.join()
            got = _collect(server, len(reqs))
    assert len(got) == len(reqs)
    sizes = [c.batch_size for c in got.values()]
    assert max(sizes) > 1 and max(sizes) <= 16
    served = [None] * len(reqs)
    for t, c in got.items():
        assert c.status == 0
        assert c.submit_ms <= c.start_ms <= c.done_ms
        served[tickets[t]] = c.answers
    for i in range(len(reqs)):
        assert _same(served[i], alone[i]), i
    _check(x, reqs, served)


def test_memory_budget_and_batch_cap():
    """A budget below one request's estimate admits one request at a time (each still
    runs: alone); max_batch caps the batch size."""
    x = _waveform(1 << 16, 23)
    rng = np.random.default_rng(24)
    reqs = _requests(x, rng, [64, 96, 150, 300, 64, 500, 128, 40])
    with tb.Context(x) as ctx:
        with ctx.serve(workers=1, max_batch=8, memory_budget=1) as server:
            for r in reqs:
                server.submit(r)
            got = _collect(server, len(reqs))
        assert sorted(c.batch_size for c in got.values()) == [1] * len(reqs)
        with ctx.serve(workers=2, max_batch=3) as server:
            ticket = {server.submit(r): i for i, r in enumerate(reqs)}
            got2 = _collect(server, len(reqs))
        assert max(c.batch_size for c in got2.values()) <= 3
    served = [None] * len(reqs)
    for t, c in got2.items():
        served[ticket[t]] = c.answers
    _check(x, reqs, served)
    _check(x, reqs, [c.answers for c in sorted(got.values(), key=lambda c: c.ticket)])


def test_serving_state_rules():
    x = _waveform(1 << 15, 25)
    rng = np.random.default_rng(26)
    reqs = _requests(x, rng, [64, 100])
    with tb.Context(x) as ctx:
        server = ctx.serve()
        with pytest.raises(tb.TremorError):
            ctx.set_window_range(0, 1000)
        with pytest.raises(tb.TremorError):
            ctx.serve()  # already serving
        with pytest.raises(tb.TremorError):
            server.submit(tb.Request(np.ones(20000, np.float32)))  # longer than 16384
        t = [server.submit(r) for r in reqs]
        # the synchronous calls stay usable while serving
        assert _same(ctx.scan_batch([reqs[0]])[0], ctx.scan_batch([reqs[0]])[0])
        server.stop()
        with pytest.raises(tb.TremorError):
            server.submit(reqs[0])
        got = _collect(server, len(reqs), timeout_s=10)  # completions stay pollable after stop
        assert sorted(got) == sorted(t)
        pending, in_flight, nbytes, launches = server.status()
        assert (pending, in_flight, nbytes) == (0, 0, 0) and launches > 0
    _check(x, reqs, [got[i].answers for i in t])


def test_batch_time_budget():
    """batch_ms bounds a batch's modelled device time: below any one request's estimate
    every batch holds one request (a first request alone is always admitted), and the
    answers are those of the requests alone."""
    x = _waveform(1 << 16, 27)
    rng = np.random.default_rng(28)
    reqs = _requests(x, rng, [64, 96, 150, 300, 64, 500, 128, 40])
    with tb.Context(x) as ctx:
        with ctx.serve(workers=1, max_batch=8, batch_ms=1e-9) as server:
            ticket = {server.submit(r): i for i, r in enumerate(reqs)}
            got = _collect(server, len(reqs))
    assert sorted(c.batch_size for c in got.values()) == [1] * len(reqs)
    served = [None] * len(reqs)
    for t, c in got.items():
        served[ticket[t]] = c.answers
    _check(x, reqs, served)


def test_poll_without_limit_returns_once_stopped():
    """tm_poll with no time limit returns (empty) once the server is stopped and nothing is
    left to complete, instead of waiting for good."""
    x = _waveform(1 << 15, 29)
    with tb.Context(x) as ctx:
        server = ctx.serve()
        server.stop()
        out = []
        th = threading.Thread(target=lambda: out.append(server.poll(8, timeout_ms=-1)), daemon=True)
        th.start()
        th.join(timeout=10.0)
        assert not th.is_alive(), 'poll without a limit did not return after stop'
        assert out == [[]]
