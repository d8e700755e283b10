"""GPU: the continuous-batching server's request handling -- u16 and u8 requests mixed in one
stream, cancellation of queued, admitted and completed requests, a consumer that collects
its results late and out of order, and admission priced in device memory. Every served
result that is not cancelled equals the plain form of the same request, byte for byte."""
import time

import numpy as np
import pytest

import terrain_b200

pytestmark = pytest.mark.gpu


def square(cx, cz, r):
    return [(cx + dx, cz + dz) for dz in range(-r, r + 1) for dx in range(-r, r + 1)]


@pytest.fixture(scope='module')
def gen():
    g = terrain_b200.TerrainGenerator(max_batch_chunks=64)
    yield g
    g.close()


def alone(g, seed, chunks):
    g.set_seed(seed)
    return g.generate(chunks)


def test_u16_and_u8_requests_mixed(gen, ref_model):
    reqs = [(3, square(100, -40, 2)), (5, square(-7000, 9000, 3)), (3, square(6128, 6128, 1)), (11, square(0, 0, 4))]
    want = [alone(gen, s, c) for s, c in reqs]
    with terrain_b200.TerrainServer(gen, batch_chunks=48) as srv:
        tickets = [srv.submit(s, c, u8=(i % 2 == 1)) for i, (s, c) in enumerate(reqs)]
        got = [srv.wait(t) for t in tickets]
    for i, ((b, q), (wb, wq)) in enumerate(zip(got, want)):
        assert b.dtype == (np.uint8 if i % 2 else np.uint16)
        assert (b.astype(np.uint16) == wb).all() and (q == wq).all(), i
    rb, rq = ref_model.seed(5).generate(reqs[1][1])
    assert (got[1][0].astype(np.uint16) == rb).all() and (got[1][1] == rq).all()


def test_cancellation(gen):
    """A budget of one batch keeps most requests queued: a queued request cancels at once,
    the others are unaffected, a completed request's cancel returns False and its result
    stands, and an admitted request either completes or reports TG_ERR_CANCELLED."""
    reqs = [(7, square(40 * i, -40 * i, 3)) for i in range(6)]
    want = [alone(gen, s, c) for s, c in reqs]
    price = None
    with terrain_b200.TerrainServer(gen, batch_chunks=16, hbm_budget_bytes=1) as srv:
        price = srv.stats()['device_bytes_per_chunk']
        tickets = [srv.submit(s, c) for s, c in reqs]
        assert srv.cancel(tickets[5]) is True                 # still queued behind 5 requests of 49 chunks
        first = srv.cancel(tickets[0])                        # admitted (maybe already in flight)
        with pytest.raises(terrain_b200.TerrainError) as e:
            srv.wait(tickets[5])
        assert e.value.status == 10
        for i in (1, 2, 3, 4):
            b, q = srv.wait(tickets[i])
            assert (b == want[i][0]).all() and (q == want[i][1]).all(), i
        if first:
            with pytest.raises(terrain_b200.TerrainError) as e:
                srv.wait(tickets[0])
            assert e.value.status == 10
        else:
            b, q = srv.wait(tickets[0])
            assert (b == want[0][0]).all()
        t = srv.submit(*reqs[2])
        b, q = srv.wait(t)
        assert (b == want[2][0]).all()
        st = srv.stats()
        assert st['cancelled_requests'] >= 1 and st['max_active_chunks'] == 16
    assert price > 100000                                     # HBM per chunk of batch capacity


def test_late_consumer_and_latencies(gen):
    """Results are collected late and in reverse order; the server completes every request
    without the consumer, and reports one latency per completed request."""
    reqs = [(9, square(-300 * i, 17, 1 + i % 3)) for i in range(8)]
    want = [alone(gen, s, c) for s, c in reqs]
    with terrain_b200.TerrainServer(gen, batch_chunks=32) as srv:
        tickets = [srv.submit(s, c) for s, c in reqs]
        last_done = False
        for _ in range(1000):
            if not last_done:
                last_done = srv.poll(tickets[-1], 50)         # wait on the last one only
            elif srv.stats()['completed_requests'] == len(reqs):
                break
            else:
                time.sleep(0.01)
        assert last_done and srv.stats()['completed_requests'] == len(reqs)
        lat = srv.latencies()
        assert lat.shape[0] == len(reqs) and (lat > 0).all()
        for i in reversed(range(len(reqs))):
            if i == len(reqs) - 1:
                _, b, q = srv.pending.pop(tickets[i])         # released by the poll that saw it done
            else:
                b, q = srv.wait(tickets[i])
            assert (b == want[i][0]).all() and (q == want[i][1]).all(), i
