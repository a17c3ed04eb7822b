"""Served-loop scheduling on a simulated clock (no GPU): launch policies,
per-graph ordering, budgets, and the request trace."""
import numpy as np

import dyncolor_b200 as dc
from dyncolor_b200.serve import Request, Server, make_trace


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-6)


class FakeStats:
    def __init__(self, ms):
        self.device_ms = ms


class FakePool:
    """Applies nothing; a launch costs 2 ms plus 10 ns per line."""

    def __init__(self, clock, sizes):
        self.clock = clock
        self.sizes = sizes
        self.launches = []
        self.per_graph = {g: [] for g in range(len(sizes))}

    def apply(self, batch):
        graphs = [g for g, _ in batch]
        assert len(set(graphs)) == len(graphs), "two batches for one graph in a launch"
        lines = sum(len(x) for _, x in batch)
        cost = 2e-3 + 1e-8 * lines
        self.clock.t += cost
        self.launches.append(batch)
        for g, x in batch:
            self.per_graph[g].append(int(x["node1"][0]) if len(x) else -1)
        return FakeStats(cost * 1e3), np.arange(len(batch)), np.zeros(len(batch), np.int32)

    def graph_size(self, g):
        n, s = self.sizes[g]
        return n, s, True


def trace(count, ngraphs, rate, seed=1):
    arr, gr, ks = make_trace(count, ngraphs, rate, seed, kmin=10, kmax=20_000)
    reqs = []
    for i, (t, g, k) in enumerate(zip(arr, gr, ks)):
        x = np.zeros(int(k), dtype=dc.CHANGE_DTYPE)
        x["node1"] = i  # tags the request
        reqs.append(Request(i, int(g), x, float(t)))
    return reqs


def run(policy, reqs, sizes, max_lines=1 << 16, vcap=10_000, slots=1 << 20):
    clk = FakeClock()
    pool = FakePool(clk, sizes)
    st = Server(pool, policy, vcap, slots, max_lines=max_lines, clock=clk, sleep=clk.sleep).run(reqs)
    return st, pool


def test_plain_one_request_per_launch_in_arrival_order():
    sizes = [(100, 1000)] * 8
    reqs = trace(200, 8, rate=5000)
    st, pool = run("plain", reqs, sizes)
    assert st.launches == 200 and all(len(b) == 1 for b in pool.launches)
    order = [int(b[0][1]["node1"][0]) for b in pool.launches]
    assert order == sorted(order)
    assert all(r.latency >= 0 for r in reqs)


def test_batched_keeps_per_graph_order_and_budgets():
    sizes = [(100 + 50 * g, 2000 + 500 * g) for g in range(16)]
    reqs = trace(400, 16, rate=20_000)
    st, pool = run("batched", reqs, sizes, max_lines=50_000, vcap=600, slots=12_000)
    assert sum(len(b) for b in pool.launches) == 400
    for b in pool.launches:
        if len(b) > 1:
            assert sum(len(x) for _, x in b) <= 50_000
            assert sum(sizes[g][0] for g, _ in b) <= 600
            assert sum(sizes[g][1] for g, _ in b) <= int(12_000 * 0.9)
    # every graph saw its requests in arrival order, as under the plain policy
    reqs2 = trace(400, 16, rate=20_000)
    _, plain = run("plain", reqs2, sizes)
    for g in range(16):
        assert pool.per_graph[g] == plain.per_graph[g]
        assert pool.per_graph[g] == sorted(pool.per_graph[g])
    assert st.launches < 400
    assert all(r.done >= r.arrival for r in reqs)


def test_batched_beats_plain_under_overload():
    sizes = [(100, 1000)] * 64
    a = trace(600, 64, rate=50_000)
    b = trace(600, 64, rate=50_000)
    sp, _ = run("plain", a, sizes)
    sb, _ = run("batched", b, sizes, max_lines=1 << 20)
    lp = np.percentile([r.latency for r in a], 99)
    lb = np.percentile([r.latency for r in b], 99)
    assert sb.launches < sp.launches and lb < lp
    assert sb.summary(b)["updates_per_s"] > sp.summary(a)["updates_per_s"]


def test_trace_shape():
    arr, g1, k1 = make_trace(20_000, 256, rate=1000, seed=3)
    arr2, g2, k2 = make_trace(20_000, 256, rate=50_000, seed=3)
    assert np.array_equal(g1, g2) and np.array_equal(k1, k2)  # rate only stretches time
    assert np.allclose(arr2 * 50, arr)
    assert k1.min() >= 10 and k1.max() <= 1_000_000
    assert abs(np.median(np.log10(k1)) - 3.5) < 0.1  # log-uniform over [10, 1e6]
    counts = np.bincount(g1, minlength=256)
    top = np.sort(counts)[::-1]
    assert top[0] > 0.12 * len(g1) and top[0] > 10 * top[50]  # Zipf(1.1)
    gaps = np.diff(arr)
    assert abs(gaps.mean() - 1e-3) < 5e-5


class SleepPool(FakePool):
    """A launch takes (real) time: 1 ms plus 20 ns per line, spent in
    time.sleep, which lets other lanes' threads run meanwhile."""

    def __init__(self, sizes):
        super().__init__(None, sizes)

    def apply(self, batch):
        import time

        graphs = [g for g, _ in batch]
        assert len(set(graphs)) == len(graphs), "two batches for one graph in a launch"
        lines = sum(len(x) for _, x in batch)
        dt = 1e-3 + 2e-8 * lines
        time.sleep(dt)
        self.busy = getattr(self, "busy", 0.0) + dt
        self.launches.append(batch)
        for g, x in batch:
            self.per_graph[g].append(int(x["node1"][0]) if len(x) else -1)
        return FakeStats(1.0), np.arange(len(batch)), np.zeros(len(batch), np.int32)


def test_lanes_overlap_and_keep_each_graphs_order():
    from dyncolor_b200.serve import LanedServer, assign_lanes

    ng = 24
    sizes = [(100 + 10 * g, 1000) for g in range(ng)]

    def lanes_run(nl):
        which = assign_lanes([n for n, _ in sizes], nl)
        lanes = []
        for j in range(nl):
            gl = sorted(g for g in range(ng) if which[g] == j)
            gmap = {g: i for i, g in enumerate(gl)}
            pool = SleepPool([sizes[g] for g in gl])
            lanes.append((pool, gmap, 10_000, 1 << 20))
        reqs = trace(240, ng, rate=100_000)
        st = LanedServer(lanes, max_lines=4_000).run(reqs)
        return st, reqs, lanes, which

    st1, r1, lanes1, _ = lanes_run(1)
    st4, r4, lanes4, which = lanes_run(4)
    assert sorted(set(which.values())) == [0, 1, 2, 3]
    assert all(r.done >= r.arrival for r in r4) and st4.lines == st1.lines
    # every graph saw its requests in arrival order, in its own lane
    for g in range(ng):
        pool, gmap, _, _ = lanes4[which[g]]
        tags = pool.per_graph[gmap[g]]
        assert tags == sorted(tags) and len(tags) == sum(1 for r in r4 if r.graph == g)
    # the four lanes' launches overlap: together they were busy for much
    # longer than the run took
    busy = sum(getattr(pool, "busy", 0.0) for pool, _, _, _ in lanes4)
    assert busy > 1.5 * st4.makespan
    assert st4.makespan < st1.makespan
