"""Served loop: update-batch requests for many resident graphs, recoloured
as they arrive.

Requests (graph, lines, arrival time) arrive over time.  Two launch
policies run over the same ResidentPool interface:

  plain     one request per launch, oldest first: the reference's model of
            one graph and one batch per run (HI/Color_main.cu:146-216), kept
            resident instead of re-read from files;
  batched   continuous batching: every launch takes the oldest waiting
            request of each graph that has one (a graph's requests stay in
            arrival order, at most one per launch), oldest first, while the
            launch stays under a line budget and the graphs fit the pool
            together.  Requests that arrive during a launch join the next.

Both give every graph the same sequence of batches, so every graph ends
with the same colours under either policy.  A request's latency is the time
from its arrival to the return of the launch that applied it.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    rid: int
    graph: int
    lines: np.ndarray
    arrival: float               # seconds after the start of the run
    done: float = float("nan")   # seconds after the start of the run
    iterations: int = -1
    launch: int = -1

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclass
class RunStats:
    launches: int = 0
    lines: int = 0
    makespan: float = 0.0        # first arrival to last completion, seconds
    device_ms: float = 0.0       # sum of the launches' device time
    per_launch_requests: list = field(default_factory=list)

    def summary(self, requests) -> dict:
        lat = np.array([r.latency for r in requests]) * 1e3
        return {
            "requests": len(requests),
            "launches": self.launches,
            "lines": self.lines,
            "makespan_s": self.makespan,
            "updates_per_s": self.lines / self.makespan if self.makespan > 0 else 0.0,
            "device_updates_per_s": self.lines / (self.device_ms / 1e3) if self.device_ms > 0 else 0.0,
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else 0.0,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else 0.0,
            "mean_ms": float(lat.mean()) if len(lat) else 0.0,
            "requests_per_launch": float(np.mean(self.per_launch_requests)) if self.per_launch_requests else 0.0,
        }


def choose_plain(queues, heads_order, sizes, vertex_capacity, pool_slots, max_lines):
    """The oldest waiting request alone."""
    return [queues[heads_order[0]][0]]


def choose_batched(queues, heads_order, sizes, vertex_capacity, pool_slots, max_lines):
    """Oldest head requests of distinct graphs while the launch stays under
    max_lines and its graphs fit the pool together (the first always goes)."""
    out, lines, nsum, slots = [], 0, 0, 0
    for g in heads_order:
        r = queues[g][0]
        n, s = sizes(g)
        if out and (lines + len(r.lines) > max_lines or nsum + n > vertex_capacity or slots + s > pool_slots):
            continue
        out.append(r)
        lines += len(r.lines)
        nsum += n
        slots += s
    return out


POLICIES = {"plain": choose_plain, "batched": choose_batched}


class Server:
    """Runs a request trace against `pool` (anything with apply() and
    graph_size() like ResidentPool) in real time."""

    def __init__(self, pool, policy: str, vertex_capacity: int, pool_slots: int, max_lines: int = 1 << 22,
                 clock=time.perf_counter, sleep=time.sleep):
        if policy not in POLICIES:
            raise ValueError(f"unknown policy {policy!r}")
        self.pool = pool
        self.choose = POLICIES[policy]
        self.vertex_capacity = vertex_capacity
        # leave room for rows that grow while resident
        self.pool_slots = int(pool_slots * 0.9)
        self.max_lines = max_lines
        self.clock = clock
        self.sleep = sleep

    def run(self, requests, t0: float | None = None) -> RunStats:
        """Serves `requests` (arrival times in seconds after t0; t0 = now by
        default) and fills in each one's completion time."""
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        queues: dict[int, deque] = {}
        size_cache: dict[int, tuple] = {}

        def sizes(g):
            if g not in size_cache:
                n, s, _ = self.pool.graph_size(g)
                size_cache[g] = (n, s)
            return size_cache[g]

        st = RunStats()
        nxt = 0
        if t0 is None:
            t0 = self.clock()
        remaining = len(reqs)
        while remaining:
            now = self.clock() - t0
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                r = reqs[nxt]
                queues.setdefault(r.graph, deque()).append(r)
                nxt += 1
            active = [g for g, q in queues.items() if q]
            if not active:
                self.sleep(max(0.0, reqs[nxt].arrival - now))
                continue
            heads_order = sorted(active, key=lambda g: (queues[g][0].arrival, queues[g][0].rid))
            batch = self.choose(queues, heads_order, sizes, self.vertex_capacity, self.pool_slots,
                                self.max_lines)
            stats, its, _ = self.pool.apply([(r.graph, r.lines) for r in batch])
            done = self.clock() - t0
            for r, it in zip(batch, its):
                queues[r.graph].popleft()
                r.done = done
                r.iterations = int(it)
                r.launch = st.launches
                size_cache.pop(r.graph, None)
                st.lines += len(r.lines)
            st.launches += 1
            st.device_ms += float(stats.device_ms)
            st.per_launch_requests.append(len(batch))
            remaining -= len(batch)
        if reqs:
            st.makespan = max(r.done for r in reqs) - reqs[0].arrival
        return st


class LanedServer:
    """Continuous batching over several lanes that run side by side on the
    device.  Each lane is its own pool (its own stream, and a share of the
    SMs for its persistent launches), holds a fixed subset of the graphs and
    serves their requests with its own host thread under the `batched`
    policy, so a long launch in one lane does not hold up the requests of
    the others: requests that arrive while other lanes' launches are on the
    device start as soon as their own lane is free, and the lanes' launches
    overlap.  A graph's requests stay in arrival order within its lane, so
    every graph gets the same sequence of batches, and the same colours, as
    under the single-lane policies.

    lanes: [(pool, {global graph id: lane-local graph id}, vertex_capacity,
    pool_slots), ...]."""

    def __init__(self, lanes, max_lines: int = 1 << 22, clock=time.perf_counter, sleep=time.sleep):
        self.lanes = [(Server(pool, "batched", vcap, slots, max_lines=max_lines, clock=clock, sleep=sleep), gmap)
                      for pool, gmap, vcap, slots in lanes]
        self.clock = clock

    def run(self, requests) -> RunStats:
        import threading

        parts = []
        for srv, gmap in self.lanes:
            mine = [r for r in requests if r.graph in gmap]
            local = [Request(r.rid, gmap[r.graph], r.lines, r.arrival) for r in mine]
            parts.append((srv, mine, local))
        if sum(len(m) for _, m, _ in parts) != len(requests):
            raise ValueError("a request names a graph that no lane holds")
        results, errors = [None] * len(parts), []
        t0 = self.clock()

        def work(i, srv, local):
            try:
                results[i] = srv.run(local, t0=t0)
            except BaseException as e:  # reported after every lane has stopped
                errors.append(e)

        threads = [threading.Thread(target=work, args=(i, srv, local)) for i, (srv, _, local) in enumerate(parts)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
        st = RunStats()
        for (srv, mine, local), rs in zip(parts, results):
            for r, l in zip(mine, local):
                r.done, r.iterations, r.launch = l.done, l.iterations, l.launch
            st.launches += rs.launches
            st.lines += rs.lines
            st.device_ms += rs.device_ms
            st.per_launch_requests += rs.per_launch_requests
        done = [r for r in requests if r.done == r.done]
        if done:
            st.makespan = max(r.done for r in done) - min(r.arrival for r in requests)
        return st


def assign_lanes(sizes, lanes: int):
    """Graph -> lane, balancing the lanes' total vertices (largest graphs
    first, each to the lightest lane)."""
    load = [0] * lanes
    out = {}
    for g in sorted(range(len(sizes)), key=lambda g: -sizes[g]):
        j = min(range(lanes), key=lambda x: load[x])
        out[g] = j
        load[j] += sizes[g]
    return out


def make_trace(count: int, ngraphs: int, rate: float, seed: int, kmin: int = 10, kmax: int = 1_000_000,
               zipf_s: float = 1.1):
    """Arrival times (Poisson, `rate` per second), target graphs (Zipf(s)
    over a seeded random ranking of the graphs) and batch sizes (log-uniform
    in [kmin, kmax]) of `count` requests."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, count))
    ranks = np.arange(1, ngraphs + 1, dtype=np.float64)
    p = ranks ** -zipf_s
    p /= p.sum()
    perm = rng.permutation(ngraphs)
    graphs = perm[rng.choice(ngraphs, size=count, p=p)]
    sizes = np.exp(rng.uniform(np.log(kmin), np.log(kmax), count)).astype(np.int64)
    return arrivals, graphs, sizes
