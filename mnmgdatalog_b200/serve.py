"""Served form: a request loop over union sessions (continuous batching).

Requests (TC, SG or WCC queries, each an edge relation) arrive over time.
The server keeps one union session per program on the device and, between
two iterations, admits every waiting request that fits the HBM budget, so
requests that arrive while others are running join the running fixpoints
instead of waiting for them. Each session step advances every active
instance of its program by one iteration; a request finishes at its own
fixpoint, its result rows are copied to the host and its device memory is
released. Latency = completion time - arrival time.

Admission is by an HBM budget: a request is admitted when the bytes the
sessions hold plus the estimated peak bytes of the admitted, unfinished
requests plus its own estimate stay within the budget. The estimate scales
with the input (rows x bytes-per-row per program); it is corrected upward
whenever a finished request turns out larger than estimated. Requests are
admitted in arrival order (no overtaking), and a request that does not fit
an empty server is still admitted alone.

The reference has no served form: each of its drivers runs one program on
one edge file per process (tc.cu:42-423, sg.cu:40-477, wcc.cu:58-585).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

PROGRAMS = ("tc", "sg", "wcc")

# Initial peak device bytes per input row of a request (full relation runs in
# two buffers, the delta and the join output), corrected by observation.
ROW_BYTES = {"tc": 8 * 8 * 64, "sg": 8 * 8 * 8, "wcc": 8 * 8 * 2}


@dataclass
class Request:
    id: int
    program: str
    edges: np.ndarray
    arrival: float = 0.0            # seconds after the start of the run
    admitted: float = -1.0
    done: float = -1.0
    result: object = None           # RunResult (rows on the host)
    est_bytes: int = 0

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclass
class ServeStats:
    requests: int
    seconds: float
    queries_per_s: float
    latency_p50: float
    latency_p95: float
    latency_p99: float
    latency_max: float
    steps: int
    max_active: int
    peak_device_bytes: int
    budget_bytes: int
    waits_on_budget: int
    extra: dict = field(default_factory=dict)

    def as_dict(self) -> dict:
        d = {k: v for k, v in self.__dict__.items() if k != "extra"}
        d.update(self.extra)
        return d


def percentiles(lat: list[float]) -> tuple[float, float, float, float]:
    a = np.asarray(lat, dtype=np.float64)
    if a.size == 0:
        return 0.0, 0.0, 0.0, 0.0
    return (float(np.percentile(a, 50)), float(np.percentile(a, 95)), float(np.percentile(a, 99)),
            float(a.max()))


class Server:
    """Continuous-batching server over one session per program.

    `backend` maps a program name to a session factory; by default the
    sessions come from `engine.session(program)`. Each session object needs
    admit(edges) -> id, step() -> active, poll() -> [ids],
    result(id) -> RunResult, release(id) and memory() -> (bytes, active)."""

    def __init__(self, engine=None, *, budget_bytes: int = 150 * 10**9, wcc_stop: str = "reference",
                 max_active: int = 0, backend=None, clock=time.perf_counter, keep_results: bool = True):
        self.budget = int(budget_bytes)
        self.max_active = max_active
        self.clock = clock
        self.keep_results = keep_results
        if backend is None:
            backend = {p: (lambda p=p: engine.session(p, wcc_stop=wcc_stop)) for p in PROGRAMS}
        self._factory = backend
        self.sessions = {}
        self.row_bytes = dict(ROW_BYTES)
        self.queue: list[Request] = []       # arrived, waiting for admission (arrival order)
        self.running: dict[tuple[str, int], Request] = {}
        self.finished: list[Request] = []
        self.steps = 0
        self.max_active_seen = 0
        self.peak_bytes = 0
        self.budget_waits = 0
        self._t0 = 0.0

    def close(self):
        for s in self.sessions.values():
            s.close()
        self.sessions.clear()

    def _session(self, program: str):
        s = self.sessions.get(program)
        if s is None:
            s = self.sessions[program] = self._factory[program]()
        return s

    def now(self) -> float:
        return self.clock() - self._t0

    def estimate(self, req: Request) -> int:
        return int(len(req.edges) * self.row_bytes[req.program]) + (1 << 20)

    def device_bytes(self) -> int:
        return sum(s.memory()[0] for s in self.sessions.values())

    def _reserved(self) -> int:
        return sum(r.est_bytes for r in self.running.values())

    def admit_waiting(self) -> int:
        """Admits waiting requests in arrival order while they fit."""
        n = 0
        held = self.device_bytes()
        while self.queue:
            req = self.queue[0]
            est = self.estimate(req)
            if self.max_active and len(self.running) >= self.max_active:
                break
            # held bytes already include what running requests allocated, so
            # the reservation of the running requests is an upper bound on top
            if self.running and max(held, self._reserved()) + est > self.budget:
                self.budget_waits += 1
                break
            self.queue.pop(0)
            req.est_bytes = est
            req.admitted = self.now()
            i = self._session(req.program).admit(req.edges)
            self.running[(req.program, i)] = req
            n += 1
            self._collect(req.program)  # instances with no work finish at admission
        return n

    def _collect(self, program: str) -> None:
        s = self.sessions[program]
        for i in s.poll():
            req = self.running.pop((program, i))
            res = s.result(i)  # rows copied to the host
            req.done = self.now()
            req.result = res if self.keep_results else None
            used = s.memory()[0]
            self.peak_bytes = max(self.peak_bytes, used)
            observed = (res.output_tuples * 8 * 3) / max(len(req.edges), 1)
            if observed > self.row_bytes[program]:
                self.row_bytes[program] = observed
            s.release(i)
            self.finished.append(req)

    def step(self) -> int:
        """One iteration of every session with active instances."""
        active = 0
        for p, s in list(self.sessions.items()):
            if s.memory()[1] == 0:
                continue
            s.step()
            self.steps += 1
            self._collect(p)
            active += s.memory()[1]
        self.peak_bytes = max(self.peak_bytes, self.device_bytes())
        self.max_active_seen = max(self.max_active_seen, active)
        return active

    def serve(self, requests: list[Request], *, idle_sleep: float = 0.0002) -> ServeStats:
        """Runs the request stream (arrival times relative to the start)."""
        pending = sorted(requests, key=lambda r: r.arrival)
        k = 0
        self._t0 = self.clock()
        while k < len(pending) or self.queue or self.running:
            t = self.now()
            while k < len(pending) and pending[k].arrival <= t:
                self.queue.append(pending[k])
                k += 1
            self.admit_waiting()
            if self.running:
                self.step()
            elif k < len(pending) and not self.queue:
                wait = pending[k].arrival - self.now()
                if wait > 0:
                    time.sleep(min(wait, idle_sleep) if wait < 0.01 else wait - 0.005)
        total = self.now()
        lat = [r.latency for r in requests]
        p50, p95, p99, mx = percentiles(lat)
        return ServeStats(len(requests), total, len(requests) / total if total > 0 else 0.0, p50, p95, p99, mx,
                          self.steps, self.max_active_seen, self.peak_bytes, self.budget, self.budget_waits)


def poisson_arrivals(count: int, rate: float, rng: np.random.Generator) -> np.ndarray:
    """Arrival times of a Poisson process of `rate` requests/s."""
    return np.cumsum(rng.exponential(1.0 / rate, size=count))


def mixed_requests(count: int, *, lo: int = 1000, hi: int = 500_000, pool: int = 48, seed: int = 0,
                   programs=PROGRAMS) -> list[Request]:
    """A mixed TC/SG/WCC request list: programs uniform, edge counts
    log-uniform in [lo, hi]. Inputs are drawn from a pool of `pool` seeded
    graphs per program (generating every request's graph afresh would take
    longer than serving it); the server keeps no result cache, so a repeated
    input is computed again like any other."""
    from . import graphs
    rng = np.random.default_rng(seed)
    bank = {}
    for p in programs:
        sizes = graphs.log_uniform(pool, lo, hi, rng)
        bank[p] = [graphs.sized(p, int(m), seed=seed * 7919 + j) for j, m in enumerate(sizes)]
    out = []
    for i in range(count):
        p = programs[int(rng.integers(len(programs)))]
        out.append(Request(i, p, bank[p][int(rng.integers(pool))]))
    return out


def serve_plain(engine, requests: list[Request], *, wcc_stop: str = "reference",
                clock=time.perf_counter) -> tuple[float, list[float], list]:
    """One request at a time through the plain engine (no batching): returns
    (total seconds, per-request service seconds, results)."""
    svc, res = [], []
    t0 = clock()
    for r in requests:
        a = clock()
        res.append(engine.run(r.program, r.edges, wcc_stop=wcc_stop))
        svc.append(clock() - a)
    return clock() - t0, svc, res
