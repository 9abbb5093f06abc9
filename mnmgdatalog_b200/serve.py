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
requests plus its own estimate stay within the budget. The budget is capped
at construction by the device memory then free, less what each worker
context may keep cached for reuse (`cache_gib`), so that the sessions'
buffers always fit beside everything else on the device. The estimate scales
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


class PinnedPool:
    """Reusable page-locked host buffers for result rows.

    A device-to-host copy into freshly allocated pageable memory runs at a
    small fraction of the link rate (page faults and an extra staging copy),
    so results are delivered into pooled pinned buffers instead; a consumer
    done with a result hands its buffer back with give(). Buffers come in
    power-of-two row classes; past `limit_bytes` of pinned memory, take()
    returns None and the caller falls back to pageable memory."""

    def __init__(self, limit_bytes: int = 8 << 30):
        self.limit = limit_bytes
        self.total = 0
        self.free: dict[int, list] = {}
        self._keep = {}

    def take(self, rows: int):
        if rows <= 0:
            return None
        cls = max(1024, 1 << (int(rows) - 1).bit_length())
        lst = self.free.get(cls)
        if lst:
            return lst.pop()
        if self.total + cls * 8 > self.limit:
            return None
        import torch
        t = torch.empty((cls, 2), dtype=torch.int32, pin_memory=True)
        a = t.numpy()
        self._keep[id(a)] = t
        self.total += cls * 8
        return a

    def give(self, arr) -> None:
        if arr is not None and id(arr) in self._keep:
            self.free.setdefault(len(arr), []).append(arr)


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


def device_headroom(device: int, workers: int, cache_gib: int, margin_gib: int = 2) -> int:
    """Bytes the sessions may hold on `device`: the memory free now, less
    `cache_gib` GiB of reuse cache per worker context and a margin for the
    contexts' small fixed buffers."""
    import torch
    free, _ = torch.cuda.mem_get_info(device)
    return max(0, int(free) - (workers * int(cache_gib) + margin_gib) * (1 << 30))


class Server:
    """Continuous-batching server over one session per program.

    `backend` maps a program name to a session factory; by default the
    sessions come from `engine.session(program)`. Each session object needs
    admit_many([edges]) -> [ids], step() -> active, poll() -> [ids],
    result(id) -> RunResult, release(id) and memory() -> (bytes, active)."""

    def __init__(self, engine=None, *, budget_bytes: int = 150 * 10**9, wcc_stop: str = "reference",
                 max_active: int = 0, backend=None, clock=time.perf_counter, keep_results: bool = True,
                 concurrent: bool = False, output: str = "host", pinned: bool = False, tuning: dict | None = None,
                 cache_gib: int = 4):
        self.budget = int(budget_bytes)
        self.output = output  # where result rows go: "host" (delivered), "device" or "none"
        self.pool = PinnedPool() if (pinned and output == "host") else None
        self.max_active = max_active
        self.clock = clock
        self.keep_results = keep_results
        self.concurrent = concurrent
        self._engines = []
        if backend is None:
            if concurrent:
                # one context (and stream) per program: the programs' union
                # fixpoints run side by side on the device
                from .engine import Engine
                backend = {}
                for p in PROGRAMS:
                    e = Engine(engine.device)
                    if tuning:
                        e.set_tuning(tuning)
                    # buffers a worker keeps for reuse are outside the sessions'
                    # accounting: keep them small and leave room for them below
                    e.set_tuning(cache_max_gib=cache_gib)
                    self._engines.append(e)
                    backend[p] = (lambda p=p, e=e: e.session(p, wcc_stop=wcc_stop))
            else:
                backend = {p: (lambda p=p: engine.session(p, wcc_stop=wcc_stop)) for p in PROGRAMS}
            if self._engines:
                room = device_headroom(engine.device, len(self._engines), cache_gib)
            else:  # the sessions share the caller's context and its cache limit
                room = device_headroom(engine.device, 1, engine.tuning()["cache_max_gib"])
            self.budget = min(self.budget, room)
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
        import threading
        self._pool_lock = threading.Lock()

    def reset_stats(self) -> None:
        """Forgets the counters of previous serve() calls (sessions stay)."""
        self.finished = []
        self.steps = 0
        self.max_active_seen = 0
        self.peak_bytes = 0
        self.budget_waits = 0

    def close(self):
        for s in self.sessions.values():
            s.close()
        self.sessions.clear()
        for e in self._engines:
            e.close()
        self._engines = []

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
        """Admits waiting requests in arrival order while they fit; the
        admitted requests of each program join their session in one call."""
        take: list[Request] = []
        held = self.device_bytes()
        reserved = self._reserved()
        while self.queue:
            req = self.queue[0]
            est = self.estimate(req)
            if self.max_active and len(self.running) + len(take) >= self.max_active:
                break
            # held bytes already include what running requests allocated, so
            # the reservation of the running requests is an upper bound on top
            if (self.running or take) and max(held, reserved) + est > self.budget:
                self.budget_waits += 1
                break
            self.queue.pop(0)
            req.est_bytes = est
            reserved += est
            take.append(req)
        now = self.now()
        for p in PROGRAMS:
            group = [r for r in take if r.program == p]
            if not group:
                continue
            ids = self._session(p).admit_many([r.edges for r in group])
            for r, i in zip(group, ids):
                r.admitted = now
                self.running[(p, i)] = r
            self._collect(p)  # instances with no work finish at admission
        return len(take)

    def _collect(self, program: str) -> None:
        s = self.sessions[program]
        for i in s.poll():
            req = self.running.pop((program, i))
            res, buf = self._result(s, i)
            req.done = self.now()
            req.result = res if self.keep_results else None
            if not self.keep_results and self.pool is not None:
                self.pool.give(buf)
            used = s.memory()[0]
            self.peak_bytes = max(self.peak_bytes, used)
            observed = (res.output_tuples * 8 * 3) / max(len(req.edges), 1)
            if observed > self.row_bytes[program]:
                self.row_bytes[program] = observed
            s.release(i)
            self.finished.append(req)

    def _result(self, s, i):
        """(RunResult, pooled buffer or None) of a finished instance."""
        if self.pool is None:
            return s.result(i, output=self.output), None
        got = []

        def take(n):
            with self._pool_lock:
                got.append(self.pool.take(n))
            return got[0]

        res = s.result(i, output=self.output, out=take)
        return res, (got[0] if got else None)

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
        self.reset_stats()
        if self.concurrent:
            return self._serve_threads(requests)
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
        return self._stats(requests, self.now())

    def _stats(self, requests, total) -> ServeStats:
        lat = [r.latency for r in requests]
        p50, p95, p99, mx = percentiles(lat)
        return ServeStats(len(requests), total, len(requests) / total if total > 0 else 0.0, p50, p95, p99, mx,
                          self.steps, self.max_active_seen, self.peak_bytes, self.budget, self.budget_waits)

    # ---- one worker thread per program ---------------------------------------
    def _serve_threads(self, requests: list[Request]) -> ServeStats:
        """The same loop with one worker per program. The main thread moves
        arrivals into the queue and admits them (arrival order, budget) into
        per-program inboxes; each worker admits its inbox into its session
        between two steps and steps its session; the library releases the
        interpreter lock inside every call, so the programs' steps overlap on
        the device."""
        import threading
        pending = sorted(requests, key=lambda r: r.arrival)
        cond = threading.Condition()
        inbox = {p: [] for p in PROGRAMS}
        held = {p: 0 for p in PROGRAMS}
        active = {p: 0 for p in PROGRAMS}
        admitting = {p: [] for p in PROGRAMS}  # taken from the inbox, not yet in self.running
        state = {"stop": False, "error": None}
        sessions = {p: self._session(p) for p in PROGRAMS}

        def worker(p):
            s = sessions[p]
            try:
                while True:
                    with cond:
                        while not inbox[p] and active[p] == 0 and not state["stop"]:
                            cond.wait()
                        if state["stop"] and not inbox[p] and active[p] == 0:
                            return
                        batch, inbox[p] = inbox[p], []
                        admitting[p] = batch
                    if batch:
                        ids = s.admit_many([r.edges for r in batch])
                        now = self.now()
                        with cond:
                            for r, i in zip(batch, ids):
                                r.admitted = now
                                self.running[(p, i)] = r
                            admitting[p] = []
                    done = self._collect_unlocked(p, s, cond)
                    if s.memory()[1]:
                        s.step()
                        done += self._collect_unlocked(p, s, cond)
                    b, a = s.memory()
                    with cond:
                        self.steps += 1
                        held[p], active[p] = b, a
                        self.peak_bytes = max(self.peak_bytes, sum(held.values()))
                        self.max_active_seen = max(self.max_active_seen, sum(active.values()))
                        if done or batch:
                            cond.notify_all()
            except BaseException as exc:  # surfaced by serve()
                with cond:
                    state["error"] = exc
                    state["stop"] = True
                    cond.notify_all()

        threads = [threading.Thread(target=worker, args=(p,), daemon=True) for p in PROGRAMS]
        k = 0
        self._t0 = self.clock()
        for t in threads:
            t.start()
        try:
            with cond:
                while not state["error"]:
                    t = self.now()
                    while k < len(pending) and pending[k].arrival <= t:
                        self.queue.append(pending[k])
                        k += 1
                    queued = [r for q in inbox.values() for r in q] + [r for q in admitting.values() for r in q]
                    reserved = sum(r.est_bytes for r in self.running.values()) + sum(r.est_bytes for r in queued)
                    waiting = len(queued)
                    while self.queue:
                        req = self.queue[0]
                        est = self.estimate(req)
                        busy = len(self.running) + waiting
                        if self.max_active and busy >= self.max_active:
                            break
                        if busy and max(sum(held.values()), reserved) + est > self.budget:
                            self.budget_waits += 1
                            break
                        self.queue.pop(0)
                        req.est_bytes = est
                        reserved += est
                        waiting += 1
                        inbox[req.program].append(req)
                    cond.notify_all()
                    if k == len(pending) and not self.queue and not self.running and not any(inbox.values()) \
                            and not any(admitting.values()) and not any(active.values()):
                        break
                    timeout = 0.05
                    if k < len(pending):
                        timeout = min(timeout, max(pending[k].arrival - self.now(), 0.0))
                    if timeout > 0:
                        cond.wait(timeout)
                state["stop"] = True
                cond.notify_all()
        finally:
            with cond:
                state["stop"] = True
                cond.notify_all()
            for t in threads:
                t.join()
        if state["error"] is not None:
            raise state["error"]
        return self._stats(requests, self.now())

    def _collect_unlocked(self, program: str, s, cond) -> int:
        """Finished instances of one session: result rows to the host, then
        bookkeeping under the lock. Returns how many finished."""
        n = 0
        for i in s.poll():
            res, buf = self._result(s, i)
            done = self.now()
            s.release(i)
            with cond:
                req = self.running.pop((program, i))
                req.done = done
                req.result = res if self.keep_results else None
                if not self.keep_results and self.pool is not None:
                    self.pool.give(buf)
                observed = (res.output_tuples * 8 * 3) / max(len(req.edges), 1)
                if observed > self.row_bytes[program]:
                    self.row_bytes[program] = observed
                self.finished.append(req)
            n += 1
        return n


def poisson_arrivals(count: int, rate: float, rng: np.random.Generator) -> np.ndarray:
    """Arrival times of a Poisson process of `rate` requests/s."""
    return np.cumsum(rng.exponential(1.0 / rate, size=count))


def relabel(edges: np.ndarray, seed: int) -> np.ndarray:
    """The same graph under a seeded injective map of node ids,
    id -> (a * id + b) mod (2^31 - 1) (a prime modulus, a != 0): a distinct
    input with the same structure, the same closure sizes and different
    result rows. Ids stay in [0, 2^31 - 2], so never the reference's -1."""
    P = 2**31 - 1
    rng = np.random.default_rng(seed)
    a = int(rng.integers(1, P))
    b = int(rng.integers(0, P))
    e = np.asarray(edges, dtype=np.int64)
    return ((e * a + b) % P).astype(np.int32)


def mixed_requests(count: int, *, lo: int = 1000, hi: int = 500_000, pool: int = 48, seed: int = 0,
                   programs=PROGRAMS, distinct: bool = False) -> list[Request]:
    """A mixed TC/SG/WCC request list: programs uniform, edge counts
    log-uniform in [lo, hi]. Inputs come from a pool of `pool` seeded graphs
    per program (generating every request's graph afresh would take longer
    than serving it); with `distinct`, every request relabels its pool graph
    by its own seeded id map (relabel), so no two requests carry the same
    input. The server keeps no result cache either way."""
    from . import graphs
    rng = np.random.default_rng(seed)
    bank = {}
    for p in programs:
        sizes = graphs.log_uniform(pool, lo, hi, rng)
        bank[p] = [graphs.sized(p, int(m), seed=seed * 7919 + j) for j, m in enumerate(sizes)]
    out = []
    for i in range(count):
        p = programs[int(rng.integers(len(programs)))]
        e = bank[p][int(rng.integers(pool))]
        out.append(Request(i, p, relabel(e, seed * 1_000_003 + i) if distinct else e))
    return out


def serve_plain(engine, requests: list[Request], *, wcc_stop: str = "reference", clock=time.perf_counter,
                pinned: bool = False, keep_results: bool = True) -> tuple[float, list[float], list]:
    """One request at a time through the plain engine (no batching): returns
    (total seconds, per-request service seconds, results). With `pinned`,
    rows land in one reused page-locked buffer (grown on demand), the same
    delivery the server uses; results then hold row counts only unless
    keep_results copies them out."""
    svc, res = [], []
    buf = None
    t0 = clock()
    for r in requests:
        a = clock()
        if pinned:
            def grow(n):
                nonlocal buf
                if buf is None or len(buf) < n:
                    import torch
                    cap = max(1024, 1 << max(int(n) - 1, 1).bit_length())
                    buf = torch.empty((cap, 2), dtype=torch.int32, pin_memory=True).numpy()
                return buf
            x = engine.run(r.program, r.edges, wcc_stop=wcc_stop, out=grow)
            if keep_results:
                x.rows = x.rows.copy()
        else:
            x = engine.run(r.program, r.edges, wcc_stop=wcc_stop)
        res.append(x)
        svc.append(clock() - a)
    return clock() - t0, svc, res
