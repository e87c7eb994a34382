"""A request loop of steady solves on one GPU (the served configuration):
open-loop Poisson arrivals of terrain tiles, each either a mass-consistent
initial field only (gust::initialize_state, init.first_guess = profile,
steady.stage = none) or a full SIMPLEC solve to the steady criterion.

Continuous batching. A request is admitted as soon as it has arrived and
its device footprint fits the memory budget beside the requests already
running. Each admitted request gets its own CUDA stream, gb_ctx and
resident state, and a host thread drives it, so requests that arrive while
others are on the GPU start at once and their kernels overlap the others'.
A finished request frees its memory, and the queued requests are admitted
in arrival order (backfill). Latency runs from arrival to completion.
Results do not depend on the mix (batch.Member: nothing shared on the
device).

    python -m ablsteadyrans_b200.serve --rate 2 --requests 40

prints one JSON line: requests/s, the p50 and p99 latency, and the counts.
"""
import json
import threading
import time
from collections import deque

import numpy as np


class Request:
    def __init__(self, rid, kind, inst, arrival):
        self.id = rid
        self.kind = kind            # "init" (mass-consistent only) or "rans" (SIMPLEC to the criterion)
        self.inst = inst
        self.arrival = arrival      # seconds after the start
        self.start = None
        self.done = None
        self.status = None
        self.iterations = 0
        self.bytes = 0
        self.result = None

    @property
    def latency(self):
        return None if self.done is None else self.done - self.arrival


def requests_config4(count, rate, seed=0, init_fraction=0.7, precision=1, sizes=None, layers=None):
    """count requests with exponential inter-arrival times at `rate` per
    second; tiles drawn as in the batched configuration; 70 % mass-consistent
    only, 30 % full solves."""
    from . import workloads
    from .batch import CONFIG3_LAYERS, CONFIG3_SIZES
    sizes = sizes or CONFIG3_SIZES
    layers = layers or CONFIG3_LAYERS
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for n in range(count):
        t += rng.exponential(1.0 / rate)
        size = int(rng.choice(sizes))
        nz = int(rng.choice(layers))
        kind = "init" if rng.random() < init_fraction else "rans"
        out.append(Request(n, kind, workloads.tile(size, nz, 5000 + n, precision=precision), t))
    return out


class Server:
    """Admission by device footprint under `budget` bytes, one driving
    thread per admitted request, retire and backfill."""

    def __init__(self, budget, footprint, max_iterations=2000, poll=0.002):
        self.budget = budget
        self.model = footprint      # (a, b): bytes = a + b * padded points
        self.max_iterations = max_iterations
        self.poll = poll
        self.lock = threading.Lock()
        self.in_use = 0
        self.peak = 0
        self.active = 0
        self.peak_active = 0

    def footprint(self, req):
        a, b = self.model
        return int(1.1 * (a + b * req.inst.grid.volume))

    def _serve_one(self, req, t0):
        from .batch import Member
        try:
            m = Member(req.inst)
            if req.kind == "init":
                res = m.stage.initialize()
                m.stream.synchronize()
                req.status = "initialized"
                req.result = {"divergence_before": res.divergence_before, "divergence_after": res.divergence_after,
                              "poisson_iterations": res.poisson_iterations}
            else:
                # the application's order: the mass-consistent initial state, then the
                # stage, driven to the criterion by the C++ driver (one native call)
                from .simplec import run_drivers
                m.stage.initialize()
                (status, n), = run_drivers([m.native], self.max_iterations, 1)
                m.stream.synchronize()
                req.status = status
                req.iterations = n
            m.close()
        except Exception as e:  # the request fails; the server carries on
            req.status = f"error: {e}"
        import torch
        with self.lock:
            torch.cuda.empty_cache()   # the member's stream-bound blocks go back to the device
        req.done = time.perf_counter() - t0
        with self.lock:
            self.in_use -= req.bytes
            self.active -= 1

    def run(self, requests):
        """Serves the requests (sorted by arrival); returns the wall time (s)."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        queue = deque()
        threads = []
        t0 = time.perf_counter()
        while pending or queue:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            while queue:
                req = queue[0]
                need = self.footprint(req)
                with self.lock:
                    fits = self.in_use + need <= self.budget or self.active == 0
                    if fits:
                        self.in_use += need
                        self.active += 1
                        self.peak = max(self.peak, self.in_use)
                        self.peak_active = max(self.peak_active, self.active)
                if not fits:
                    break
                queue.popleft()
                req.bytes = need
                req.start = time.perf_counter() - t0
                th = threading.Thread(target=self._serve_one, args=(req, t0), daemon=True)
                th.start()
                threads.append(th)
            time.sleep(self.poll)
        for th in threads:
            th.join()
        return time.perf_counter() - t0


def sequential_latencies(arrivals, services):
    """FIFO one-at-a-time service of requests arriving at `arrivals` (sorted)
    with service times `services`: each starts when it has arrived and the
    one before it is done. Returns the latencies (done - arrival)."""
    done = 0.0
    out = []
    for a, sv in zip(arrivals, services):
        start = max(a, done)
        done = start + sv
        out.append(done - a)
    return out


def sequential_services(count, seed=0, sizes=None, layers=None, max_iterations=1500):
    """The plain FP64 sequential path's service time of each request (the
    same tiles and kinds as requests_config4 at any rate: the arrival draws
    do not move the tile draws), each one alone: the initializer, then the
    C++ driver to the criterion or the cap. Returns (services, statuses)."""
    import torch

    from .batch import Member
    from .simplec import run_drivers
    seq = requests_config4(count, 1.0, seed, precision=0, sizes=sizes, layers=layers)
    services = []
    for req in seq:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m = Member(req.inst)
        m.stage.initialize()
        if req.kind == "rans":
            (req.status, req.iterations), = run_drivers([m.native], max_iterations, 1)
        m.stream.synchronize()
        services.append(time.perf_counter() - t0)
        m.close()
        del m
        torch.cuda.empty_cache()
    return services, [r.status for r in seq]


def serve_sweep(rates, count=12, seed=0, sizes=None, layers=None, max_iterations=1500, budget=150e9):
    """The served form against the plain FP64 sequential path on the same
    requests, at each arrival rate of `rates`: (1) the server (continuous
    batching, FP32 inner solves), latencies from arrival to completion;
    (2) the requests in plain FP64 served one at a time in arrival order:
    each one's service time measured alone once (sequential_services), its
    latency from the FIFO queue over that rate's arrivals. Returns one dict
    per rate with p50/p99 latency and solves/s of each form."""
    model = calibrate_footprint()
    services, statuses = sequential_services(count, seed, sizes, layers, max_iterations)
    out = []
    for rate in rates:
        served = requests_config4(count, rate, seed, precision=1, sizes=sizes, layers=layers)
        srv = Server(budget, model, max_iterations=max_iterations)
        wall = srv.run(served)
        lat = np.array([r.latency for r in served])
        arrivals = [r.arrival for r in served]
        slat = np.array(sequential_latencies(arrivals, services))
        makespan = max(a + l for a, l in zip(arrivals, slat))
        out.append({
            "requests": count, "rate_per_s": rate, "full_solves": sum(1 for r in served if r.kind == "rans"),
            "served_fp32_inner": {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                                  "solves_per_s": count / wall, "wall_s": wall,
                                  "steady": sum(1 for r in served if r.status == "steady"),
                                  "capped": sum(1 for r in served if r.kind == "rans" and r.status == "running"),
                                  "peak_concurrent": srv.peak_active},
            "sequential_fp64": {"p50_s": float(np.percentile(slat, 50)), "p99_s": float(np.percentile(slat, 99)),
                                "solves_per_s": count / makespan, "makespan_s": makespan,
                                "service_s_total": float(sum(services)),
                                "steady": sum(1 for st in statuses if st == "steady")},
        })
    return out


def serve_vs_sequential(count=12, rate=2.0, seed=0, sizes=None, layers=None, max_iterations=1500, budget=150e9):
    """serve_sweep at one rate."""
    return serve_sweep([rate], count, seed, sizes, layers, max_iterations, budget)[0]


def measure_peak_bytes(n, nz):
    """Peak device bytes of one request on an n x n x nz tile: the resident
    member plus the initializer's Poisson solver, which lives only while the
    initial state is projected."""
    import torch

    import ablsteadyrans_b200 as gb
    from . import workloads
    from .batch import Member
    inst = workloads.tile(n, nz, 0)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    m = Member(inst)
    opts = gb.PoissonOptions.default(precision=inst.options.precision)
    ps = gb.PoissonSolver(m.ctx, inst.grid, m.case.z, m.case.J, [1, 1, 1, 2, 2, 1], opts)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    ps.close()
    m.close()
    del m
    torch.cuda.empty_cache()
    return max(free0 - free1, 1), inst.grid.volume


def calibrate_footprint():
    """(a, b) of the footprint model bytes = a + b * volume (padded points),
    fitted on a small and a large tile (fixed per-request costs dominate
    small tiles)."""
    b1, v1 = measure_peak_bytes(64, 48)
    b2, v2 = measure_peak_bytes(128, 64)
    b = max((b2 - b1) / (v2 - v1), 1.0)
    a = max(b1 - b * v1, 0.0)
    return a, b


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--rate", type=float, default=2.0, help="arrivals per second (open loop)")
    ap.add_argument("--requests", type=int, default=40)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--max-iterations", type=int, default=300, help="cap of a full solve's outer iterations")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", type=int, default=1, choices=[0, 1])
    args = ap.parse_args(argv)
    model = calibrate_footprint()
    reqs = requests_config4(args.requests, args.rate, args.seed, precision=args.precision)
    srv = Server(args.budget_gb * 1e9, model, max_iterations=args.max_iterations)
    wall = srv.run(reqs)
    lat = np.array([r.latency for r in reqs if r.latency is not None])
    by_kind = {k: np.array([r.latency for r in reqs if r.kind == k and r.latency is not None]) for k in ("init", "rans")}
    line = {
        "metric": "requests/s", "unit": "requests/s", "value": len(lat) / wall,
        "rate": args.rate, "requests": len(reqs), "wall_s": wall,
        "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
        "p50_init_s": float(np.percentile(by_kind["init"], 50)) if len(by_kind["init"]) else None,
        "p50_rans_s": float(np.percentile(by_kind["rans"], 50)) if len(by_kind["rans"]) else None,
        "steady": sum(1 for r in reqs if r.status == "steady"),
        "diverged": sum(1 for r in reqs if r.status == "diverged"),
        "capped": sum(1 for r in reqs if r.kind == "rans" and r.status == "running"),
        "errors": [r.status for r in reqs if r.status and r.status.startswith("error")][:3],
        "peak_concurrent": srv.peak_active, "peak_bytes": srv.peak,
        "footprint_model": {"fixed_bytes": model[0], "bytes_per_point": model[1]},
        "max_iterations": args.max_iterations,
    }
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
