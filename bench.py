"""Benchmark of the overworld TERRAIN step on B200 (one JSON line on rank 0).

Workload (the reference's ladder size): one seed, three 64x64-chunk regions of 4,096
chunks each -- at the origin, at block -1,000,000 (chunk -62,500) and touching the
+1,874,999-block border (chunk 117,187 is the region's last chunk). A step is the full
TERRAIN step over all 12,288 chunks: biomes, density with caves, aquifers, ore veins and
material rules, u16 block states and u8 quart biomes out.

  value      chunks/s with the chunk lists already in HBM and the outputs left in HBM
             (tg_generate_device, the step's 12,288 chunks as one batch), device time from
             CUDA events on the launching stream
  e2e        chunks/s through tg_generate_u8 -- the reference generator's own call and output
             type (u8 palette index per block) -- with host buffers: the chunk list is copied
             in and every block and biome byte copied out to pinned memory inside the step;
             e2e_u16 is the same through tg_generate (u16 block states, the CPU port's type)
  roofline   the channel-corner kernel against the issue rate: its work counted on the host
             twin of the kernel bodies (octave samples per distinct corner point) times a
             minimal instruction recipe per sample, over its CUDA-event launch time;
             roofline_walk_hbm gives the column walk's HBM fraction (417,792 B per chunk over
             its launch time, against the measured HBM copy peak)
  reference_gpu  the reference's own GPU generator built for sm_100a on the same step and
             model (baseline/): end to end and kernels only, with our ratios
  cpu_baseline  the reference's own C++ port (oracle/_ref) on this host's cores: a 16x16
             region on 1 thread and a 32x32 region on all threads, as its bench does

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, 'minecraft-terrain-cuda_b200'))
sys.path.insert(0, os.path.join(REPO, 'oracle'))

SEED = 0x5445525241494E31   # "TERRAIN1"
REGIONS = [('origin', 0, 0), ('negative', -62500, -62500), ('border', 117124, 117124)]
SIDE = 64
BYTES_PER_CHUNK = 98304 * 2 + 1536
BYTES_PER_CHUNK_U8 = 98304 + 1536
# data the walk-rules kernel touches once per chunk: the u8 biome and u8 ore-vein bits of each
# block read, its u16 state written, and the column air / fluid masks (2 x 12 words x 256 columns)
WALK_BYTES_PER_CHUNK = 98304 * (1 + 1 + 2) + 2 * 12 * 4 * 256
# dram__bytes_read.sum + dram__bytes_write.sum of one 12,288-chunk launch of the walk-rules
# kernel in this workload: a one-pass ncu capture of a 4,096-chunk launch (515.35 MB + 288.65
# MB) scaled by the chunks a launch processes (the traffic is per block, so it grows with
# them)
WALK_TRAFFIC_PER_LAUNCH = 3 * 803998464
# Instructions (per thread) one octave sample needs at least, by pipe, following the
# reference's perlin_volume (cpu/include/mccuda/noise_eval.h:163-178): per axis the coordinate
# in FP64 (scale multiply, wrap test, offset add, floor, floor back to double, subtract,
# double-to-float: 7; the block coordinate's conversion is shared by a stack's layers) and
# its smoothstep (7 FP32); 7 loads of a paired permutation table (both neighbours of a
# lattice step in one entry) with an add and a mask each and 8 byte extracts; 8 lattice
# gradients of two non-zero unit components (a sign flip and an add each in FP32, 3 integer
# selects); the corner offsets (3 FP32), the trilinear lerp (7 x 3 FP32) and the amplitude
# accumulate (3 FP32).
VOL_OCTAVE_INSTR = {'fp64': 21, 'fp32': 21 + 16 + 3 + 21 + 3, 'alu': 14 + 8 + 24, 'lsu': 7}
OP_COUNTS = os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'model', 'op_counts.json')
METRIC = 'bit-exact TERRAIN chunks/s on 1 B200, served vs plain; p50/p99 request latency'


def json_default(o):
    """numpy scalars and arrays in the bench line as plain JSON values."""
    if isinstance(o, np.generic):
        return o.item()
    if isinstance(o, np.ndarray):
        return o.tolist()
    raise TypeError('not JSON serializable: %r' % type(o))


def model_sha256():
    """SHA-256 of the world model files the library is built from (the workload's definition)."""
    import hashlib
    d = os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'model')
    return {f: hashlib.sha256(open(os.path.join(d, f), 'rb').read()).hexdigest() for f in ('overworld_ir.json', 'overworld_terrain.json')}


def samples_per_chunk():
    """Octave and simplex samples the kernels evaluate per chunk of a large region, counted on
    the kernel bodies (op_counts.json): the work behind each chunk/s figure of this model."""
    try:
        with open(OP_COUNTS) as f:
            doc = json.load(f)['kernels']
    except (OSError, KeyError):
        return None
    u = doc['units_in_sample']
    # units per chunk of a 64 x 64 region (distinct corner columns and biome chunks of the square;
    # distinct surface-level quarts as in the counted sample)
    per = {'corner': 257 * 257 * 49 / 4096.0, 'corner_col': 257 * 257 / 4096.0, 'climate_col': 66 * 66 / 4096.0, 'climate_quart': 66 * 66 / 4096.0,
           'surface_level': u['surface_quarts'] / float(u['chunks'])}
    total = 0.0
    for name, rec in doc['per_kernel'].items():
        total += sum(rec['samples_per_unit'].values()) * per.get(name, 1.0)
    return round(total, 1)


def region_chunks(x0, z0, side=SIDE):
    return np.array([(x0 + x, z0 + z) for z in range(side) for x in range(side)], np.int32)


def peaks():
    try:
        with open(os.path.join(REPO, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
        return float(p['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


class ClockSampler:
    """SM clock and clock-event reasons of the GPU sampled during the timed region: NVML
    queries (read only) every 5 ms on a thread, from before the region starts to its end;
    nvidia-smi at 100 ms when NVML cannot be loaded. dev is the CUDA device ordinal; the
    NVML handle is found by its PCI address."""

    REASONS = (('hw_slowdown', 0x8), ('hw_thermal_slowdown', 0x40), ('sw_thermal_slowdown', 0x20), ('sw_power_cap', 0x4))

    def __init__(self, dev):
        self.dev = dev
        self.samples = []          # (sm MHz, reason bits)
        self.max_mhz = None
        self.stop = threading.Event()
        self.proc = None
        self.lines = []
        self.t = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.dev)
        try:
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId('%08x:%02x:%02x.0' % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id))
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def _poll(self, nv, h):
        while not self.stop.is_set():
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
            except Exception:
                pass
            self.stop.wait(0.005)

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.t.start()
            while not self.samples and self.t.is_alive():   # the first sample precedes the region
                time.sleep(0.001)
            return self
        except Exception:
            self.t = None
        cmd = ['nvidia-smi', '-i', str(self.dev), '--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
               'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
               'clocks_event_reasons.sw_power_cap', '--format=csv,noheader,nounits', '-lms', '100']
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        elif self.t:
            self.t.join(timeout=1)

    def summary(self):
        sm, mx, reasons = [], self.max_mhz, set()
        for mhz, bits in self.samples:
            sm.append(float(mhz))
            for name, bit in self.REASONS:
                if bits & bit:
                    reasons.add(name)
        for l in self.lines:
            f = [x.strip() for x in l.split(',')]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for (n, _), v in zip(self.REASONS, f[4:8]):
                if v.lower() == 'active':
                    reasons.add(n)
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': mx, 'reasons': sorted(reasons), 'samples': len(sm),
                'source': 'nvml 5 ms' if self.samples else 'nvidia-smi 100 ms'}


def host_cores():
    """(hardware threads usable by this process, physical cores of the host)."""
    try:
        threads = len(os.sched_getaffinity(0))
    except AttributeError:
        threads = os.cpu_count()
    try:
        import psutil
        physical = psutil.cpu_count(logical=False)
    except Exception:
        physical = None
    return threads, physical


def cpu_baseline(threads=None):
    """The reference C++ port on this host, sized as the reference's own bench times it
    (bench/bench_main.cpp:253-304, README.md:30-31): region form (biomes of the region plus a
    one-chunk border computed once per chunk, then fill + surface per chunk), a 16x16-chunk
    region on one thread and a 32x32-chunk region on all hardware threads, each at the corner
    of the ladder's origin region."""
    import ref_oracle
    if not ref_oracle.available():
        return None
    m = ref_oracle.RefModel()
    s = m.seed(SEED)
    hw, physical = host_cores()
    threads = threads or hw
    big = region_chunks(0, 0, 32)
    s.generate(big[:threads], threads=threads)   # warm the caches / page in
    t0 = time.perf_counter()
    s.generate(big, threads=threads)
    dt = time.perf_counter() - t0
    one = region_chunks(0, 0, 16)
    t0 = time.perf_counter()
    s.generate(one, threads=1)
    dt1 = time.perf_counter() - t0
    return {'value': round(len(big) / dt, 2), 'unit': 'chunks/s', 'cores': threads, 'kind': 'reference',
            'value_1_thread': round(len(one) / dt1, 2), 'hardware_threads': hw, 'physical_cores': physical,
            'sample': '32x32-chunk region at the origin on %d threads (%d chunks, %.1f s); 1-thread figure from the 16x16-chunk '
                      'region at the origin (%d chunks, %.1f s); region form, biomes of the region plus a one-chunk border'
                      % (threads, len(big), dt, len(one), dt1)}


def run_reference(args, rank):
    """Reference arm: the reference's own C++ port (oracle/_ref) on all host threads. Each step
    is a 32x32-chunk region (the size the reference's own bench times on all threads), in
    region form, taken in turn from a quadrant of each of the three ladder regions."""
    if rank != 0:
        return
    import ref_oracle
    if not ref_oracle.available():
        print(json.dumps({'impl': 'reference', 'unavailable': 'oracle/_ref not built (the reference C++ port compiles only where its sources are)'}))
        return
    m = ref_oracle.RefModel()
    s = m.seed(SEED)
    threads, physical = host_cores()
    sets = []
    for k in range(args.warmup + args.steps):
        _, x0, z0 = REGIONS[k % len(REGIONS)]
        q = (k // len(REGIONS)) % 4
        sets.append(region_chunks(x0 + 32 * (q % 2), z0 + 32 * (q // 2), 32))
    per_step = sets[0].shape[0]
    for k in range(args.warmup):
        s.generate(sets[k], threads=threads)
    t0 = time.perf_counter()
    for k in range(args.steps):
        s.generate(sets[args.warmup + k], threads=threads)
    dt = time.perf_counter() - t0
    v = per_step * args.steps / dt
    line = {'metric': METRIC, 'value': round(v, 2), 'unit': 'chunks/s', 'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': round(1000 * dt / args.steps, 3), 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32+f64+int',
            'data': 'synthetic world model (project-authored, reference JSON formats); seeded chunk lists', 'impl': 'reference',
            'config': {'workload': 'ladder: one seed, three 64x64-chunk regions (origin, -1,000,000 blocks, +1,874,999-block border)',
                       'per_step_sample': '%d chunks: a 32x32-chunk quadrant of one ladder region per step, in turn, region form, '
                                          'the reference C++ port on %d host threads' % (per_step, threads)},
            'cpu_baseline': {'value': round(v, 2), 'unit': 'chunks/s', 'cores': threads, 'kind': 'reference', 'hardware_threads': threads,
                             'physical_cores': physical, 'sample': '%d chunks per step (a 32x32 region)' % per_step},
            'e2e': {'value': round(v, 2), 'unit': 'chunks/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line))


def pcie_d2h_gbs(nbytes=1 << 30, reps=5):
    """Device-to-pinned-host copy bandwidth of this box (GB/s), one 1 GiB copy at a time."""
    import torch
    d = torch.empty(nbytes, dtype=torch.uint8, device='cuda')
    h = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    h.copy_(d, non_blocking=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        h.copy_(d, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    return round(reps * nbytes / (e0.elapsed_time(e1) / 1000.0) / 1e9, 2)


def max_over_ranks(value, world, device=None):
    """The step time every rank reports: the maximum over ranks (all_reduce MAX)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], device=device) if device is not None else torch.tensor([float(value)])
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def serving_requests(n, rng):
    """View-distance requests: a (2r+1)^2 square or the ring of radius r (r in 2..12) around a
    uniform centre within +/-117,187 chunks; seeds from a pool of 64."""
    seeds = [int(v) for v in rng.integers(-(1 << 62), 1 << 62, 64)]
    reqs = []
    for _ in range(n):
        r = int(rng.integers(2, 13))
        cx, cz = (int(v) for v in rng.integers(-117187 + r, 117187 - r, 2))
        if rng.random() < 0.5:
            chunks = [(cx + dx, cz + dz) for dz in range(-r, r + 1) for dx in range(-r, r + 1)]
        else:
            chunks = [(cx + dx, cz + dz) for dz in range(-r, r + 1) for dx in range(-r, r + 1) if max(abs(dx), abs(dz)) == r]
        reqs.append((seeds[int(rng.integers(0, 64))], np.array(chunks, np.int32)))
    return seeds, reqs


def p99_interval(lat):
    """(p99, low, high): the 99th percentile of the latencies and its 95 % interval from the
    order statistics (binomial ranks n * 0.99 -/+ 1.96 sqrt(n * 0.99 * 0.01))."""
    v = np.sort(np.asarray(lat))
    n = v.shape[0]
    if n == 0:
        return None, None, None
    sd = 1.96 * np.sqrt(n * 0.99 * 0.01)
    lo = int(max(0, np.floor(n * 0.99 - sd) - 1))
    hi = int(min(n - 1, np.ceil(n * 0.99 + sd) - 1))
    return float(np.quantile(v, 0.99)), float(v[lo]), float(v[hi])


def served_bench(g, n_unique=96, batch_chunks=768, loads=(0.6, 0.7, 0.8), seed=2024, p99_target_ms=20.0, seconds=10.0, min_requests=5000):
    """Plain against served on a stream of view-distance requests (squares and rings of radius
    2-12 around centres within +/-117,187 chunks, seeds from a resident pool): the plain
    form is one synchronous tg_generate per request, in order; the server runs the same
    stream in both output forms (u16, and u8 through tg_server_submit_u8). For each form: the
    saturated throughput (everything submitted at once), then Poisson arrivals at each
    fraction in `loads` of it, each point lasting at least `seconds` and `min_requests`
    requests, with p50 and p99 (and the p99's 95 % interval) of submit -> last byte on the
    host. A point is steady when it served at least 97 % of what was offered; the best
    steady point under the p99 target is reported. Outputs go to pinned host memory (a
    request re-submitted reuses its buffers)."""
    import torch
    import terrain_b200
    rng = np.random.default_rng(seed)
    seeds, reqs = serving_requests(n_unique, rng)
    h = g.height
    sizes = [len(c) for _, c in reqs]
    per16 = 256 * h + 768
    pool = torch.empty(sum(sizes) * per16, dtype=torch.int16, pin_memory=True).numpy().view(np.uint16)
    offs, at = [], 0
    for n in sizes:
        offs.append(at)
        at += n * per16

    def bufs(i, u8):
        n = sizes[i]
        base = pool[offs[i]:offs[i] + n * per16]
        q = base[n * 256 * h:].view(np.uint8)[:n * 1536].reshape(n, 1536)
        b = base[:n * 256 * h]
        return (b.view(np.uint8)[:n * 256 * h].reshape(n, h, 16, 16) if u8 else b.reshape(n, h, 16, 16)), q

    mean_chunks = float(np.mean(sizes))
    for sd in seeds:                      # resident tables for the whole pool
        g.set_seed(sd)
    g.generate(reqs[0][1][:1])
    # plain: synchronous calls in order for about `seconds / 2`
    done, t0 = 0, time.perf_counter()
    k = 0
    while time.perf_counter() - t0 < seconds / 2 or k < n_unique:
        i = k % n_unique
        b, q = bufs(i, False)
        g.set_seed(reqs[i][0])
        g.generate(reqs[i][1], blocks_out=b, biomes_out=q)
        done += sizes[i]
        k += 1
    plain_cps = done / (time.perf_counter() - t0)
    out = {'seed_pool': 64, 'unique_requests': n_unique, 'mean_request_chunks': round(mean_chunks, 1), 'plain_chunks_per_s': round(plain_cps, 1),
           'plain_requests': k, 'batch_chunks': batch_chunks, 'p99_target_ms': p99_target_ms, 'forms': {}}
    for form in ('u16', 'u8'):
        u8 = form == 'u8'
        res = {'points': []}
        with terrain_b200.TerrainServer(g, batch_chunks=batch_chunks) as srv:
            for t in [srv.submit(reqs[i][0], reqs[i][1], *bufs(i, u8), u8=u8) for i in range(4)]:
                srv.wait(t)
            # saturated: about seconds / 2 of work submitted at once
            n_sat = max(n_unique, int(seconds / 2 * 250000 / mean_chunks))
            stream = [i % n_unique for i in range(n_sat)]
            srv.reset_stats()
            t0 = time.perf_counter()
            tickets = [srv.submit(reqs[i][0], reqs[i][1], *bufs(i, u8), u8=u8) for i in stream]
            for t in tickets:
                srv.wait(t)
            sat = sum(sizes[i] for i in stream) / (time.perf_counter() - t0)
            res['saturated_chunks_per_s'] = round(sat, 1)
            res['saturated_over_plain'] = round(sat / plain_cps, 3)
            for frac in loads:
                rate = frac * sat / mean_chunks                         # requests per second
                n_req = int(max(min_requests, rate * seconds))
                order = rng.integers(0, n_unique, n_req)
                gaps = rng.exponential(1.0 / rate, n_req)
                srv.reset_stats()
                tickets = []
                due = t_start = time.perf_counter()
                for k2 in range(n_req):
                    due += gaps[k2]
                    wait = due - time.perf_counter()
                    if wait > 0:
                        time.sleep(wait)
                    i = int(order[k2])
                    tickets.append(srv.submit(reqs[i][0], reqs[i][1], *bufs(i, u8), u8=u8))
                for t in tickets:
                    srv.wait(t)
                span = time.perf_counter() - t_start
                st = srv.stats()
                lat = srv.latencies()
                p99, lo, hi = p99_interval(lat)
                offered = sum(sizes[int(i)] for i in order) / (due - t_start)
                pt = {'load': frac, 'requests': n_req, 'seconds': round(span, 2), 'offered_chunks_per_s': round(offered, 1),
                      'served_chunks_per_s': round(st['chunks_per_s'], 1), 'p50_ms': round(st['p50_ms'], 2), 'p99_ms': round(p99, 2),
                      'p99_ci95_ms': [round(lo, 2), round(hi, 2)], 'max_ms': round(st['max_ms'], 2)}
                pt['steady'] = pt['served_chunks_per_s'] >= 0.97 * pt['offered_chunks_per_s']
                res['points'].append(pt)
        steady = [p for p in res['points'] if p['steady'] and p['p99_ms'] < p99_target_ms]
        if steady:
            best = max(steady, key=lambda p: p['served_chunks_per_s'])
            res['best_steady_under_target'] = dict(best, served_over_plain=round(best['served_chunks_per_s'] / plain_cps, 3))
        out['forms'][form] = res
    return out


def batched_lists(n_seeds=256, seed=3):
    """The batched workload: n_seeds random seeds, each with a chunk list of log-uniform size in
    [1, 1024]; each list a contiguous square, scattered chunks within +/-117,187, or chunks
    straddling the noise-lattice wrap at chunk 6128 / -6129. Returns (seeds, lists)."""
    rng = np.random.default_rng(seed)
    seeds = [int(v) for v in rng.integers(-(1 << 62), 1 << 62, n_seeds)]
    lists = []
    for k in range(n_seeds):
        n = int(min(1024, max(1, round(np.exp(rng.uniform(0, np.log(1024)))))))
        kind = k % 3
        if kind == 0:
            side = int(np.ceil(np.sqrt(n)))
            x0, z0 = (int(v) for v in rng.integers(-117187, 117187 - side, 2))
            c = [(x0 + i % side, z0 + i // side) for i in range(n)]
        elif kind == 1:
            c = [(int(a), int(b)) for a, b in rng.integers(-117187, 117188, (n, 2))]
        else:
            xs = rng.choice(np.array([6127, 6128, 6129, -6128, -6129, -6130]), n)
            c = [(int(a), int(b)) for a, b in zip(xs, rng.integers(-117187, 117188, n))]
        lists.append(np.array(c, np.int32))
    return seeds, lists


def batched_bench(g, n_seeds=256, seed=3):
    """Many seeds and uneven chunk lists in one tg_generate_batch call (batched_lists). Outputs
    to pinned host memory (requests share one pool; only the time is used)."""
    import ctypes
    import torch
    import terrain_b200
    seeds, lists = batched_lists(n_seeds, seed)
    total = sum(len(c) for c in lists)
    biggest = max(len(c) for c in lists)
    pool_b = torch.empty(biggest * 98304, dtype=torch.int16, pin_memory=True).numpy().view(np.uint16)
    pool_q = torch.empty(biggest * 1536, dtype=torch.uint8, pin_memory=True).numpy()
    reqs = (terrain_b200.TgRequest * n_seeds)()
    for i, c in enumerate(lists):
        reqs[i].seed = seeds[i]
        reqs[i].chunks = c.ctypes.data_as(ctypes.POINTER(terrain_b200.TgChunk))
        reqs[i].count = len(c)
        reqs[i].blocks_out = pool_b.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))
        reqs[i].biomes_out = pool_q.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
    for sd in seeds:
        g.set_seed(sd)
    t = terrain_b200.TgTiming()
    g._check(g.L.tg_generate_batch(g.h, reqs, n_seeds, ctypes.byref(t)))          # warm-up (graphs)
    best = None
    for _ in range(3):
        t0 = time.perf_counter()
        g._check(g.L.tg_generate_batch(g.h, reqs, n_seeds, None))
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    out = {'seeds': n_seeds, 'chunks': total, 'chunks_per_s': round(total / best, 1), 'ms': round(best * 1000, 2),
           'form': 'tg_generate_batch, device batches of up to 4,096 chunks mixing seeds, outputs copied to pinned host memory',
           'lists': 'log-uniform sizes 1..1024; squares, scattered within +/-117,187, and wrap-straddling chunks 6127..6129 / -6128..-6130'}
    out['device_queue'] = batched_device_bench(g, seeds, lists)
    return out


def batched_device_bench(g, seeds, lists, reps=3):
    """The same 256-seed workload with every list and output in HBM (tg_generate_batch_device):
    the requests form one device work queue drained by one graph launch (a WHILE loop on the
    device), against one graph launch per batch from the host; CUDA events on the stream."""
    import torch
    chunks = [torch.from_numpy(c).cuda() for c in lists]
    total = sum(len(c) for c in lists)
    blocks = torch.empty(total * 98304, dtype=torch.int16, device='cuda')
    biomes = torch.empty(total * 1536, dtype=torch.uint8, device='cuda')
    reqs, at = [], 0
    for sd, c in zip(seeds, chunks):
        n = c.shape[0]
        reqs.append((sd, c.data_ptr(), n, blocks.data_ptr() + 2 * 98304 * at, biomes.data_ptr() + 1536 * at))
        at += n
    res = {}
    for name, host_loop in (('device_loop', False), ('host_loop', True)):
        g.generate_batch_device(reqs, host_loop=host_loop)                     # warm-up: graphs
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            g.generate_batch_device(reqs, host_loop=host_loop)
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        res[name] = {'chunks_per_s': round(total / (min(ms) / 1000.0), 1), 'ms': round(min(ms), 2)}
    res['form'] = ('tg_generate_batch_device: lists and outputs in HBM, one device work queue of (chunk, seed) items, 4,096-chunk '
                   'batches; device_loop = one graph launch with a WHILE node, host_loop = one graph launch per batch')
    del blocks, biomes
    torch.cuda.empty_cache()
    return res


def biome_stream_bench(g, n_seeds=1024, per_seed=16384, seed=5):
    """Biome-only lookups: n_seeds seeds x per_seed positions (x, z uniform in +/-1,874,999,
    y uniform in [-64, 319]) through tg_biome_lookup; the per-seed tables are built inside the
    call as seeds arrive (more seeds than stay resident), so their setup is part of the time."""
    rng = np.random.default_rng(seed)
    seeds = np.repeat(np.array([int(v) for v in rng.integers(-(1 << 62), 1 << 62, n_seeds)], np.int64), per_seed)
    n = n_seeds * per_seed
    xyz = np.empty((n, 3), np.int32)
    xyz[:, 0] = rng.integers(-1874999, 1875000, n)
    xyz[:, 1] = rng.integers(-64, 320, n)
    xyz[:, 2] = rng.integers(-1874999, 1875000, n)
    g.biome_lookup(seeds[:per_seed], xyz[:per_seed])                                      # warm-up
    t0 = time.perf_counter()
    g.biome_lookup(seeds, xyz)
    dt = time.perf_counter() - t0
    # resident tables: the first 512 seeds' positions, once to load their tables, then timed
    k = min(n_seeds, 512) * per_seed
    g.biome_lookup(seeds[:k], xyz[:k])
    t0 = time.perf_counter()
    g.biome_lookup(seeds[:k], xyz[:k])
    dt_res = time.perf_counter() - t0
    return {'lookups': n, 'seeds': n_seeds, 'lookups_per_s': round(n / dt, 1), 'ms': round(dt * 1000, 1),
            'resident_lookups_per_s': round(k / dt_res, 1),
            'form': 'tg_biome_lookup: one thread per position, zoom corner then that quart\'s climate, R-tree minimum and tie test, '
                    'replaying the chunk chain only from the nearest earlier quart whose result is fixed'}


def reference_gpu_bench(steps=3, warmup=2):
    """The reference's own GPU generator (FullTerrainGenerator, built unchanged for sm_100a by
    baseline/Makefile, evaluators generated by its own code generator from the same model
    files) on this B200, on the same 12,288-chunk ladder step: end to end as the reference's
    bench runs it (one generate() call per step, u8 blocks and u8 biomes into pinned host
    memory, 2,048-chunk batches, 2 pipeline slots: its headline setting), and kernels only
    (the sum of its per-stage CUDA-event times at 4,096-chunk batches, 1 slot). Returns None
    when the side arm is not built."""
    sys.path.insert(0, os.path.join(REPO, 'baseline'))
    import refgpu
    if not refgpu.available():
        return None
    import torch
    chunks = np.concatenate([region_chunks(x0, z0) for _, x0, z0 in REGIONS])
    n = chunks.shape[0]
    t8 = torch.empty(n * 98304, dtype=torch.uint8, pin_memory=True).numpy().reshape(n, 384, 16, 16)
    b8 = torch.empty(n * 1536, dtype=torch.uint8, pin_memory=True).numpy().reshape(n, 1536)
    out = {'form': 'mcc::cuda::FullTerrainGenerator of the reference, compiled for sm_100a with its exactness flags, '
                   'evaluators from its gen_router.py over the same model files'}
    g = refgpu.RefGpuGenerator(max_batch_chunks=2048, pipeline_slots=2)
    try:
        g.set_seed(SEED)
        for _ in range(warmup):
            g.generate(chunks, t8, b8)
        t0 = time.perf_counter()
        for _ in range(steps):
            g.generate(chunks, t8, b8)
        dt = (time.perf_counter() - t0) / steps
        out['e2e_chunks_per_s'] = round(n / dt, 1)
        out['e2e_setting'] = 'batch 2048, 2 slots, pinned u8 blocks + biomes'
    finally:
        g.close()
    g = refgpu.RefGpuGenerator(max_batch_chunks=4096, pipeline_slots=1)
    try:
        g.set_seed(SEED)
        g.generate(chunks, t8, b8, timing=True)
        ks = []
        for _ in range(steps):
            _, _, st = g.generate(chunks, t8, b8, timing=True)
            ks.append(sum(st[k] for k in ('biome_ms', 'noise_ms', 'aquifer_ms', 'fill_ms', 'surface_ms')))
            stages = st
        ms = min(ks)
        out['kernel_chunks_per_s'] = round(n / (ms / 1000.0), 1)
        out['kernel_ms_per_step'] = round(ms, 3)
        out['stage_ms_per_step'] = {k: round(v, 3) for k, v in stages.items()}
        out['kernel_setting'] = 'batch 4096, 1 slot, sum of the per-stage CUDA-event times'
    finally:
        g.close()
    return out


def corner_roofline(stats, n, regions, sms, clocks):
    """Issue roofline of the channel-corner kernel, the largest kernel of the step. Its work is
    counted, not guessed: the octave samples the kernel evaluates per corner point, counted
    on the host twin of the kernel bodies (tests/hostcheck/count_kernels.py: volume, smeared
    volume and point samples, lazy per-point evaluation), times the distinct corner points of
    one launch (257 x 257 columns x 49 rows, each computed once, per 64 x 64-chunk region), times the
    minimal instruction recipe of one sample (VOL_OCTAVE_INSTR). Peak: 4 warp instructions per
    clock per SM (32 threads each) at the SM clock sampled during the timed steps; the FP64
    pipe (64 lanes per SM per clock) is reported beside it. The reference port's eager volume
    path (both branches of every choice node over a whole volume) samples more per point;
    its count (oracle/count_ops.py) is given beside."""
    try:
        with open(OP_COUNTS) as f:
            oc = json.load(f)
    except OSError:
        return None
    per_point = sum(oc['kernels']['per_kernel']['corner']['samples_per_unit'].values())
    port_per_point = (oc['per_chunk']['corners']['vol_octave'] + oc['per_chunk']['corners']['point_octave']) / (25 * 49)
    side = int(round(n ** 0.5))
    points = (side * 4 + 1) ** 2 * 49 * regions
    samples = points * per_point
    per_sample = sum(VOL_OCTAVE_INSTR.values())
    instr = samples * per_sample
    launch_ms = sum(t['corner_ms'] for t in stats) / len(stats)
    mhz = clocks.get('sm_mhz') or 1965.0
    peak = sms * 4 * 32 * mhz * 1e6 / 1e12                      # T thread-instructions / s
    achieved = instr / (launch_ms / 1000.0) / 1e12
    fp64_peak = sms * 64 * mhz * 1e6 / 1e12
    fp64 = samples * VOL_OCTAVE_INSTR['fp64'] / (launch_ms / 1000.0) / 1e12
    return {'bound': 'issue', 'kernel': 'corner (k_body<&body_corner>)', 'achieved': round(achieved, 3), 'peak': round(peak, 3),
            'unit': 'T thread-instructions/s', 'frac': round(achieved / peak, 4), 'traffic': None, 'launch_ms': round(launch_ms, 3),
            'octave_samples_per_launch': int(samples), 'samples_per_corner_point': round(per_point, 3),
            'port_samples_per_corner_point': round(port_per_point, 3), 'instructions_per_sample': VOL_OCTAVE_INSTR,
            'fp64_pipe': {'achieved': round(fp64, 3), 'peak': round(fp64_peak, 3), 'frac': round(fp64 / fp64_peak, 4), 'unit': 'T FP64 ops/s'},
            'peak_source': 'issue rate at the sampled SM clock (%s MHz), %d SMs' % (mhz, sms),
            'note': '%.2f octave samples per corner point (counted on the kernel bodies) x %d distinct corner points of one %d-chunk launch '
                    'x %d instructions per sample; the DRAM traffic is negligible (the kernel reads L2-resident tables)' %
                    (per_point, points, n * regions, per_sample)}


def flythrough_bench(g, frames=90, radius=24, width=1280, height=720, speed=15.0):
    """Live flythrough (tg_viewer_*): a 64 x 64-chunk window, the camera flying along +x at
    `speed` blocks per frame at 110 blocks up, looking ahead and 12 degrees down; every frame
    generates the chunks within `radius` that the window lacks (nearest first, at most 512)
    straight into the window on the device, then ray traces a width x height frame (4 rays
    per pixel, shadow rays). The first frame fills the window and is left out of the means.
    Times are CUDA events of the generation and window update, and of the render kernel."""
    import terrain_b200
    g.set_seed(SEED)
    gen_ms, chunks, render_ms = [], [], []
    with terrain_b200.TerrainViewer(g, window_chunks=64, width=width, height=height) as v:
        x, z = 8.0, 8.0
        for f in range(frames + 1):
            n, ms = v.update(int(np.floor(x / 16)), int(np.floor(z / 16)), radius, cap=512, frame=f)
            _, _, rms = v.render(terrain_b200.camera(x, 110.0, z, yaw_deg=90.0, pitch_deg=-12.0, fog=radius * 16.0), f, rgb=f == frames)
            if f > 0:
                gen_ms.append(ms)
                chunks.append(n)
                render_ms.append(rms)
            x += speed
    return {'frames': frames, 'frame': '%dx%d' % (width, height), 'radius_chunks': radius, 'speed_blocks_per_frame': speed,
            'chunks_per_frame': round(float(np.mean(chunks)), 1), 'generate_ms_per_frame': round(float(np.mean(gen_ms)), 3),
            'render_ms_per_frame': round(float(np.mean(render_ms)), 3), 'render_ms_p99': round(float(np.quantile(render_ms, 0.99)), 3),
            'frames_per_s_render_and_generate': round(1000.0 / (float(np.mean(gen_ms)) + float(np.mean(render_ms))), 1),
            'form': 'tg_viewer_update (chunks generated on the device into the voxel window) + tg_viewer_render (2x2 rays per pixel, '
                    'shadow rays, 4x4-column empty-space skipping)'}


def run_ours(args, rank, world, local_rank):
    import torch
    import terrain_b200
    dev = local_rank
    torch.cuda.set_device(dev)
    nreg = len(REGIONS)
    n = SIDE * SIDE
    # The step's three regions go to the kernels as one 12,288-chunk batch (fewer kernel
    # tails and launches than three 4,096-chunk batches: 29 against 31 ms per step)
    g = terrain_b200.TerrainGenerator(max_batch_chunks=n * nreg, device=dev)
    stream = torch.cuda.current_stream()
    g.set_stream(stream.cuda_stream)
    g.set_seed(SEED)
    host_chunks = [region_chunks(x0, z0) for _, x0, z0 in REGIONS]
    d_chunks = torch.from_numpy(np.concatenate(host_chunks)).cuda()
    d_blocks = torch.empty(n * nreg * 98304, dtype=torch.int16, device='cuda')
    d_biomes = torch.empty(n * nreg * 1536, dtype=torch.uint8, device='cuda')

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def step_device(stats=None):
        # the timed steps run without stage events; one extra step records the stage times
        t = g.generate_device(d_chunks.data_ptr(), n * nreg, d_blocks.data_ptr(), d_biomes.data_ptr(), timing=stats is not None)
        if stats is not None:
            stats.append(t)

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    stats = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step_device()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    step_device(stats)               # stage and walk-rules times (events between the stages), untimed
    barrier()
    torch.cuda.synchronize()
    ms_max = max_over_ranks(ms, world, 'cuda')
    chunks_total = n * nreg * args.steps * world
    value = chunks_total / (ms_max / 1000.0)

    # end to end through the host API: pinned host outputs, copies inside the step
    all_chunks = np.concatenate(host_chunks)
    pin_all_blocks = torch.empty(n * nreg * 98304, dtype=torch.int16, pin_memory=True).numpy().view(np.uint16).reshape(n * nreg, -1, 16, 16)
    pin_all_biomes = torch.empty(n * nreg * 1536, dtype=torch.uint8, pin_memory=True).numpy().reshape(n * nreg, -1)
    pin_all_blocks8 = torch.empty(n * nreg * 98304, dtype=torch.uint8, pin_memory=True).numpy().reshape(n * nreg, -1, 16, 16)

    def step_e2e():
        # one call per step: the library pipelines its batches (copies of batch k overlap batch k + 1)
        g.generate_u8(all_chunks, blocks_out=pin_all_blocks8, biomes_out=pin_all_biomes)

    def step_e2e_u16():
        g.generate(all_chunks, blocks_out=pin_all_blocks, biomes_out=pin_all_biomes)

    def time_e2e(step):
        for _ in range(max(1, min(args.warmup, 2))):
            step()
        torch.cuda.synchronize()
        barrier()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for _ in range(args.steps):
            step()
        e3.record(stream)
        torch.cuda.synchronize()
        return chunks_total / (max_over_ranks(e2.elapsed_time(e3), world, 'cuda') / 1000.0)

    e2e_value = time_e2e(step_e2e)
    e2e_u16 = time_e2e(step_e2e_u16)
    pcie = pcie_d2h_gbs()

    if rank != 0:
        return
    stage = {k: sum(t[k] for t in stats) for k in ('biome_ms', 'noise_ms', 'aquifer_ms', 'fill_ms', 'surface_ms', 'kernel_ms')}
    launches = sum(t['launches'] for t in stats) * args.steps   # per step (the stats step) x timed steps
    calls = len(stats)
    clocks = clk.summary()
    # the column walk with the rule tree, timed by its own CUDA events: its HBM fraction
    per_launch_ms = sum(t['walk_rules_ms'] for t in stats) / calls
    algo_bytes = WALK_BYTES_PER_CHUNK * n * nreg
    achieved = algo_bytes / (per_launch_ms / 1000.0) / 1e9
    peak, peak_kind = peaks()
    roofline = corner_roofline(stats, n, nreg, torch.cuda.get_device_properties(dev).multi_processor_count, clocks)
    line = {
        'metric': METRIC, 'value': round(value, 1), 'unit': 'chunks/s', 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': round(ms_max / args.steps, 3), 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32+f64+int',
        'data': 'synthetic world model (project-authored, reference JSON formats); seeded chunk lists',
        'config': {'workload': 'ladder: one seed, three 64x64-chunk regions (origin, -1,000,000 blocks, +1,874,999-block border), 12,288 chunks per step',
                   'seed': SEED, 'chunks_per_step': n * nreg, 'batch_chunks': n * nreg, 'l2': 'outputs (2.4 GB per step) larger than L2',
                   'model_sha256': model_sha256(), 'samples_per_chunk': samples_per_chunk(),
                   'parallelism': 'replicas: each GPU runs the full workload' if world > 1 else 'single GPU'},
        'stage_ms_per_step': {k: round(v, 3) for k, v in stage.items()},
        'roofline': roofline,
        'roofline_walk_hbm': {'bound': 'hbm', 'kernel': 'surface_walk_rules and its deferred pass (walk_deferred)', 'achieved': round(achieved, 2), 'peak': peak, 'unit': 'GB/s',
                              'frac': round(achieved / peak, 5), 'traffic': WALK_TRAFFIC_PER_LAUNCH, 'peak_source': peak_kind,
                              'launch_ms': round(per_launch_ms, 3), 'share_of_step': round(per_launch_ms * calls / stage['kernel_ms'], 3),
                              'note': 'algorithmic bytes = 417,792 B per chunk (per block the u8 biome and u8 ore bits read and the u16 state '
                                      'written, plus the column air / fluid masks) x 12,288 chunks per launch, over the time of the walk and its '
                                      'deferred pass; traffic = dram read + write bytes of one walk launch (ncu capture of a 4,096-chunk launch scaled to '
                                      '12,288 chunks; the deferred pass moves 16 B per deferred block, about 10 MB). The kernels are issue- and latency-bound, so their HBM fraction is small'},
        'e2e': {'value': round(e2e_value, 1), 'unit': 'chunks/s', 'h2d_bytes_per_step': int(n * nreg * 8),
                'd2h_bytes_per_step': int(n * nreg * BYTES_PER_CHUNK_U8), 'd2h_gbs': round(e2e_value * BYTES_PER_CHUNK_U8 / 1e9, 2),
                'pcie_d2h_gbs_measured': pcie, 'pcie_frac': round(e2e_value * BYTES_PER_CHUNK_U8 / 1e9 / pcie, 3) if pcie else None,
                'api': 'tg_generate_u8 (u8 palette index per block and u8 quart biomes to pinned host memory)'},
        'e2e_u16': {'value': round(e2e_u16, 1), 'unit': 'chunks/s', 'h2d_bytes_per_step': int(n * nreg * 8),
                    'd2h_bytes_per_step': int(n * nreg * BYTES_PER_CHUNK), 'd2h_gbs': round(e2e_u16 * BYTES_PER_CHUNK / 1e9, 2),
                    'api': 'tg_generate (u16 block states and u8 quart biomes to pinned host memory)'},
        'gpu_launches': int(launches),
        'clocks': clocks,
    }
    if not (args.no_serve and args.no_extra):
        # the other forms on a generator of 4,096-chunk batches, as their workloads are quoted
        g.close()
        torch.cuda.empty_cache()
        g = terrain_b200.TerrainGenerator(max_batch_chunks=n, device=dev)
        g.set_seed(SEED)
    if not args.no_serve:
        g.set_stream(0)
        line['served'] = served_bench(g)
    if not args.no_extra:
        g.set_stream(0)
        line['batched'] = batched_bench(g)
        line['biome_stream'] = biome_stream_bench(g)
        line['flythrough'] = flythrough_bench(g)
    if not args.no_reference_gpu:
        line['reference_gpu'] = reference_gpu_bench()
        if line['reference_gpu']:
            rg = line['reference_gpu']
            rg['ours_over_reference_kernels'] = round(value / rg['kernel_chunks_per_s'], 3)
            rg['ours_over_reference_e2e'] = round(e2e_value / rg['e2e_chunks_per_s'], 3)
    if not args.no_cpu_baseline:
        line['cpu_baseline'] = cpu_baseline()
    print(json.dumps(line, default=json_default))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-serve', action='store_true', help='skip the served-versus-plain request-stream measurement')
    ap.add_argument('--no-extra', action='store_true', help='skip the batched-seeds and biome-stream measurements')
    ap.add_argument('--no-reference-gpu', action='store_true', help='skip the reference GPU generator side arm')
    ap.add_argument('--profile-small', action='store_true',
                    help='one untimed step over a 32x32-chunk corner of each region, 1,024-chunk batches (a small case for ncu captures), '
                         'then the first corner again in the u8 form')
    ap.add_argument('--profile-lookup', action='store_true',
                    help='three untimed tg_biome_lookup calls of one 2^20-position sub-batch (64 seeds x 16,384 positions), for ncu launch lists')
    args = ap.parse_args()
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local_rank = int(os.environ.get('LOCAL_RANK', '0'))
    if args.impl == 'reference':
        run_reference(args, rank)
        return
    if args.profile_lookup:
        import terrain_b200
        g = terrain_b200.TerrainGenerator(max_batch_chunks=64)
        rng = np.random.default_rng(5)
        ns, per = 64, 16384
        seeds = np.repeat(rng.integers(-(1 << 62), 1 << 62, ns).astype(np.int64), per)
        xyz = np.empty((ns * per, 3), np.int32)
        xyz[:, 0] = rng.integers(-1874999, 1875000, ns * per)
        xyz[:, 1] = rng.integers(-64, 320, ns * per)
        xyz[:, 2] = rng.integers(-1874999, 1875000, ns * per)
        for _ in range(3):
            g.biome_lookup(seeds, xyz)
        g.close()
        return
    if args.profile_small:
        import terrain_b200
        g = terrain_b200.TerrainGenerator(max_batch_chunks=1024)
        g.set_seed(SEED)
        for _, x0, z0 in REGIONS:
            g.generate(region_chunks(x0, z0, 32))
        g.generate_u8(region_chunks(0, 0, 32))   # last, so the launches before it are unchanged
        g.close()
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == '__main__':
    main()
