"""Autotuner of the TERRAIN step's launch shapes (runs on the target GPU).

    python minecraft-terrain-cuda_b200/autotune.py [--out tuning/launch_table.txt] [--report autotune.json]

For every tunable kernel of a batch, in order of its share of the step, it tries launch
shapes -- threads per block {64, 128, 256}, resident-block grid cap {1 .. 16} blocks per SM
(at most 2,048 threads per SM), and the kernel form: grid-stride loop (grab 0) or persistent
work queue taking runs of grab * threads items (grab 1, 2, 4) -- with the other kernels held
at their current best, measuring the kernel's own CUDA-event time (tg_kernel_times) over
timed batches of the ladder workload (three 64x64-chunk regions, at the origin, at block
-1,000,000 and at the +1,874,999-block border, as one 12,288-chunk batch, the form the
benchmark times), and keeps the fastest. Kernels under 2 % of the step try a
reduced set. Then the dedupe hash-table load (capacity >= 2 or 4 x the keys) is chosen by
the whole step's time. Last, the batch schedule of calls with host outputs (the host_u8
and host_u16 lines: largest batch, tail, head) is chosen per output form by timing tg_generate_u8 and tg_generate
into pinned host memory over the same 12,288 chunks. The table is written for build.py to compile in, with the
step time of the table in use before and of the tuned one, each timed through the
graph-launched device-resident form (tg_generate_device).
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import terrain_b200  # noqa: E402

SEED = 0x5445525241494E31
REGIONS = [(0, 0), (-62500, -62500), (117124, 117124)]
HOST_REGIONS = REGIONS
THREADS = (64, 128, 256)
BLOCKS_PER_SM = (1, 2, 3, 4, 6, 8, 12, 16)
GRABS = (0, 1, 2, 4)


SCHED_KEYS = ('host_u8', 'host_u16')
OTHER_KEYS = ('walk_defer',)   # carried through unchanged


def parse(text):
    """(kernel shapes, table load, other lines {host_u8 / host_u16: (batch, tail_min, tail_pct, head_min, head_pct),
    walk_defer: (blocks per chunk,)})"""
    table, load, sched = {}, 2, {}
    for line in text.splitlines():
        line = line.split('#')[0].split()
        if not line:
            continue
        if line[0] == 'table_load':
            load = int(line[1])
        elif line[0] in SCHED_KEYS or line[0] in OTHER_KEYS:
            sched[line[0]] = tuple(int(v) for v in line[1:6])
        else:
            table[line[0]] = tuple(int(v) for v in line[1:4])
    return table, load, sched


def fmt(table, load, sched=None, header=''):
    lines = [header] if header else []
    lines.append('table_load %d' % load)
    lines += ['%s %s' % (k, ' '.join('%d' % v for v in sched[k])) for k in SCHED_KEYS + OTHER_KEYS if sched and k in sched]
    lines += ['%s %d %d %d' % ((k,) + table[k]) for k in terrain_b200.KERNELS]
    return '\n'.join(lines) + '\n'


class Bench:
    def __init__(self, side=64):
        import torch
        self.torch = torch
        self.n = side * side * len(REGIONS)
        self.g = terrain_b200.TerrainGenerator(max_batch_chunks=self.n)
        self.g.set_seed(SEED)
        grid = lambda x0, z0: np.array([(x0 + x, z0 + z) for z in range(side) for x in range(side)], np.int32)
        # the regions as one batch (a list of one device chunk list)
        self.chunks = [torch.from_numpy(np.concatenate([grid(x0, z0) for x0, z0 in REGIONS])).cuda()]
        self.blocks = torch.empty(self.n * 98304, dtype=torch.int16, device='cuda')
        self.biomes = torch.empty(self.n * 1536, dtype=torch.uint8, device='cuda')
        self.sched = {}
        self.host_chunks = np.concatenate([grid(x0, z0) for x0, z0 in HOST_REGIONS])
        nh = len(self.host_chunks)
        self.pin8 = torch.empty(nh * 98304, dtype=torch.uint8, pin_memory=True).numpy().reshape(nh, -1, 16, 16)
        self.pin16 = torch.empty(nh * 98304, dtype=torch.int16, pin_memory=True).numpy().view(np.uint16).reshape(nh, -1, 16, 16)
        self.pinb = torch.empty(nh * 1536, dtype=torch.uint8, pin_memory=True).numpy().reshape(nh, -1)

    def set(self, table, load, sched=None):
        self.g.set_launch_table(fmt(table, load, self.sched if sched is None else sched))

    def kernel_ms(self, table, load, reps=2):
        """{kernel: ms per batch}: medians over reps timed batches of each region."""
        g = self.g
        self.set(table, load)
        for c in self.chunks:                                     # warm-up (tables, caches)
            g.generate_device(c.data_ptr(), self.n, self.blocks.data_ptr(), self.biomes.data_ptr(), timing=False)
        g.kernel_times(enable=True)
        per = {k: [] for k in terrain_b200.KERNELS}
        for _ in range(reps):
            for c in self.chunks:
                g.generate_device(c.data_ptr(), self.n, self.blocks.data_ptr(), self.biomes.data_ptr(), timing=True)
                for k, (ms, calls) in g.kernel_times(enable=True).items():
                    per[k].append(ms / max(calls, 1))
        g.kernel_times(enable=False)
        return {k: float(np.median(v)) for k, v in per.items()}

    def step_ms(self, table, load, reps=5, sched=None):
        """Device time of the graph-launched steps (all regions), median of reps."""
        torch = self.torch
        g = self.g
        self.set(table, load, sched)
        for c in self.chunks:
            g.generate_device(c.data_ptr(), self.n, self.blocks.data_ptr(), self.biomes.data_ptr(), timing=False)
        out = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for c in self.chunks:
                g.generate_device(c.data_ptr(), self.n, self.blocks.data_ptr(), self.biomes.data_ptr(), timing=False)
            e1.record()
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1))
        return float(np.median(out))

    def host_ms(self, table, load, sched, u8, reps=5):
        """Wall time of one call with pinned host outputs over the host regions, median of reps
        (the call returns when its outputs are in host memory)."""
        g = self.g
        self.set(table, load, sched)
        call = ((lambda: g.generate_u8(self.host_chunks, blocks_out=self.pin8, biomes_out=self.pinb)) if u8 else
                (lambda: g.generate(self.host_chunks, blocks_out=self.pin16, biomes_out=self.pinb)))
        call()
        out = []
        for _ in range(reps):
            t0 = time.perf_counter()
            call()
            out.append((time.perf_counter() - t0) * 1e3)
        return float(np.median(out))


def candidates(kernel, big):
    if not big:
        shapes = [(t, b, 0) for t in (128, 256) for b in (4, 8, 16) if t * b <= 2048]
    else:
        shapes = [(t, b, gr) for t in THREADS for b in BLOCKS_PER_SM for gr in GRABS if t * b <= 2048]
    if kernel == 'chain':
        shapes = [s for s in shapes if s[2] == 0]
    return shapes


# batch schedules of calls with host outputs, per form: largest batch, tail (min, pct), head (min, pct)
HOST_BATCH = {'host_u8': (2048, 3072, 4096, 6144), 'host_u16': (1024, 2048, 3072, 4096)}
TAILS = ((0, 0), (512, 50), (1024, 50), (256, 50), (512, 67), (512, 75))
HEADS = ((0, 0), (512, 200), (1024, 200), (256, 200))


def tune_schedule(b, table, load, sched, reps):
    """Per output form: the largest batch, then the tail, then the head, each with the others
    held at their best; returns the schedule lines and the timings."""
    sched = dict(sched)
    report = {}
    for key in SCHED_KEYS:
        u8 = key == 'host_u8'
        cur = list(sched[key])
        before = b.host_ms(table, load, sched, u8, reps * 2)
        tried = []
        for what, opts in (('batch', HOST_BATCH[key]), ('tail', TAILS), ('head', HEADS)):
            best, best_ms = None, None
            for o in opts:
                c = list(cur)
                if what == 'batch':
                    c[0] = o
                elif what == 'tail':
                    c[1:3] = o
                else:
                    c[3:5] = o
                ms = b.host_ms(table, load, dict(sched, **{key: tuple(c)}), u8, reps)
                tried.append((what, o, round(ms, 3)))
                if best_ms is None or ms < best_ms:
                    best, best_ms = c, ms
            cur = best
        after = b.host_ms(table, load, dict(sched, **{key: tuple(cur)}), u8, reps * 2)
        keep = after < 0.99 * before                  # a new schedule only for a clear gain
        report[key] = {'before': sched[key], 'before_ms': round(before, 3), 'tuned': tuple(cur), 'tuned_ms': round(after, 3),
                       'kept': 'tuned' if keep else 'before', 'chosen_ms': round(after if keep else before, 3), 'tried': tried}
        print('%s: %s %.3f ms -> %s %.3f ms (%s)' % (key, sched[key], before, tuple(cur), after, report[key]['kept']), flush=True)
        if keep:
            sched[key] = tuple(cur)
    return sched, report


def main(argv):
    ap = argparse.ArgumentParser()
    ap.add_argument('--out', default=os.path.join(HERE, 'tuning', 'launch_table.txt'))
    ap.add_argument('--report', default=None)
    ap.add_argument('--reps', type=int, default=2)
    ap.add_argument('--schedule-only', action='store_true', help='keep the kernel shapes; tune only the host-output schedule')
    args = ap.parse_args(argv)
    t_start = time.time()
    b = Bench()
    default_text = b.g.launch_table()
    table, load, sched = parse(default_text)
    b.sched = sched
    base, base_load, base_sched = dict(table), load, dict(sched)
    report = {'kernels': {}}
    if not args.schedule_only:
        ms0 = b.kernel_ms(table, load, args.reps)
        total0 = sum(ms0.values())
        order = sorted(terrain_b200.KERNELS, key=lambda k: -ms0[k])
        report['default_kernel_ms'] = ms0
        for k in order:
            big = ms0[k] >= 0.02 * total0
            best, best_ms, tried = table[k], None, []
            for shape in candidates(k, big):
                table[k] = shape
                ms = b.kernel_ms(table, load, args.reps)[k]
                tried.append((shape, round(ms, 4)))
                if best_ms is None or ms < best_ms:
                    best, best_ms = shape, ms
            table[k] = best
            report['kernels'][k] = {'default': base[k], 'default_ms': round(ms0[k], 4), 'best': best, 'best_ms': round(best_ms, 4),
                                    'tried': len(tried), 'top': sorted(tried, key=lambda x: x[1])[:5]}
            print('%-15s %s %.4f ms -> %s %.4f ms (%d shapes)' % (k, base[k], ms0[k], best, best_ms, len(tried)), flush=True)
        loads = {}
        for ld in (2, 4):
            loads[ld] = b.step_ms(table, ld)
        load = 4 if loads[4] < 0.99 * loads[2] else 2     # the larger tables only for a clear gain
        report['table_load_step_ms'] = loads
    step_default = b.step_ms(base, base_load, reps=9, sched=base_sched)
    step_tuned = b.step_ms(table, load, reps=9)
    keep_tuned = step_tuned < step_default
    if not keep_tuned:
        table, load = base, base_load
    sched, report['host_schedule'] = tune_schedule(b, table, load, sched, max(3, args.reps + 1))
    report.update({'table_load': load, 'step_ms_default': round(step_default, 3), 'step_ms_tuned': round(step_tuned, 3),
                   'regions': REGIONS, 'host_regions': HOST_REGIONS, 'batch_chunks': b.n, 'seconds': round(time.time() - t_start, 1)})
    hs = report['host_schedule']
    header = ('# Launch shapes of the TERRAIN step\'s kernels, compiled into libterrain_b200.so by build.py.\n'
              '# Written by autotune.py on a B200; a line per kernel: name threads blocks_per_sm grab\n'
              '# (grab 0: grid-stride loop; grab g > 0: persistent work queue, g * threads items per take),\n'
              '# table_load: dedupe hash tables of at least table_load x the most keys of a batch;\n'
              '# host_u8 / host_u16: batch tail_min tail_pct head_min head_pct of calls with host outputs.\n'
              '# Three 64x64-chunk ladder regions as one 12,288-chunk batch, device-resident step:\n'
              '# %s.\n'
              '# Three ladder regions in one call to pinned host memory: u8 %.3f -> %.3f ms, u16 %.3f -> %.3f ms.'
              % (('%.3f ms per step (kernel shapes not re-tuned in this run)' % step_default) if args.schedule_only else
                 ('the table in use before %.3f ms, tuned %.3f ms per step%s' % (step_default, step_tuned, '' if keep_tuned else ' (tuned slower: the previous shapes kept)')),
                 hs['host_u8']['before_ms'], hs['host_u8']['chosen_ms'], hs['host_u16']['before_ms'], hs['host_u16']['chosen_ms']))
    text = fmt(table, load, sched, header)
    with open(args.out, 'w') as f:
        f.write(text)
    report['kept'] = 'tuned' if keep_tuned else 'default'
    report['schedule'] = sched
    if args.report:
        with open(args.report, 'w') as f:
            json.dump(report, f, indent=1)
    print(json.dumps({k: report[k] for k in ('step_ms_default', 'step_ms_tuned', 'table_load', 'kept', 'schedule', 'seconds')}))
    b.g.close()


if __name__ == '__main__':
    main(sys.argv[1:])
