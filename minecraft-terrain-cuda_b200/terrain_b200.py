"""Python binding of the C ABI in include/terrain_b200.h (ctypes, no torch types).

    g = TerrainGenerator()                 # loads lib/libterrain_b200.so, device 0
    g.set_seed(123456789)
    blocks, biomes = g.generate([(0, 0), (1, 0)])   # numpy u16 (n, height, 16, 16), u8 (n, 1536)

The library must have been built (python build.py); a missing library raises, there is
no fallback path.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'lib', 'libterrain_b200.so')

STATUS = {0: 'TG_OK', 1: 'TG_ERR_INVALID_ARGUMENT', 2: 'TG_ERR_MODEL_MISMATCH', 3: 'TG_ERR_CUDA', 4: 'TG_ERR_OUT_OF_MEMORY', 5: 'TG_ERR_RANGE',
          6: 'TG_ERR_NO_SEED', 7: 'TG_ERR_DEVICE_TIMEOUT', 8: 'TG_ERR_INTERNAL', 9: 'TG_ERR_IO', 10: 'TG_ERR_CANCELLED'}


class TgChunk(ctypes.Structure):
    _fields_ = [('x', ctypes.c_int32), ('z', ctypes.c_int32)]


class TgConfig(ctypes.Structure):
    _fields_ = [('max_batch_chunks', ctypes.c_int32), ('pipeline_slots', ctypes.c_int32), ('device', ctypes.c_int32)]


class TgTiming(ctypes.Structure):
    _fields_ = [(k, ctypes.c_float) for k in ('h2d_ms', 'biome_ms', 'noise_ms', 'aquifer_ms', 'fill_ms', 'surface_ms', 'd2h_ms', 'kernel_ms',
                                               'wall_ms')] + [('batches', ctypes.c_int32), ('launches', ctypes.c_int32), ('walk_rules_ms', ctypes.c_float),
                                               ('corner_ms', ctypes.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TgRequest(ctypes.Structure):
    _fields_ = [('seed', ctypes.c_int64), ('chunks', ctypes.POINTER(TgChunk)), ('count', ctypes.c_int32),
                ('blocks_out', ctypes.POINTER(ctypes.c_uint16)), ('biomes_out', ctypes.POINTER(ctypes.c_uint8))]


class TgRequestDevice(ctypes.Structure):
    _fields_ = [('seed', ctypes.c_int64), ('chunks', ctypes.c_void_p), ('count', ctypes.c_int32), ('blocks_out', ctypes.c_void_p),
                ('biomes_out', ctypes.c_void_p)]


TG_BATCH_HOST_LOOP = 1


class TgViewerConfig(ctypes.Structure):
    _fields_ = [('window_chunks', ctypes.c_int32), ('width', ctypes.c_int32), ('height', ctypes.c_int32), ('reserved', ctypes.c_int32)]


class TgCamera(ctypes.Structure):
    _fields_ = [(k, ctypes.c_float) for k in ('x', 'y', 'z', 'yaw_deg', 'pitch_deg', 'fov_deg', 'sun_x', 'sun_y', 'sun_z', 'fog')]


class TgServerConfig(ctypes.Structure):
    _fields_ = [('batch_chunks', ctypes.c_int32), ('hbm_budget_bytes', ctypes.c_int64), ('reserved', ctypes.c_int32)]


class TgServerStats(ctypes.Structure):
    _fields_ = [('completed_requests', ctypes.c_int64), ('completed_chunks', ctypes.c_int64)] + \
               [(k, ctypes.c_double) for k in ('p50_ms', 'p99_ms', 'mean_ms', 'max_ms', 'chunks_per_s')] + \
               [(k, ctypes.c_int32) for k in ('batches', 'queued_requests', 'active_requests')] + \
               [('cancelled_requests', ctypes.c_int64), ('device_bytes_per_chunk', ctypes.c_double), ('max_active_chunks', ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


EXPORTS = ['tg_create', 'tg_destroy', 'tg_set_stream', 'tg_set_seed', 'tg_generate', 'tg_generate_u8', 'tg_write_region', 'tg_generate_device',
           'tg_generate_density', 'tg_generate_batch', 'tg_generate_batch_device', 'tg_biome_lookup',
           'tg_biome_lookup_noalloc',
           'tg_server_create', 'tg_server_submit', 'tg_server_submit_u8', 'tg_server_wait', 'tg_server_cancel', 'tg_server_get_stats',
           'tg_server_latencies', 'tg_server_reset_stats', 'tg_server_destroy', 'tg_set_launch_table', 'tg_get_launch_table', 'tg_kernel_times',
           'tg_host_schedule', 'tg_viewer_create', 'tg_viewer_update', 'tg_viewer_render', 'tg_viewer_state', 'tg_viewer_params', 'tg_viewer_destroy',
           'tg_alloc_pinned', 'tg_free_pinned', 'tg_model_info', 'tg_last_error_string']

# the tunable kernels of a batch, in pipeline order (tg_kernel_times order)
KERNELS = ['nb_insert', 'nb_resolve', 'climate_col', 'climate_quart', 'chain', 'cc_insert', 'cc_resolve', 'corner_col', 'corner', 'zoom_table',
           'zoom_uniform', 'sg_insert', 'sg_resolve', 'surface_level', 'aquifer_cell', 'aquifer_query', 'aquifer_skip', 'init_heights', 'fill',
           'surface1', 'block_biome', 'walk_rules', 'surface_frozen', 'gather', 'axis_insert', 'axis_number', 'axis_fill', 'walk_deferred']


class TerrainError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__('%s: %s' % (STATUS.get(status, status), msg))
        self.status = status


_lib = None


def load(path=LIB_PATH):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError('terrain_b200 library not built: %s (run python minecraft-terrain-cuda_b200/build.py)' % path)
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    L.tg_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(TgConfig), ctypes.POINTER(vp)]
    L.tg_destroy.argtypes = [vp]
    L.tg_set_seed.argtypes = [vp, ctypes.c_int64]
    L.tg_set_stream.argtypes = [vp, vp]
    L.tg_generate.argtypes = [vp, ctypes.POINTER(TgChunk), ctypes.c_int32, vp, vp, vp, ctypes.POINTER(TgTiming)]
    L.tg_generate_u8.argtypes = [vp, ctypes.POINTER(TgChunk), ctypes.c_int32, vp, vp, vp, ctypes.POINTER(TgTiming)]
    L.tg_write_region.argtypes = [vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_char_p, ctypes.c_char_p]
    L.tg_generate_device.argtypes = [vp, vp, ctypes.c_int32, vp, vp, ctypes.POINTER(TgTiming)]
    L.tg_generate_density.argtypes = [vp, vp, ctypes.c_int32, vp]
    L.tg_generate_batch.argtypes = [vp, ctypes.POINTER(TgRequest), ctypes.c_int32, ctypes.POINTER(TgTiming)]
    L.tg_generate_batch_device.argtypes = [vp, ctypes.POINTER(TgRequestDevice), ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(TgTiming)]
    L.tg_biome_lookup.argtypes = [vp, vp, vp, ctypes.c_int32, vp]
    L.tg_biome_lookup_noalloc.argtypes = [vp, vp, ctypes.c_int32, vp]
    L.tg_server_create.argtypes = [vp, ctypes.POINTER(TgServerConfig), ctypes.POINTER(vp)]
    L.tg_server_submit.argtypes = [vp, ctypes.c_int64, vp, ctypes.c_int32, vp, vp, ctypes.POINTER(ctypes.c_uint64)]
    L.tg_server_submit_u8.argtypes = [vp, ctypes.c_int64, vp, ctypes.c_int32, vp, vp, ctypes.POINTER(ctypes.c_uint64)]
    L.tg_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]
    L.tg_server_cancel.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32)]
    L.tg_server_latencies.argtypes = [vp, vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]
    L.tg_server_get_stats.argtypes = [vp, ctypes.POINTER(TgServerStats)]
    L.tg_server_reset_stats.argtypes = [vp]
    L.tg_server_destroy.argtypes = [vp]
    L.tg_set_launch_table.argtypes = [vp, ctypes.c_char_p]
    L.tg_get_launch_table.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    L.tg_kernel_times.argtypes = [vp, ctypes.c_int32, vp, vp, ctypes.c_int32]
    L.tg_host_schedule.argtypes = [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]
    L.tg_viewer_create.argtypes = [vp, ctypes.POINTER(TgViewerConfig), ctypes.POINTER(vp)]
    L.tg_viewer_update.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                   ctypes.POINTER(ctypes.c_float)]
    L.tg_viewer_render.argtypes = [vp, ctypes.POINTER(TgCamera), ctypes.c_int32, vp, vp, ctypes.POINTER(ctypes.c_float)]
    L.tg_viewer_state.argtypes = [vp, vp, vp, vp, vp]
    L.tg_viewer_params.argtypes = [vp, ctypes.POINTER(TgCamera), vp, vp, vp, vp, vp]
    L.tg_viewer_destroy.argtypes = [vp]
    L.tg_alloc_pinned.argtypes = [ctypes.c_size_t]
    L.tg_alloc_pinned.restype = vp
    L.tg_free_pinned.argtypes = [vp]
    L.tg_model_info.argtypes = [ctypes.POINTER(ctypes.c_int32)] * 5
    L.tg_last_error_string.restype = ctypes.c_char_p
    for f in ('tg_create', 'tg_destroy', 'tg_set_stream', 'tg_set_seed', 'tg_generate', 'tg_generate_u8', 'tg_write_region', 'tg_generate_device',
              'tg_generate_density', 'tg_generate_batch', 'tg_generate_batch_device', 'tg_biome_lookup', 'tg_biome_lookup_noalloc',
              'tg_server_create', 'tg_server_submit', 'tg_server_submit_u8', 'tg_server_wait', 'tg_server_cancel', 'tg_server_get_stats',
              'tg_server_latencies', 'tg_server_reset_stats', 'tg_server_destroy',
              'tg_set_launch_table', 'tg_get_launch_table', 'tg_kernel_times', 'tg_host_schedule', 'tg_model_info',
              'tg_viewer_create', 'tg_viewer_update', 'tg_viewer_render', 'tg_viewer_state', 'tg_viewer_params', 'tg_viewer_destroy'):
        getattr(L, f).restype = ctypes.c_int
    _lib = L
    return L


def model_info():
    L = load()
    v = [ctypes.c_int32() for _ in range(5)]
    L.tg_model_info(*[ctypes.byref(x) for x in v])
    return dict(zip(('min_y', 'height', 'sea_level', 'palette_size', 'biome_count'), [x.value for x in v]))


def host_schedule(count, max_batch_chunks, u8=True, table=None):
    """The batch sizes of a call with host outputs (tg_generate_u8 when u8, else tg_generate)
    over count chunks on a generator of max_batch_chunks, under a launch table (text; None:
    the compiled-in one). Host only."""
    L = load()
    n = ctypes.c_int32()
    st = L.tg_host_schedule(table.encode() if table is not None else None, 1 if u8 else 0, count, max_batch_chunks, None, 0, ctypes.byref(n))
    if st != 0:
        raise TerrainError(st, L.tg_last_error_string().decode())
    out = np.zeros(n.value, np.int32)
    L.tg_host_schedule(table.encode() if table is not None else None, 1 if u8 else 0, count, max_batch_chunks, _ptr(out), n.value, ctypes.byref(n))
    return out.tolist()


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def chunk_array(chunks):
    a = np.ascontiguousarray(np.asarray(chunks, dtype=np.int32).reshape(-1, 2))
    return a


class TerrainGenerator:
    def __init__(self, max_batch_chunks=2048, device=0, ir_path=None, terrain_path=None, pipeline_slots=2):
        self.L = load()
        self.h = ctypes.c_void_p()
        cfg = TgConfig(max_batch_chunks, pipeline_slots, device)
        self._check(self.L.tg_create(ir_path.encode() if ir_path else None, terrain_path.encode() if terrain_path else None, ctypes.byref(cfg),
                                     ctypes.byref(self.h)))
        info = model_info()
        self.height = info['height']
        self.min_y = info['min_y']
        self.per = 256 * self.height
        self.qper = 16 * (self.height // 4)

    def _check(self, st):
        if st != 0:
            raise TerrainError(st, self.L.tg_last_error_string().decode())

    def close(self):
        if self.h:
            self.L.tg_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle):
        """cudaStream_t as an int (e.g. torch.cuda.current_stream().cuda_stream); 0 = own stream."""
        self._check(self.L.tg_set_stream(self.h, ctypes.c_void_p(stream_handle) if stream_handle else None))

    def set_seed(self, seed):
        self._check(self.L.tg_set_seed(self.h, int(seed)))

    def generate(self, chunks, blocks_out=None, biomes_out=None, aquifer=False, timing=False):
        a = chunk_array(chunks)
        n = a.shape[0]
        blocks = blocks_out if blocks_out is not None else np.empty((n, self.height, 16, 16), np.uint16)
        biomes = biomes_out if biomes_out is not None else np.empty((n, self.qper), np.uint8)
        aq = np.empty((n, self.height, 16, 16), np.uint16) if aquifer else None
        # stage timing records events between the kernels and waits for each batch, so it is
        # requested only when asked for; without it batches run as CUDA graphs and overlap
        t = TgTiming() if timing else None
        self._check(self.L.tg_generate(self.h, a.ctypes.data_as(ctypes.POINTER(TgChunk)), n, _ptr(blocks), _ptr(biomes), _ptr(aq),
                                       ctypes.byref(t) if timing else None))
        out = (blocks, biomes) + ((aq,) if aquifer else ())
        return out + (t.as_dict(),) if timing else out

    def generate_u8(self, chunks, blocks_out=None, biomes_out=None, aquifer=False, timing=False):
        """The reference generator's output form: u8 palette index per block (tg_generate_u8)."""
        a = chunk_array(chunks)
        n = a.shape[0]
        blocks = blocks_out if blocks_out is not None else np.empty((n, self.height, 16, 16), np.uint8)
        biomes = biomes_out if biomes_out is not None else np.empty((n, self.qper), np.uint8)
        aq = np.empty((n, self.height, 16, 16), np.uint8) if aquifer else None
        t = TgTiming() if timing else None
        self._check(self.L.tg_generate_u8(self.h, a.ctypes.data_as(ctypes.POINTER(TgChunk)), n, _ptr(blocks), _ptr(biomes), _ptr(aq),
                                          ctypes.byref(t) if timing else None))
        out = (blocks, biomes) + ((aq,) if aquifer else ())
        return out + (t.as_dict(),) if timing else out

    def write_region(self, seed, x0, z0, region, dump_dir=None, topdown_path=None):
        """Region dump (terrain.u8, biomes.u8, meta.json in dump_dir) and / or top-down map
        (topdown_path) of the region x region chunks from (x0, z0); sets the seed."""
        enc = lambda p: os.fsencode(p) if p is not None else None
        self._check(self.L.tg_write_region(self.h, int(seed), int(x0), int(z0), int(region), enc(dump_dir), enc(topdown_path)))

    def generate_device(self, chunks_ptr, count, blocks_ptr, biomes_ptr=None, timing=True):
        """Device pointers (ints); returns the stage timing dict (None with timing=False, which
        leaves out the stage events)."""
        t = TgTiming() if timing else None
        self._check(self.L.tg_generate_device(self.h, ctypes.c_void_p(chunks_ptr), count, ctypes.c_void_p(blocks_ptr),
                                              ctypes.c_void_p(biomes_ptr) if biomes_ptr else None, ctypes.byref(t) if timing else None))
        return t.as_dict() if timing else None

    def generate_density(self, chunks):
        """Final density per block, f32 (n, height, 16, 16) (tg_generate_density)."""
        a = chunk_array(chunks)
        n = a.shape[0]
        out = np.empty((n, self.height, 16, 16), np.float32)
        self._check(self.L.tg_generate_density(self.h, _ptr(a), n, _ptr(out)))
        return out

    def set_launch_table(self, text=None):
        """Launch shapes as text (None: the compiled-in, autotuned table)."""
        self._check(self.L.tg_set_launch_table(self.h, text.encode() if text is not None else None))

    def launch_table(self):
        need = ctypes.c_size_t()
        self._check(self.L.tg_get_launch_table(self.h, None, 0, ctypes.byref(need)))
        buf = ctypes.create_string_buffer(need.value)
        self._check(self.L.tg_get_launch_table(self.h, buf, need.value, None))
        return buf.value.decode()

    def kernel_times(self, enable=True):
        """{kernel: (ms, launches)} gathered from timed batches since the last call; enable
        switches the per-kernel events on or off from now on."""
        ms = np.zeros(len(KERNELS), np.float32)
        calls = np.zeros(len(KERNELS), np.int32)
        self._check(self.L.tg_kernel_times(self.h, 1 if enable else 0, _ptr(ms), _ptr(calls), len(KERNELS)))
        return {k: (float(ms[i]), int(calls[i])) for i, k in enumerate(KERNELS)}

    def generate_batch(self, requests, timing=False):
        """requests: list of (seed, chunks). Returns list of (blocks, biomes)."""
        outs, keep, reqs = [], [], (TgRequest * max(1, len(requests)))()
        for i, (seed, chunks) in enumerate(requests):
            a = chunk_array(chunks)
            n = a.shape[0]
            b = np.empty((n, self.height, 16, 16), np.uint16)
            bi = np.empty((n, self.qper), np.uint8)
            keep.append(a)
            outs.append((b, bi))
            reqs[i].seed = int(seed)
            reqs[i].chunks = a.ctypes.data_as(ctypes.POINTER(TgChunk))
            reqs[i].count = n
            reqs[i].blocks_out = b.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))
            reqs[i].biomes_out = bi.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        t = TgTiming() if timing else None
        self._check(self.L.tg_generate_batch(self.h, reqs, len(requests), ctypes.byref(t) if timing else None))
        return (outs, t.as_dict()) if timing else outs

    def generate_batch_device(self, requests, host_loop=False, timing=False):
        """requests: list of (seed, chunks_ptr, count, blocks_ptr, biomes_ptr or 0), device
        pointers as ints (tg_generate_batch_device). Returns the timing dict with timing=True."""
        reqs = (TgRequestDevice * max(1, len(requests)))()
        for i, (seed, cp, n, bp, qp) in enumerate(requests):
            reqs[i].seed, reqs[i].chunks, reqs[i].count = int(seed), cp, int(n)
            reqs[i].blocks_out, reqs[i].biomes_out = bp, (qp or None)
        t = TgTiming() if timing else None
        self._check(self.L.tg_generate_batch_device(self.h, reqs, len(requests), TG_BATCH_HOST_LOOP if host_loop else 0,
                                                    ctypes.byref(t) if timing else None))
        return t.as_dict() if timing else None

    def biome_lookup(self, seeds, xyz):
        xyz = np.ascontiguousarray(np.asarray(xyz, np.int32).reshape(-1, 3))
        seeds = np.ascontiguousarray(np.broadcast_to(np.asarray(seeds, np.int64), (xyz.shape[0],)))
        out = np.empty(xyz.shape[0], np.uint8)
        self._check(self.L.tg_biome_lookup(self.h, _ptr(seeds), _ptr(xyz), xyz.shape[0], _ptr(out)))
        return out

    def biome_lookup_noalloc(self, xyz):
        """Lookups for the current seed through the fixed device scratch (at most 4,096)."""
        xyz = np.ascontiguousarray(np.asarray(xyz, np.int32).reshape(-1, 3))
        out = np.empty(xyz.shape[0], np.uint8)
        self._check(self.L.tg_biome_lookup_noalloc(self.h, _ptr(xyz), xyz.shape[0], _ptr(out)))
        return out


class TerrainServer:
    """Continuous-batching server over one generator (tg_server_*).

        srv = TerrainServer(gen, batch_chunks=512)
        t = srv.submit(seed, chunks)          # returns a ticket; outputs allocated here
        blocks, biomes = srv.wait(t)
    """

    def __init__(self, gen, batch_chunks=0, hbm_budget_bytes=0):
        self.gen = gen
        self.L = gen.L
        self.h = ctypes.c_void_p()
        cfg = TgServerConfig(batch_chunks, hbm_budget_bytes, 0)
        gen._check(self.L.tg_server_create(gen.h, ctypes.byref(cfg), ctypes.byref(self.h)))
        self.pending = {}

    def submit(self, seed, chunks, blocks_out=None, biomes_out=None, u8=False):
        """Queues a request; u8=True asks for the u8 palette-index form (tg_server_submit_u8)."""
        a = chunk_array(chunks)
        n = a.shape[0]
        g = self.gen
        blocks = blocks_out if blocks_out is not None else np.empty((n, g.height, 16, 16), np.uint8 if u8 else np.uint16)
        biomes = biomes_out if biomes_out is not None else np.empty((n, g.qper), np.uint8)
        t = ctypes.c_uint64()
        f = self.L.tg_server_submit_u8 if u8 else self.L.tg_server_submit
        g._check(f(self.h, int(seed), _ptr(a), n, _ptr(blocks), _ptr(biomes), ctypes.byref(t)))
        self.pending[t.value] = (a, blocks, biomes)
        return t.value

    def poll(self, ticket, timeout_ms=0):
        done = ctypes.c_int32()
        st = self.L.tg_server_wait(self.h, ctypes.c_uint64(ticket), int(timeout_ms), ctypes.byref(done))
        if st == 10:
            self.pending.pop(ticket, None)
        self.gen._check(st)
        return bool(done.value)

    def wait(self, ticket):
        self.poll(ticket, -1)
        _, blocks, biomes = self.pending.pop(ticket)
        return blocks, biomes

    def cancel(self, ticket):
        """True when the request was still pending (it will report TG_ERR_CANCELLED)."""
        p = ctypes.c_int32()
        self.gen._check(self.L.tg_server_cancel(self.h, ctypes.c_uint64(ticket), ctypes.byref(p)))
        return bool(p.value)

    def latencies(self):
        n = ctypes.c_int32()
        self.gen._check(self.L.tg_server_latencies(self.h, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1))
        self.gen._check(self.L.tg_server_latencies(self.h, _ptr(out), out.shape[0], ctypes.byref(n)))
        return out[:n.value]

    def stats(self):
        st = TgServerStats()
        self.gen._check(self.L.tg_server_get_stats(self.h, ctypes.byref(st)))
        return st.as_dict()

    def reset_stats(self):
        self.gen._check(self.L.tg_server_reset_stats(self.h))

    def close(self):
        if self.h:
            self.L.tg_server_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def camera(x, y, z, yaw_deg=0.0, pitch_deg=-10.0, fov_deg=70.0, sun=(-0.45, 0.62, -0.64), fog=0.0):
    return TgCamera(x, y, z, yaw_deg, pitch_deg, fov_deg, sun[0], sun[1], sun[2], fog)


class TerrainViewer:
    """Live flythrough renderer over a generator (tg_viewer_*).

        v = TerrainViewer(gen, window_chunks=64, width=1280, height=720)
        n, ms = v.update(cx, cz, radius=24)             # generate what the window lacks
        rgb, hits, ms = v.render(camera(x, y, z, yaw, pitch), frame)
    """

    def __init__(self, gen, window_chunks=64, width=1280, height=720):
        self.gen = gen
        self.L = gen.L
        self.h = ctypes.c_void_p()
        self.W, self.width, self.height = window_chunks, width, height
        cfg = TgViewerConfig(window_chunks, width, height, 0)
        gen._check(self.L.tg_viewer_create(gen.h, ctypes.byref(cfg), ctypes.byref(self.h)))

    def update(self, cx, cz, radius, cap=0, frame=0):
        n, ms = ctypes.c_int32(), ctypes.c_float()
        self.gen._check(self.L.tg_viewer_update(self.h, int(cx), int(cz), int(radius), int(cap), int(frame), ctypes.byref(n), ctypes.byref(ms)))
        return n.value, ms.value

    def render(self, cam, frame=0, hits=False, rgb=True):
        out = np.empty((self.height, self.width, 3), np.uint8) if rgb else None
        hit = np.empty((self.height, self.width, 4), np.int32) if hits else None
        ms = ctypes.c_float()
        self.gen._check(self.L.tg_viewer_render(self.h, ctypes.byref(cam), int(frame), _ptr(out), _ptr(hit), ctypes.byref(ms)))
        return out, hit, ms.value

    def state(self):
        wb = self.W * 16
        info = model_info()
        vox = np.empty((info['height'], wb, wb), np.uint8)
        cells = np.empty((self.W * 4, self.W * 4), np.uint32)
        slots = np.empty((self.W * self.W, 2), np.int32)
        born = np.empty(self.W * self.W, np.int32)
        self.gen._check(self.L.tg_viewer_state(self.h, _ptr(vox), _ptr(cells), _ptr(slots), _ptr(born)))
        return vox, cells, slots, born

    def params(self, cam):
        c = np.empty(18, np.float32)
        top = np.empty((64, 3), np.float32)
        side = np.empty((64, 3), np.float32)
        caps = np.empty(64, np.int32)
        ids = np.empty(7, np.int32)
        self.gen._check(self.L.tg_viewer_params(self.h, ctypes.byref(cam), _ptr(c), _ptr(top), _ptr(side), _ptr(caps), _ptr(ids)))
        return c, top, side, caps, ids

    def close(self):
        if self.h:
            self.L.tg_viewer_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
