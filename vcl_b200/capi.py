"""ctypes binding of the vcl C ABI (include/vcl.h) in libvcl.so.

This is the reference-side binding a Python caller uses: every function of
vcl.h is declared here with its argument types.  Buffers are passed as raw
device addresses (for example ``tensor.data_ptr()`` of a CUDA tensor) and
streams as raw ``cudaStream_t`` handles.  There is no fallback: if the
library is missing or a call fails, an exception is raised.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# the in-tree build; VCL_LIB names another build of the same library
LIB_PATH = os.environ.get("VCL_LIB") or os.path.join(HERE, "libvcl.so")

c_int, c_ll, c_size, c_float, c_double, c_void_p, c_char_p = (
    ctypes.c_int, ctypes.c_longlong, ctypes.c_size_t, ctypes.c_float, ctypes.c_double, ctypes.c_void_p, ctypes.c_char_p)
P = c_void_p

MODE_COMPAT = 0
MODE_EXACT = 1

# name: (restype, [argtypes])
SIGNATURES = {
    "vcl_version": (c_char_p, []),
    "vcl_create": (c_int, [c_int, ctypes.POINTER(c_void_p)]),
    "vcl_destroy": (None, [P]),
    "vcl_last_error": (c_char_p, [P]),
    "vcl_set_mode": (c_int, [P, c_int]),
    "vcl_get_mode": (c_int, [P]),
    "vcl_set_raster_config": (c_int, [P, c_int, c_ll]),
    "vcl_set_raster_areas": (c_int, [P, c_int, c_int]),
    "vcl_set_raster_autotune": (c_int, [P, c_int]),
    "vcl_get_raster_config": (c_int, [P, ctypes.POINTER(c_int), ctypes.POINTER(c_ll)]),
    "vcl_raster_overflow_count": (c_int, [P, P, ctypes.POINTER(c_ll)]),
    "vcl_check_indices": (c_int, [P, P, ctypes.POINTER(c_int)]),
    "vcl_reserve_raster": (c_int, [P, c_int, c_int, c_int, c_int]),
    "vcl_tex_levels": (c_int, [c_int, c_int, c_int]),
    "vcl_tex_level_offset": (c_size, [c_int, c_int, c_int, c_int]),
    "vcl_project_fwd": (c_int, [P, P, c_int, P, c_int, c_int, P, P]),
    "vcl_project_bwd": (c_int, [P, P, c_int, P, c_int, c_int, P, P]),
    "vcl_rasterize_fwd": (c_int, [P, P, c_int, P, c_int, c_int, c_int, c_int, P, P, P]),
    "vcl_raster_scratch_bytes": (c_size, []),
    "vcl_raster_scratch_init": (c_int, [P]),
    "vcl_rasterize_fwd_static": (c_int, [P, P, c_int, P, c_int, c_int, c_int, c_int, P, P, P]),
    "vcl_rasterize_bwd": (c_int, [P, P, c_int, P, c_int, c_int, c_int, c_int, P, P, P, P]),
    "vcl_raster_ties": (c_int, [P, P, c_int, P, c_int, c_int, c_int, c_int, P, P, P, P]),
    "vcl_probe_red_throughput": (c_int, [P, P, c_ll, c_int, ctypes.POINTER(c_ll), P]),
    "vcl_probe_mufu_threads": (c_ll, [P]),
    "vcl_probe_mufu_throughput": (c_int, [P, P, c_int, ctypes.POINTER(c_ll), P]),
    "vcl_probe_fma_throughput": (c_int, [P, P, c_int, ctypes.POINTER(c_ll), P]),
    "vcl_interpolate_fwd": (c_int, [P, P, P, c_int, c_int, c_int, P, c_int, c_int, P, c_int, P, P, P]),
    "vcl_interpolate_bwd": (c_int, [P, P, c_int, c_int, c_int, P, c_int, c_int, P, c_int, P, P, P, P]),
    "vcl_texture_fwd": (c_int, [P, P, P, P, c_int, c_int, c_int, P, c_int, c_int, c_int, c_int, P, P]),
    "vcl_texture_bwd": (c_int, [P, P, P, P, c_int, c_int, c_int, P, c_int, c_int, c_int, c_int, P, P, P, P, P]),
    "vcl_texture_build_mips": (c_int, [P, P, c_int, c_int, c_int, c_int, P]),
    "vcl_texture_grad_pushdown": (c_int, [P, P, c_int, c_int, c_int, c_int, P]),
    "vcl_clamp": (c_int, [P, P, c_size, c_float, c_float, P]),
    "vcl_antialias_fwd": (c_int, [P, P, c_int, P, c_int, P, c_int, c_int, c_int, c_int, P, P, P]),
    "vcl_antialias_bwd": (c_int, [P, P, c_int, P, c_int, P, c_int, c_int, c_int, c_int, P, P, P, P, P]),
    "vcl_normal_axis_fwd": (c_int, [P, P, c_int, c_int, c_int, P, P, c_int, P, c_int, P, P]),
    "vcl_view_axis_fwd": (c_int, [P, c_int, c_int, c_int, P, P, P]),
    "vcl_sg_specular_fwd": (c_int, [P, P, c_int, c_int, c_int, P, P, P, c_float, P, P, P, P]),
    "vcl_sg_specular_bwd": (c_int, [P, P, c_int, c_int, c_int, P, P, P, c_float, P, P, P, P]),
    "vcl_sg_fwd": (c_int, [P, P, c_int, c_int, c_int, c_int, c_int, P, P, P, P, P, P, P, P, P, P, P, P]),
    "vcl_sg_bwd": (c_int, [P, P, c_int, c_int, c_int, c_int, c_int, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P,
                           P]),
    "vcl_mse": (c_int, [P, P, P, c_size, P, P, P]),
    "vcl_adam_step": (c_int, [P, P, P, P, P, c_size, c_double, c_double, c_double, c_double, c_int, P]),
    "vcl_fit_create": (c_int, [P, P, ctypes.POINTER(c_void_p)]),
    "vcl_fit_destroy": (None, [P]),
    "vcl_fit_set_strategy": (c_int, [P, c_int]),
    "vcl_fit_set_target": (c_int, [P, P, c_int, P]),
    "vcl_fit_set_cameras": (c_int, [P, P, P, P]),
    "vcl_fit_step": (c_int, [P, P]),
    "vcl_fit_render": (c_int, [P, P, P]),
    "vcl_fit_loss_device": (c_void_p, [P]),
    "vcl_fit_read_loss": (c_int, [P, P, P]),
    "vcl_fit_read_loss_async": (c_int, [P, P, P]),
    "vcl_fit_state_bytes": (ctypes.c_size_t, [P]),
    "vcl_fit_save_state": (c_int, [P, P, ctypes.c_size_t, P]),
    "vcl_fit_load_state": (c_int, [P, P, ctypes.c_size_t, P]),
    "vcl_fit_read_params": (c_int, [P, P, P, P, P, P, P]),
    "vcl_fit_footprint": (c_size, [P]),
    "vcl_fit_raster_tuning": (c_int, [P, P, P]),
    "vcl_fit_launches_per_step": (c_int, [P]),
    "vcl_fit_raster_schedule": (c_int, [P, P, P, P, P, P]),
    "vcl_raster_tuning_cache_clear": (None, []),
    "vcl_fit_stage_target": (c_int, [P, P, P]),
    "vcl_fit_prepare": (c_int, [P, P]),
    "vcl_fit_destroy_async": (None, [P, P]),
    "vcl_fit_kernel_count": (c_int, []),
    "vcl_fit_kernel_name": (c_char_p, [c_int]),
    "vcl_fit_time_kernels": (c_int, [P, P, c_int, P, c_int]),
    "vcl_asset_error": (c_char_p, []),
    "vcl_obj_load": (c_int, [P, c_char_p, ctypes.POINTER(c_void_p)]),
    "vcl_obj_free": (None, [P]),
    "vcl_obj_counts": (c_int, [P, P, P, P, P, P]),
    "vcl_obj_arrays": (c_int, [P, P, P, P, P, P, P]),
    "vcl_obj_welded": (c_int, [P, P, P, P, P]),
    "vcl_bmp_load": (c_int, [P, c_char_p, P, P, P, P]),
    "vcl_sg_load": (c_int, [P, c_char_p, c_int, P, P, P, P]),
    "vcl_batch_create": (c_int, [P, ctypes.POINTER(c_void_p)]),
    "vcl_batch_destroy": (None, [P]),
    "vcl_batch_add": (c_int, [P, P]),
    "vcl_batch_remove": (c_int, [P, P]),
    "vcl_batch_size": (c_int, [P]),
    "vcl_batch_set_repeat": (c_int, [P, P, c_int]),
    "vcl_batch_step": (c_int, [P, P]),
    "vcl_batch_launches_per_step": (c_int, [P]),
    "vcl_batch_rebuild_stats": (c_int, [P, P, P]),
    "vcl_server_host_stats": (c_int, [P, P, P, P, P]),
    "vcl_server_create": (c_int, [P, c_size, c_int, ctypes.POINTER(c_void_p)]),
    "vcl_server_destroy": (None, [P]),
    "vcl_server_last_error": (c_char_p, [P]),
    "vcl_server_submit": (c_int, [P, P, P, c_int, c_int, P]),
    "vcl_server_tick": (c_int, [P, P, P, P]),
    "vcl_server_drain": (c_int, [P, P]),
    "vcl_server_pending": (c_int, [P]),
    "vcl_server_now_ms": (c_double, [P]),
    "vcl_server_job_status": (c_int, [P, c_ll, P, P, P, P, P]),
    "vcl_server_job_result": (c_int, [P, c_ll, P, P, P, P, P, P]),
    "vcl_server_stats": (c_int, [P, P, P, P, P, P, P]),
}

FIT_PLAIN = 0
FIT_FUSED = 1


class FitDesc(ctypes.Structure):
    """vcl_fit_desc of include/vcl.h."""
    _fields_ = [("W", c_int), ("H", c_int), ("views", c_int), ("C", c_int), ("K", c_int), ("nv", c_int),
                ("nt", c_int), ("tex_w", c_int), ("tex_h", c_int), ("levels", c_int),
                ("pos", c_void_p), ("tri", c_void_p), ("uv", c_void_p), ("normal", c_void_p), ("tex", c_void_p),
                ("lobe_axis", c_void_p), ("lobe_sharp", c_void_p), ("lobe_amp", c_void_p), ("mvp", c_void_p),
                ("pvinv", c_void_p), ("rot", c_void_p), ("roughness", c_float), ("ior", c_float),
                ("lr", c_double), ("beta1", c_double), ("beta2", c_double), ("eps", c_double),
                ("learn_pos", c_int), ("learn_tex", c_int), ("learn_lobes", c_int),
                ("lr_pos", c_double), ("lr_tex", c_double), ("lr_lobes", c_double)]


class VclError(RuntimeError):
    pass


_lib = None


def lib():
    """Load libvcl.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise VclError(f"{LIB_PATH} is missing: build it with `python -m vcl_b200.build` (nvcc, sm_100a)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(SIGNATURES)


def _addr(x):
    """Device address of a torch tensor / int / None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return x.data_ptr()


class Context:
    """Owns one vcl_ctx.  Methods mirror the C functions without the ``vcl_``
    prefix; tensor arguments may be torch CUDA tensors or raw addresses."""

    def __init__(self, device=0, mode=MODE_COMPAT):
        self.lib = lib()
        h = c_void_p()
        st = self.lib.vcl_create(device, ctypes.byref(h))
        if st != 0:
            raise VclError(f"vcl_create(device={device}) failed with status {st}")
        self.h = h
        self.device = device
        self.set_mode(mode)

    def close(self):
        if self.h:
            self.lib.vcl_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, name):
        if st != 0:
            msg = self.lib.vcl_last_error(self.h)
            raise VclError(f"{name} failed (status {st}): {msg.decode() if msg else ''}")

    def set_mode(self, mode):
        self._check(self.lib.vcl_set_mode(self.h, mode), "vcl_set_mode")

    def set_raster_config(self, tile, bin_capacity=0):
        self._check(self.lib.vcl_set_raster_config(self.h, tile, bin_capacity), "vcl_set_raster_config")

    def raster_overflow_count(self, stream=None):
        c = c_ll()
        self._check(self.lib.vcl_raster_overflow_count(self.h, stream, ctypes.byref(c)), "vcl_raster_overflow_count")
        return c.value

    def check_indices(self, stream=None):
        c = c_int()
        self._check(self.lib.vcl_check_indices(self.h, stream, ctypes.byref(c)), "vcl_check_indices")
        return c.value

    def call(self, name, *args):
        fn = getattr(self.lib, "vcl_" + name)
        conv = []
        for a, t in zip(args, fn.argtypes[1:]):
            conv.append(_addr(a) if t is P else a)
        self._check(fn(self.h, *conv), "vcl_" + name)

    def __getattr__(self, name):
        if name.startswith("_") or "vcl_" + name not in SIGNATURES:
            raise AttributeError(name)
        return lambda *a: self.call(name, *a)


def fit_desc(S, tex=None, pos=None, lobes=None, learn=(1, 1, 1)):
    """vcl_fit_desc for scene S (starting values default to the scene's
    initial ones).  Returns (desc, arrays): the arrays back the descriptor's
    host pointers and must outlive its use."""
    import numpy as np
    tex = S.tex_init if tex is None else tex
    pos = S.pos if pos is None else pos
    axis, sharp, amp = lobes if lobes is not None else (S.lobe_axis_init, S.lobe_sharp_init, S.lobe_amp_init)
    keep = [np.ascontiguousarray(a, dtype=dt) for a, dt in (
        (pos, np.float32), (S.tri, np.uint32), (S.uv, np.float32), (S.normal, np.float32), (tex, np.float32),
        (axis, np.float32), (sharp, np.float32), (amp, np.float32), (S.mvp, np.float32), (S.pvinv, np.float32),
        (S.rot, np.float32))]
    d = FitDesc()
    d.W, d.H, d.views, d.C, d.K = S.W, S.H, S.views, S.C, S.K
    d.nv, d.nt, d.tex_w, d.tex_h, d.levels = S.nv, S.nt, S.tex_w, S.tex_h, S.levels
    (d.pos, d.tri, d.uv, d.normal, d.tex, d.lobe_axis, d.lobe_sharp, d.lobe_amp, d.mvp, d.pvinv,
     d.rot) = [a.ctypes.data for a in keep]
    d.roughness, d.ior = S.roughness, S.ior
    d.lr, d.beta1, d.beta2, d.eps = S.lr, 0.9, 0.999, 1e-8
    d.learn_pos, d.learn_tex, d.learn_lobes = learn
    d.lr_pos = getattr(S, "lr_pos", 0.0) or 0.0
    d.lr_tex = d.lr_lobes = 0.0
    return d, keep


def footprint(S):
    """Device bytes a fit job for scene S holds at most."""
    d, keep = fit_desc(S)
    return lib().vcl_fit_footprint(ctypes.byref(d))


class Fit:
    """A resident fit job (vcl_fit_*).  `scene` is a vcl_b200.scenes.Scene;
    its host arrays are uploaded at creation."""

    def __init__(self, ctx, scene, tex=None, pos=None, lobes=None, learn=(1, 1, 1), strategy=FIT_PLAIN):
        self.ctx = ctx
        self.scene = scene
        d, keep = fit_desc(scene, tex, pos, lobes, learn)
        self.desc = d
        h = c_void_p()
        ctx._check(ctx.lib.vcl_fit_create(ctx.h, ctypes.byref(d), ctypes.byref(h)), "vcl_fit_create")
        self.h = h
        self.set_strategy(strategy)

    def close(self):
        if self.h:
            self.ctx.lib.vcl_fit_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, st, name):
        self.ctx._check(st, name)

    def set_strategy(self, s):
        self._c(self.ctx.lib.vcl_fit_set_strategy(self.h, s), "vcl_fit_set_strategy")

    def set_target(self, src, stream=None, is_device=None):
        if is_device is None:
            is_device = not hasattr(src, "ctypes")
        addr = src.ctypes.data if hasattr(src, "ctypes") else _addr(src)
        self._c(self.ctx.lib.vcl_fit_set_target(self.h, addr, int(is_device), stream), "vcl_fit_set_target")

    def stage_target(self, host, copy_stream=None):
        """Upload the next step's target (host memory; pinned for overlap) on `copy_stream`."""
        addr = host.ctypes.data if hasattr(host, "ctypes") else _addr(host)
        self._c(self.ctx.lib.vcl_fit_stage_target(self.h, addr, copy_stream), "vcl_fit_stage_target")

    def set_cameras(self, mvp, pvinv, stream=None):
        a = mvp.ctypes.data if hasattr(mvp, "ctypes") else _addr(mvp)
        b = pvinv.ctypes.data if hasattr(pvinv, "ctypes") else _addr(pvinv)
        self._c(self.ctx.lib.vcl_fit_set_cameras(self.h, a, b, stream), "vcl_fit_set_cameras")

    def step(self, stream=None):
        self._c(self.ctx.lib.vcl_fit_step(self.h, stream), "vcl_fit_step")

    def render(self, out, stream=None):
        self._c(self.ctx.lib.vcl_fit_render(self.h, _addr(out), stream), "vcl_fit_render")

    def read_loss(self, stream=None):
        out = ctypes.c_float()
        self._c(self.ctx.lib.vcl_fit_read_loss(self.h, ctypes.byref(out), stream), "vcl_fit_read_loss")
        return out.value

    def read_loss_async(self, host_address, stream=None):
        """Queue the copy of the last step's loss to `host_address` (pinned
        host memory, e.g. a pinned torch tensor's data_ptr()) without waiting."""
        self._c(self.ctx.lib.vcl_fit_read_loss_async(self.h, ctypes.c_void_p(host_address), stream),
                "vcl_fit_read_loss_async")

    def save_state(self, stream=None):
        """The job's resumable state (parameters, Adam moments and step) as bytes."""
        n = self.ctx.lib.vcl_fit_state_bytes(self.h)
        buf = ctypes.create_string_buffer(n)
        self._c(self.ctx.lib.vcl_fit_save_state(self.h, buf, n, stream), "vcl_fit_save_state")
        return buf.raw

    def load_state(self, state, stream=None):
        buf = ctypes.create_string_buffer(bytes(state), len(state))
        self._c(self.ctx.lib.vcl_fit_load_state(self.h, buf, len(state), stream), "vcl_fit_load_state")

    def loss_address(self):
        return self.ctx.lib.vcl_fit_loss_device(self.h)

    def raster_tuning(self):
        t = ctypes.c_int()
        ms = (ctypes.c_float * 3)()
        self._c(self.ctx.lib.vcl_fit_raster_tuning(self.h, ctypes.byref(t), ms), "vcl_fit_raster_tuning")
        return t.value, list(ms)

    def launches_per_step(self):
        return self.ctx.lib.vcl_fit_launches_per_step(self.h)

    def read_params(self, stream=None):
        import numpy as np
        S = self.scene
        pos = np.zeros((S.nv, 3), np.float32)
        tex = np.zeros((S.tex_h, S.tex_w, S.C), np.float32)
        ax = np.zeros((S.K, 3), np.float32); sh = np.zeros(S.K, np.float32); am = np.zeros((S.K, S.C), np.float32)
        self._c(self.ctx.lib.vcl_fit_read_params(self.h, pos.ctypes.data, tex.ctypes.data, ax.ctypes.data,
                                                 sh.ctypes.data, am.ctypes.data, stream), "vcl_fit_read_params")
        return pos, tex, (ax, sh, am)

    def time_kernels(self, stream=None, reps=5):
        """{stage name: ms per launch} of the fused step's stages (clears the gradients)."""
        L = self.ctx.lib
        n = L.vcl_fit_kernel_count()
        ms = (ctypes.c_float * n)()
        self._c(L.vcl_fit_time_kernels(self.h, stream, reps, ms, n), "vcl_fit_time_kernels")
        return {L.vcl_fit_kernel_name(i).decode(): ms[i] for i in range(n)}

    def raster_schedule(self):
        """(tile, direct-raster box area, bin capacity, from cache, overflowed tiles of the last step)."""
        t, sa, cached = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        cap, ov = c_ll(), c_ll()
        self._c(self.ctx.lib.vcl_fit_raster_schedule(self.h, ctypes.byref(t), ctypes.byref(sa), ctypes.byref(cap),
                                                     ctypes.byref(cached), ctypes.byref(ov)),
                "vcl_fit_raster_schedule")
        return t.value, sa.value, cap.value, bool(cached.value), ov.value


class Batch:
    """vcl_batch: fit jobs advanced together by one graph launch per step."""

    def __init__(self, ctx):
        self.ctx = ctx
        h = c_void_p()
        ctx._check(ctx.lib.vcl_batch_create(ctx.h, ctypes.byref(h)), "vcl_batch_create")
        self.h = h
        self.jobs = []

    def add(self, fit):
        self.ctx._check(self.ctx.lib.vcl_batch_add(self.h, fit.h), "vcl_batch_add")
        self.jobs.append(fit)

    def remove(self, fit):
        self.ctx._check(self.ctx.lib.vcl_batch_remove(self.h, fit.h), "vcl_batch_remove")
        self.jobs.remove(fit)

    def step(self, stream=None):
        self.ctx._check(self.ctx.lib.vcl_batch_step(self.h, stream), "vcl_batch_step")

    def set_repeat(self, fit, iterations):
        self.ctx._check(self.ctx.lib.vcl_batch_set_repeat(self.h, fit.h, int(iterations)), "vcl_batch_set_repeat")

    def launches_per_step(self):
        return self.ctx.lib.vcl_batch_launches_per_step(self.h)

    def __len__(self):
        return self.ctx.lib.vcl_batch_size(self.h)

    def close(self):
        if self.h:
            self.ctx.lib.vcl_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


JOB_QUEUED, JOB_LIVE, JOB_DONE, JOB_FAILED = 0, 1, 2, 3


class Server:
    """vcl_server: admission by device footprint, continuous batching of the
    live jobs' iterations, p50/p99 job latency."""

    def __init__(self, ctx, budget_bytes, max_live=64):
        self.ctx = ctx
        h = c_void_p()
        st = ctx.lib.vcl_server_create(ctx.h, int(budget_bytes), int(max_live), ctypes.byref(h))
        if st:
            raise VclError(f"vcl_server_create failed with status {st}")
        self.h = h
        self.scenes = {}

    def _c(self, st, name):
        if st:
            msg = self.ctx.lib.vcl_server_last_error(self.h)
            raise VclError(f"{name} failed (status {st}): {msg.decode() if msg else ''}")

    def submit(self, scene, target, iterations, keep_result=False):
        """target: host float32 array [views][H][W][4]."""
        import numpy as np
        d, keep = fit_desc(scene)
        t = np.ascontiguousarray(target, dtype=np.float32)
        jid = c_ll()
        self._c(self.ctx.lib.vcl_server_submit(self.h, ctypes.byref(d), t.ctypes.data, int(iterations),
                                               int(keep_result), ctypes.byref(jid)), "vcl_server_submit")
        self.scenes[jid.value] = scene
        return jid.value

    def tick(self, stream=None):
        live, done = ctypes.c_int(), ctypes.c_int()
        self._c(self.ctx.lib.vcl_server_tick(self.h, stream, ctypes.byref(live), ctypes.byref(done)),
                "vcl_server_tick")
        return live.value, done.value

    def drain(self, stream=None):
        self._c(self.ctx.lib.vcl_server_drain(self.h, stream), "vcl_server_drain")

    def pending(self):
        return self.ctx.lib.vcl_server_pending(self.h)

    def now_ms(self):
        return self.ctx.lib.vcl_server_now_ms(self.h)

    def status(self, jid):
        st, it = ctypes.c_int(), ctypes.c_int()
        sub, adm, done = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._c(self.ctx.lib.vcl_server_job_status(self.h, jid, ctypes.byref(st), ctypes.byref(it), ctypes.byref(sub),
                                                   ctypes.byref(adm), ctypes.byref(done)), "vcl_server_job_status")
        return dict(state=st.value, iters=it.value, submit_ms=sub.value, admit_ms=adm.value, done_ms=done.value)

    def result(self, jid):
        import numpy as np
        S = self.scenes[jid]
        pos = np.zeros((S.nv, 3), np.float32)
        tex = np.zeros((S.tex_h, S.tex_w, S.C), np.float32)
        ax = np.zeros((S.K, 3), np.float32); sh = np.zeros(S.K, np.float32); am = np.zeros((S.K, S.C), np.float32)
        loss = ctypes.c_float()
        self._c(self.ctx.lib.vcl_server_job_result(self.h, jid, pos.ctypes.data, tex.ctypes.data, ax.ctypes.data,
                                                   sh.ctypes.data, am.ctypes.data, ctypes.byref(loss)),
                "vcl_server_job_result")
        return pos, tex, (ax, sh, am), loss.value

    def stats(self):
        p50, p99 = ctypes.c_double(), ctypes.c_double()
        iters, ticks = c_ll(), c_ll()
        comp = ctypes.c_int()
        res = c_size()
        self._c(self.ctx.lib.vcl_server_stats(self.h, ctypes.byref(p50), ctypes.byref(p99), ctypes.byref(iters),
                                              ctypes.byref(comp), ctypes.byref(ticks), ctypes.byref(res)),
                "vcl_server_stats")
        return dict(p50_ms=p50.value, p99_ms=p99.value, iterations=iters.value, completed=comp.value,
                    ticks=ticks.value, resident_bytes=res.value)

    def host_stats(self):
        h, w, r = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        n = c_ll()
        self._c(self.ctx.lib.vcl_server_host_stats(self.h, ctypes.byref(h), ctypes.byref(w), ctypes.byref(n),
                                                   ctypes.byref(r)), "vcl_server_host_stats")
        return dict(host_ms=h.value, wait_ms=w.value, rebuilds=n.value, rebuild_ms=r.value)

    def close(self):
        if self.h:
            self.ctx.lib.vcl_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ assets
class _Loader:
    """Runs loader calls (no device needed) and raises with their message."""

    def __init__(self, ctx):
        self.lib = lib()
        self.h = ctx.h if ctx is not None else None

    def check(self, st, name):
        if st:
            msg = self.lib.vcl_asset_error()
            raise VclError(f"{name} failed (status {st}): {msg.decode() if msg else ''}")

    def close(self):
        pass


def load_obj(path, ctx=None):
    """OBJ mesh: dict with the file's arrays (pos, pos_idx, texel, texel_idx,
    normal, normal_idx; absent attributes None) and the welded arrays
    (w_pos, w_uv, w_normal, w_tri) with one shared index."""
    import numpy as np
    ld = _Loader(ctx)
    L = ld.lib
    try:
        o = c_void_p()
        ld.check(L.vcl_obj_load(ld.h, str(path).encode(), ctypes.byref(o)), "vcl_obj_load")
        cnt = [ctypes.c_int() for _ in range(5)]
        L.vcl_obj_counts(o, *[ctypes.byref(c) for c in cnt])
        npos, ntri, ntex, nnrm, nw = [c.value for c in cnt]
        ptr = [c_void_p() for _ in range(6)]
        L.vcl_obj_arrays(o, *[ctypes.byref(p) for p in ptr])
        wp = [c_void_p() for _ in range(4)]
        L.vcl_obj_welded(o, *[ctypes.byref(p) for p in wp])

        def arr(p, n, cols, dt):
            if not p.value or n == 0:
                return None
            ct = ctypes.c_float if dt == np.float32 else ctypes.c_uint32
            return np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ct)), shape=(n, cols)).copy()

        out = dict(pos=arr(ptr[0], npos, 3, np.float32), pos_idx=arr(ptr[1], ntri, 3, np.uint32),
                   texel=arr(ptr[2], ntex, 2, np.float32), texel_idx=arr(ptr[3], ntri if ntex else 0, 3, np.uint32),
                   normal=arr(ptr[4], nnrm, 3, np.float32), normal_idx=arr(ptr[5], ntri if nnrm else 0, 3, np.uint32),
                   w_pos=arr(wp[0], nw, 3, np.float32), w_uv=arr(wp[1], nw, 2, np.float32),
                   w_normal=arr(wp[2], nw, 3, np.float32), w_tri=arr(wp[3], ntri, 3, np.uint32))
        L.vcl_obj_free(o)
        return out
    finally:
        ld.close()


def load_bmp(path, ctx=None):
    """BMP image as float32 [height][width][channels] in [0, 1], rows bottom-up."""
    import numpy as np
    ld = _Loader(ctx)
    L = ld.lib
    try:
        w, h, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ld.check(L.vcl_bmp_load(ld.h, str(path).encode(), ctypes.byref(w), ctypes.byref(h), ctypes.byref(c), None),
                 "vcl_bmp_load")
        out = np.zeros((h.value, w.value, c.value), np.float32)
        ld.check(L.vcl_bmp_load(ld.h, str(path).encode(), ctypes.byref(w), ctypes.byref(h), ctypes.byref(c),
                                out.ctypes.data), "vcl_bmp_load")
        return out
    finally:
        ld.close()


def load_sg(path, ctx=None):
    """Lobe list: (axis [K][3], sharpness [K], amplitude [K][3])."""
    import numpy as np
    ld = _Loader(ctx)
    L = ld.lib
    try:
        k = ctypes.c_int()
        ld.check(L.vcl_sg_load(ld.h, str(path).encode(), 0, ctypes.byref(k), None, None, None), "vcl_sg_load")
        K = k.value
        ax, sh, am = np.zeros((K, 3), np.float32), np.zeros(K, np.float32), np.zeros((K, 3), np.float32)
        ld.check(L.vcl_sg_load(ld.h, str(path).encode(), K, ctypes.byref(k), ax.ctypes.data, sh.ctypes.data,
                               am.ctypes.data), "vcl_sg_load")
        return ax, sh, am
    finally:
        ld.close()
