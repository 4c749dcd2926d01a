"""Python host API over the C-ABI, mirroring the reference's scene/solver surface.

  SolarScene          -> SolarScene (solar_scene.h:19-50) + SceneProcessor
  SolarScene.trace    -> results_with_given_normal's tracing loop (Gtest.cu:10-46)
  SolarScene.trace_tables -> recthelio_ray_tracing / map_tracing on explicit
                          sample tables (recthelio_tracing.cpp:46-80)
  image_smooth        -> ImageSmoother::image_smooth (image_smooth.cuh:17-23)

Device memory comes from torch (plumbing only); every computation runs in
libqmcrt.so.  Errors raise capi.QmcrtError carrying the library's status.
"""
import ctypes as C

import numpy as np
import torch

from . import capi


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class SolarScene:
    def __init__(self, pos, size, receiver, grid, sigma=0.002, aim=None, normal=None, slope_sigma=None, tilt=None):
        self.pos = np.ascontiguousarray(pos, np.float32)
        self.size = np.ascontiguousarray(size, np.float32)
        self.aim = None if aim is None else np.ascontiguousarray(aim, np.float32)
        self.normal = None if normal is None else np.ascontiguousarray(normal, np.float32)
        self.slope_sigma = None if slope_sigma is None else np.ascontiguousarray(slope_sigma, np.float32)
        self.tilt = None if tilt is None else np.ascontiguousarray(tilt, np.float32)
        self.sigma = float(sigma)
        self.receiver = receiver
        self.grid = grid
        self.res = (receiver.res_y, receiver.res_x)
        h = C.c_void_p()
        capi.check(capi.lib().qmcrt_scene_create(C.byref(self.field()), C.byref(receiver), C.byref(grid), C.byref(h)))
        self.h = h

    @classmethod
    def from_workload(cls, w):
        return cls(w.pos, w.size, w.receiver, w.grid, sigma=w.sigma, aim=w.aim)

    @property
    def n(self):
        return self.pos.shape[0]

    def field(self):
        f = capi.Field()
        f.n = self.n
        f.pos = capi.as_fp(self.pos)
        f.size = capi.as_fp(self.size)
        f.aim = capi.as_fp(self.aim)
        f.normal = capi.as_fp(self.normal)
        f.slope_sigma = capi.as_fp(self.slope_sigma)
        f.sigma = self.sigma
        f.tilt = capi.as_fp(self.tilt)
        return f

    def close(self):
        if getattr(self, "h", None):
            capi.lib().qmcrt_scene_destroy(self.h)
            self.h = None

    def update_field(self):
        """Upload the (modified) host arrays pos/size/aim/normal/tilt/slope_sigma."""
        capi.check(capi.lib().qmcrt_scene_set_field(self.h, C.byref(self.field()), _stream()))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_sun(self, sun, quirks=0):
        capi.check(capi.lib().qmcrt_scene_set_sun(self.h, C.byref(sun), quirks, _stream()))

    def grid_info(self):
        gi = capi.GridInfo()
        capi.check(capi.lib().qmcrt_scene_grid_info(self.h, C.byref(gi)))
        return gi

    def read_grid(self):
        gi = self.grid_info()
        start = np.zeros(gi.cells + 1, np.int32)
        ent = np.zeros(max(gi.entries, 1), np.int32)
        capi.check(capi.lib().qmcrt_scene_read_grid(self.h, capi.as_i32p(start), capi.as_i32p(ent), _stream()))
        return start, ent[: start[-1]]

    def read_candidates(self, exhaustive=False):
        """Occluder candidates of the current sun: counts [n, 2] (shadow,
        block) and ids [n, 2, 32] (-1 past the count)."""
        counts = np.zeros((self.n, 2), np.int32)
        ids = np.zeros((self.n, 2, capi.CAND_CAP), np.int32)
        capi.check(capi.lib().qmcrt_scene_read_candidates(self.h, int(bool(exhaustive)), capi.as_i32p(counts),
                                                          capi.as_i32p(ids), _stream()))
        return counts, ids

    def read_geometry(self):
        nrm = np.zeros((self.n, 3))
        vert = np.zeros((self.n, 9))
        capi.check(capi.lib().qmcrt_scene_read_geometry(self.h, nrm.ctypes.data_as(capi.dp),
                                                        vert.ctypes.data_as(capi.dp), _stream()))
        return nrm, vert

    def sample_points(self, params):
        n = C.c_int64()
        capi.check(capi.lib().qmcrt_scene_sample_points(self.h, C.byref(params), C.byref(n), _stream()))
        return n.value

    def read_points(self):
        n = self.sample_points_count
        xz = np.zeros((n, 2), np.float32)
        helio = np.zeros(n, np.int32)
        capi.check(capi.lib().qmcrt_scene_read_points(self.h, capi.as_fp(xz), capi.as_i32p(helio), _stream()))
        return xz, helio

    def points(self, params):
        self.sample_points_count = self.sample_points(params)
        return self.read_points()

    def _outputs(self, rays, records, maps=True):
        dev = torch.device("cuda")
        r = {}
        o = capi.Outputs()
        if maps:
            r["counts"] = torch.zeros(self.res, dtype=torch.int32, device=dev)
            r["energy"] = torch.zeros(self.res, dtype=torch.float32, device=dev)
            r["flux"] = torch.zeros(self.res, dtype=torch.float32, device=dev)
            o.d_counts, o.d_energy, o.d_flux = (r[k].data_ptr() for k in ("counts", "energy", "flux"))
        if records:
            r["flags"] = torch.zeros(rays, dtype=torch.uint8, device=dev)
            r["pixel"] = torch.zeros(rays, dtype=torch.int32, device=dev)
            o.d_ray_flags, o.d_ray_pixel = r["flags"].data_ptr(), r["pixel"].data_ptr()
        return o, r

    def trace(self, sun, params, records=False, stats=True, outputs=None):
        """Full trace; returns device maps (and per-ray records) plus stats."""
        rays = int(params.rays)
        if params.point_mode == capi.POINTS_GRID:
            rays = self.sample_points(params) * params.rays_per_point
        self.sample_points_count = rays // params.rays_per_point
        if outputs is None:
            o, r = self._outputs(rays, records)
        else:
            o, r = outputs
        st = capi.TraceStats() if stats else None
        capi.check(capi.lib().qmcrt_trace(self.h, C.byref(sun), C.byref(params), C.byref(o),
                                          C.byref(st) if stats else None, _stream()))
        r["stats"] = st
        return r

    def trace_tables(self, sun, params, sun_local, turb_local, start, point_xz, point_helio, records=True,
                     stats=True):
        dev = torch.device("cuda")
        t = {k: torch.as_tensor(np.ascontiguousarray(v), device=dev)
             for k, v in (("sl", np.asarray(sun_local, np.float32)), ("tl", np.asarray(turb_local, np.float32)),
                          ("st", np.asarray(start, np.int32)), ("xz", np.asarray(point_xz, np.float32)),
                          ("ph", np.asarray(point_helio, np.int32)))}
        ti = capi.TableInputs()
        ti.d_sun_local, ti.d_turb_local = t["sl"].data_ptr(), t["tl"].data_ptr()
        ti.table_size = t["sl"].shape[0]
        ti.d_start, ti.d_point_xz, ti.d_point_helio = t["st"].data_ptr(), t["xz"].data_ptr(), t["ph"].data_ptr()
        ti.points = t["st"].shape[0]
        ti.rays_per_point = params.rays_per_point
        rays = ti.points * ti.rays_per_point
        o, r = self._outputs(rays, records)
        st = capi.TraceStats() if stats else None
        capi.check(capi.lib().qmcrt_trace_tables(self.h, C.byref(sun), C.byref(ti), C.byref(params), C.byref(o),
                                                 C.byref(st) if stats else None, _stream()))
        torch.cuda.current_stream().synchronize()
        r["stats"] = st
        return r

    def adjoint_forward(self, sun, params, target, state_bytes_max=0, want_loss=True, flux=True, tape=None):
        """Bilinear forward pass + loss against `target` (device [res] W/m^2).
        Returns (tape, loss or None, flux map or None); pass the tape of an
        earlier call back in to reuse its device buffers."""
        tape = C.c_void_p(tape.value if isinstance(tape, C.c_void_p) else tape)
        loss = C.c_double()
        fl = torch.zeros(self.res, dtype=torch.float32, device="cuda") if flux else None
        capi.check(capi.lib().qmcrt_adjoint_forward(self.h, C.byref(sun), C.byref(params), _ptr(target),
                                                    state_bytes_max, _ptr(fl), C.byref(loss) if want_loss else None,
                                                    C.byref(tape), _stream()))
        return tape, (loss.value if want_loss else None), fl

    def adjoint_backward(self, tape):
        ga = torch.empty((self.n, 2), dtype=torch.float32, device="cuda")
        gt = torch.empty((self.n, 2), dtype=torch.float32, device="cuda")
        capi.check(capi.lib().qmcrt_adjoint_backward(tape, _ptr(ga), _ptr(gt), _stream()))
        return ga, gt

    def adjoint_replay(self, tape, target, want_loss=True, flux=False):
        """The forward pass at the current aim points and tilts with the
        visibility recorded in `tape` (qmcrt_adjoint_replay).  Returns
        (loss or None, flux map or None)."""
        loss = C.c_double()
        fl = torch.zeros(self.res, dtype=torch.float32, device="cuda") if flux else None
        capi.check(capi.lib().qmcrt_adjoint_replay(tape, _ptr(target), _ptr(fl), C.byref(loss) if want_loss else None,
                                                   _stream()))
        return (loss.value if want_loss else None), fl

    def tape_energy(self, tape):
        """The tape's energy map (device float32 [res], a copy):
        qmcrt_tape_energy."""
        e = torch.empty(self.res, dtype=torch.float32, device="cuda")
        capi.check(capi.lib().qmcrt_tape_energy(tape, _ptr(e), _stream()))
        return e

    def adjoint_loss(self, tape, target, energy=None, want_loss=True, flux=False):
        """Flux, loss and adjoint map re-formed from `energy` (e.g. the sum of
        the ranks' energy maps; None: the tape's own): qmcrt_adjoint_loss.
        Returns (loss or None, flux map or None)."""
        loss = C.c_double()
        fl = torch.zeros(self.res, dtype=torch.float32, device="cuda") if flux else None
        capi.check(capi.lib().qmcrt_adjoint_loss(tape, _ptr(energy), _ptr(target), _ptr(fl),
                                                 C.byref(loss) if want_loss else None, _stream()))
        return (loss.value if want_loss else None), fl

    @staticmethod
    def tape_free(tape):
        capi.lib().qmcrt_tape_free(tape)

    def set_timing(self, stages):
        """Which stages later traces time (capi.TIMING_* bits; 0: none, the default)."""
        capi.check(capi.lib().qmcrt_scene_set_timing(self.h, stages))

    def timing(self):
        t = capi.Timing()
        capi.check(capi.lib().qmcrt_scene_timing(self.h, C.byref(t)))
        return t

    def trace_host(self, sun, params, stats=True):
        """End-to-end call on host buffers (uploads the field, downloads maps)."""
        counts = np.zeros(self.res, np.uint32)
        flux = np.zeros(self.res, np.float32)
        st = capi.TraceStats()
        capi.check(capi.lib().qmcrt_trace_host(self.h, C.byref(self.field()), C.byref(sun), C.byref(params),
                                               capi.as_u32p(counts), capi.as_fp(flux),
                                               C.byref(st) if stats else None, _stream()))
        return counts, flux, st


    def results_host(self, sun, params, radius=2, ratio=0.2, method=capi.TRIM_SORTED, source=capi.SMOOTH_COUNTS,
                     stats=False, upload=True, out=None):
        """One sun position end to end on host buffers (qmcrt_results_host,
        the work of results_with_given_normal, Gtest.cu:10-63): upload the
        field, trace, scale, smooth, download counts, flux and the smoothed
        map.  `out` may hold preallocated (pinned) host arrays."""
        if out is None:
            out = {"counts": np.zeros(self.res, np.uint32), "flux": np.zeros(self.res, np.float32),
                   "smoothed": np.zeros(self.res, np.float32)}
        sm = capi.SmoothParams(radius, ratio, method, source)
        st = capi.TraceStats() if stats else None
        capi.check(capi.lib().qmcrt_results_host(self.h, C.byref(self.field()) if upload else None, C.byref(sun),
                                                 C.byref(params), C.byref(sm), out["counts"].ctypes.data_as(capi.u32p),
                                                 capi.as_fp(out["flux"]), capi.as_fp(out["smoothed"]),
                                                 C.byref(st) if stats else None, _stream()))
        out["stats"] = st
        return out


class Batch:
    """Many (field, sun) items traced in one persistent launch (qmcrt_batch_*)."""

    def __init__(self, scenes, items, params):
        self.scenes = list(scenes)
        self.n_items = len(items)
        arr = (C.c_void_p * len(self.scenes))(*[s.h for s in self.scenes])
        its = (capi.BatchItem * len(items))()
        for k, (si, sun) in enumerate(items):
            its[k].scene = si
            its[k].sun = sun
        self.items = list(items)
        self.params = params
        h = C.c_void_p()
        capi.check(capi.lib().qmcrt_batch_create(arr, len(self.scenes), its, len(items), C.byref(params), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            capi.lib().qmcrt_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def autotune(self):
        t = capi.BatchTuning()
        capi.check(capi.lib().qmcrt_batch_autotune(self.h, C.byref(t), _stream()))
        return t

    def set_tuning(self, chunk_rays, ctas_per_sm, tile):
        t = capi.BatchTuning(chunk_rays, ctas_per_sm, tile, 0.0)
        capi.check(capi.lib().qmcrt_batch_set_tuning(self.h, C.byref(t)))

    def run(self):
        capi.check(capi.lib().qmcrt_batch_run(self.h, _stream()))

    def capture(self):
        capi.check(capi.lib().qmcrt_batch_capture(self.h))

    def launch(self):
        capi.check(capi.lib().qmcrt_batch_launch(self.h, _stream()))

    def read(self, i):
        sc = self.scenes[self.items[i][0]]
        counts = np.zeros(sc.res, np.uint32)
        flux = np.zeros(sc.res, np.float32)
        st = capi.TraceStats()
        capi.check(capi.lib().qmcrt_batch_read(self.h, i, capi.as_u32p(counts), capi.as_fp(flux), C.byref(st),
                                               _stream()))
        return counts, flux, st


def write_flux_csv(path, flux, precision=2, append=True):
    """Flux map [res_y, res_x] (host array or tensor) as the reference's text
    file (ImageSaver::savetxt, image_save.cpp:5-24)."""
    m = _host_map(flux)
    capi.check(capi.lib().qmcrt_write_flux_csv(str(path).encode(), capi.as_fp(m), m.shape[1], m.shape[0],
                                               precision, 1 if append else 0))


def write_intercept_ratio(path, flux, total_energy, append=True):
    """Sum of the flux map over total_energy, written as the reference's
    intercept-ratio line (image_save.cpp:26-48); returns the ratio.  path=None
    writes nothing."""
    m = _host_map(flux)
    r = C.c_float()
    capi.check(capi.lib().qmcrt_write_intercept_ratio(None if path is None else str(path).encode(), capi.as_fp(m),
                                                      m.shape[1], m.shape[0], C.c_float(total_energy),
                                                      1 if append else 0, C.byref(r)))
    return r.value


def _host_map(flux):
    if isinstance(flux, torch.Tensor):
        flux = flux.detach().cpu().numpy()
    m = np.ascontiguousarray(flux, np.float32)
    if m.ndim != 2:
        raise ValueError("map must be 2-D [rows, cols]")
    return m


def image_smooth(d_map, radius, ratio, method=capi.TRIM_SORTED):
    """Trimmed-mean smoothing of a device map (uint32/int32 counts or float32)."""
    assert d_map.is_cuda and d_map.is_contiguous() and d_map.dim() == 2
    out = torch.empty(d_map.shape, dtype=torch.float32, device=d_map.device)
    h, w = d_map.shape
    if d_map.dtype in (torch.int32, torch.uint32):
        f = capi.lib().qmcrt_smooth_trimmed_u32
    elif d_map.dtype == torch.float32:
        f = capi.lib().qmcrt_smooth_trimmed_f32
    else:
        raise TypeError("map must be int32/uint32 counts or float32")
    capi.check(f(_ptr(d_map), _ptr(out), w, h, radius, C.c_float(ratio), method, _stream()))
    return out
