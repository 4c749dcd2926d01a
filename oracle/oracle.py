"""ctypes binding of the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker of the CUDA path.  Nothing in the
product package imports this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

fp = C.POINTER(C.c_float)
dp = C.POINTER(C.c_double)
i32p = C.POINTER(C.c_int32)
u32p = C.POINTER(C.c_uint32)
u8p = C.POINTER(C.c_uint8)


class OrcScene(C.Structure):
    _fields_ = [("n", C.c_int), ("pos", fp), ("size", fp), ("sigma", fp), ("normal", dp), ("frame", dp),
                ("vert", dp), ("recv_type", C.c_int), ("recv_v", C.c_double * 12), ("recv_focus", C.c_double * 3),
                ("res_x", C.c_int), ("res_y", C.c_int), ("cyl", C.c_double * 5), ("gpos", C.c_double * 3),
                ("gcell", C.c_double * 3), ("gdims", C.c_int * 3), ("cell_start", i32p), ("entries", i32p),
                ("fine_div", C.c_int)]


class OrcTraceCfg(C.Structure):
    _fields_ = [("sun_dir", C.c_double * 3), ("dni", C.c_double), ("rho", C.c_double), ("cdf_x", fp),
                ("cdf_y", fp), ("slope", fp), ("bparams", fp), ("seed", C.c_uint64), ("item", C.c_uint32),
                ("rays", C.c_int64), ("rays_per_point", C.c_int), ("point_xz", fp), ("point_helio", i32p),
                ("helio_weight", dp), ("quirks", C.c_uint32), ("threads", C.c_int), ("ray_begin", C.c_int64),
                ("ray_end", C.c_int64), ("deposit", C.c_int), ("atten", C.c_int)]


class OrcTraceOut(C.Structure):
    _fields_ = [("flags", u8p), ("pixel", i32p), ("counts", u32p), ("energy", dp), ("stats", C.c_uint64 * 7)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_philox4x32_10.argtypes = [u32p, u32p, u32p]
        L.orc_buie_table.argtypes = [C.c_float, fp, fp, fp, fp]
        L.orc_max_less_index.argtypes = [fp, C.c_double, C.c_int]
        L.orc_max_less_index.restype = C.c_int
        L.orc_buie_sample.argtypes = [C.c_double, fp, fp, fp, fp]
        L.orc_buie_sample.restype = C.c_double
        L.orc_local2world.argtypes = [dp, dp, C.c_uint32, dp]
        L.orc_scene_aim.argtypes = [C.POINTER(OrcScene), dp, fp, fp, fp, C.c_uint32]
        L.orc_receiver_flat.argtypes = [C.POINTER(OrcScene), fp, fp, fp, C.c_int, C.c_int, C.c_int]
        L.orc_receiver_cylinder.argtypes = [C.POINTER(OrcScene), fp, C.c_float, C.c_float, C.c_int, C.c_int]
        L.orc_grid_bounds.argtypes = [fp, fp, C.c_int, fp, C.c_float, dp, C.POINTER(C.c_int)]
        L.orc_grid_build.argtypes = [C.POINTER(OrcScene), C.c_uint32, i32p, i32p]
        L.orc_grid_build.restype = C.c_int64
        L.orc_ray_parallelogram.argtypes = [dp, dp, dp, dp, dp, dp, dp, dp]
        L.orc_ray_parallelogram.restype = C.c_int
        L.orc_dda_blocked.argtypes = [C.POINTER(OrcScene), dp, dp, C.c_int, C.c_uint32, C.POINTER(C.c_uint64)]
        L.orc_dda_blocked.restype = C.c_int
        L.orc_brute_blocked.argtypes = [C.POINTER(OrcScene), dp, dp, C.c_int, C.c_uint32]
        L.orc_brute_blocked.restype = C.c_int
        L.orc_receiver_hit.argtypes = [C.POINTER(OrcScene), dp, dp, C.c_uint32, i32p, dp]
        L.orc_receiver_hit.restype = C.c_int
        L.orc_points_poisson.argtypes = [fp, C.c_int, C.c_int64, C.c_float, C.c_uint64, fp, i32p]
        L.orc_points_poisson.restype = C.c_int
        L.orc_points_grid.argtypes = [fp, C.c_int, C.c_float, fp, i32p]
        L.orc_points_grid.restype = C.c_int64
        L.orc_trace_philox.argtypes = [C.POINTER(OrcScene), C.POINTER(OrcTraceCfg), C.POINTER(OrcTraceOut)]
        L.orc_trace_tables.argtypes = [C.POINTER(OrcScene), C.POINTER(OrcTraceCfg), fp, fp, C.c_int64, i32p,
                                       C.c_int64, C.POINTER(OrcTraceOut)]
        L.orc_ray_samples.argtypes = [C.POINTER(OrcTraceCfg), C.c_double, C.c_uint64, dp, dp]
        L.orc_adjoint.argtypes = [C.POINTER(OrcScene), C.POINTER(OrcTraceCfg), fp, fp, fp, dp, dp, dp, C.c_double,
                                  C.c_double, dp, dp, dp]
        L.orc_smooth_u32.argtypes = [u32p, fp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int]
        L.orc_smooth_f32.argtypes = [fp, fp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def philox(ctr, key):
    c = np.asarray(ctr, np.uint32)
    k = np.asarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    lib().orc_philox4x32_10(_p(c, u32p), _p(k, u32p), _p(o, u32p))
    return o


def buie_table(csr):
    x = np.zeros(1025, np.float32)
    y = np.zeros(1025, np.float32)
    s = np.zeros(1024, np.float32)
    p = np.zeros(6, np.float32)
    lib().orc_buie_table(C.c_float(csr), _p(x, fp), _p(y, fp), _p(s, fp), _p(p, fp))
    return x, y, s, p


def smooth_u32(img, radius, ratio, method):
    img = np.ascontiguousarray(img, np.uint32)
    out = np.zeros(img.shape, np.float32)
    lib().orc_smooth_u32(_p(img, u32p), _p(out, fp), img.shape[1], img.shape[0], radius, C.c_float(ratio), method)
    return out


def smooth_f32(img, radius, ratio, method):
    img = np.ascontiguousarray(img, np.float32)
    out = np.zeros(img.shape, np.float32)
    lib().orc_smooth_f32(_p(img, fp), _p(out, fp), img.shape[1], img.shape[0], radius, C.c_float(ratio), method)
    return out


def points_poisson(size, total_points, spacing, seed):
    size = np.ascontiguousarray(size, np.float32)
    xz = np.zeros((total_points, 2), np.float32)
    helio = np.zeros(total_points, np.int32)
    r = lib().orc_points_poisson(_p(size, fp), size.shape[0], total_points, C.c_float(spacing), seed, _p(xz, fp),
                                 _p(helio, i32p))
    if r != 0:
        raise RuntimeError("Poisson sampling failed for heliostat %d" % (-1 - r))
    return xz, helio


def points_grid(size, pl):
    size = np.ascontiguousarray(size, np.float32)
    n = lib().orc_points_grid(_p(size, fp), size.shape[0], C.c_float(pl), None, None)
    xz = np.zeros((n, 2), np.float32)
    helio = np.zeros(n, np.int32)
    lib().orc_points_grid(_p(size, fp), size.shape[0], C.c_float(pl), _p(xz, fp), _p(helio, i32p))
    return xz, helio


class Scene:
    """Oracle copy of a scene: geometry for one sun, grid CSR, receiver."""

    def __init__(self, pos, size, sigma, receiver, cell, margin, sun_dir, quirks=0, aim=None, normal=None,
                 tilt=None, grid_csr=None, grid_bounds=None):
        self.pos = np.ascontiguousarray(pos, np.float32)
        self.size = np.ascontiguousarray(size, np.float32)
        n = self.pos.shape[0]
        self.sigma = np.ascontiguousarray(np.broadcast_to(np.asarray(sigma, np.float32), (n,)))
        self.normal = np.zeros((n, 3))
        self.frame = np.zeros((n, 9))
        self.vert = np.zeros((n, 9))
        s = OrcScene()
        s.n = n
        s.pos, s.size, s.sigma = _p(self.pos, fp), _p(self.size, fp), _p(self.sigma, fp)
        s.normal, s.frame, s.vert = _p(self.normal, dp), _p(self.frame, dp), _p(self.vert, dp)
        L = lib()
        rpos = np.array(receiver.pos[:], np.float32)
        if receiver.type == 1:
            L.orc_receiver_cylinder(C.byref(s), _p(rpos, fp), C.c_float(receiver.size[0]), C.c_float(receiver.size[1]),
                                    receiver.res_x, receiver.res_y)
        else:
            rsize = np.array(receiver.size[:], np.float32)
            rn = np.array(receiver.normal[:], np.float32)
            L.orc_receiver_flat(C.byref(s), _p(rpos, fp), _p(rsize, fp), _p(rn, fp), receiver.face, receiver.res_x,
                                receiver.res_y)
        self.aim = None if aim is None else np.ascontiguousarray(aim, np.float32)
        self.normal_in = None if normal is None else np.ascontiguousarray(normal, np.float32)
        self.tilt = None if tilt is None else np.ascontiguousarray(tilt, np.float32)
        sd = (C.c_double * 3)(*sun_dir)
        L.orc_scene_aim(C.byref(s), sd, _p(self.aim, fp), _p(self.normal_in, fp), _p(self.tilt, fp), quirks)
        if grid_bounds is not None:
            gpos, gcell, gdims = grid_bounds
            s.gpos[:] = list(gpos)
            s.gcell[:] = list(gcell)
            s.gdims[:] = list(gdims)
        else:
            cellv = np.array([cell, cell, cell], np.float32)
            gd = (C.c_int * 3)()
            gp = (C.c_double * 3)()
            L.orc_grid_bounds(_p(self.pos, fp), _p(self.size, fp), n, _p(cellv, fp), C.c_float(margin), gp, gd)
            s.gpos[:] = gp[:]
            s.gcell[:] = [float(cellv[0])] * 3
            s.gdims[:] = gd[:]
        if grid_csr is not None:
            self.cell_start, self.entries = (np.ascontiguousarray(a, np.int32) for a in grid_csr)
        else:
            cnt = L.orc_grid_build(C.byref(s), quirks, None, None)
            cells = s.gdims[0] * s.gdims[1] * s.gdims[2]
            self.cell_start = np.zeros(cells + 1, np.int32)
            self.entries = np.zeros(max(cnt, 1), np.int32)
            L.orc_grid_build(C.byref(s), quirks, _p(self.cell_start, i32p), _p(self.entries, i32p))
        s.cell_start = _p(self.cell_start, i32p)
        s.entries = _p(self.entries, i32p)
        self.s = s
        self.quirks = quirks
        self.sun_dir = list(sun_dir)
        self.res = (receiver.res_y, receiver.res_x)

    def cfg(self, csr, seed, rays, rpp, point_xz, point_helio, weight=None, threads=0, ray_begin=0, ray_end=0,
            quirks=None, dni=1000.0, rho=0.88, item=0, atten=0):
        c = OrcTraceCfg()
        c.sun_dir[:] = self.sun_dir
        c.dni, c.rho = dni, rho
        self._tab = buie_table(csr)
        x, y, s, p = self._tab
        c.cdf_x, c.cdf_y, c.slope, c.bparams = _p(x, fp), _p(y, fp), _p(s, fp), _p(p, fp)
        c.seed = seed
        c.item = item
        c.rays = rays
        c.rays_per_point = rpp
        self._pxz = np.ascontiguousarray(point_xz, np.float32)
        self._ph = np.ascontiguousarray(point_helio, np.int32)
        c.point_xz, c.point_helio = _p(self._pxz, fp), _p(self._ph, i32p)
        self._w = None if weight is None else np.ascontiguousarray(weight, np.float64)
        c.helio_weight = _p(self._w, dp)
        c.quirks = self.quirks if quirks is None else quirks
        c.threads = threads
        c.ray_begin, c.ray_end = ray_begin, ray_end
        c.deposit = 0
        c.atten = atten
        return c

    def _out(self, nrec, records, maps):
        o = OrcTraceOut()
        res = self.res[0] * self.res[1]
        r = {}
        if records:
            r["flags"] = np.zeros(nrec, np.uint8)
            r["pixel"] = np.zeros(nrec, np.int32)
            o.flags, o.pixel = _p(r["flags"], u8p), _p(r["pixel"], i32p)
        if maps:
            r["counts"] = np.zeros(res, np.uint32)
            r["energy"] = np.zeros(res, np.float64)
            o.counts, o.energy = _p(r["counts"], u32p), _p(r["energy"], dp)
        return o, r

    def trace_philox(self, cfg, records=True, maps=True):
        end = cfg.ray_end if cfg.ray_end > 0 else cfg.rays
        o, r = self._out(end - cfg.ray_begin, records, maps)
        lib().orc_trace_philox(C.byref(self.s), C.byref(cfg), C.byref(o))
        r["stats"] = list(o.stats)
        return r

    def trace_tables(self, cfg, sun_local, turb_local, start, records=True, maps=True):
        end = cfg.ray_end if cfg.ray_end > 0 else cfg.rays
        o, r = self._out(end - cfg.ray_begin, records, maps)
        sl = np.ascontiguousarray(sun_local, np.float32)
        tl = np.ascontiguousarray(turb_local, np.float32)
        st = np.ascontiguousarray(start, np.int32)
        lib().orc_trace_tables(C.byref(self.s), C.byref(cfg), _p(sl, fp), _p(tl, fp), sl.shape[0], _p(st, i32p),
                               st.shape[0], C.byref(o))
        r["stats"] = list(o.stats)
        return r

    def adjoint(self, cfg, target, scale, fd_h=1e-7):
        """FP64 loss, bilinear energy map and per-heliostat gradients [n, 4]
        (aim along the receiver width, along its height, tilt u, tilt v)."""
        rv = np.array(self.s.recv_v[:]).reshape(4, 3)
        ew = rv[3] - rv[0]
        eh = rv[1] - rv[0]
        ew = np.ascontiguousarray(ew / np.linalg.norm(ew))
        eh = np.ascontiguousarray(eh / np.linalg.norm(eh))
        tgt = np.ascontiguousarray(target, np.float64).ravel()
        energy = np.zeros(self.res[0] * self.res[1])
        grad = np.zeros((self.s.n, 4))
        loss = C.c_double()
        lib().orc_adjoint(C.byref(self.s), C.byref(cfg), _p(self.aim, fp), _p(self.normal_in, fp), _p(self.tilt, fp),
                          _p(ew, dp), _p(eh, dp), _p(tgt, dp), scale, fd_h, _p(energy, dp), C.byref(loss),
                          _p(grad, dp))
        return loss.value, energy.reshape(self.res), grad

    def dda(self, o, d, own, brute=False):
        ov = (C.c_double * 3)(*o)
        dv = (C.c_double * 3)(*d)
        if brute:
            return lib().orc_brute_blocked(C.byref(self.s), ov, dv, own, self.quirks)
        ctr = (C.c_uint64 * 2)()
        return lib().orc_dda_blocked(C.byref(self.s), ov, dv, own, self.quirks, ctr)
