"""Synthetic heliostat-field workloads with the shapes the tracer is measured on.

No public dataset is involved: every field is generated by the library's
radial-staggered layout generator from a fixed seed.  Sizes:

  small  100 heliostats 2x2 m, tower 80 m, flat 5x5 m receiver at 128x128,
         sun 45 deg elevation / 180 deg azimuth, CSR 0.1, slope 2 mrad,
         16 Poisson points (0.3 m spacing) x 256 rays, 10 m cells.
  mid    1000 heliostats 10x10 m out to 600 m, tower 150 m, flat 12x12 m
         receiver at 256x256, aim offsets N(0, 0.5 m), sun 30 deg, CSR 0.05,
         slope 2.5 mrad, 2^28 rays, 25 m cells.
  large  10000 heliostats 11x11 m surround field out to 1300 m, tower 200 m,
         cylinder R 8 m x H 18 m unrolled to 512x256, sun 20 deg, CSR 0.2,
         slope 3 mrad, 2^31 rays, two-level grid of 50 m coarse / 12.5 m
         fine cells.
"""
import ctypes as C
from dataclasses import dataclass, field as dfield

import numpy as np

from . import capi

FIELD_SEED = 20261203


@dataclass
class Workload:
    name: str
    pos: np.ndarray
    size: np.ndarray
    sigma: float
    receiver: capi.Receiver
    grid: capi.GridParams
    sun: capi.Sun
    params: capi.TraceParams
    aim: np.ndarray = None
    smooth_radius: int = 2
    smooth_ratio: float = 0.2
    extra: dict = dfield(default_factory=dict)

    @property
    def n(self):
        return self.pos.shape[0]

    @property
    def res(self):
        return (self.receiver.res_y, self.receiver.res_x)

    def field_struct(self):
        """ctypes Field pointing into this workload's arrays (keep self alive)."""
        f = capi.Field()
        f.n = self.n
        f.pos = capi.as_fp(self.pos)
        f.size = capi.as_fp(self.size)
        f.aim = capi.as_fp(self.aim) if self.aim is not None else None
        f.normal = None
        f.slope_sigma = None
        f.sigma = self.sigma
        f.tilt = None
        return f


def layout(n, w, h, r_min, r_max, az_center=0.0, az_span=120.0, spacing=0.0, jitter=0.0, mount=None, seed=FIELD_SEED):
    p = capi.LayoutParams()
    p.n = n
    p.helio_w, p.helio_h = w, h
    p.thickness = 0.05
    p.r_min, p.r_max = r_min, r_max
    p.az_center_deg, p.az_span_deg = az_center, az_span
    p.spacing = spacing
    p.jitter = jitter
    p.mount_height = mount if mount is not None else 0.5 * h + 0.5
    p.seed = seed
    pos = np.zeros((n, 3), np.float32)
    got = C.c_int32()
    capi.check(capi.lib().qmcrt_layout_radial_staggered(C.byref(p), capi.as_fp(pos), n, C.byref(got)))
    return pos


def paraboloid_facets(a, b, normal, centre, rows=3, cols=3, facet=2 ** 0.5 / 3, gap=0.1, thickness=0.1,
                      reference_frame=False):
    """Facets of one paraboloid heliostat (qmcrt_layout_paraboloid_facets):
    pos, size and unit normals [rows*cols, 3]; the defaults are the
    reference's own 3 x 3 heliostat."""
    p = capi.FacetParams()
    p.a, p.b = a, b
    p.normal[:] = list(normal)
    p.centre[:] = list(centre)
    p.rows, p.cols, p.facet, p.gap, p.thickness = rows, cols, facet, gap, thickness
    p.reference_frame = 1 if reference_frame else 0
    n = rows * cols
    pos, size, nrm = (np.zeros((n, 3), np.float32) for _ in range(3))
    got = C.c_int32()
    capi.check(capi.lib().qmcrt_layout_paraboloid_facets(C.byref(p), capi.as_fp(pos), capi.as_fp(size),
                                                         capi.as_fp(nrm), n, C.byref(got)))
    return pos, size, nrm


def sun_dir(elev, azim):
    d = (C.c_float * 3)()
    capi.check(capi.lib().qmcrt_sun_direction(elev, azim, d))
    return [d[0], d[1], d[2]]


def make_sun(elev, azim, dni=1000.0, csr=0.1):
    s = capi.Sun()
    s.dir[:] = sun_dir(elev, azim)
    s.dni = dni
    s.csr = csr
    return s


def flat_receiver(tower, w, h, res_x, res_y, normal=(0.0, 0.0, -1.0)):
    r = capi.Receiver()
    r.type = capi.RECEIVER_FLAT
    r.pos[:] = [0.0, tower, 0.0]
    r.size[:] = [w, h, 0.0]
    r.normal[:] = list(normal)
    r.face = 0
    r.res_x, r.res_y = res_x, res_y
    return r


def cylinder_receiver(tower, radius, height, res_x, res_y):
    r = capi.Receiver()
    r.type = capi.RECEIVER_CYLINDER
    r.pos[:] = [0.0, tower - height / 2.0, 0.0]
    r.size[:] = [radius, height, 0.0]
    r.normal[:] = [0.0, 0.0, -1.0]
    r.face = 0
    r.res_x, r.res_y = res_x, res_y
    return r


def grid(cell, margin=1.0, fine_div=1):
    """Grid of `cell` m cells; fine_div > 1 makes `cell` the coarse cell of a
    two-level grid whose fine cells are cell / fine_div."""
    g = capi.GridParams()
    g.cell[:] = [cell, cell, cell]
    g.margin = margin
    g.explicit_bounds = 0
    g.fine_div = fine_div
    return g


def params(rays, rpp, spacing, seed=7, quirks=0, mode=capi.POINTS_POISSON):
    p = capi.TraceParams()
    p.seed = seed
    p.rays = rays
    p.rays_per_point = rpp
    p.point_mode = mode
    p.point_spacing = spacing
    p.reflectivity = 0.88
    p.quirks = quirks
    p.deposit = capi.DEPOSIT_NEAREST
    p.accumulate = 0
    p.kernel_variant = 0
    return p


def small(rays=None, seed=7):
    """100 heliostats, 16 points x 256 rays (409 600 rays)."""
    n = 100
    pos = layout(n, 2.0, 2.0, 40.0, 200.0, spacing=3.4, jitter=0.2, mount=1.6)
    size = np.tile(np.array([[2.0, 0.05, 2.0]], np.float32), (n, 1))
    rays = rays or n * 16 * 256
    return Workload("small", pos, size, 0.002, flat_receiver(80.0, 5.0, 5.0, 128, 128), grid(10.0),
                    make_sun(45.0, 180.0, 1000.0, 0.1), params(rays, 256, 0.3, seed))


def mid(rays=1 << 28, seed=7):
    """1000 heliostats 10x10 m to 600 m, 2^28 rays."""
    n = 1000
    pos = layout(n, 10.0, 10.0, 100.0, 600.0, jitter=0.0, mount=6.0)
    size = np.tile(np.array([[10.0, 0.1, 10.0]], np.float32), (n, 1))
    rec = flat_receiver(150.0, 12.0, 12.0, 256, 256)
    rng = np.random.default_rng(FIELD_SEED + 1)
    off = rng.normal(0.0, 0.5, (n, 2)).astype(np.float32)
    # receiver plane basis: width along x, height along y (normal -z)
    aim = np.zeros((n, 3), np.float32)
    aim[:, 0] = off[:, 0]
    aim[:, 1] = 150.0 + off[:, 1]
    aim[:, 2] = 0.0
    w = Workload("mid", pos, size, 0.0025, rec, grid(25.0), make_sun(30.0, 180.0, 1000.0, 0.05),
                 params(rays, 256, 0.18, seed), aim=aim)
    return w


def large(rays=1 << 31, seed=7):
    """10 000 heliostats 11x11 m surround field to 1300 m, cylinder receiver, 2^31 rays."""
    n = 10000
    pos = layout(n, 11.0, 11.0, 120.0, 1300.0, az_center=0.0, az_span=360.0, mount=6.5)
    size = np.tile(np.array([[11.0, 0.1, 11.0]], np.float32), (n, 1))
    rec = cylinder_receiver(200.0, 8.0, 18.0, 512, 256)
    return Workload("large", pos, size, 0.003, rec, grid(50.0, fine_div=4), make_sun(20.0, 180.0, 1000.0, 0.2),
                    params(rays, 256, 0.22, seed))


def equinox_suns(latitude=37.0, step_min=15.0, min_elevation=5.0, dni=1000.0, csr=0.1):
    """Sun positions over one equinox day (declination 0) every step_min
    minutes of solar time, keeping elevations >= min_elevation."""
    out = []
    L = capi.lib()
    el, az = C.c_float(), C.c_float()
    for k in range(int(24 * 60 / step_min)):
        hour = k * step_min / 60.0
        capi.check(L.qmcrt_solar_position(latitude, 0.0, 15.0 * (hour - 12.0), C.byref(el), C.byref(az)))
        if el.value >= min_elevation:
            out.append((hour, el.value, az.value, make_sun(el.value, az.value, dni, csr)))
    return out


def batched(rays_per_item=1 << 24, seed=11):
    """Three fields of 300, 1000 and 4000 heliostats (10x10 m, flat 12x12 m
    receivers at 256x256 on 150 m towers) over every sun position of an
    equinox day at 37 N (15-minute steps, elevation >= 5 deg)."""
    fields = []
    for n, rmax in ((300, 350.0), (1000, 600.0), (4000, 1100.0)):
        pos = layout(n, 10.0, 10.0, 100.0 if n > 300 else 80.0, rmax, mount=6.0, seed=FIELD_SEED + n)
        size = np.tile(np.array([[10.0, 0.1, 10.0]], np.float32), (n, 1))
        fields.append(Workload("batch_%d" % n, pos, size, 0.0025, flat_receiver(150.0, 12.0, 12.0, 256, 256),
                               grid(25.0), make_sun(45.0, 180.0), params(rays_per_item, 256, 0.4, seed)))
    suns = equinox_suns()
    items = [(f, s[3]) for f in range(len(fields)) for s in suns]
    return fields, suns, items, params(rays_per_item, 256, 0.4, seed)


def differentiable(n=2000, rays=1 << 26, seed=13):
    """2000 heliostats 10x10 m, flat 12x12 m receiver at 128x128 on a 150 m
    tower, sun at 40 deg; explicit aim points (the receiver centre) and zero
    tilts are the parameters; target: a uniform 800 kW/m^2 disk of radius 4 m
    whose centre is offset by a seeded N(0, 0.5 m) in the receiver plane."""
    pos = layout(n, 10.0, 10.0, 100.0, 800.0, mount=6.0, seed=FIELD_SEED + 7)
    size = np.tile(np.array([[10.0, 0.1, 10.0]], np.float32), (n, 1))
    rec = flat_receiver(150.0, 12.0, 12.0, 128, 128)
    aim = np.tile(np.array([[0.0, 150.0, 0.0]], np.float32), (n, 1))
    p = params(rays, 256, 0.5, seed)
    p.deposit = capi.DEPOSIT_BILINEAR
    w = Workload("differentiable", pos, size, 0.0025, rec, grid(25.0), make_sun(40.0, 180.0, 1000.0, 0.1), p, aim=aim)
    w.extra["tilt"] = np.zeros((n, 2), np.float32)
    w.extra["target"] = target_disk(rec, 800e3, 4.0, np.random.default_rng(FIELD_SEED + 9).normal(0, 0.5, 2))
    return w


def target_disk(rec, level, radius, centre_offset):
    """Target flux map [res_y, res_x]: `level` W/m^2 inside a disk of `radius` m
    centred at the receiver centre + centre_offset (width, height), 0 outside."""
    ny, nx = rec.res_y, rec.res_x
    # pixel centres in receiver-plane coordinates: column along the width, row along the height
    xs = (np.arange(nx) + 0.5) / nx * rec.size[0] - rec.size[0] / 2
    ys = (np.arange(ny) + 0.5) / ny * rec.size[1] - rec.size[1] / 2
    X, Y = np.meshgrid(xs, ys)
    inside = (X - centre_offset[0]) ** 2 + (Y - centre_offset[1]) ** 2 <= radius ** 2
    return np.where(inside, level, 0.0).astype(np.float32)


BUILDERS = {"small": small, "mid": mid, "large": large}
