"""Generates tests/golden/ref_host_vectors.npz from the REFERENCE's own
host-callable code (oracle/_ref/libref.so, built by oracle/ref.mk from the
reference sources).  Inputs are seeded; outputs are what the reference code
returns.  Run here (needs the reference tree only at build time):

    make -C oracle -f ref.mk && python tests/golden/gen_ref_vectors.py
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref.so")
fp = C.POINTER(C.c_float)


def P(a):
    return a.ctypes.data_as(fp)


def main():
    L = C.CDLL(LIB)
    L.ref_ray_parallelogram.restype = C.c_int
    L.ref_max_less_index.restype = C.c_int
    L.ref_heap_trimmed.restype = C.c_float
    L.ref_heap_trimmed.argtypes = [fp, C.c_int, C.c_float]
    L.ref_angle2xyz.argtypes = [C.c_float, C.c_float, fp]
    L.ref_buie_table.argtypes = [C.c_float, fp, fp, fp, fp]
    L.ref_max_less_index.argtypes = [fp, fp, C.c_float]
    rng = np.random.default_rng(20261203)
    out = {}

    # local2world (global_function.cuh:14-52)
    d = rng.normal(size=(300, 3)).astype(np.float32)
    n = rng.normal(size=(300, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    n[:5] = [[0, 1, 0], [0, -1, 0], [1e-7, 1, 0], [0.3, 0.0, 0.954], [-1, 0, 0]]
    n = n.astype(np.float32)
    r = np.zeros_like(d)
    for i in range(len(d)):
        L.ref_local2world(P(d[i]), P(n[i]), P(r[i]))
    out.update(l2w_d=d, l2w_n=n, l2w_out=r)

    # rayParallelogramIntersect (global_function.cuh:78-105)
    m = 2000
    A = rng.uniform(-5, 5, (m, 3)).astype(np.float32)
    B = (A + rng.uniform(-3, 3, (m, 3))).astype(np.float32)
    Cc = (A + rng.uniform(-3, 3, (m, 3))).astype(np.float32)
    tgt = A + rng.uniform(-0.3, 1.3, (m, 1)) * (B - A) + rng.uniform(-0.3, 1.3, (m, 1)) * (Cc - A)
    o = (tgt + rng.normal(0, 6, (m, 3))).astype(np.float32)
    dr = (tgt - o) * rng.choice([1.0, -1.0], (m, 1), p=[0.85, 0.15])
    dr = (dr / np.linalg.norm(dr, axis=1, keepdims=True)).astype(np.float32)
    hit = np.zeros(m, np.int32)
    tuv = np.zeros((m, 3), np.float32)
    for i in range(m):
        hit[i] = L.ref_ray_parallelogram(P(o[i]), P(dr[i]), P(A[i]), P(B[i]), P(Cc[i]), P(tuv[i]))
    out.update(rp_o=o, rp_d=dr, rp_A=A, rp_B=B, rp_C=Cc, rp_hit=hit, rp_tuv=tuv)

    # angle2xyz (global_function.cuh:175-180)
    ang = np.stack([rng.uniform(-0.02, 0.02, 200), rng.uniform(0, 2 * np.pi, 200)], 1).astype(np.float32)
    a2x = np.zeros((200, 3), np.float32)
    for i in range(200):
        L.ref_angle2xyz(C.c_float(ang[i, 0]), C.c_float(ang[i, 1]), P(a2x[i]))
    out.update(a2x_in=ang, a2x_out=a2x)

    # rotateY (global_function.cuh:61-74) for the receiver faces' normals
    ro = rng.uniform(-3, 3, (100, 3)).astype(np.float32)
    ra = np.array([[0, 0, 1], [1, 0, 0], [0, 0, -1], [-1, 0, 0]] * 25, np.float32)
    th = rng.uniform(0, 2 * np.pi, 100)
    rb = np.stack([np.sin(th), np.zeros(100), np.cos(th)], 1).astype(np.float32)
    rr = np.zeros_like(ro)
    for i in range(100):
        L.ref_rotate_y(P(ro[i]), P(ra[i]), P(rb[i]), P(rr[i]))
    out.update(roty_o=ro, roty_a=ra, roty_b=rb, roty_out=rr)

    # Buie tables (set_samplelights / parameters_generate) and max_less_index
    for csr in (0.05, 0.1, 0.2, 0.3):
        x = np.zeros(1025, np.float32)
        y = np.zeros(1025, np.float32)
        s = np.zeros(1024, np.float32)
        p = np.zeros(6, np.float32)
        L.ref_buie_table(C.c_float(csr), P(x), P(y), P(s), P(p))
        key = "buie_%03d" % int(round(csr * 100))
        out.update({key + "_x": x, key + "_y": y, key + "_slope": s, key + "_params": p})
        if csr == 0.1:
            vals = np.concatenate([rng.uniform(0, y[-1], 500), y[[0, 1, 7, 512, 1023, 1024]]]).astype(np.float32)
            idx = np.array([L.ref_max_less_index(P(x), P(y), C.c_float(v)) for v in vals], np.int32)
            out.update(mli_values=vals, mli_index=idx)

    # the heap trimmed mean over windows (heap.cuh, image_smooth.cu:22-57)
    wins, cnts, ratios, res = [], [], [], []
    for i in range(400):
        side = int(rng.choice([3, 5, 7, 9, 11]))
        cnt = side * int(rng.choice([side, side - 1, (side + 1) // 2]))
        w = rng.integers(0, 40, cnt).astype(np.float32)
        if i % 3 == 0:
            w = rng.uniform(0, 100, cnt).astype(np.float32)
        if i % 7 == 0:
            w[:] = np.round(w / 20)
        ratio = float(rng.choice([0.02, 0.05, 0.1, 0.2, 0.3]))
        buf = np.zeros(121, np.float32)
        buf[:cnt] = w
        wins.append(buf)
        cnts.append(cnt)
        ratios.append(ratio)
        res.append(L.ref_heap_trimmed(P(buf), cnt, C.c_float(ratio)))
    out.update(heap_win=np.array(wins), heap_cnt=np.array(cnts, np.int32), heap_ratio=np.array(ratios, np.float32),
               heap_out=np.array(res, np.float32))

    # RectangleHelio::CRotate (heliostat.cpp:16-58): given normals and aimed
    hp = rng.uniform(-200, 200, (60, 3)).astype(np.float32)
    hp[:, 1] = rng.uniform(1, 8, 60)
    hs = np.stack([rng.uniform(1, 11, 60), rng.uniform(0, 0.2, 60), rng.uniform(1, 11, 60)], 1).astype(np.float32)
    hn = rng.normal(size=(60, 3))
    hn[:, 1] = np.abs(hn[:, 1]) + 0.2
    hn = hn.astype(np.float32)
    focus = np.array([0, 80, 0], np.float32)
    sun = np.array([0.1, -0.7, -0.6], np.float32)
    v_given = np.zeros((60, 12), np.float32)
    v_aimed = np.zeros((60, 12), np.float32)
    n_given = np.zeros((60, 3), np.float32)
    n_aimed = np.zeros((60, 3), np.float32)
    for i in range(60):
        L.ref_helio_vertices(P(hp[i]), P(hs[i]), P(hn[i]), None, None, P(v_given[i]), P(n_given[i]))
        L.ref_helio_vertices(P(hp[i]), P(hs[i]), None, P(focus), P(sun), P(v_aimed[i]), P(n_aimed[i]))
    out.update(helio_pos=hp, helio_size=hs, helio_normal_in=hn, helio_v_given=v_given, helio_n_given=n_given,
               helio_focus=focus, helio_sun=sun, helio_v_aimed=v_aimed, helio_n_aimed=n_aimed)

    # ImageSaver::savetxt (image_save.cpp:5-48): the flux file at two
    # precisions and the intercept-ratio file, each appended twice to a fresh
    # file (the reference opens with ios::app)
    import tempfile
    fmap = rng.uniform(0, 9e5, (9, 13)).astype(np.float32)
    fmap[rng.random((9, 13)) < 0.3] = 0
    fmap[0, :4] = [1e-7, 9.9e-7, 1e-6, 1.00001e-6]
    fmap[1, :3] = [-3.5, 0.125, 2.5]
    fmap[2, :3] = [123456.789, 0.004999, 0.005]
    L.ref_save_flux_txt.argtypes = [C.c_char_p, C.c_int, C.c_int, fp, C.c_int]
    L.ref_save_ratio_txt.argtypes = [C.c_char_p, C.c_int, C.c_int, fp, C.c_float]
    total = float(np.float32(fmap[fmap >= 1e-6].astype(np.float64).sum() * 1.37))
    with tempfile.TemporaryDirectory() as td:
        for key, call in (("save_flux_p2", lambda p: L.ref_save_flux_txt(p, 13, 9, P(fmap), 2)),
                          ("save_flux_p4", lambda p: L.ref_save_flux_txt(p, 13, 9, P(fmap), 4)),
                          ("save_ratio", lambda p: L.ref_save_ratio_txt(p, 13, 9, P(fmap), C.c_float(total)))):
            path = os.path.join(td, key + ".txt")
            call(path.encode())
            call(path.encode())
            out[key] = np.frombuffer(open(path, "rb").read(), np.uint8)
    out.update(save_map=fmap, save_total=np.float32(total))
    np.savez_compressed(os.path.join(HERE, "ref_host_vectors.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
