"""Helpers that run the product's host-side topology builder (tc_mesh_*)."""
import ctypes as C

import numpy as np

from taremincloth_b200 import _lib

_f, _u = np.float32, np.uint32


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def host_build(positions, edges, faces=None, inv_masses=None, layer_ids=None, thicknesses=None, layer_id=0,
               thickness=0.005, stiffness=1000.0, bending_stiffness=10.0, compression_stiffness=None,
               shear_stiffness=None, sewing_springs=None, sewing_shrink_speed=1.0):
    L = _lib.load()
    pos = np.ascontiguousarray(positions, _f).reshape(-1, 3)
    e = np.ascontiguousarray(edges, _u).reshape(-1, 2)
    f = None if faces is None else np.ascontiguousarray(faces, _u).reshape(-1, 3)
    im = None if inv_masses is None else np.ascontiguousarray(inv_masses, _f)
    li = None if layer_ids is None else np.ascontiguousarray(layer_ids, _u)
    th = None if thicknesses is None else np.ascontiguousarray(thicknesses, _f)
    comp = stiffness if compression_stiffness is None else compression_stiffness
    shear = stiffness * 0.5 if shear_stiffness is None else shear_stiffness
    h = C.c_void_p()
    sew = None if sewing_springs is None else np.ascontiguousarray(sewing_springs, _u).reshape(-1, 2)
    _lib.check(L.tc_mesh_build_sewn(C.byref(h), _p(pos), pos.shape[0], _p(e), e.shape[0], _p(f),
                                    0 if f is None else f.shape[0], _p(im), _p(li), _p(th), layer_id, thickness,
                                    stiffness, comp, shear, bending_stiffness, _p(sew),
                                    0 if sew is None else sew.shape[0], sewing_shrink_speed, float("nan"), 1))
    try:
        c = np.zeros(10, _u)
        cell = C.c_float()
        _lib.check(L.tc_mesh_counts(h, _p(c), C.byref(cell)))
        n, nd, nb, ne, kd, kb = (int(x) for x in c[:6])
        out = dict(n=n, nd=nd, nb=nb, n_edges=ne, n_dist_colors=kd, n_bend_colors=kb, table_size=int(c[6]),
                   multi_layer=int(c[7]), num_virtual=int(c[8]), cell=cell.value)
        dv, dp = np.zeros((max(nd, 1), 2), _u), np.zeros((max(nd, 1), 4), _f)
        bv, bp = np.zeros((max(nb, 1), 4), _u), np.zeros((max(nb, 1), 4), _f)
        do, dc = np.zeros(max(kd, 1), _u), np.zeros(max(kd, 1), _u)
        bo, bc = np.zeros(max(kb, 1), _u), np.zeros(max(kb, 1), _u)
        _lib.check(L.tc_mesh_constraints(h, _p(dv), _p(dp), _p(do), _p(dc), _p(bv), _p(bp), _p(bo), _p(bc)))
        out.update(dist_v=dv[:nd], dist_par=dp[:nd], dist_off=do[:kd], dist_cnt=dc[:kd], bend_v=bv[:nb],
                   bend_par=bp[:nb], bend_off=bo[:kb], bend_cnt=bc[:kb])
        a, t, s = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _lib.check(L.tc_mesh_topology_sizes(h, C.byref(a), C.byref(t), C.byref(s)))
        topo = dict(adj_off=np.zeros(n + 1, _u), adj_idx=np.zeros(max(a.value, 1), _u), th_off=np.zeros(n + 1, _u),
                    th_idx=np.zeros(max(t.value, 1), _u), th_rest=np.zeros(max(t.value, 1), _f),
                    local_len=np.zeros(max(n, 1), _f), star_off=np.zeros(n + 1, _u),
                    star_idx=np.zeros((max(s.value, 1), 2), _u), island=np.zeros(max(n, 1), _u),
                    layer=np.zeros(max(n, 1), _u), edges=np.zeros((max(ne, 1), 2), _u),
                    edge_bits=np.zeros(max((ne + 31) // 32, 1), _u))
        _lib.check(L.tc_mesh_topology(h, *[_p(topo[k]) for k in ["adj_off", "adj_idx", "th_off", "th_idx", "th_rest",
                                                                   "local_len", "star_off", "star_idx", "island",
                                                                   "layer", "edges", "edge_bits"]]))
        topo["adj_idx"] = topo["adj_idx"][:a.value]
        topo["th_idx"] = topo["th_idx"][:t.value]
        topo["th_rest"] = topo["th_rest"][:t.value]
        topo["star_idx"] = topo["star_idx"][:s.value]
        topo["edges"] = topo["edges"][:ne]
        topo["edge_bits"] = topo["edge_bits"][:(ne + 31) // 32]
        out.update(topo)
        ns, nc = C.c_uint32(), C.c_uint32()
        _lib.check(L.tc_mesh_sewing(h, C.byref(ns), C.byref(nc), None, None, None, None, None))
        sv, sp = np.zeros((max(ns.value, 1), 2), _u), np.zeros((max(ns.value, 1), 5), _f)
        so, sc, rep = np.zeros(max(nc.value, 1), _u), np.zeros(max(nc.value, 1), _u), np.zeros(max(n, 1), _u)
        _lib.check(L.tc_mesh_sewing(h, None, None, _p(sv), _p(sp), _p(so), _p(sc), _p(rep)))
        out.update(sew_v=sv[:ns.value], sew_par=sp[:ns.value], sew_off=so[:nc.value], sew_cnt=sc[:nc.value],
                   sew_rep=rep[:n])
        return out
    finally:
        L.tc_mesh_destroy(h)
