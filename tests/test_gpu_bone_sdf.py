"""Bone SDF collider on the GPU against the oracle (bit-exact expected).

* The GPU bake (bake_bone_sdf_gpu) against the oracle's sequential bake of
  the same bone-local triangles, which this file prepares in numpy following
  sdf_baker.rs:494-700 (layout, padded AABBs, triangle lists, normals).
* The dynamic path (skinning, triangle preparation, rebake of all bones, then
  of dirty bones only) against the oracle's restatement of the same kernels.
* Cloth colliding with the baked atlas (static and posed) against the oracle.

The reference pins none of these (no fixture holds atlas values), so this row
is parity unpinned against the reference; against the oracle the stated
tolerance is 1e-5 of the cloth extent and the measured result is bit-exact.
"""
import numpy as np
import pytest

from gpu_common import extent
from oracle import oracle as O
from taremincloth_b200 import ClothSimulator, scenes
from taremincloth_b200.simulator import bake_bone_sdf_gpu

pytestmark = pytest.mark.gpu
F = np.float32


def _tp(M, p):
    """Row-major transform with the projective divide (float32, sdf_baker.rs:167-177)."""
    M = M.astype(F)
    x = ((M[0, 0] * p[:, 0] + M[0, 1] * p[:, 1]) + M[0, 2] * p[:, 2]) + M[0, 3]
    y = ((M[1, 0] * p[:, 0] + M[1, 1] * p[:, 1]) + M[1, 2] * p[:, 2]) + M[1, 3]
    z = ((M[2, 0] * p[:, 0] + M[2, 1] * p[:, 1]) + M[2, 2] * p[:, 2]) + M[2, 3]
    w = ((M[3, 0] * p[:, 0] + M[3, 1] * p[:, 1]) + M[3, 2] * p[:, 2]) + M[3, 3]
    div = (np.abs(w) > F(1e-7)) & (np.abs(w - F(1)) > F(1e-5))
    iw = np.where(div, F(1) / np.where(div, w, F(1)), F(1))
    return np.stack([np.where(div, x * iw, x), np.where(div, y * iw, y), np.where(div, z * iw, z)], 1).astype(F)


def _normal(p0, p1, p2):
    a, b = (p1 - p0).astype(F), (p2 - p0).astype(F)
    c = np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1], a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                  a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], 1).astype(F)
    l2 = (c[:, 0] * c[:, 0] + c[:, 1] * c[:, 1]) + c[:, 2] * c[:, 2]
    ok = l2 > F(1e-12)
    inv = F(1) / np.sqrt(np.where(ok, l2, F(1)))
    n = (c * inv[:, None]).astype(F)
    n[~ok] = [0, 1, 0]
    return n


def _open_edges(tris, nv):
    from collections import Counter
    cnt = Counter()
    for t in tris:
        i0, i1, i2 = (int(x) for x in t)
        if min(i0, i1, i2) < 0 or max(i0, i1, i2) >= nv or i0 == i1 or i1 == i2 or i2 == i0:
            continue
        for u, v in ((i0, i1), (i1, i2), (i2, i0)):
            cnt[(min(u, v), max(u, v))] += 1
    return {k for k, c in cnt.items() if c == 1}


def _prepare_bake(verts, tris, W, bind, res_req, margin=0.2, thr=0.02, thickness=0.005):
    """numpy restatement of the host part of bake_bone_sdf_gpu (closed meshes)."""
    active = [b for b in range(W.shape[0]) if float(W[b].max(initial=0.0)) > thr]
    n = len(active)
    ncols = max(int(np.ceil(n ** (1.0 / 3.0))), 1)
    nrows = max(int(np.ceil(np.sqrt(-(-n // ncols)))), 1)
    nlay = max(-(-n // (ncols * nrows)), 1)
    mt = max(ncols, nrows, nlay)
    res = max(2048 // mt, 16) if mt * res_req > 2048 else res_req
    dims = (ncols * res, nrows * res, nlay * res)
    open_e = _open_edges(tris, len(verts))
    params, all_tris = [], []
    for ob, b in enumerate(active):
        M = bind[b]
        sel = W[b] > F(thr)
        if sel.any():
            pl = _tp(M, verts[sel])
            mn, mx = pl.min(0), pl.max(0)
        else:
            mn, mx = np.full(3, -0.1, F), np.full(3, 0.1, F)
        mn, mx = mn.astype(F).copy(), mx.astype(F).copy()
        size = np.maximum(mx - mn, F(0.05)).astype(F)
        pad = (size * F(margin) + F(max(thickness, 0.0))).astype(F)
        mn, mx = (mn - pad).astype(F), (mx + pad).astype(F)
        l, rem = divmod(ob, ncols * nrows)
        r, c = divmod(rem, ncols)
        start = len(all_tris)
        w = W[b][tris]
        has = (w > 0).any(1)
        p0, p1, p2 = (_tp(M, verts[tris[:, k]]) for k in range(3))
        tmin = np.minimum(np.minimum(p0, p1), p2)
        tmax = np.maximum(np.maximum(p0, p1), p2)
        ov = has & (tmin <= mx).all(1) & (tmax >= mn).all(1)
        nrm = _normal(p0, p1, p2)
        for t in np.nonzero(ov)[0]:
            i0, i1, i2 = (int(x) for x in tris[t])
            bm = (1 if (min(i0, i1), max(i0, i1)) in open_e else 0) | \
                 (2 if (min(i1, i2), max(i1, i2)) in open_e else 0) | \
                 (4 if (min(i2, i0), max(i2, i0)) in open_e else 0)
            all_tris.append(np.r_[p0[t], w[t, 0], p1[t], w[t, 1], p2[t], w[t, 2], nrm[t], F(bm)].astype(F))
        params.append(O.bake_params_words(mn, start, mx, len(all_tris) - start, c, r, l, res, *dims))
    return active, dims, np.asarray(params), np.asarray(all_tris, F).reshape(-1, 16)


@pytest.fixture(scope="module")
def small_body():
    return scenes.mannequin(body_vertices=4000, seed=3)


def test_static_bake_matches_oracle(small_body):
    b = small_body
    bake = bake_bone_sdf_gpu(b["verts"], b["tris"], b["names"], list(b["weights"]), b["bind_inv"], resolution=16)
    active, dims, params, tris = _prepare_bake(b["verts"], b["tris"], b["weights"], b["bind_inv"], 16)
    assert (bake["width"], bake["height"], bake["depth"]) == dims
    assert bake["active_bones"] == [b["names"][i] for i in active]
    tex = np.frombuffer(bake["texture_bytes"], np.uint32)
    ref = O.bone_bake(params, tris, dims)
    assert np.array_equal(tex, ref), int((tex != ref).sum())
    # the atlas holds real distances: inside a capsule negative, far away positive
    dist = (tex & 0xFFFF).astype(np.uint16).view(np.float16).astype(np.float32)
    assert dist.min() < 0.0 < dist.max()


def _dyn_sim(body, bake, order):
    sc = dict(positions=np.zeros((3, 3), F), edges=np.array([[0, 1], [1, 2]], np.uint32),
              faces=np.array([[0, 1, 2]], np.uint32))
    s = ClothSimulator(np.array([[5.0, 5.0, 5.0], [5.1, 5.0, 5.0], [5.0, 5.0, 5.1]], F), sc["edges"], sc["faces"])
    s.set_gravity(0.0, 0.0, 0.0)
    src, tw = scenes.bone_tri_sources(body, bake)
    W = body["weights"][order]
    top = np.argsort(-W, axis=0)[:4].T
    bw = np.take_along_axis(W.T, top, axis=1).astype(F)
    res = int(bake["bone_infos"][0][7])
    s.setup_dynamic_bone_sdf(bake["width"], bake["height"], bake["depth"], res, bake["bone_infos"], body["verts"],
                             top.astype(np.uint32), bw, src, tw, body["bind_inv"][order])
    return s, src, tw, top.astype(np.uint32), bw, res


def _oracle_rebake(body, bake, order, src, tw, top, bw, res, world, inv, bones=None, prev=None):
    skin = O.bone_skin_mats(world, body["bind_inv"][order])
    skinned = O.bone_skin(body["verts"], top, bw, skin)
    from taremincloth_b200.simulator import ClothSimulator as _C  # noqa: F401
    srcw = np.zeros((len(src), 4), F)
    srcw[:, :3] = tw  # closed meshes: no open-boundary bits
    tris = O.bone_prep(skinned, inv.reshape(-1, 16), src, srcw)
    nb = len(order)
    dims = (bake["width"], bake["height"], bake["depth"])
    ncols, nrows = max(dims[0] // res, 1), max(dims[1] // res, 1)
    starts = {}
    for i, bb in enumerate(src[:, 3]):
        starts.setdefault(int(bb), [i, 0])[1] += 1
    params = []
    for bb in (range(nb) if bones is None else bones):
        l, rem = divmod(bb, ncols * nrows)
        r, c = divmod(rem, ncols)
        info = bake["bone_infos"][bb]
        st, cnt = starts.get(bb, [0, 0])
        params.append(O.bake_params_words(info[0:3], st, info[4:7], cnt, c, r, l, res, *dims))
    out = np.zeros(dims[0] * dims[1] * dims[2], np.uint32) if prev is None else prev.copy()
    new = O.bone_bake(np.asarray(params), tris, dims)
    if prev is None:
        return new
    # a partial rebake overwrites only the listed bones' tiles
    mask = np.zeros(len(out), bool)
    W, H = dims[0], dims[1]
    for bb in bones:
        l, rem = divmod(bb, ncols * nrows)
        r, c = divmod(rem, ncols)
        z, y, x = np.meshgrid(np.arange(l * res, l * res + res), np.arange(r * res, r * res + res),
                              np.arange(c * res, c * res + res), indexing="ij")
        mask[((z * H + y) * W + x).ravel()] = True
    out[mask] = new[mask]
    return out


def test_dynamic_rebake_matches_oracle(small_body):
    body = small_body
    bake = bake_bone_sdf_gpu(body["verts"], body["tris"], body["names"], list(body["weights"]), body["bind_inv"],
                             resolution=16)
    order = [body["names"].index(n) for n in bake["active_bones"]]
    s, src, tw, top, bw, res = _dyn_sim(body, bake, order)
    world, inv = scenes.shader_mats(scenes.pose(body, 17)[order])
    s.update_bone_transforms(world, inv)
    s.step(1.0 / 60.0, 1)
    _, tex = s.get_bone_sdf_atlas()
    ref = _oracle_rebake(body, bake, order, src, tw, top, bw, res, world, inv)
    assert np.array_equal(tex, ref), int((tex != ref).sum())
    # world bounding spheres in the infos' .w slots (mod.rs:1889-1931)
    infos = s.get_bone_infos()
    Mw = world.astype(np.float64)
    for bb in range(len(order)):
        mn, mx = infos[bb, 0:3].astype(np.float64), infos[bb, 4:7].astype(np.float64)
        cw = (Mw[bb][:3, :3].T @ ((mn + mx) / 2)) + Mw[bb][3, :3]
        assert np.allclose([infos[bb, 3], infos[bb, 7], infos[bb, 11]], cw, atol=1e-5)
    # dirty bones: [] keeps the atlas, [k] rebakes bone k's tile only
    world2, inv2 = scenes.shader_mats(scenes.pose(body, 40)[order])
    s.update_bone_transforms(world2, inv2, dirty_bone_indices=[])
    s.step(1.0 / 60.0, 1)
    assert np.array_equal(s.get_bone_sdf_atlas()[1], tex)
    k = 7 if len(order) > 7 else 0
    s.update_bone_transforms(world2, inv2, dirty_bone_indices=[k])
    s.step(1.0 / 60.0, 1)
    ref2 = _oracle_rebake(body, bake, order, src, tw, top, bw, res, world2, inv2, bones=[k], prev=tex)
    got2 = s.get_bone_sdf_atlas()[1]
    assert np.array_equal(got2, ref2), int((got2 != ref2).sum())
    assert not np.array_equal(got2, tex)


@pytest.mark.parametrize("frame", [0, 25])
def test_cloth_on_bone_sdf_matches_oracle(small_body, frame):
    body = small_body
    bake = bake_bone_sdf_gpu(body["verts"], body["tris"], body["names"], list(body["weights"]), body["bind_inv"],
                             resolution=24)
    order = [body["names"].index(n) for n in bake["active_bones"]]
    # a 24 x 24 sheet, 0.4 m, 5 cm above the left upper arm and forearm
    pos, edges, faces, _ = scenes.tri_grid(24, 0.4, 1.50, 0)
    pos = pos.astype(F)
    pos[:, 0] += F(0.2)
    pos[:, 2] -= F(0.2)
    inv_m = scenes.areal_inv_masses(pos, faces, 0.15)
    tex = np.frombuffer(bake["texture_bytes"], np.uint32)
    dims = (bake["width"], bake["height"], bake["depth"])
    sims = []
    for cls in (ClothSimulator, O.OracleSim):
        s = cls(pos, edges, faces, inv_m, thickness=0.004)
        s.set_gravity(0.0, -9.81, 0.0)
        s.set_solver_iterations(3)
        sims.append(s)
    g, o = sims
    g.set_bone_sdf_colliders(dims[0], dims[1], dims[2], bake["texture_bytes"], bake["bone_infos"])
    world, inv = scenes.shader_mats(scenes.pose(body, frame)[order])
    g.update_bone_transforms(world, inv)
    infos = g.get_bone_infos()
    xf = np.zeros((len(order), 32), F)
    xf[:, :16] = world.reshape(-1, 16)
    xf[:, 16:] = inv.reshape(-1, 16)
    o.set_bone_sdf(dims, tex, infos, xf)
    ext = extent(pos)
    for _ in range(12):
        g.step(1.0 / 60.0, 10)
        o.step(1.0 / 60.0, 10)
        xg, _, _ = g.get_state()
        xo, _, _ = o.get_state()
        assert float(np.abs(xg - xo).max()) <= 1e-5 * ext
    assert np.array_equal(xg, xo)
    if frame == 0:  # arm horizontal at rest: part of the sheet lies on it
        assert int((xg[:, 1] > 1.44).sum()) > 20, "the cloth never met the bone SDF"


def _grid_box(n, lo, hi):
    """Closed box [lo, hi] with every face split into an n x n grid of quads
    (two triangles each), vertices shared along the edges."""
    lo, hi = np.asarray(lo, F), np.asarray(hi, F)
    verts, index, tris = [], {}, []

    def vid(p):
        key = tuple(np.round(p, 7))
        if key not in index:
            index[key] = len(verts)
            verts.append(p)
        return index[key]

    for ax in range(3):
        u, v = (ax + 1) % 3, (ax + 2) % 3
        for side in (0, 1):
            for i in range(n):
                for j in range(n):
                    c = []
                    for di, dj in ((0, 0), (1, 0), (1, 1), (0, 1)):
                        p = np.empty(3, F)
                        p[ax] = hi[ax] if side else lo[ax]
                        p[u] = lo[u] + (hi[u] - lo[u]) * F((i + di) / n)
                        p[v] = lo[v] + (hi[v] - lo[v]) * F((j + dj) / n)
                        c.append(vid(p))
                    a, b, cc, d = c
                    tris += [[a, b, cc], [a, cc, d]] if side else [[a, cc, b], [a, d, cc]]
    return np.asarray(verts, F), np.asarray(tris, np.int32)


def _slab(ncol, length=0.1, width=0.002, height=0.01):
    """Closed thin slab along x whose long faces are strips of ncol quads in x
    order: for a voxel above a face the squared distances of successive
    triangles fall by steps far below the tie tolerance's scale."""
    xs = np.linspace(0.0, length, ncol + 1).astype(F)
    corners = [(0.0, 0.0), (width, 0.0), (width, height), (0.0, height)]  # (y, z) around the section
    verts = np.asarray([[x, y, z] for x in xs for (y, z) in corners], F)
    tris = []
    for i in range(ncol):
        for k in range(4):
            a, b = 4 * i + k, 4 * i + (k + 1) % 4
            c, d = a + 4, b + 4
            tris += [[a, b, d], [a, d, c]]
    last = 4 * ncol
    tris += [[0, 2, 1], [0, 3, 2], [last, last + 1, last + 2], [last, last + 2, last + 3]]
    return verts, np.asarray(tris, np.int32)


def _single_bone_bake(verts, tris, res):
    W = np.ones((1, len(verts)), F)
    bind = np.eye(4, dtype=F)[None]
    bake = bake_bone_sdf_gpu(verts, tris, ["b"], list(W), bind, resolution=res)
    _, dims, params, btris = _prepare_bake(verts, tris, W, bind, res)
    tex = np.frombuffer(bake["texture_bytes"], np.uint32)
    return tex, O.bone_bake(params, btris, dims)


@pytest.mark.parametrize("shuffle", [False, True])
def test_bake_many_ties_matches_oracle(shuffle):
    """Grid faces give many exactly equal distances (shared vertices and edges),
    decided by the |projection| tie rule; a shuffled triangle order changes
    which triangle wins, and the GPU must follow the order."""
    verts, tris = _grid_box(10, (-0.05, -0.03, -0.02), (0.05, 0.03, 0.02))
    if shuffle:
        tris = tris[np.random.default_rng(5).permutation(len(tris))]
    tex, ref = _single_bone_bake(verts, tris, 24)
    assert np.array_equal(tex, ref), int((tex != ref).sum())


def test_bake_slowly_descending_order_matches_oracle():
    """Triangles ordered along the slab, so that above a face the distances
    descend in steps well inside the tie tolerance's window: these voxels take
    the kernel's full sequential scan."""
    verts, tris = _slab(1000)
    tex, ref = _single_bone_bake(verts, tris, 20)
    assert np.array_equal(tex, ref), int((tex != ref).sum())


def test_static_bake_default_resolution_matches_oracle(small_body):
    b = small_body
    bake = bake_bone_sdf_gpu(b["verts"], b["tris"], b["names"], list(b["weights"]), b["bind_inv"], resolution=40)
    _, dims, params, tris = _prepare_bake(b["verts"], b["tris"], b["weights"], b["bind_inv"], 40)
    tex = np.frombuffer(bake["texture_bytes"], np.uint32)
    ref = O.bone_bake(params, tris, dims)
    assert np.array_equal(tex, ref), int((tex != ref).sum())
