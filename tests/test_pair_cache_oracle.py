"""The oracle's contact-pair cache (self-collision algorithm 1), on the CPU.

Pins the semantics the GPU parity tests rely on:
* the per-vertex top-K: with the broad phase at the first substep on the
  same positions, each vertex's quota-2 lists are the heads of its quota-8
  lists (distance, then key), and slot order is vertex-major;
* stored pairs are canonical: a V-T triangle starts at its smallest vertex
  with its winding kept, an E-E pair lists the far edge as (min, max), and no
  pair repeats;
* the reference's pinned-lower-layer test
  (crates/cloth_core/src/simulation/tests.rs:2061-2148) on the oracle.
"""
import numpy as np

from taremincloth_b200 import scenes


def _collect(oracle_lib, sc, max_pairs):
    o = scenes.build(oracle_lib.OracleSim, sc)
    o.set_pair_cache(True, False)
    o.set_pair_cache_options(max_pairs, max_pairs)
    o.step(sc["dt"], sc["substeps"])
    return o.active_pairs()


def _by_vertex(pairs):
    d = {}
    for p in pairs:
        d.setdefault(int(p[0]), []).append(tuple(int(x) for x in p[1:]))
    return d


def test_quota_lists_are_heads_of_larger_quota(oracle_lib):
    sc = scenes.config2(n=24, subdiv=2)
    n = len(sc["positions"])
    big = _collect(oracle_lib, sc, 8 * n)
    small = _collect(oracle_lib, sc, 2 * n)
    for k in (2, 3):
        b, s = _by_vertex(big[k]), _by_vertex(small[k])
        assert s and set(s) == set(b)
        for v, lst in s.items():
            assert len(lst) <= 2 and lst == b[v][:2], v
        # slot order is vertex-major
        ids = np.asarray(small[k])[:, 0]
        assert (np.diff(ids.astype(np.int64)) >= 0).all()
    # counts: accepted candidates >= stored pairs; drops only at the smaller quota
    assert big[0] >= len(big[2]) and big[1] >= len(big[3])


def test_stored_pairs_are_canonical_and_unique(oracle_lib):
    sc = scenes.config2(n=24, subdiv=2)
    vt_n, ee_n, vt, ee = _collect(oracle_lib, sc, 8 * len(sc["positions"]))
    assert len(vt) and len(ee)
    assert (vt[:, 1] < vt[:, 2]).all() and (vt[:, 1] < vt[:, 3]).all()
    assert (ee[:, 2] < ee[:, 3]).all()
    for arr in (vt, ee):
        assert len({tuple(r) for r in arr.tolist()}) == len(arr)
        assert all(len(set(r)) == 4 for r in arr.tolist())
    faces = {frozenset(f) for f in np.asarray(sc["faces"]).tolist()}
    assert all(frozenset(r[1:]) in faces for r in vt.tolist())
    edges = {tuple(sorted(e)) for e in np.asarray(sc["edges"]).tolist()}
    assert all(tuple(sorted(r[:2])) in edges and tuple(r[2:]) in edges for r in ee.tolist())


def test_pinned_lower_layer_pushes_upper_layer(oracle_lib):
    nx, ny, sp = 8, 7, 0.15
    per = nx * ny
    pos, edges, faces, layers, inv = [], [], [], [], []
    for layer in range(2):
        off = layer * per
        for iy in range(ny):
            for ix in range(nx):
                pos.append([ix * sp, iy * sp, 0.0 if layer == 0 else 0.005])
                layers.append(layer)
                inv.append(0.0 if layer == 0 else 1.0)
        for iy in range(ny):
            for ix in range(nx):
                v0 = off + iy * nx + ix
                if ix + 1 < nx:
                    edges.append([v0, v0 + 1])
                if iy + 1 < ny:
                    edges.append([v0, v0 + nx])
                if ix + 1 < nx and iy + 1 < ny:
                    edges.append([v0, v0 + nx + 1])
                    faces += [[v0, v0 + 1, v0 + nx + 1], [v0, v0 + nx + 1, v0 + nx]]
    o = oracle_lib.OracleSim(np.array(pos, np.float32), np.array(edges), np.array(faces),
                             inv_masses=np.array(inv, np.float32), layer_ids=np.array(layers, np.uint32),
                             thickness=0.04, stiffness=10000.0, compression_stiffness=10000.0,
                             shear_stiffness=5000.0, bending_stiffness=0.0)
    o.set_enable_self_collision(True)
    o.set_pair_cache(True, True)
    o.set_gravity(0.0, 0.0, 0.0)
    o.step(1.0 / 60.0, 4)
    x, _, _ = o.get_state()
    assert (x[per:, 2] > 0.02).sum() > per // 2
