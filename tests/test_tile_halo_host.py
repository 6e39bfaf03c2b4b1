"""Host-side checks of the tensor-core mixed stage's tiles and halos (no GPU).

dgk_tile_halo cuts each partition into tiles of consecutive elements and lists, per tile, the faces whose
neighbour lies outside it (the halo the kernel gathers into shared memory).  The test restates the kernel's
shared-memory slot in numpy: the tile's own values at the slot's start, halo face j's values at
halo_floats + j Nfp in the face's point order; every face trace read through the tile-local connectivity
(position | code << 16, the identity row for halo faces) must equal the gather map's values bit for bit.
Layouts: padded partitions, partitions that are not multiples of the tile, halo limits that force short
tiles, and a shuffled element order.
"""
import numpy as np
import pytest

from dgkernel_b200 import mesh as M
from dgkernel_b200._lib import DGKError
from oracle import burgers_ref as b

from test_mixed_host import _gmap_padded, _layout


def _setup(N, n, nslab):
    prob = b.Problem(N, n, nslab, "sine")
    el = prob.el
    node_off, total = _layout(prob.Kpart, el.Np, 64)
    gmap, face_off = _gmap_padded(prob, node_off, 32)
    conn, table = M.compact_faces(prob.Kpart, node_off, face_off, el.Np, el.Nfp, gmap)
    return prob, el, node_off, total, gmap, face_off, conn, table


def _check(prob, el, node_off, total, gmap, face_off, conn, table, max_elems, max_halo, seed=0):
    Np, Nfp = el.Np, el.Nfp
    hf = max_elems * Np + 40  # halo values start past the tile's own values (any such position works)
    th = M.tile_halo(prob.Kpart, node_off, Np, Nfp, conn, max_elems=max_elems, max_halo=max_halo, halo_floats=hf,
                     identity_code=len(table))
    ident = np.concatenate([table, np.arange(Nfp, dtype=np.uint8)[None, :]])
    u = np.random.default_rng(seed).standard_normal(total)
    slots = np.cumsum([0] + [(k + 31) // 32 * 32 for k in prob.Kpart])
    covered = [np.zeros(k, dtype=bool) for k in prob.Kpart]
    NF = 4 * Nfp
    for t in range(len(th["nelem"])):
        p, s0, ne = int(th["part"][t]), int(th["first"][t]), int(th["nelem"][t])
        assert 1 <= ne <= max_elems and s0 % 4 == 0
        assert not covered[p][s0:s0 + ne].any()
        covered[p][s0:s0 + ne] = True
        h0, h1 = int(th["halo_off"][t]), int(th["halo_off"][t + 1])
        assert (h1 - h0) % 2 == 0 and h1 - h0 <= max_halo
        slot = np.full(hf + max_halo * Nfp, np.nan)
        base = node_off[p] + s0 * Np
        slot[:ne * Np] = u[base:base + ne * Np]
        for j, (nb, code) in enumerate(th["halo_list"][h0:h1]):
            slot[hf + j * Nfp:hf + (j + 1) * Nfp] = u[nb + table[code].astype(np.int64)]
        nhalo = 0
        for e in range(ne):
            words = th["tconn"][slots[p] + s0 + e].astype(np.int64)
            for f in range(4):
                off, code = int(words[f] & 0xFFFF), int((words[f] >> 16) & 0xFF)
                nhalo += off >= hf
                got = slot[off + ident[code].astype(np.int64)]
                want = u[gmap[face_off[p] + (s0 + e) * NF + f * Nfp:face_off[p] + (s0 + e) * NF + (f + 1) * Nfp]]
                assert np.array_equal(got, want), (t, e, f)
        assert nhalo <= h1 - h0 <= nhalo + 1  # one repeated entry pads an odd count
    assert all(c.all() for c in covered)
    return th


@pytest.mark.parametrize("N,n,nslab", [(1, 6, 3), (2, 6, 2), (3, 4, 4), (4, 6, 2)])
def test_tile_traces_reproduce_gather_map(N, n, nslab):
    args = _setup(N, n, nslab)
    th = _check(*args, max_elems=128, max_halo=256)
    prob = args[0]
    # with room for every halo the tiles are the plain 128-element cuts
    for p, k in enumerate(prob.Kpart):
        sizes = th["nelem"][th["part"] == p]
        assert list(sizes) == [min(128, k - s) for s in range(0, k, 128)]


def test_short_tiles_when_the_halo_limit_binds():
    args = _setup(2, 6, 2)
    th = _check(*args, max_elems=128, max_halo=40)
    assert th["nelem"].max() < 128  # the limit cut the tiles short
    assert np.diff(th["halo_off"]).max() <= 40


def test_shuffled_element_order():
    # a face matching computed on a shuffled element order: the halos are large and the tiles short
    prob, el, node_off, total, gmap, face_off, conn, table = _setup(3, 4, 1)
    rng = np.random.default_rng(3)
    K, Np, NF = prob.Kpart[0], el.Np, 4 * el.Nfp
    perm = rng.permutation(K)  # new element i is old element perm[i]
    inv = np.argsort(perm)
    g_old = gmap[:K * NF].astype(np.int64).reshape(K, NF)[perm]
    e_old, node = g_old // Np, g_old % Np
    g_new = (inv[e_old] * Np + node).astype(np.int32).reshape(-1)
    conn2, table2 = M.compact_faces([K], node_off[:1], face_off[:1], Np, el.Nfp, g_new)
    th = _check(prob, el, node_off, total, g_new, face_off, conn2, table2, max_elems=128, max_halo=256, seed=5)
    assert th["nelem"].max() < 128


def test_bad_limits_are_refused():
    prob, el, node_off, total, gmap, face_off, conn, table = _setup(2, 4, 2)
    with pytest.raises(DGKError):  # odd halo capacity
        M.tile_halo(prob.Kpart, node_off, el.Np, el.Nfp, conn, max_halo=255)
    with pytest.raises(DGKError):  # halo positions overlapping the tile's own values
        M.tile_halo(prob.Kpart, node_off, el.Np, el.Nfp, conn, halo_floats=10)
    with pytest.raises(DGKError):  # positions past 16 bits
        M.tile_halo(prob.Kpart, node_off, el.Np, el.Nfp, conn, halo_floats=65000)
