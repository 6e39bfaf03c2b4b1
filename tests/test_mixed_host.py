"""Host-side checks of the mixed stage's compact face connectivity (no GPU).

The compact form replaces each face's Nfp gather indices by one neighbour base and a face-order code; the
test rebuilds every gather index from (base, table[code]) and requires bit-exact equality with the gather
map (the FaceConnector pick/place lists fused over partition offsets), on partitioned layouts with padding
between partitions and with partitions whose size is not a multiple of the 32-element slot.
"""
import numpy as np
import pytest

from dgkernel_b200 import mesh as M
from dgkernel_b200._lib import DGKError
from oracle import burgers_ref as b


def _layout(K, per, align):
    """Partition starts (npart + 1 entries, the last one the total) with each start aligned to `align` values."""
    off, o = [], 0
    for k in K:
        off.append(o)
        o = (o + k * per + align - 1) // align * align
    off.append(o)
    return np.array(off, dtype=np.int64), o


def _gmap_padded(prob, node_off, face_pad):
    el = prob.el
    NF = 4 * el.Nfp
    packed = M.face_gather_map(prob.K, 4, el.Nfp, el.Np, prob.vmapP, prob.EToP, node_off)
    face_off, total = _layout(prob.Kpart, NF, face_pad)
    g = np.full(total, -7, dtype=np.int32)
    o = 0
    for p, k in enumerate(prob.Kpart):
        g[face_off[p]:face_off[p] + k * NF] = packed[o:o + k * NF]
        o += k * NF
    return g, face_off


def _rebuild(conn, table, Kpart, NF, Nfp):
    out, s0 = [], 0
    for k in Kpart:
        c = conn[s0:s0 + k]
        codes = np.stack([(c[:, 4].astype(np.int64) >> (8 * f)) & 0xFF for f in range(4)], axis=1)
        idx = c[:, :4, None].astype(np.int64) + table[codes].astype(np.int64)  # [k, 4, Nfp]
        out.append(idx.reshape(-1))
        s0 += (k + 31) // 32 * 32
    return out


@pytest.mark.parametrize("N,n,nslab", [(2, 4, 2), (3, 5, 5), (4, 4, 4), (1, 6, 3)])
def test_compact_faces_reproduce_gather_map(N, n, nslab):
    prob = b.Problem(N, n, nslab, "sine")
    el = prob.el
    node_off, _ = _layout(prob.Kpart, el.Np, 64)
    gmap, face_off = _gmap_padded(prob, node_off, 32)
    conn, table = M.compact_faces(prob.Kpart, node_off, face_off, el.Np, el.Nfp, gmap)
    assert table.shape[0] <= 24  # 4 faces x 6 orientations of a triangle
    assert conn.shape[0] == sum((k + 31) // 32 * 32 for k in prob.Kpart)
    NF = 4 * el.Nfp
    got = _rebuild(conn, table, prob.Kpart, NF, el.Nfp)
    for p, k in enumerate(prob.Kpart):
        want = gmap[face_off[p]:face_off[p] + k * NF].astype(np.int64)
        assert np.array_equal(got[p], want)
    # every base is the first node of an element of the state layout
    bases = np.concatenate([conn[s:s + k, :4].reshape(-1) for s, k in
                            zip(np.cumsum([0] + [(k + 31) // 32 * 32 for k in prob.Kpart])[:-1], prob.Kpart)])
    part = np.searchsorted(node_off[:-1], bases, side="right") - 1
    assert np.all((bases - node_off[part]) % el.Np == 0)


def test_compact_faces_rejects_a_face_spanning_two_elements():
    prob = b.Problem(2, 4, 2, "sine")
    el = prob.el
    node_off, _ = _layout(prob.Kpart, el.Np, 64)
    gmap, face_off = _gmap_padded(prob, node_off, 32)
    bad = gmap.copy()
    bad[face_off[1] + 3] = bad[face_off[1] + 3] + el.Np  # one face point moved into the next element
    with pytest.raises(DGKError):
        M.compact_faces(prob.Kpart, node_off, face_off, el.Np, el.Nfp, bad)
    outside = gmap.copy()
    outside[face_off[0]] = 10 ** 8
    with pytest.raises(DGKError):
        M.compact_faces(prob.Kpart, node_off, face_off, el.Np, el.Nfp, outside)
