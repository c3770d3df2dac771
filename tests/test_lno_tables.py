"""Host logic of the LNO orbit tiles (no GPU): the gather tables and the
de-duplication patterns the library builds on the host
(triples_lno_tables), checked against their definitions.

A candidate region c = 6 pi + rho of a tile holds the positions with occupied
triple (ijk[pi0], ijk[pi1], ijk[pi2]) and virtual sub-ranges (U[rho0],
U[rho1], U[rho2]); a slot (l0, l1, l2) indexes the position inside it.
  * sigma (simultaneous permutation of the orbit sums): the position
    (occ[s0], occ[s1], occ[s2]; vir[s0], vir[s1], vir[s2]);
  * r3 term s (forward): Z(j) gathers X(i) with i[s[k]] = j[k];
    adjoint: Xbar(i) gathers Zbar(j) with j[k] = i[s[k]];
  * pattern: candidates with equal (occupied triple, ranges) share a slab.
"""
import ctypes
import itertools

import numpy as np

from pyscfad_b200 import _lib

R3 = [(0, 1, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0), (0, 2, 1), (1, 0, 2)]


def perm_of(s):
    first = s >> 1
    lo = 1 if first == 0 else 0
    hi = 1 if first == 2 else 2
    return (first, hi if s & 1 else lo, lo if s & 1 else hi)


def pad(slot):
    return slot + 3 * (slot >> 4)


def _tables():
    lib = _lib.load()
    fn = lib.triples_lno_tables
    fn.restype = ctypes.c_size_t
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
    n = fn(None, 0)
    buf = (ctypes.c_ubyte * n)()
    assert fn(buf, n) == n
    b = np.frombuffer(bytes(buf), dtype=np.uint8)
    symsl = b[0:384].reshape(6, 64)
    r3sl = b[384:1152].reshape(2, 6, 64)
    symc = b[1152:1368].reshape(36, 6)
    r3c = b[1368:1800].reshape(2, 36, 6)
    pats = b[1808:1808 + 16 * 73].reshape(16, 73)
    return symsl, r3sl, symc, r3c, pats


def _key(c, occ, vr):
    pp, pr = perm_of(c // 6), perm_of(c % 6)
    return tuple(occ[pp[k]] for k in range(3)), tuple(vr[pr[k]] for k in range(3))


def test_perm_order_is_lexicographic():
    assert [perm_of(s) for s in range(6)] == sorted(itertools.permutations(range(3)))


def test_slot_maps():
    symsl, r3sl, _, _, _ = _tables()
    for sl in range(64):
        l = (sl // 16, (sl // 4) % 4, sl % 4)
        for s in range(6):
            ps = perm_of(s)
            t = (l[ps[0]], l[ps[1]], l[ps[2]])
            assert symsl[s][sl] == pad((t[0] * 4 + t[1]) * 4 + t[2])
            # forward r3: i[m] = j[sinv[m]]; adjoint: j[k] = i[s[k]]
            inv = [0] * 3
            for k in range(3):
                inv[R3[s][k]] = k
            f = (l[inv[0]], l[inv[1]], l[inv[2]])
            a = (l[R3[s][0]], l[R3[s][1]], l[R3[s][2]])
            assert r3sl[0][s][sl] == pad((f[0] * 4 + f[1]) * 4 + f[2])
            assert r3sl[1][s][sl] == pad((a[0] * 4 + a[1]) * 4 + a[2])


def test_candidate_maps_follow_the_keys():
    _, _, symc, r3c, _ = _tables()
    occ, vr = (7, 5, 2), (30, 20, 10)          # all distinct: every candidate is its own key
    for c in range(36):
        o3, v3 = _key(c, occ, vr)
        for s in range(6):
            ps = perm_of(s)
            assert _key(int(symc[c][s]), occ, vr) == (tuple(o3[ps[k]] for k in range(3)),
                                                      tuple(v3[ps[k]] for k in range(3)))
            inv = [0] * 3
            for k in range(3):
                inv[R3[s][k]] = k
            assert _key(int(r3c[0][c][s]), occ, vr) == (o3, tuple(v3[inv[k]] for k in range(3)))
            assert _key(int(r3c[1][c][s]), occ, vr) == (o3, tuple(v3[R3[s][k]] for k in range(3)))


def test_patterns_deduplicate_exactly():
    *_, pats = _tables()
    for pid in range(16):
        eo01, eo12, ev01, ev12 = (pid >> 3) & 1, (pid >> 2) & 1, (pid >> 1) & 1, pid & 1
        occ, vr = [2, 1, 0], [2, 1, 0]
        if eo12:
            occ[1] = occ[2]
        if eo01:
            occ[0] = occ[1]
        if ev12:
            vr[1] = vr[2]
        if ev01:
            vr[0] = vr[1]
        keys = [_key(c, occ, vr) for c in range(36)]
        nslab, cand, prim = int(pats[pid][0]), pats[pid][1:37], pats[pid][37:73]
        assert nslab == len(set(keys))
        assert len({keys[int(cand[g])] for g in range(nslab)}) == nslab
        for c in range(36):
            assert keys[int(cand[int(prim[c])])] == keys[c]
