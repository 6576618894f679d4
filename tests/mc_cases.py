"""Independent restatement of the marching-cubes case table (test side).

Derives the 256 cases from cube geometry in numpy, without sharing code with
the library's C generator, so the two can be checked against each other:
faces are found from corner coordinates and ordered counter-clockwise seen
from outside; each maximal run of inside corners around a face is cut off by
one directed segment (leave edge -> enter edge); segments chain into loops;
a loop is started at its smallest edge and fanned, hexagons split into the
alternate-vertex triangle plus three ears.

Corner / edge numbering is the reference's (MarchingCubes.cu:264-285).
"""
import numpy as np

CORNERS = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
EDGES = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]
_EID = {}
for _e, (_a, _b) in enumerate(EDGES):
    _EID[(_a, _b)] = _EID[(_b, _a)] = _e


def _faces():
    out = []
    for axis in range(3):
        for side in (0, 1):
            cs = [c for c in range(8) if CORNERS[c][axis] == side]
            ctr = np.mean([CORNERS[c] for c in cs], axis=0)
            nrm = np.zeros(3)
            nrm[axis] = 1.0 if side else -1.0
            u = np.zeros(3)
            u[(axis + 1) % 3] = 1.0
            v = np.cross(nrm, u)

            def ang(c):
                d = np.array(CORNERS[c], float) - ctr
                return np.arctan2(d @ v, d @ u)

            cs.sort(key=ang)
            p = [np.array(CORNERS[c], float) for c in cs]
            assert np.cross(p[1] - p[0], p[3] - p[0]) @ nrm > 0
            out.append(cs)
    return out


FACES = _faces()


def edge_mask(c: int) -> int:
    return sum(1 << e for e, (a, b) in enumerate(EDGES) if ((c >> a) & 1) != ((c >> b) & 1))


def loops(c: int):
    nxt = {}
    for cyc in FACES:
        ins = [(c >> k) & 1 for k in cyc]
        if sum(ins) in (0, 4):
            continue
        for i in range(4):
            if ins[i] and not ins[i - 1]:
                j = i
                while ins[(j + 1) % 4]:
                    j = (j + 1) % 4
                enter = _EID[(cyc[i - 1], cyc[i])]
                leave = _EID[(cyc[j], cyc[(j + 1) % 4])]
                assert leave not in nxt
                nxt[leave] = enter
    out, seen = [], set()
    for s in sorted(nxt):
        if s in seen:
            continue
        lp = [s]
        seen.add(s)
        while nxt[lp[-1]] != s:
            lp.append(nxt[lp[-1]])
            seen.add(lp[-1])
        out.append(lp)
    return out


def triangles(c: int):
    tris = []
    for lp in loops(c):
        if len(lp) == 6:
            tris += [(lp[0], lp[1], lp[2]), (lp[2], lp[3], lp[4]), (lp[4], lp[5], lp[0]), (lp[0], lp[2], lp[4])]
        else:
            tris += [(lp[0], lp[i], lp[i + 1]) for i in range(1, len(lp) - 1)]
    return tris


def generated_table() -> np.ndarray:
    """(256, 16) uint8: triangle edge indices, count in column 15, 0xFF unused."""
    t = np.full((256, 16), 0xFF, np.uint8)
    for c in range(256):
        tr = triangles(c)
        assert len(tr) <= 5
        flat = [e for tri in tr for e in tri]
        t[c, :len(flat)] = flat
        t[c, 15] = len(tr)
    return t


def boundary(tris):
    """Directed triangle edges whose reverse is absent: the segments on the
    cube faces, with their orientation."""
    d = set()
    for t in tris:
        for i in range(3):
            d.add((t[i], t[(i + 1) % 3]))
    return {e for e in d if (e[1], e[0]) not in d}
