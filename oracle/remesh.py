"""The soup subdivision's checkers.  TEST INFRASTRUCTURE ONLY.

* `reference_split` runs the reference's own CPU remeshers
  (src/remesh.cpp, src/remesh_clip.cpp, compiled unmodified into
  oracle/_ref/libremesh_ref.so by oracle/Makefile, wrapper oracle/ref_remesh.cpp).
* `restated_split` restates them in numpy single precision (every operation
  rounded, no fused multiply-add, as the reference's host build computes) with
  the output numbering of the GPU remesher: per input face, the top TOP_LEVELS
  levels of its split tree breadth first (left to right, first child before
  second), then the subtrees below them left to right, each depth first.  It is pinned to the reference through
  `families`, which compares the two as sets of triangles per input face.
"""

from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libremesh_ref.so")
_lib = None
f32 = np.float32


def reference_available() -> bool:
    return os.path.exists(REF_LIB)


def _ref():
    global _lib
    if _lib is None:
        L = C.CDLL(REF_LIB)
        vp, i, f = C.c_void_p, C.c_int, C.c_float
        L.remref_split_world.restype = vp
        L.remref_split_world.argtypes = [vp, vp, i, i, i, f]
        L.remref_split_clip.restype = vp
        L.remref_split_clip.argtypes = [vp, vp, vp, vp, i, i, i, f, f]
        L.remref_sizes.argtypes = [vp, C.POINTER(i), C.POINTER(i)]
        L.remref_export.argtypes = [vp, vp, vp, vp, vp]
        L.remref_free.argtypes = [vp]
        _lib = L
    return _lib


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def reference_split(verts, faces, num_splits: int, tau: float, mvp=None, valid=None, aspect_wh: float = 1.0):
    """The reference's split_triangle_soup (mvp None) or split_triangle_soup_clip
    (src/main.cpp:308-388): (verts, faces, face_mapping, face_flags)."""
    L = _ref()
    v = np.ascontiguousarray(verts, np.float32)
    f = np.ascontiguousarray(faces, np.int32)
    if mvp is None:
        h = L.remref_split_world(_p(v), _p(f), v.shape[0], f.shape[0], int(num_splits), float(tau))
    else:
        m = np.ascontiguousarray(mvp, np.float32)
        ok = np.ascontiguousarray(valid, np.int32)
        h = L.remref_split_clip(_p(m), _p(v), _p(f), _p(ok), v.shape[0], f.shape[0], int(num_splits), float(tau),
                                float(aspect_wh))
    nv, nt = C.c_int(0), C.c_int(0)
    L.remref_sizes(h, C.byref(nv), C.byref(nt))
    ov = np.empty((nv.value, 3), np.float32)
    of = np.empty((nt.value, 3), np.int32)
    om = np.empty(nt.value, np.int32)
    ofl = np.empty(nt.value, np.int32)
    L.remref_export(h, _p(ov), _p(of), _p(om), _p(ofl))
    L.remref_free(h)
    return ov, of, om, ofl


# ---------------------------------------------------------------------------
# restatement
# ---------------------------------------------------------------------------

def _hom(m, v):
    """((m0 x + m1 y) + m2 z) + m3 per row (remesh_clip.cpp:19-29)."""
    return [f32(f32(f32(f32(m[r, 0] * v[0]) + f32(m[r, 1] * v[1])) + f32(m[r, 2] * v[2])) + m[r, 3])
            for r in range(4)]


def _clip(m, v):
    c = _hom(m, v)
    ok = c[3] > 0
    n = [f32(c[k] / c[3]) if ok else f32(0) for k in range(3)]
    inside = ok and all(f32(-1) <= n[k] <= f32(1) for k in range(3))
    return c, n, inside


def _len2(mode, m, aspect, A, B):
    if mode == 0:
        d = [f32(B[k] - A[k]) for k in range(3)]
        return f32(f32(f32(d[0] * d[0]) + f32(d[1] * d[1])) + f32(d[2] * d[2]))
    _, na, ia = _clip(m, A)
    _, nb, ib = _clip(m, B)
    if not (ia and ib):
        return f32(0)
    dx = f32(f32(na[0] - nb[0]) * aspect)
    dy = f32(na[1] - nb[1])
    return f32(f32(dx * dx) + f32(dy * dy))


def _split_point(mode, m, A, B):
    if mode == 0:
        return [f32(f32(0.5) * f32(A[k] + B[k])) for k in range(3)]
    ca, na, _ = _clip(m, A)
    cb, nb, _ = _clip(m, B)
    nx = f32(f32(0.5) * f32(na[0] + nb[0]))
    ny = f32(f32(0.5) * f32(na[1] + nb[1]))
    dx, dy, dw = f32(cb[0] - ca[0]), f32(cb[1] - ca[1]), f32(cb[3] - ca[3])
    ax, ay = f32(ca[0] - f32(nx * ca[3])), f32(ca[1] - f32(ny * ca[3]))
    bx, by = f32(dx - f32(nx * dw)), f32(dy - f32(ny * dw))
    den = f32(f32(bx * bx) + f32(by * by))
    tB = f32(-f32(f32(ax * bx) + f32(ay * by)) / den) if den != 0 else f32(0.5)
    tA = f32(f32(1) - tB)
    return [f32(f32(tA * A[k]) + f32(tB * B[k])) for k in range(3)]


TOP_LEVELS = 5  # split levels of a family numbered breadth first (csrc/remesh.cu kTopLevels)


def restated_split(verts, faces, tau: float, mvp=None, valid=None, aspect_wh: float = 1.0):
    """Threshold mode (num_splits = -1) of either remesher, numbered per input
    face depth first: (verts, faces, face_mapping, face_flags)."""
    mode = 0 if mvp is None else 1
    v = np.asarray(verts, np.float32)
    fc = np.asarray(faces, np.int32)
    m = None if mvp is None else np.asarray(mvp, np.float32)
    aspect = f32(aspect_wh)
    t = f32(tau) if mode == 0 else f32(f32(2) * f32(tau))
    tau2 = f32(t * t)
    N, M = v.shape[0], fc.shape[0]
    fam_splits: List[list] = []  # per face: list of (kind, data) in walk order
    leaves: List[list] = []
    for face in range(M):
        ids = [int(x) for x in fc[face]]
        P = [v[i].copy() for i in ids]
        splittable = tau > 0 and (mode == 0 or valid is None or int(valid[face]) > 0)
        new_verts, fam_leaves = [], []

        def split(node):
            """The node's children (first, second) if it splits, else None (a leaf)."""
            slot, cid, cp = node
            e, best = -1, f32(0)
            if splittable:
                for q in range(3):
                    l2 = _len2(mode, m, aspect, cp[q], cp[(q + 1) % 3])
                    if (mode == 0 or l2 > 0) and (e < 0 or l2 > best):
                        e, best = q, l2
            if not (e >= 0 and best >= tau2 and best > 0):
                fam_leaves.append((slot, cid))
                return None
            k = len(new_verts) // 3
            ia, ib, ic = e, (e + 1) % 3, (e + 2) % 3
            Cp = np.array(_split_point(mode, m, cp[ia], cp[ib]), np.float32)
            new_verts.extend([Cp, Cp, cp[ic].copy()])
            mA = -(3 * k + 1)  # placeholders, resolved once the family's offset is known
            second = (("new", k), [mA - 1, cid[ib], cid[ic]], [Cp, cp[ib], cp[ic]])
            first = (slot, [cid[ia], mA, mA - 2], [cp[ia], Cp, cp[ic]])
            return first, second

        front = [(face, ids, P)]
        for _ in range(TOP_LEVELS):  # top levels breadth first
            nxt = []
            for node in front:
                ch = split(node)
                if ch is not None:
                    nxt.extend(ch)
            front = nxt
        for root in front:  # then each subtree depth first, left to right
            stack = [root]
            while stack:
                cur = stack.pop()
                while True:
                    ch = split(cur)
                    if ch is None:
                        break
                    stack.append(ch[1])
                    cur = ch[0]
        fam_splits.append(new_verts)
        leaves.append(fam_leaves)
    counts = np.array([len(nv) // 3 for nv in fam_splits], np.int64)
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    S = int(off[-1])
    ov = np.concatenate([v] + [np.stack(nv) for nv in fam_splits if nv], 0) if S else v.copy()
    of = np.empty((M + S, 3), np.int32)
    om = np.empty(M + S, np.int32)
    ofl = np.empty(M + S, np.int32)
    for face in range(M):
        vb = N + 3 * int(off[face])
        for slot, cid in leaves[face]:
            s = face if not isinstance(slot, tuple) else M + int(off[face]) + slot[1]
            of[s] = [c if c >= 0 else vb + (-c - 1) for c in cid]
            om[s] = face
            ofl[s] = 1 if counts[face] == 0 else 0
    return ov, of, om, ofl


def families(verts, faces, mapping, flags) -> Dict[int, List[Tuple]]:
    """Per input face: the sorted list of its triangles, each as the bit
    patterns of its three corners in order, with the face's flag."""
    v = np.asarray(verts, np.float32).view(np.uint32)
    out: Dict[int, List[Tuple]] = {}
    for s in range(faces.shape[0]):
        tri = tuple(tuple(int(x) for x in v[int(i)]) for i in faces[s])
        out.setdefault(int(mapping[s]), []).append((tri, int(flags[s])))
    for k in out:
        out[k].sort()
    return out
