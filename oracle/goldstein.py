"""Oracle: CPU restatement of the Goldstein branch-cut phase unwrapper
(Codes/sub_code/goldstein_GPU: unwrapp2_gpu.m, goldstein_branch_cut.m and the
kernels / host code it calls).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  The branch linker of this
module is additionally pinned against the reference's own C++ linker,
compiled from its sources into oracle/_ref (see oracle/ref_goldstein/).

One behaviour of the reference is made defined here: the neighbour search
(search_universal.cpp:35-39) checks its box indices only against the upper
bound, so a box left of or above the grid reads the lookup table at a lower
index -- the previous row's or the previous slice's entries, which this
restatement reads as well -- and, at the very start of the table, before the
array.  Such reads return -1 (an empty box) here.

Arrays: MATLAB column-major order, indexed a[d1, d2, z]; residue tables are
[6, R] int32 rows (idx, value, case, x, y, z) as in goldstein_branch_cut.m:30.
"""
from __future__ import annotations

import math

import numpy as np

PI_F = np.float32(3.141592654)          # CUDART_PI_F of the reference kernels
TWO_PI_F = np.float32(2.0) * PI_F
F32 = np.float32


def modulo_float(a, b):
    """fmodf(fmodf(a, b) + b, b) (get_residue_cuda.cu:28-31)."""
    return np.fmod(np.fmod(a, b) + b, b).astype(F32)


def roundf(x):
    return (np.sign(x) * np.floor(np.abs(x) + F32(0.5))).astype(F32)


# ---------------------------------------------------------------- a11
def get_residue(phase):
    """get_residue_cuda.cu:34-66: residue of each 2x2 loop, [N1-1, N2-1, n]."""
    p = np.asarray(phase, dtype=F32)
    v11, v21 = p[:-1, :-1], p[1:, :-1]
    v12, v22 = p[:-1, 1:], p[1:, 1:]
    d1_1 = modulo_float((v11 - v12) + PI_F, TWO_PI_F)
    d1_2 = modulo_float((v21 - v22) + PI_F, TWO_PI_F)
    d2_1 = modulo_float((v11 - v21) + PI_F, TWO_PI_F)
    d2_2 = modulo_float((v12 - v22) + PI_F, TWO_PI_F)
    s = ((d1_1 + d2_2) - d1_2) - d2_1
    return roundf(s / TWO_PI_F)


# ---------------------------------------------------------------- a12
def remove_dipoles(residue):
    """remove_dipoles_cuda.cu:52-146 driven as unwrapp2_gpu.m:3 does (positive
    residues in column-major find() order, directions 0..3 in turn).  Within
    one direction every positive residue pairs with a distinct neighbour, so
    the reference kernel's result does not depend on thread order.  Returns
    (residue', step1 [N1, N2, n] single, step2 [N2, n] single (never written:
    remove_dipoles_mex.cpp:117 aliases it to step1))."""
    r = np.array(residue, dtype=F32, copy=True)
    M1, M2, n = r.shape
    step1 = np.zeros((M1 + 1, M2 + 1, n), dtype=F32)
    flat = r.reshape(-1, order="F")
    pos = list(np.nonzero(flat > 0)[0])
    alive = [True] * len(pos)
    for direction in range(4):
        for k, idr in enumerate(pos):
            if not alive[k]:
                continue
            d12 = idr % (M1 * M2)
            d3 = idr // (M1 * M2)
            d2, d1 = d12 // M1, d12 % M1
            p1 = d1 - (direction == 0) + (direction == 2)
            p2 = d2 - (direction == 1) + (direction == 3)
            if not (0 <= p1 < M1 and 0 <= p2 < M2):
                continue
            idp = d3 * M1 * M2 + p2 * M1 + p1
            pv = flat[idp]
            if pv < 0:
                v = flat[idr]
                rm = F32(min(v, -pv))
                v = roundf(F32(v - rm))
                pv = roundf(F32(pv + rm))
                flat[idr] = v
                flat[idp] = pv
                if v == 0:
                    alive[k] = False
                if direction in (1, 3):
                    step1[p1 + 1, min(d2, p2) + 1, d3] = rm if direction == 1 else -rm
    r = flat.reshape((M1, M2, n), order="F")
    step2 = np.zeros((M2 + 1, n), dtype=F32)
    return r, step1, step2


# ---------------------------------------------------------------- a13
def residue_table(residue):
    """goldstein_branch_cut.m:10-33: residue list sorted by (z, case),
    square sizes, lookup table and per-slice lookup offsets."""
    M1, M2, n = residue.shape
    flat = residue.reshape(-1, order="F")
    idx = np.nonzero(flat)[0].astype(np.int64)
    z = idx // (M1 * M2)
    counts = np.bincount(z, minlength=n)[:n].astype(np.float64)
    ss = np.ceil(np.sqrt((counts + 1) / 16)).astype(np.int32)
    # create_sort_value_cuda.cu:52-86
    d12 = idx % (M1 * M2)
    x = (d12 % M1).astype(np.int32)
    y = (d12 // M1).astype(np.int32)
    sz = ss[z]
    cs1 = np.ceil(np.float32(M1) / sz.astype(np.float32)).astype(np.int32)
    cs2 = np.ceil(np.float32(M2) / sz.astype(np.float32)).astype(np.int32)
    case = (x // cs1) + (y // cs2) * sz
    tab = np.stack([idx.astype(np.int32), flat[idx].astype(np.int32), case.astype(np.int32), x, y,
                    z.astype(np.int32)])
    order = np.lexsort((np.arange(idx.size), tab[2], tab[5]))   # stable sortrows([6, 3])
    tab = np.ascontiguousarray(tab[:, order])
    zstart = np.zeros(n, dtype=np.int32)
    total = 0
    for i in range(n):
        zstart[i] = total
        total += int(ss[i]) * int(ss[i])
    lookup = np.full(total, -1, dtype=np.int32)
    for i in range(tab.shape[1]):                      # get_lookup_cuda.cu:60-88
        if i == 0 or tab[2, i] != tab[2, i - 1] or tab[5, i] != tab[5, i - 1]:
            lookup[zstart[tab[5, i]] + tab[2, i]] = i
    return tab, ss, lookup, zstart


def _look(lookup, i):
    return int(lookup[i]) if 0 <= i < lookup.size else -1


def _bsearch(arr, x, low, high):
    """binarySearch_array_2_size (search_universal.cpp:1-27)."""
    mid = 0
    while low < high:
        mid = (high + low) // 2 if high + low >= 0 else -((-(high + low)) // 2)
        if arr[2 * mid + 1] == x:
            break
        elif arr[2 * mid + 1] > x:
            high = mid - 1
        else:
            low = mid + 1
    s = high + low
    mid = s // 2 if s >= 0 else -((-s) // 2)
    return mid if x <= arr[2 * mid + 1] else mid + 1


def _search_in_case(tab, lookup, cur, ss, b1, b2, start, R, xc, yc, K, id1, states):
    """search_in_case (search_universal.cpp:28-100)."""
    if b1 >= ss or b2 >= ss:
        return
    cid = start + b1 + b2 * ss
    sl = _look(lookup, cid)
    if sl == -1:
        return
    el = R
    nf = 1
    while cid + nf < lookup.size and el == R:
        v = _look(lookup, cid + nf)
        if v >= 0:
            el = v
            break
        nf += 1
    for i in range(sl, el):
        if states is not None and (states[i] & 2):
            continue
        xx = abs(xc - int(tab[3, i]))
        yy = abs(yc - int(tab[4, i]))
        dist = int(np.sqrt(np.float32(xx * xx + yy * yy)))
        if dist < cur[2 * K - 1] and i != id1:
            ins = _bsearch(cur, dist, 0, K - 1)
            if ins < K:
                for k in range(K - 1, ins, -1):
                    cur[2 * k] = cur[2 * (k - 1)]
                    cur[2 * k + 1] = cur[2 * (k - 1) + 1]
                cur[2 * ins] = i
                cur[2 * ins + 1] = dist


def shortest(id1, tab, lookup, zstart, ss_arr, K, dims, states=None):
    """shortest_compute_kernel (search_universal.cpp:102-271): the K nearest
    residues of residue id1 within its distance to the border (states != None:
    the host variant used by the linker, skipping active residues)."""
    R = tab.shape[1]
    M1, M2 = dims[0], dims[1]
    case = int(tab[2, id1]); xc = int(tab[3, id1]); yc = int(tab[4, id1]); z = int(tab[5, id1])
    start = int(zstart[z])
    ss = int(ss_arr[z])
    cs1 = int(math.ceil(np.float32(M1) / np.float32(ss)))
    cs2 = int(math.ceil(np.float32(M2) / np.float32(ss)))
    c1, c2 = case % ss, case // ss
    maxb = max(max(ss - c1, ss - c2), max(c1, c2))
    dmax = min(min(xc, yc), min(M1 - xc, M2 - yc))
    cur = []
    for _ in range(K):
        cur += [-1, dmax]
    last = dmax
    d = 0
    while d < maxb and d < ss:
        if d == 0:
            _search_in_case(tab, lookup, cur, ss, c1, c2, start, R, xc, yc, K, id1, states)
        else:
            for ii in range(1 - d, d + 1):
                b1 = [c1 - d, c1 + ii, c1 - ii, c1 + d]
                b2 = [c2 - ii, c2 - d, c2 + d, c2 + ii]
                md = [
                    max(abs((b1[0] + 1) * cs1 - xc), abs(((b2[0] + (1 if ii > 0 else 0)) * cs2 - yc) * (0 if ii == 0 else 1))),
                    max(abs(((b1[1] + (0 if ii > 0 else 1)) * cs1 - xc) * (0 if ii == 0 else 1)), abs((b2[1] + 1) * cs2 - yc)),
                    max(abs(((b1[2] + (1 if ii > 0 else 0)) * cs1 - xc) * (0 if ii == 0 else 1)), abs(b2[2] * cs2 - yc)),
                    max(abs(b1[3] * cs1 - xc), abs(((b2[3] + (0 if ii > 0 else 1)) * cs2 - yc) * (0 if ii == 0 else 1))),
                ]
                to_eval = [m < last for m in md]
                for e in range(4):
                    if to_eval[e]:
                        _search_in_case(tab, lookup, cur, ss, b1[e], b2[e], start, R, xc, yc, K, id1, states)
                last = cur[2 * K - 1]
        last = cur[2 * K - 1]
        if d * cs1 >= last and d * cs2 >= last:
            break
        d += 1
    return cur


def shortest_list(tab, lookup, zstart, ss, K, dims):
    """get_shortest_sort_gpu (K = 8): [2, K, R] int32 (id, distance)."""
    R = tab.shape[1]
    out = np.zeros((2, K, R), dtype=np.int32)
    for i in range(R):
        cur = shortest(i, tab, lookup, zstart, ss, K, dims)
        out[0, :, i] = cur[0::2]
        out[1, :, i] = cur[1::2]
    return out


# ---------------------------------------------------------------- a14
BALANCED, ACTIVE = 1, 2


def get_branches(tab, sl, ss, lookup, zstart, dims):
    """get_branches_goldstein_compute (get_branches_goldstein_compute_v2.cpp
    :12-203) with update_min_distance / get_shortest_id
    (get_branches_goldstein_update_v2.cpp:13-61).  Returns [6, B] int32 rows
    (x1, y1, x2, y2, z, jump)."""
    R = tab.shape[1]
    K = sl.shape[1]
    DMAX = 200000
    state = [0] * R
    branches = []

    def shortest_id(a):
        if a["idx"] < K:
            return int(sl[0, a["idx"], a["res"]])
        return a["ovf"]

    def update(a):
        nxt = 1 + a["idx"]
        while True:
            if nxt < K:
                cand = int(sl[0, nxt, a["res"]])
                if cand == -1 or nxt == K - 1 or not (state[cand] & ACTIVE):
                    a["idx"] = nxt
                    a["dist"] = int(sl[1, nxt, a["res"]])
                    return
            else:
                a["idx"] = K
                res = shortest(a["res"], tab, lookup, zstart, ss, 1, dims, states=state)
                a["ovf"], a["dist"] = res[0], res[1]
                return
            nxt += 1

    for i in range(R):
        if state[i] & BALANCED:
            continue
        act = [dict(res=i, parent=0, pb=0, dist=0, idx=0, ovf=0)]
        state[i] |= ACTIVE
        load = int(tab[1, i])
        cur_min = 0
        next_min = 0
        while load != 0:
            cur_min = next_min
            next_min = DMAX
            ai = 0
            while ai < len(act):
                if act[ai]["dist"] == cur_min:
                    sid = shortest_id(act[ai])
                    if sid == -1 or not (state[sid] & ACTIVE):
                        old = load
                        if sid != -1 and not (state[sid] & BALANCED):
                            load += int(tab[1, sid])
                        if sid == -1:
                            load = 0
                        new = dict(res=sid, parent=ai, dist=0, idx=-1, ovf=0, pb=len(branches))
                        act.append(new)
                        if sid != -1:
                            state[sid] |= ACTIVE
                        src = act[ai]["res"]
                        br = [int(tab[3, sid]) if sid != -1 else -1, int(tab[4, sid]) if sid != -1 else -1,
                              int(tab[3, src]), int(tab[4, src]), int(tab[5, src]), 0]
                        branches.append(br)
                        if sid == -1 or not (state[sid] & BALANCED):
                            jump = int(tab[1, sid]) if sid != -1 else -old
                            p = len(act) - 1
                            while p != 0:
                                branches[act[p]["pb"]][5] += jump
                                p = act[p]["parent"]
                        update(act[ai])
                        if sid != -1:
                            update(act[-1])
                        # the reference compares its local copy (min distance 0)
                        if 0 < cur_min:
                            cur_min = 0
                        if 0 < next_min:
                            next_min = 0
                    else:
                        update(act[ai])
                if act[ai]["dist"] < next_min:
                    next_min = act[ai]["dist"]
                if load == 0:
                    break
                ai += 1
        for a in act:
            if a["res"] != -1:
                state[a["res"]] &= ~ACTIVE
                state[a["res"]] |= BALANCED
    return np.array(branches, dtype=np.int32).T.reshape(6, -1)


# ---------------------------------------------------------------- a15
def raster_branches(branches, step1, step2):
    """raster_branches_cuda.cu:68-131 (integer adds: order-free)."""
    s1 = np.array(step1, dtype=np.int32, copy=True)
    s2 = np.array(step2, dtype=np.int32, copy=True)
    N1, N2, _ = s1.shape
    f1 = s1.reshape(-1, order="F")
    f2 = s2.reshape(-1, order="F")
    for b in range(branches.shape[1]):
        x1, y1, x2, y2, z, jump = [int(v) for v in branches[:, b]]
        if x1 == -1:
            xs = x2 < N1 - x2
            ys = y2 < N2 - y2
            mdx = x2 if xs else N1 - x2
            mdy = y2 if ys else N2 - y2
            x1 = x2 if mdx > mdy else (-1 if xs else N1 - 1)
            y1 = y2 if mdx < mdy else (-1 if ys else N2 - 1)
            if x1 == -1:
                f2[N2 * z + y2 + 1] += jump
                continue
            if x1 == N1:
                continue
        if y1 != y2:
            if y2 > y1:
                x1, x2 = x2, x1
                y1, y2 = y2, y1
                jump = -jump
            steps = y1 - y2
            for i in range(steps):
                cy = y2 + i + 1
                cx = x2 + int((np.float32(i) / np.float32(steps)) * np.float32(x1 - x2)) + 1
                f1[N1 * N2 * z + N1 * cy + cx] += jump
    return f1.reshape(s1.shape, order="F"), f2.reshape(s2.shape, order="F")


# ---------------------------------------------------------------- a16
def unwrap_phase(wrapped, step1, step2):
    """unwrapp_phase_goldstein_cuda.cu:63-115: integrate along dimension 2 at
    row 0 of each slice (with step2), then down every column (with step1)."""
    p = np.array(wrapped, dtype=F32, copy=True)
    N1, N2, n = p.shape
    for z in range(n):
        last = p[0, 0, z]
        for i in range(1, N2):
            cur = p[0, i, z]
            d = F32(modulo_float(F32((cur - last) + PI_F), TWO_PI_F) - PI_F)
            cur = F32(F32(last + d) - F32(F32(F32(step2[i, z]) * F32(2.0)) * PI_F))
            p[0, i, z] = cur
            last = cur
    for z in range(n):
        for j in range(N2):
            last = p[0, j, z]
            for i in range(1, N1):
                cur = p[i, j, z]
                d = F32(modulo_float(F32((cur - last) + PI_F), TWO_PI_F) - PI_F)
                cur = F32(F32(last + d) - F32(F32(F32(step1[i, j, z]) * F32(2.0)) * PI_F))
                p[i, j, z] = cur
                last = cur
    return p


def unwrapp2(wrapped, return_intermediates=False):
    """unwrapp2_gpu.m:1-6."""
    res = get_residue(wrapped)
    res, step1, step2 = remove_dipoles(res)
    inter = {"residue": res}
    if np.any(res != 0):
        M = res.shape
        tab, ss, lookup, zstart = residue_table(res)
        sl = shortest_list(tab, lookup, zstart, ss, 8, M)
        br = get_branches(tab, sl, ss, lookup, zstart, M)
        step1, step2 = raster_branches(br, step1, step2)
        inter.update(table=tab, square_size=ss, lookup=lookup, lookup_z_start=zstart,
                     shortest=sl, branches=br)
    else:
        step1 = step1.astype(np.int32)
        step2 = step2.astype(np.int32)
        inter["branches"] = np.zeros((6, 0), dtype=np.int32)
    inter.update(step1=step1, step2=step2)
    out = unwrap_phase(wrapped, step1, step2)
    return (out, inter) if return_intermediates else out


# ---------------------------------------------------------------- reference
def ref_lib():
    """The reference's own linker and nearest-residue search built from its
    sources by oracle/ref_goldstein/Makefile into oracle/_ref (None when
    that library has not been built)."""
    import ctypes as C
    import os

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libref_goldstein.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    P = C.POINTER(C.c_int32)
    lib.ref_nearest.argtypes = [P, P, P, P] + [C.c_int] * 6 + [P]
    lib.ref_nearest.restype = C.c_int
    lib.ref_branches.argtypes = [P, P, P, P, P] + [C.c_int] * 7 + [P, C.c_longlong]
    lib.ref_branches.restype = C.c_longlong
    return lib


def _p(a):
    import ctypes as C

    return a.ctypes.data_as(C.POINTER(C.c_int32))


def ref_nearest(lib, tab, lookup, zstart, ss, K, dims):
    """shortest_compute_kernel of the reference, on the host: [2, K, R]."""
    R = tab.shape[1]
    tab = np.ascontiguousarray(tab.T)      # [R, 6] rows of 6 = the reference's [6, R] column-major
    out = np.zeros((R, K, 2), dtype=np.int32)
    lib.ref_nearest(_p(tab), _p(np.ascontiguousarray(lookup, np.int32)), _p(np.ascontiguousarray(zstart, np.int32)),
                    _p(np.ascontiguousarray(ss, np.int32)), R, K, int(dims[0]), int(dims[1]), int(len(ss)),
                    int(lookup.size), _p(out))
    return np.ascontiguousarray(out.transpose(2, 1, 0))


def ref_branches(lib, tab, sl, ss, lookup, zstart, dims):
    """get_branches_goldstein_compute of the reference: [6, B]."""
    R = tab.shape[1]
    K = sl.shape[1]
    rows = np.ascontiguousarray(tab.T)
    near = np.ascontiguousarray(sl.transpose(2, 1, 0))   # [R, K, 2]
    cap = 4 * R + 16
    out = np.zeros((cap, 6), dtype=np.int32)
    dz = int(dims[2]) if len(dims) > 2 else 1
    n = lib.ref_branches(_p(rows), _p(near), _p(np.ascontiguousarray(ss, np.int32)),
                         _p(np.ascontiguousarray(lookup, np.int32)), _p(np.ascontiguousarray(zstart, np.int32)),
                         R, int(len(ss)), int(lookup.size), K, int(dims[0]), int(dims[1]), dz, _p(out), cap)
    if n > cap:
        raise RuntimeError("branch capacity exceeded")
    return np.ascontiguousarray(out[:n].T)
