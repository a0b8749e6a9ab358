"""Executable model of the round scheduling used by the insert and remove
kernels (flash-map_b200/csrc/fm_kernels.cu), for CPU tests.

Each round applies the kernels' decision rules (segment registration, leader
choice, forward flow walks / potential-target windows).  The ops a round
selects are then applied one after another in a RANDOM order: the kernels run
them concurrently, so the scheduling is correct only if any order gives the
sequential (oracle) result.  Table semantics follow src/rayon_cpu.rs.
"""
from __future__ import annotations

import numpy as np

import oracle as O

EMPTY, OCC, TOMB = 0, 1, 2
IDLE = 0xFFFFFFFF


class ModelTable:
    def __init__(self, cap, ks, vs, mode=0):
        self.cap, self.mask, self.ks, self.vs, self.mode = cap, cap - 1, ks, vs, mode
        self.flags = np.zeros(cap, np.uint64)
        self.keys = [bytes(ks)] * cap
        self.vals = [bytes(vs)] * cap
        self.dmax = 0
        self.len = 0
        self.max_rounds = 0

    def h(self, k: bytes) -> int:
        return O.hash_key(k, self.mode) & self.mask

    def free(self, s):
        return int(self.flags[s]) & 0xF in (EMPTY, TOMB)

    # sequential insert of one key (rayon_cpu.rs:157-264), with the step limit
    def exec_insert(self, k, v):
        h, p = self.h(k), 0
        ck, cv = k, v
        limit = 2 * self.cap + 2
        step = 0
        while True:
            if p > self.mask or step > limit:
                return 0
            step += 1
            idx = (h + p) & self.mask
            f = int(self.flags[idx])
            st, d = f & 0xF, f >> 4
            if st == OCC:
                if self.keys[idx] == ck:
                    self.vals[idx] = cv
                    return 0
                if p > d:
                    self.keys[idx], ck = ck, self.keys[idx]
                    self.vals[idx], cv = cv, self.vals[idx]
                    self.flags[idx] = ((p & 0x0FFFFFFF) << 4) | OCC
                    self.dmax = max(self.dmax, p)
                    h, p = self.h(ck), d + 1
                    continue
                p += 1
                continue
            if st in (EMPTY, TOMB):
                self.keys[idx], self.vals[idx] = ck, cv
                self.flags[idx] = ((p & 0x0FFFFFFF) << 4) | OCC
                self.dmax = max(self.dmax, p)
                return 1
            p += 1

    def bulk_insert(self, keys, vals, rng):
        n = len(keys)
        if self.len + n > self.cap:
            raise O.TableFull(self.len, self.cap)
        pend = list(range(n))
        added = 0
        rounds = 0
        while pend:
            rounds += 1
            seg_min, seg_cnt, opF = {}, {}, {}
            serial = False
            for j in pend:  # phase 1
                h = self.h(keys[j])
                F = None
                for p in range(self.cap):
                    s = (h + p) & self.mask
                    if self.free(s):
                        F = s
                        break
                opF[j] = F
                if F is None:
                    serial = True
                else:
                    seg_min[F] = min(seg_min.get(F, IDLE), j)
                    seg_cnt[F] = seg_cnt.get(F, 0) + 1
            gmin = min(pend)
            leader, block = {}, {j: IDLE for j in pend}
            for j in pend:  # phase 2
                F = opF[j]
                leader[j] = F is not None and seg_min[F] == j
                if not leader[j] or seg_cnt[F] < 2:
                    continue
                flow, L, pos, walked = seg_cnt[F] - 1, j, F + 1, 0
                while True:
                    F2 = None
                    while walked < self.mask:
                        s = pos & self.mask
                        pos += 1
                        walked += 1
                        if self.free(s):
                            F2 = s
                            break
                    if F2 is None:
                        serial = True
                        break
                    c2 = seg_cnt.get(F2, 0)
                    if c2:
                        l2 = seg_min[F2]
                        block[l2] = min(block[l2], L)
                        L = min(L, l2)
                    flow += c2 - 1
                    if flow == 0:
                        break
            run = [j for j in pend if (j == gmin if serial else (leader[j] and block[j] > j))]
            assert run, "no progress"
            order = list(run)
            rng.shuffle(order)
            for j in order:  # phase 3, in an arbitrary order
                added += self.exec_insert(keys[j], vals[j])
            rs = set(run)
            pend = [j for j in pend if j not in rs]
        self.max_rounds = max(self.max_rounds, rounds)
        self.len += added
        return added

    def bulk_remove(self, keys, rng):
        n = len(keys)
        pend = list(range(n))
        removed = 0
        while pend:
            marks = {}
            info = {}
            for j in pend:  # phase 1: probe and mark potential targets
                k = keys[j]
                h = self.h(k)
                tp, p, empty_hit = None, 0, False
                while p <= self.mask:
                    s = (h + p) & self.mask
                    f = int(self.flags[s])
                    st, d = f & 0xF, f >> 4
                    if st == EMPTY:
                        empty_hit = True
                        break
                    if st == OCC:
                        if p > d:
                            break
                        if d == (p & 0x0FFFFFFF) and self.keys[s] == k:
                            tp = p
                            break
                    p += 1
                lim = min((tp if tp is not None else 0) + self.dmax, self.mask)
                pts = []
                if empty_hit:
                    wend = None if p == 0 else min(p - 1, lim)
                else:
                    if tp is not None:
                        pts.append(tp)
                    q = (tp if tp is not None else p) + 1
                    wend = min(p, lim)
                    while q <= lim:
                        s = (h + q) & self.mask
                        f = int(self.flags[s])
                        if f & 0xF == EMPTY:
                            break
                        wend = q
                        if f & 0xF == OCC and (f >> 4) == (q & 0x0FFFFFFF) and self.keys[s] == k:
                            pts.append(q)
                        q += 1
                for q in pts:
                    s = (h + q) & self.mask
                    marks[s] = min(marks.get(s, IDLE), j)
                info[j] = (h, tp, wend)
            run = []
            for j in pend:  # phase 2: window check
                h, tp, wend = info[j]
                ok = True
                if wend is not None:
                    for q in range(wend + 1):
                        if marks.get((h + q) & self.mask, IDLE) < j:
                            ok = False
                            break
                if ok:
                    run.append(j)
            assert run, "no progress"
            order = list(run)
            rng.shuffle(order)
            for j in order:
                h, tp, _ = info[j]
                if tp is not None:
                    self.flags[(h + tp) & self.mask] = TOMB
                    removed += 1
            rs = set(run)
            pend = [j for j in pend if j not in rs]
        self.len -= removed
        return removed

    def snapshot(self):
        f = self.flags.astype(np.uint32)
        occ = (f & 0xF) == OCC
        k = np.array([np.frombuffer(x, np.uint8) for x in self.keys], np.uint8).reshape(self.cap, self.ks)
        v = np.array([np.frombuffer(x, np.uint8) for x in self.vals], np.uint8).reshape(self.cap, self.vs)
        k[~occ] = 0
        v[~occ] = 0
        return f, k, v
