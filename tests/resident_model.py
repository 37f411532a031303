"""A pure-Python model of the resident coherency planner (xkb_planner_create_resident), for the
tests: the canonical block partition of each (ld, sizeof) frame -- x-slabs are the elementary
intervals of every x-boundary inserted so far; a slab's blocks are cut at the y-boundaries of
every rect inserted over it (the partition of the reference's memory tree,
include/xkrt/memory/access/blas/memory-tree.hpp:1765-1776) -- and the resident rules: a block is
coherent on the host when no device bit is set or the host bit is, on the GPU when the GPU bit
is; a read copies the blocks the target lacks (whole blocks, host pitch), a write leaves the
target as the only coherent copy; virtual accesses move nothing. Copies are listed per access in
the order of its rects, slabs by x, blocks by y, with the library's record layout
(task, access, kind, src_dev, src_alloc, src_off, src_ld, dst_dev, dst_alloc, dst_off, dst_ld,
m, n, sizeof)."""
import bisect

H2D, D2H = 0, 1
HOST, GPU = 1, 2
SEGMENT, MATRIX = 1, 2
R, W, V = 1, 2, 4
SEG_LD = (1 << 64) - 1


class Slab:
    def __init__(self, x1, ys=None, ends=None, st=None):
        self.x1 = x1
        self.ys = list(ys or [])       # block starts, ascending
        self.ends = list(ends or [])   # block ends
        self.st = list(st or [])       # block states

    def copy(self, x1):
        return Slab(x1, self.ys, self.ends, self.st)

    def split_y(self, y):
        i = bisect.bisect_right(self.ys, y) - 1
        if i >= 0 and self.ys[i] < y < self.ends[i]:
            self.ys.insert(i + 1, y)
            self.ends.insert(i + 1, self.ends[i])
            self.st.insert(i + 1, self.st[i])
            self.ends[i] = y

    def fill(self, y0, y1):
        """split at y0, y1 and create blocks over the y-gaps of [y0, y1)"""
        self.split_y(y0)
        self.split_y(y1)
        y = y0
        i = bisect.bisect_left(self.ys, y0)
        while y < y1:
            if i < len(self.ys) and self.ys[i] == y:
                y = self.ends[i]
                i += 1
                continue
            end = self.ys[i] if i < len(self.ys) and self.ys[i] < y1 else y1
            self.ys.insert(i, y)
            self.ends.insert(i, end)
            self.st.insert(i, 0)
            i += 1
            y = end


class Frame:
    def __init__(self):
        self.xs = []       # slab starts, ascending
        self.slabs = []

    def split_x(self, x):
        i = bisect.bisect_right(self.xs, x) - 1
        if i >= 0 and self.xs[i] < x < self.slabs[i].x1:
            right = self.slabs[i].copy(self.slabs[i].x1)
            self.slabs[i].x1 = x
            self.xs.insert(i + 1, x)
            self.slabs.insert(i + 1, right)

    def insert(self, x0, x1, y0, y1):
        self.split_x(x0)
        self.split_x(x1)
        x = x0
        i = bisect.bisect_left(self.xs, x0)
        while x < x1:
            if i < len(self.xs) and self.xs[i] == x:
                x = self.slabs[i].x1
                i += 1
                continue
            end = self.xs[i] if i < len(self.xs) and self.xs[i] < x1 else x1
            self.xs.insert(i, x)
            self.slabs.insert(i, Slab(end))
            i += 1
            x = end
        i = bisect.bisect_left(self.xs, x0)
        while i < len(self.xs) and self.xs[i] < x1:
            self.slabs[i].fill(y0, y1)
            i += 1

    def partites(self, x0, x1, y0, y1):
        """(x0, x1, y0, y1, slab, block index) of every block inside the rect"""
        out = []
        i = bisect.bisect_left(self.xs, x0)
        while i < len(self.xs) and self.xs[i] < x1:
            sl = self.slabs[i]
            j = bisect.bisect_left(sl.ys, y0)
            while j < len(sl.ys) and sl.ys[j] < y1:
                out.append((self.xs[i], sl.x1, sl.ys[j], sl.ends[j], sl, j))
                j += 1
            i += 1
        return out


class ResidentModel:
    def __init__(self):
        self.frames = {}
        self.regions = []    # (base, size, id), sorted by base
        self.nalloc = 0
        self.copies = []

    def add_region(self, base, size):
        rid = self.nalloc
        self.nalloc += 1
        self.regions.append((base, size, rid))
        self.regions.sort()
        return rid

    def fetch(self, rec, access_index, device):
        typ, mode = int(rec["type"]), int(rec["mode"])
        addr, ld, om, on = int(rec["addr"]), int(rec["ld"]), int(rec["offset_m"]), int(rec["offset_n"])
        m, n, s = int(rec["m"]), int(rec["n"]), int(rec["sizeof_type"])
        if typ == SEGMENT:
            key, seg = (SEG_LD, 1), True
            rects = [(addr, ld, 0, 1)]
            begin, end, stride = addr, ld, 0
            fld, fs = SEG_LD, 1
        else:
            key, seg = (ld, s), False
            LDs = ld * s
            A = addr + (on * ld + om) * s
            x0, y0 = A % LDs, A // LDs
            if x0 + m * s <= LDs:
                rects = [(x0, x0 + m * s, y0, y0 + n)]
            else:
                rects = [(x0, LDs, y0, y0 + n), (0, m * s - (LDs - x0), y0 + 1, y0 + n + 1)]
            begin, end, stride = A, A + ((n - 1) * ld + m) * s, LDs
            fld, fs = ld, s
        reg = [r for r in self.regions if r[0] <= begin]
        assert reg, "access in no region"
        rbase, rsize, rid = reg[-1]
        assert end <= rbase + rsize, "access crosses its region"
        view = (rid, begin - rbase, (ld - addr) if seg else ld)
        f = self.frames.setdefault(key, Frame())
        for r in rects:
            f.insert(*r)
        parts = []
        for r in rects:
            parts += f.partites(*r)
        me = HOST if device == 0 else GPU
        for (px0, px1, py0, py1, sl, j) in parts:
            st = sl.st[j]
            host_ok = st == 0 or (st & HOST)
            gpu_ok = st & GPU
            if mode & R and not mode & V and not (host_ok if me == HOST else gpu_ok):
                h = px0 + py0 * stride
                if me == GPU:
                    src_alloc, src_off, dst_alloc, dst_off, kind = -1, h, rid, h - rbase, H2D
                else:
                    src_alloc, src_off, dst_alloc, dst_off, kind = rid, h - rbase, -1, h, D2H
                pitch = 0 if seg else fld
                if seg:
                    mm, nn, ss = px1 - px0, 1, 1
                else:
                    mm, nn, ss = (px1 - px0) // fs, py1 - py0, fs
                self.copies.append((int(rec["task"]), access_index, kind, 0 if me == GPU else 1, src_alloc, src_off, pitch,
                                    1 if me == GPU else 0, dst_alloc, dst_off, pitch, mm, nn, ss))
                st |= (HOST if st == 0 else 0) | me
            if mode & W and not mode & V:
                st = me
            sl.st[j] = st
        return view

    def take(self):
        c, self.copies = self.copies, []
        return c
