// Coherency and transfer planner for one host (device 0) and one GPU (device 1).
//
// Computes the same allocations, device views and copies as the reference's coherency
// controller, KBLASMemoryTree::fetch (include/xkrt/memory/access/blas/memory-tree.hpp:1805-1874),
// under the canonical schedule: accesses fetched one at a time in spawn/declaration order, each
// fetch's copies completed before the next fetch (so no block is ever "being fetched" when a
// fetch starts, and no access has to await another's copy).
//
// Model (my own data structures; the decisions are the reference's):
//  * Block partition of a (ld, sizeof) frame. The reference's tree is a partition of every rect
//    inserted so far into blocks; that partition is canonical: the x-slabs are the elementary
//    intervals of every x-boundary inserted so far, and within a slab the y-cuts are the
//    boundaries of every inserted rect covering that slab. A block never merges. Here: an
//    ordered map of slabs, each an ordered map of blocks. Inserting a rect splits the slabs
//    straddling its x-boundaries (both halves keep every block), creates slabs over x-gaps,
//    and in each slab it covers splits the blocks straddling its y-boundaries and creates
//    fresh blocks over y-gaps (fetch_list_to_device step 1, memory-tree.hpp:1765-1770).
//  * Block state: up to 8 allocation views (MEMORY_REPLICATE_ALLOCATION_VIEWS_MAX,
//    memory-tree.hpp:91), a coherent-view bitmask on the GPU, and the per-device coherent bits
//    (host = bit 0, GPU = bit 1). A view is (allocation, origin x, origin y, ld): the byte of
//    frame point p lives at alloc + (p.x - ox) + (p.y - oy) * ld * sizeof. With views stored by
//    origin, the reference's offset adjustment on split (memory_block_init, :284-339) is a copy.
//  * Device fetch: reuse the oldest allocation on which every block of the access has a view
//    (:1396-1450), else allocate m*n*sizeof bytes and give every block a view with origin at the
//    access corner and ld = m (:1326-1372); the access's device view is its corner's view
//    (:1452-1469). R: per block, nothing if that view is coherent; D2D from the block's first
//    coherent GPU view if the GPU holds it; else H2D from the host (:1471-1631). W: that view
//    becomes the only coherent copy anywhere (:1633-1667). Completion marks the fetched view
//    coherent and the GPU bit set (:2067-2105).
//  * Host fetch (write-back): no copy if no device holds the block, or the host already does;
//    else D2H from the view on the LARGEST allocation of the block (first one of maximal size,
//    coherent or not -- as the reference selects it, :1110-1160); completion sets the host bit.
//  * Registration-overflow protection (the reference's default build): a registered host range,
//    rounded out to pages, is inserted into every frame as 1-3 rects, so that no block, hence no
//    copy, straddles a registration boundary (memory-tree.hpp:2184-2240, src/memory/register.cc,
//    src/task/task.cc:88-94, 127-133). Only the partition changes; blocks keep their state.
#include "common.cuh"

#include <unistd.h>

#include <algorithm>
#include <cstring>
#include <iterator>
#include <map>
#include <memory>
#include <new>
#include <vector>

namespace {

constexpr int MAX_VIEWS = 8;
constexpr uint8_t DEV_HOST = 1, DEV_GPU = 2;

struct View { int32_t alloc; int64_t ox, oy; uint64_t ld; };
struct State {
    uint8_t nviews = 0;
    View views[MAX_VIEWS];
    uint8_t coh = 0;        // coherent GPU views (bit per view index)
    uint8_t dev = 0;        // coherent devices: DEV_HOST | DEV_GPU
};
struct Block { uint64_t y1; State st; };
struct Slab { uint64_t x1; std::map<uint64_t, Block> blocks; };
struct Frame {
    uint64_t ld, s;
    bool any = false;
    std::map<uint64_t, Slab> slabs;
};
struct Rect { uint64_t x0, x1, y0, y1; };
struct Partite { uint64_t x0, x1, y0, y1; State * st; };

void split_x(Frame & f, uint64_t x)
{
    auto it = f.slabs.upper_bound(x);
    if (it == f.slabs.begin()) return;
    --it;
    if (it->first < x && x < it->second.x1)
    {
        Slab right;
        right.x1 = it->second.x1;
        right.blocks = it->second.blocks;
        it->second.x1 = x;
        f.slabs.emplace(x, std::move(right));
    }
}

void split_y(Slab & sl, uint64_t y)
{
    auto it = sl.blocks.upper_bound(y);
    if (it == sl.blocks.begin()) return;
    --it;
    if (it->first < y && y < it->second.y1)
    {
        Block right = it->second;
        it->second.y1 = y;
        sl.blocks.emplace(y, right);
    }
}

void insert(Frame & f, const Rect & r)
{
    split_x(f, r.x0);
    split_x(f, r.x1);
    // slabs over the x-gaps of [x0, x1)
    uint64_t x = r.x0;
    auto it = f.slabs.lower_bound(r.x0);
    while (x < r.x1)
    {
        if (it != f.slabs.end() && it->first == x) { x = it->second.x1; ++it; continue; }
        const uint64_t end = (it != f.slabs.end() && it->first < r.x1) ? it->first : r.x1;
        Slab s; s.x1 = end;
        it = std::next(f.slabs.emplace(x, std::move(s)).first);
        x = end;
    }
    for (auto sit = f.slabs.lower_bound(r.x0); sit != f.slabs.end() && sit->first < r.x1; ++sit)
    {
        Slab & sl = sit->second;
        split_y(sl, r.y0);
        split_y(sl, r.y1);
        uint64_t y = r.y0;
        auto bit = sl.blocks.lower_bound(r.y0);
        while (y < r.y1)
        {
            if (bit != sl.blocks.end() && bit->first == y) { y = bit->second.y1; ++bit; continue; }
            const uint64_t end = (bit != sl.blocks.end() && bit->first < r.y1) ? bit->first : r.y1;
            Block b; b.y1 = end;
            bit = std::next(sl.blocks.emplace(y, b).first);
            y = end;
        }
    }
    f.any = true;
}

void partites(Frame & f, const Rect & r, std::vector<Partite> & out)
{
    for (auto sit = f.slabs.lower_bound(r.x0); sit != f.slabs.end() && sit->first < r.x1; ++sit)
        for (auto bit = sit->second.blocks.lower_bound(r.y0); bit != sit->second.blocks.end() && bit->first < r.y1; ++bit)
            out.push_back({sit->first, sit->second.x1, bit->first, bit->second.y1, &bit->second.st});
}

inline int64_t view_off(const View & v, uint64_t x, uint64_t y, uint64_t s)
{
    return ((int64_t) x - v.ox) + ((int64_t) y - v.oy) * (int64_t) v.ld * (int64_t) s;
}

// The same canonical partition for the resident mode, whose blocks carry only the device bits:
// an ordered map of slabs (a stream of segments can cut thousands of them), each slab's blocks
// in one sorted array (a fetch is a few binary searches over cache-resident arrays; a slab's cuts
// only grow while the first accesses of each shape arrive).
struct RBlock { uint64_t y0, y1; uint8_t st; };     // st: DEV_HOST | DEV_GPU
struct RSlab { uint64_t x1; std::vector<RBlock> b; };
struct RFrame { std::map<uint64_t, RSlab> slabs; };
struct RPartite { uint64_t x0, x1, y0, y1; uint8_t * st; };

inline size_t first_at_or_after(const std::vector<RBlock> & b, uint64_t y)
{
    return (size_t) (std::lower_bound(b.begin(), b.end(), y, [](const RBlock & q, uint64_t v) { return q.y0 < v; }) - b.begin());
}

void rsplit_y(RSlab & sl, uint64_t y)
{
    size_t i = (size_t) (std::upper_bound(sl.b.begin(), sl.b.end(), y, [](uint64_t v, const RBlock & q) { return v < q.y0; }) - sl.b.begin());
    if (i == 0) return;
    --i;
    if (sl.b[i].y0 < y && y < sl.b[i].y1)
    {
        RBlock right = sl.b[i];
        right.y0 = y;
        sl.b[i].y1 = y;
        sl.b.insert(sl.b.begin() + i + 1, right);
    }
}

// Cut the slab at `it` (which starts before x and ends after it) at x; returns the right part.
std::map<uint64_t, RSlab>::iterator rcut_x(RFrame & f, std::map<uint64_t, RSlab>::iterator it, uint64_t x)
{
    RSlab right = it->second;
    it->second.x1 = x;
    return f.slabs.emplace_hint(std::next(it), x, std::move(right));
}

// Cut the slab's blocks at y0 and y1, fill its y-gaps in [y0, y1), append its blocks there.
void rslab_fill(uint64_t x0, RSlab & sl, const Rect & r, std::vector<RPartite> & out)
{
    rsplit_y(sl, r.y0);
    rsplit_y(sl, r.y1);
    uint64_t y = r.y0;
    const size_t j0 = first_at_or_after(sl.b, r.y0);
    size_t j = j0;
    while (y < r.y1)                                   // blocks over the y-gaps of [y0, y1)
    {
        if (j < sl.b.size() && sl.b[j].y0 == y) { y = sl.b[j].y1; ++j; continue; }
        const uint64_t end = (j < sl.b.size() && sl.b[j].y0 < r.y1) ? sl.b[j].y0 : r.y1;
        sl.b.insert(sl.b.begin() + j, RBlock{y, end, 0});
        ++j;
        y = end;
    }
    for (size_t k = j0; k < j; ++k) out.push_back({x0, sl.x1, sl.b[k].y0, sl.b[k].y1, &sl.b[k].st});
}

// Insert the rect and append its blocks (x-slab by x-slab, blocks by y) to out, in one walk over
// the slabs from x0: cut the slab straddling x0, then per step either a slab starting where the
// walk is (cut at x1 if it reaches past it) or a new slab over the gap up to the next one. The
// blocks of an earlier rect of the same access stay valid: a wrapped tile's second rect ends
// left of where its first one starts, so it only cuts slabs the first one does not cover.
void rinsert(RFrame & f, const Rect & r, std::vector<RPartite> & out)
{
    auto it = f.slabs.upper_bound(r.x0);
    if (it != f.slabs.begin())
    {
        auto prev = std::prev(it);
        if (prev->first == r.x0) it = prev;
        else if (r.x0 < prev->second.x1) it = rcut_x(f, prev, r.x0);
    }
    uint64_t x = r.x0;
    while (x < r.x1)
    {
        if (it != f.slabs.end() && it->first == x)
        {
            if (it->second.x1 > r.x1) rcut_x(f, it, r.x1);
        }
        else
        {
            const uint64_t end = (it != f.slabs.end() && it->first < r.x1) ? it->first : r.x1;
            RSlab sl; sl.x1 = end;
            it = f.slabs.emplace_hint(it, x, std::move(sl));
        }
        rslab_fill(it->first, it->second, r, out);
        x = it->second.x1;
        ++it;
    }
}

// Device memory of a budget, handed out best fit from a free list: the smallest free piece that
// fits, split when what remains is at least half the request (else given whole), neighbouring
// free pieces merged again -- the reference's area allocator (src/driver/device.cc:185-280),
// with 256-byte rounding instead of 8 so that every allocation suits vector loads.
struct Arena {
    uint64_t cap = 0;
    std::map<uint64_t, uint64_t> free_at;              // offset -> size
    void init(uint64_t bytes) { cap = bytes; free_at.clear(); if (bytes) free_at[0] = bytes; }
    // offset of `size` bytes (*got: the bytes taken), or false
    bool take(uint64_t size, uint64_t & off, uint64_t & got)
    {
        size = (size + 255) & ~(uint64_t) 255;
        auto best = free_at.end();
        for (auto it = free_at.begin(); it != free_at.end(); ++it)
            if (it->second >= size && (best == free_at.end() || it->second < best->second)) best = it;
        if (best == free_at.end()) return false;
        off = best->first;
        const uint64_t rest = best->second - size;
        free_at.erase(best);
        if (rest >= size / 2 && rest > 0) { free_at[off + size] = rest; got = size; }
        else got = size + rest;
        return true;
    }
    void give(uint64_t off, uint64_t size)
    {
        auto it = free_at.emplace(off, size).first;
        auto nx = std::next(it);
        if (nx != free_at.end() && it->first + it->second == nx->first) { it->second += nx->second; free_at.erase(nx); }
        if (it != free_at.begin())
        {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) { pv->second += it->second; free_at.erase(it); }
        }
    }
    uint64_t largest() const { uint64_t m = 0; for (auto & kv : free_at) m = std::max(m, kv.second); return m; }
};

} // namespace

struct xkb_planner {
    std::map<std::pair<uint64_t, uint64_t>, std::unique_ptr<Frame>> frames;
    std::vector<uint64_t> allocs;
    // device budget (0: none): each allocation gets an offset in it; allocations not used by the
    // task being fetched are evicted, oldest first, when a new one does not fit
    uint64_t budget = 0;
    Arena arena;
    std::vector<int64_t> alloc_off;                   // offset in the budget (kept once evicted: the copies
                                                      // planned before the eviction still read it)
    std::vector<uint64_t> alloc_got;                  // bytes taken from the budget
    std::vector<uint8_t> alloc_live;                  // 0 once evicted
    int64_t cur_task = -1;
    std::vector<int32_t> pinned;                      // allocations of the current task's views
    uint64_t evicted = 0, written_back = 0;
    bool coherent_writeback = false;                  // host fetches copy from a coherent view
    std::vector<xkb_copy_t> copies;
    std::vector<Partite> scratch;
    // resident mode: one device mirror per registered host region (base -> (size, index))
    bool resident = false;
    std::map<uint64_t, std::pair<uint64_t, int32_t>> regions;
    std::map<std::pair<uint64_t, uint64_t>, std::unique_ptr<RFrame>> rframes;
    std::vector<RPartite> rscratch;
    // registration-overflow protection: the registered page intervals (start -> end, disjoint,
    // overlapping ones merged, adjacent ones not) and the pieces every new frame receives
    std::map<uint64_t, uint64_t> reg_pages;
    std::map<uint64_t, uint64_t> registered;          // start -> size
};

// The rects of the bytes [a, a + size) in a frame (interval_to_rects, access.hpp:77-139): one in
// the segment frame; in an (ld, sizeof) frame the head of the first column, the whole columns, the
// tail of the last (empty ones dropped, as the tree ignores them).
static int interval_rects(uint64_t a, uint64_t size, uint64_t ld, uint64_t s, Rect out[3])
{
    if (ld == ~0ull) { out[0] = {a, a + size, 0, 1}; return 1; }
    const uint64_t LDs = ld * s;
    const uint64_t x0 = a % LDs, x1 = std::min(x0 + size, LDs), dx10 = x1 - x0;
    const uint64_t x3 = (size - dx10) % LDs;
    const uint64_t y0 = a / LDs, y1 = y0 + 1, y3 = y0 + (size - dx10 - x3) / LDs + 2, y2 = y3 - 1;
    const Rect r[3] = {{x0, x1, y0, y1}, {0, LDs, y1, y2}, {0, x3, y2, y3}};
    int n = 0;
    for (const Rect & q : r) if (q.x0 < q.x1 && q.y0 < q.y1) out[n++] = q;
    return n;
}

static void split_frame_at(Frame & f, uint64_t a, uint64_t size)
{
    Rect r[3];
    const int n = interval_rects(a, size, f.ld, f.s, r);
    for (int k = 0; k < n; ++k) insert(f, r[k]);
}

// The access's rects in its (ld, sizeof) frame (access.hpp:204-287): one rect, or two when the
// tile wraps the leading dimension; `origin` is where each rect's view origin lies so that
// consecutive bytes of the access stay consecutive in a device allocation of ld = m
// (the wrap adjustment of fetch_access_create_allocation_views, memory-tree.hpp:1341-1347).
static int frame_rects(const xkb_access_rec_t & a, uint64_t & ld, uint64_t & s, Rect r[2], int64_t origin[2][2], int & nr)
{
    if (a.type == XKB_ACCESS_TYPE_SEGMENT)
    {
        if (a.ld <= a.addr) return xkb_set_error(XKB_EINVAL, "planner: empty segment");
        ld = ~0ull; s = 1;                          // segments: frame ld = SIZE_MAX, sizeof = 1
        r[0] = {a.addr, a.ld, 0, 1};
        origin[0][0] = (int64_t) a.addr; origin[0][1] = 0;
        nr = 1;
        return XKB_OK;
    }
    if (a.type != XKB_ACCESS_TYPE_BLAS_MATRIX || !a.ld || !a.sizeof_type || !a.m || !a.n || a.m > a.ld)
        return xkb_set_error(XKB_EINVAL, "planner: bad access");
    ld = a.ld; s = a.sizeof_type;
    const uint64_t LDs = ld * s, A = a.addr + (a.offset_n * ld + a.offset_m) * s;
    const uint64_t x0 = A % LDs, y0 = A / LDs;
    origin[0][0] = (int64_t) x0; origin[0][1] = (int64_t) y0;
    if (x0 + a.m * s <= LDs) { r[0] = {x0, x0 + a.m * s, y0, y0 + a.n}; nr = 1; return XKB_OK; }
    r[0] = {x0, LDs, y0, y0 + a.n};
    r[1] = {0, a.m * s - (LDs - x0), y0 + 1, y0 + a.n + 1};
    origin[1][0] = (int64_t) x0 - (int64_t) LDs; origin[1][1] = (int64_t) y0 + 1;
    nr = 2;
    return XKB_OK;
}

static void push_copy(xkb_planner * P, int64_t task, int64_t access, int kind, const Partite & p, uint64_t ld, uint64_t s,
                      int64_t src_alloc, int64_t src_off, int64_t src_ld, int64_t dst_alloc, int64_t dst_off, int64_t dst_ld)
{
    xkb_copy_t c;
    c.task = task; c.access = access; c.kind = kind;
    c.src_dev = kind == XKB_COPY_H2D ? 0 : 1;
    c.src_alloc = src_alloc; c.src_off = src_off; c.src_ld = src_ld;
    c.dst_dev = kind == XKB_COPY_D2H ? 0 : 1;
    c.dst_alloc = dst_alloc; c.dst_off = dst_off; c.dst_ld = dst_ld;
    if (ld == ~0ull) { c.m = (int64_t) (p.x1 - p.x0); c.n = 1; c.sizeof_type = 1; c.src_ld = c.src_ld ? c.src_ld : 0; }
    else { c.m = (int64_t) ((p.x1 - p.x0) / s); c.n = (int64_t) (p.y1 - p.y0); c.sizeof_type = (int64_t) s; }
    P->copies.push_back(c);
}

// Resident mode: every registered host region has one device mirror with the host layout
// (byte at host address h lives at mirror + (h - region base)). A block is coherent on the host
// when no device bit is set or the host bit is; on the GPU when the GPU bit is. Reads copy the
// blocks the target lacks (H2D / D2H, whole blocks, pitched like the host matrix); writes leave
// the target as the only coherent copy.
static int resident_fetch(xkb_planner * P, const xkb_access_rec_t & a, int64_t access_index, int device, xkb_view_t * view)
{
    uint64_t ld, s; Rect rr[2]; int64_t origin[2][2]; int nr = 0;
    int rc = frame_rects(a, ld, s, rr, origin, nr);
    if (rc) return rc;
    const bool seg = ld == ~0ull;
    const uint64_t stride = seg ? 0 : ld * s;
    const uint64_t begin = seg ? a.addr : a.addr + (a.offset_n * a.ld + a.offset_m) * a.sizeof_type;
    auto rit = P->regions.upper_bound(begin);
    if (rit == P->regions.begin()) return xkb_set_error(XKB_EINVAL, "planner: access at %#llx is in no registered region", (unsigned long long) begin);
    --rit;
    const uint64_t rbase = rit->first, rsize = rit->second.first;
    const int32_t region = rit->second.second;
    const uint64_t end = seg ? a.ld : begin + ((a.n - 1) * a.ld + a.m) * a.sizeof_type;
    if (begin < rbase || end > rbase + rsize) return xkb_set_error(XKB_EINVAL, "planner: access crosses the end of its region");
    if (view) { view->alloc = region; view->off = (int64_t) (begin - rbase); view->ld = seg ? (int64_t) (a.ld - a.addr) : (int64_t) a.ld; }
    std::unique_ptr<RFrame> & fp = P->rframes[{ld, s}];
    if (!fp) { fp.reset(new (std::nothrow) RFrame()); if (!fp) return xkb_set_error(XKB_ENOMEM, "planner: out of memory"); }
    P->rscratch.clear();
    for (int k = 0; k < nr; ++k) rinsert(*fp, rr[k], P->rscratch);
    const uint8_t me = device == 0 ? DEV_HOST : DEV_GPU;
    for (const RPartite & p : P->rscratch)
    {
        uint8_t & dev = *p.st;
        const bool host_ok = dev == 0 || (dev & DEV_HOST), gpu_ok = dev & DEV_GPU;
        if (a.mode & XKB_ACCESS_MODE_R && !(a.mode & XKB_ACCESS_MODE_V) && !(me == DEV_HOST ? host_ok : gpu_ok))
        {
            const uint64_t h = p.x0 + p.y0 * stride;
            xkb_copy_t c;
            c.task = a.task; c.access = access_index; c.kind = me == DEV_GPU ? XKB_COPY_H2D : XKB_COPY_D2H;
            c.src_dev = me == DEV_GPU ? 0 : 1; c.dst_dev = me == DEV_GPU ? 1 : 0;
            c.src_alloc = me == DEV_GPU ? -1 : region; c.dst_alloc = me == DEV_GPU ? region : -1;
            c.src_off = me == DEV_GPU ? (int64_t) h : (int64_t) (h - rbase);
            c.dst_off = me == DEV_GPU ? (int64_t) (h - rbase) : (int64_t) h;
            c.src_ld = c.dst_ld = seg ? 0 : (int64_t) ld;
            if (seg) { c.m = (int64_t) (p.x1 - p.x0); c.n = 1; c.sizeof_type = 1; }
            else { c.m = (int64_t) ((p.x1 - p.x0) / s); c.n = (int64_t) (p.y1 - p.y0); c.sizeof_type = (int64_t) s; }
            P->copies.push_back(c);
            dev |= (dev == 0 ? DEV_HOST : 0) | me;
        }
        if (a.mode & XKB_ACCESS_MODE_W && !(a.mode & XKB_ACCESS_MODE_V)) dev = me;
    }
    return XKB_OK;
}

// Evict allocation k: every block with a view on it loses that view; a block whose only coherent
// copy is that view (the host's is stale) is first copied back to the host (D2H, recorded for the
// fetch that needs the room). The reference only evicts blocks coherent elsewhere and gives up
// on the rest (memory-tree.hpp:1221-1324); writing them back lets any working set that fits one
// task at a time run.
static void evict(xkb_planner * P, int32_t k, int64_t task, int64_t access_index)
{
    for (auto & fk : P->frames)
    {
        Frame & f = *fk.second;
        const bool seg = f.ld == ~0ull;
        const uint64_t stride = seg ? 0 : f.ld * f.s;
        for (auto & sk : f.slabs)
            for (auto & bk : sk.second.blocks)
            {
                State & st = bk.second.st;
                int vi = -1;
                for (int q = 0; q < st.nviews; ++q) if (st.views[q].alloc == k) { vi = q; break; }
                if (vi < 0) continue;
                const View v = st.views[vi];
                if (st.coh == (1u << vi) && !(st.dev & DEV_HOST))
                {
                    Partite p{sk.first, sk.second.x1, bk.first, bk.second.y1, &st};
                    push_copy(P, task, access_index, XKB_COPY_D2H, p, f.ld, f.s, k, view_off(v, p.x0, p.y0, f.s),
                              seg ? 0 : (int64_t) v.ld, -1, (int64_t) (p.x0 + p.y0 * stride), seg ? 0 : (int64_t) f.ld);
                    st.dev |= DEV_HOST;
                    ++P->written_back;
                }
                for (int q = vi; q + 1 < st.nviews; ++q) st.views[q] = st.views[q + 1];
                --st.nviews;
                st.coh = (uint8_t) ((st.coh & ((1u << vi) - 1)) | ((st.coh >> (vi + 1)) << vi));
                if (!st.coh) st.dev = (uint8_t) ((st.dev & ~DEV_GPU) | DEV_HOST);
            }
    }
    P->arena.give((uint64_t) P->alloc_off[k], P->alloc_got[k]);
    P->alloc_live[k] = 0;
    ++P->evicted;
}

// A new allocation of `bytes` (its ordinal in *out): with a budget, room is made by evicting the
// oldest allocations the current task does not use.
static int new_allocation(xkb_planner * P, uint64_t bytes, int64_t task, int64_t access_index, int32_t * out)
{
    const int32_t id = (int32_t) P->allocs.size();
    if (P->budget)
    {
        uint64_t off = 0, got = 0;
        int32_t next = 0;
        while (!P->arena.take(bytes, off, got))
        {
            while (next < id && (!P->alloc_live[next] ||
                                 std::find(P->pinned.begin(), P->pinned.end(), next) != P->pinned.end()))
                ++next;
            if (next >= id)
                return xkb_set_error(XKB_ENOMEM, "planner: %llu bytes do not fit the device budget of %llu bytes next to the "
                                                 "current task's own allocations (largest free piece %llu)",
                                     (unsigned long long) bytes, (unsigned long long) P->budget,
                                     (unsigned long long) P->arena.largest());
            evict(P, next++, task, access_index);
        }
        P->alloc_off.push_back((int64_t) off);
        P->alloc_got.push_back(got);
        P->alloc_live.push_back(1);
    }
    P->allocs.push_back(bytes);
    *out = id;
    return XKB_OK;
}

static int fetch_one(xkb_planner * P, const xkb_access_rec_t & a, int64_t access_index, int device, xkb_view_t * view)
{
    if (P->resident) return resident_fetch(P, a, access_index, device, view);
    uint64_t ld, s; Rect rr[2]; int64_t origin[2][2]; int nr = 0;
    int rc = frame_rects(a, ld, s, rr, origin, nr);
    if (rc) return rc;
    const Rect & r = rr[0];
    std::unique_ptr<Frame> & fp = P->frames[{ld, s}];
    if (!fp)
    {
        fp.reset(new (std::nothrow) Frame());
        if (!fp) return xkb_set_error(XKB_ENOMEM, "planner: out of memory");
        fp->ld = ld; fp->s = s;
        for (const auto & kv : P->registered) split_frame_at(*fp, kv.first, kv.second);   // task.cc:88-94, 127-133
    }
    Frame & f = *fp;
    const bool seg = ld == ~0ull;
    const uint64_t host_stride = seg ? 0 : ld * s;
    auto host_addr = [&](const Partite & p) -> int64_t { return (int64_t) (p.x0 + p.y0 * host_stride); };

    if (device == 0)
    {
        if (view) { view->alloc = -1; view->off = (int64_t) a.addr; view->ld = (int64_t) a.ld; }
        if (!f.any) return XKB_OK;                 // no device access yet: nothing to write back
        for (int k = 0; k < nr; ++k) insert(f, rr[k]);
        P->scratch.clear();
        for (int k = 0; k < nr; ++k) partites(f, rr[k], P->scratch);
        for (const Partite & p : P->scratch)
        {
            State & st = *p.st;
            if (st.dev == 0 || (st.dev & DEV_HOST)) continue;
            int src = 0;
            for (int i = 1; i < st.nviews; ++i)
                if (P->allocs[st.views[src].alloc] < P->allocs[st.views[i].alloc]) src = i;
            if (P->coherent_writeback && !(st.coh & (1u << src)))
            {
                // the largest COHERENT view instead (the reference's pick may hold stale data)
                int best = -1;
                for (int i = 0; i < st.nviews; ++i)
                    if ((st.coh & (1u << i)) && (best < 0 || P->allocs[st.views[best].alloc] < P->allocs[st.views[i].alloc])) best = i;
                if (best >= 0) src = best;
            }
            const View & v = st.views[src];
            push_copy(P, a.task, access_index, XKB_COPY_D2H, p, ld, s, v.alloc, view_off(v, p.x0, p.y0, s),
                      seg ? 0 : (int64_t) v.ld, -1, host_addr(p), seg ? 0 : (int64_t) ld);
        }
        for (const Partite & p : P->scratch)
            if (p.st->dev != 0 && !(p.st->dev & DEV_HOST)) p.st->dev |= DEV_HOST;   // completion
        return XKB_OK;
    }
    if (device != 1) return xkb_set_error(XKB_EINVAL, "planner: device must be 0 (host) or 1 (GPU)");
    if ((int64_t) a.task != P->cur_task) { P->cur_task = (int64_t) a.task; P->pinned.clear(); }

    for (int k = 0; k < nr; ++k) insert(f, rr[k]);
    P->scratch.clear();
    std::vector<int> part_rect;
    for (int k = 0; k < nr; ++k)
    {
        const size_t before = P->scratch.size();
        partites(f, rr[k], P->scratch);
        part_rect.resize(P->scratch.size(), k);
        (void) before;
    }
    std::vector<Partite> & parts = P->scratch;
    // (3) oldest allocation with a view in every block, else a new one
    int32_t alloc = -1;
    {
        const State & s0 = *parts[0].st;
        for (int j = 0; j < s0.nviews && alloc < 0; ++j)
        {
            const int32_t c = s0.views[j].alloc;
            bool all = true;
            for (size_t k = 1; k < parts.size() && all; ++k)
            {
                bool has = false;
                for (int q = 0; q < parts[k].st->nviews; ++q) if (parts[k].st->views[q].alloc == c) { has = true; break; }
                all = has;
            }
            if (all) alloc = c;
        }
    }
    const uint64_t m_el = seg ? (r.x1 - r.x0) : a.m;
    if (alloc < 0)
    {
        for (const Partite & p : parts)
            if (p.st->nviews >= MAX_VIEWS)
                return xkb_set_error(XKB_ERANGE, "planner: a block would need more than %d allocations on the device "
                                                 "(the reference stops here too)", MAX_VIEWS);
        // (eviction removes views from blocks, never blocks: `parts` stays valid)
        if ((rc = new_allocation(P, seg ? (r.x1 - r.x0) : a.m * a.n * a.sizeof_type, (int64_t) a.task, access_index, &alloc)))
            return rc;
        for (size_t k = 0; k < parts.size(); ++k)
        {
            State & st = *parts[k].st;
            st.views[st.nviews++] = View{alloc, origin[part_rect[k]][0], origin[part_rect[k]][1], m_el};
        }
    }
    auto view_idx = [&](const State & st) { for (int q = 0; q < st.nviews; ++q) if (st.views[q].alloc == alloc) return q; return -1; };
    P->pinned.push_back(alloc);
    // (4) the access's device view: its corner block's view
    for (const Partite & p : parts)
        if (p.x0 == r.x0 && p.y0 == r.y0)
        {
            const View & v = p.st->views[view_idx(*p.st)];
            if (view) { view->alloc = alloc; view->off = view_off(v, r.x0, r.y0, s); view->ld = (int64_t) v.ld; }
        }
    // (5) reads: copies
    std::vector<std::pair<State *, int>> done;
    if (a.mode & XKB_ACCESS_MODE_R)
    {
        for (const Partite & p : parts)
        {
            State & st = *p.st;
            const int vi = view_idx(st);
            if (st.coh & (1u << vi)) continue;
            const View & dv = st.views[vi];
            if (st.dev & DEV_GPU)
            {
                int si = 0; while (!(st.coh & (1u << si))) ++si;
                const View & sv = st.views[si];
                push_copy(P, a.task, access_index, XKB_COPY_D2D, p, ld, s, sv.alloc, view_off(sv, p.x0, p.y0, s),
                          seg ? 0 : (int64_t) sv.ld, alloc, view_off(dv, p.x0, p.y0, s), seg ? 0 : (int64_t) dv.ld);
            }
            else
                push_copy(P, a.task, access_index, XKB_COPY_H2D, p, ld, s, -1, host_addr(p), seg ? 0 : (int64_t) ld,
                          alloc, view_off(dv, p.x0, p.y0, s), seg ? 0 : (int64_t) dv.ld);
            done.push_back({&st, vi});
        }
    }
    // (6) writes: the written view becomes the only coherent copy
    if (a.mode & XKB_ACCESS_MODE_W)
        for (const Partite & p : parts) { p.st->coh = (uint8_t) (1u << view_idx(*p.st)); p.st->dev = DEV_GPU; }
    // completion of the copies
    for (auto & d : done) { d.first->coh |= (uint8_t) (1u << d.second); d.first->dev |= DEV_GPU; }
    return XKB_OK;
}

extern "C" int xkb_planner_create(xkb_planner_t ** out)
{
    if (!out) return xkb_set_error(XKB_EINVAL, "planner_create: null output");
    *out = new (std::nothrow) xkb_planner();
    return *out ? XKB_OK : xkb_set_error(XKB_ENOMEM, "planner_create: out of memory");
}

extern "C" int xkb_planner_destroy(xkb_planner_t * P)
{
    delete P;
    return XKB_OK;
}

extern "C" int xkb_planner_fetch(xkb_planner_t * P, const xkb_access_rec_t * access, uint32_t access_index, int device,
                                 xkb_view_t * view)
{
    if (!P || !access) return xkb_set_error(XKB_EINVAL, "planner_fetch: bad arguments");
    return fetch_one(P, *access, access_index, device, view);
}

extern "C" int xkb_planner_plan(xkb_planner_t * P, const xkb_access_rec_t * recs, size_t n, int device, xkb_view_t * views)
{
    if (!P || (n && !recs)) return xkb_set_error(XKB_EINVAL, "planner_plan: bad arguments");
    size_t first = 0;
    for (size_t i = 0; i < n; ++i)
    {
        if (i == 0 || recs[i].task != recs[i - 1].task) first = i;
        int rc = fetch_one(P, recs[i], (int64_t) (i - first), device, views ? views + i : nullptr);
        if (rc) return rc;
    }
    return XKB_OK;
}

extern "C" int xkb_planner_copies(xkb_planner_t * P, xkb_copy_t * out, size_t cap, size_t * n, int take)
{
    if (!P || !n) return xkb_set_error(XKB_EINVAL, "planner_copies: bad arguments");
    *n = P->copies.size();
    if (!out) return XKB_OK;
    if (cap < P->copies.size()) return xkb_set_error(XKB_ERANGE, "planner_copies: %zu records needed", P->copies.size());
    if (!P->copies.empty()) memcpy(out, P->copies.data(), P->copies.size() * sizeof(xkb_copy_t));
    if (take) P->copies.clear();
    return XKB_OK;
}

extern "C" int xkb_planner_allocations(xkb_planner_t * P, uint64_t * sizes, size_t cap, size_t * n)
{
    if (!P || !n) return xkb_set_error(XKB_EINVAL, "planner_allocations: bad arguments");
    *n = P->allocs.size();
    if (!sizes) return XKB_OK;
    if (cap < P->allocs.size()) return xkb_set_error(XKB_ERANGE, "planner_allocations: %zu entries needed", P->allocs.size());
    if (!P->allocs.empty()) memcpy(sizes, P->allocs.data(), P->allocs.size() * sizeof(uint64_t));
    return XKB_OK;
}

extern "C" int xkb_planner_set_device_budget(xkb_planner_t * P, uint64_t bytes)
{
    if (!P || P->resident || !P->allocs.empty()) return xkb_set_error(XKB_EINVAL, "planner_set_device_budget: a fresh planner of the reference mode");
    P->budget = bytes;
    P->arena.init(bytes);
    return XKB_OK;
}

extern "C" int xkb_planner_allocation_offsets(xkb_planner_t * P, int64_t * offs, uint8_t * live, size_t cap, size_t * n)
{
    if (!P || !n || !P->budget) return xkb_set_error(XKB_EINVAL, "planner_allocation_offsets: needs a planner with a device budget");
    *n = P->alloc_off.size();
    if (!offs && !live) return XKB_OK;
    if (cap < P->alloc_off.size()) return xkb_set_error(XKB_ERANGE, "planner_allocation_offsets: %zu entries needed", P->alloc_off.size());
    if (offs && !P->alloc_off.empty()) memcpy(offs, P->alloc_off.data(), P->alloc_off.size() * sizeof(int64_t));
    if (live && !P->alloc_live.empty()) memcpy(live, P->alloc_live.data(), P->alloc_live.size());
    return XKB_OK;
}

extern "C" int xkb_planner_set_writeback_coherent(xkb_planner_t * P, int on)
{
    if (!P || P->resident) return xkb_set_error(XKB_EINVAL, "planner_set_writeback_coherent: a planner of the reference mode");
    P->coherent_writeback = on != 0;
    return XKB_OK;
}

extern "C" int xkb_planner_eviction_stats(xkb_planner_t * P, uint64_t * evicted, uint64_t * written_back)
{
    if (!P) return xkb_set_error(XKB_EINVAL, "planner_eviction_stats: null planner");
    if (evicted) *evicted = P->evicted;
    if (written_back) *written_back = P->written_back;
    return XKB_OK;
}

extern "C" int xkb_planner_create_resident(xkb_planner_t ** out)
{
    int rc = xkb_planner_create(out);
    if (rc == XKB_OK) (*out)->resident = true;
    return rc;
}

extern "C" int xkb_planner_flush_to_host(xkb_planner_t * P)
{
    if (!P || !P->resident) return xkb_set_error(XKB_EINVAL, "planner_flush_to_host: needs a resident planner");
    for (auto & kv : P->rframes)
    {
        const uint64_t ld = kv.first.first, s = kv.first.second;
        const bool seg = ld == ~0ull;
        const uint64_t stride = seg ? 0 : ld * s;
        for (auto & sk : kv.second->slabs)
        {
            const uint64_t x0 = sk.first, x1 = sk.second.x1;
            std::vector<RBlock> & b = sk.second.b;
            size_t k = 0;
            while (k < b.size())
            {
                if (!(b[k].st != 0 && !(b[k].st & DEV_HOST))) { ++k; continue; }
                // the region of the run's first block
                const uint64_t h0 = x0 + b[k].y0 * stride;
                auto rit = P->regions.upper_bound(h0);
                if (rit == P->regions.begin()) return xkb_set_error(XKB_EINVAL, "planner_flush_to_host: a block in no region");
                --rit;
                const uint64_t rbase = rit->first, rend = rit->first + rit->second.first;
                size_t e = k;
                uint64_t y1 = b[k].y1;
                b[k].st |= DEV_HOST;
                // the next blocks of the run: contiguous rows, device-only, same region
                while (e + 1 < b.size() && b[e + 1].y0 == y1 && b[e + 1].st != 0 && !(b[e + 1].st & DEV_HOST) &&
                       x0 + b[e + 1].y0 * stride >= rbase && x0 + b[e + 1].y0 * stride < rend)
                {
                    ++e;
                    y1 = b[e].y1;
                    b[e].st |= DEV_HOST;
                }
                xkb_copy_t c;
                c.task = -1; c.access = -1; c.kind = XKB_COPY_D2H;
                c.src_dev = 1; c.dst_dev = 0;
                c.src_alloc = rit->second.second; c.dst_alloc = -1;
                c.src_off = (int64_t) (h0 - rbase); c.dst_off = (int64_t) h0;
                c.src_ld = c.dst_ld = seg ? 0 : (int64_t) ld;
                if (seg) { c.m = (int64_t) (x1 - x0); c.n = 1; c.sizeof_type = 1; }
                else { c.m = (int64_t) ((x1 - x0) / s); c.n = (int64_t) (y1 - b[k].y0); c.sizeof_type = (int64_t) s; }
                P->copies.push_back(c);
                k = e + 1;
            }
        }
    }
    return XKB_OK;
}

// The page interval of [ptr, ptr + size) (pageas, include/xkrt/memory/pageas.h).
static void page_round(uint64_t ptr, uint64_t size, uint64_t & a, uint64_t & b)
{
    static const uint64_t page = (uint64_t) sysconf(_SC_PAGESIZE);
    a = ptr - ptr % page;
    const uint64_t e = ptr + size;
    b = e + (page - e % page) % page;
}

// Registered page intervals meeting [a, b), in address order.
static std::vector<std::pair<uint64_t, uint64_t>> reg_find(const xkb_planner * P, uint64_t a, uint64_t b)
{
    std::vector<std::pair<uint64_t, uint64_t>> out;
    auto it = P->reg_pages.upper_bound(a);
    if (it != P->reg_pages.begin()) { auto p = std::prev(it); if (p->second > a) out.push_back(*p); }
    for (; it != P->reg_pages.end() && it->first < b; ++it) out.push_back(*it);
    return out;
}

extern "C" int xkb_planner_register(xkb_planner_t * P, uint64_t ptr, uint64_t size)
{
    if (!P || P->resident || !size) return xkb_set_error(XKB_EINVAL, "planner_register: a planner of the reference mode and a size");
    uint64_t a, b;
    page_round(ptr, size, a, b);
    // the pieces of [a, b) not registered yet (src/memory/register.cc:121-166), each split into
    // every frame and remembered for frames made later
    const auto iv = reg_find(P, a, b);
    uint64_t p1 = a;
    for (size_t i = 0; i <= iv.size(); ++i)
    {
        const uint64_t p2 = i == iv.size() ? b : iv[i].first;
        if (p1 < p2)
        {
            P->registered[p1] = p2 - p1;
            for (auto & kv : P->frames) split_frame_at(*kv.second, p1, p2 - p1);
        }
        if (i < iv.size()) p1 = iv[i].second;
    }
    // IntervalSet::fill: merge with every interval it overlaps (adjacent ones stay apart)
    uint64_t lo = a, hi = b;
    for (const auto & v : iv) { lo = std::min(lo, v.first); hi = std::max(hi, v.second); P->reg_pages.erase(v.first); }
    P->reg_pages[lo] = hi;
    return XKB_OK;
}

extern "C" int xkb_planner_unregister(xkb_planner_t * P, uint64_t ptr, uint64_t size)
{
    if (!P || P->resident || !size) return xkb_set_error(XKB_EINVAL, "planner_unregister: a planner of the reference mode and a size");
    uint64_t a, b;
    page_round(ptr, size, a, b);
    // every registered interval it meets, whole (src/memory/register.cc:199-262), then
    // IntervalSet::unfill of [a, b)
    for (const auto & v : reg_find(P, a, b))
    {
        P->registered.erase(v.first);
        for (auto & kv : P->frames) split_frame_at(*kv.second, v.first, v.second - v.first);
        P->reg_pages.erase(v.first);
        if (v.first < a) P->reg_pages[v.first] = a;
        if (v.second > b) P->reg_pages[b] = v.second;
    }
    return XKB_OK;
}

extern "C" int xkb_planner_replace_regions(xkb_planner_t * P, uint64_t base, uint64_t size, int32_t * region)
{
    if (!P || !P->resident || !size) return xkb_set_error(XKB_EINVAL, "planner_replace_regions: needs a resident planner and a size");
    const uint64_t end = base + size;
    auto it = P->regions.lower_bound(base);          // first region starting at or after base
    if (it != P->regions.begin())
    {
        auto p = std::prev(it);
        if (p->first + p->second.first > base) return xkb_set_error(XKB_EINVAL, "planner_replace_regions: a region starts before the range");
    }
    for (auto q = it; q != P->regions.end() && q->first < end; ++q)
        if (q->first + q->second.first > end) return xkb_set_error(XKB_EINVAL, "planner_replace_regions: a region ends after the range");
    while (it != P->regions.end() && it->first < end)
        it = P->regions.erase(it);
    const int32_t id = (int32_t) P->allocs.size();
    P->allocs.push_back(size);
    P->regions[base] = {size, id};
    if (region) *region = id;
    return XKB_OK;
}

extern "C" int xkb_planner_invalidate(xkb_planner_t * P)
{
    if (!P) return xkb_set_error(XKB_EINVAL, "planner_invalidate: null planner");
    if (!P->copies.empty()) return xkb_set_error(XKB_EINVAL, "planner_invalidate: %zu planned copies not taken", P->copies.size());
    if (P->resident) { P->rframes.clear(); return XKB_OK; }       // the regions' mirrors stay, holding nothing
    P->frames.clear();
    P->allocs.clear(); P->alloc_off.clear(); P->alloc_got.clear(); P->alloc_live.clear(); P->pinned.clear();
    P->arena.init(P->budget);
    P->cur_task = -1;
    return XKB_OK;
}

extern "C" int xkb_planner_add_region(xkb_planner_t * P, uint64_t host_base, uint64_t size, int32_t * region)
{
    if (!P || !P->resident || !size) return xkb_set_error(XKB_EINVAL, "planner_add_region: needs a resident planner and a size");
    auto it = P->regions.upper_bound(host_base);
    if (it != P->regions.end() && it->first < host_base + size) return xkb_set_error(XKB_EINVAL, "planner_add_region: overlaps a region");
    if (it != P->regions.begin()) { --it; if (it->first + it->second.first > host_base) return xkb_set_error(XKB_EINVAL, "planner_add_region: overlaps a region"); }
    const int32_t id = (int32_t) P->allocs.size();
    P->allocs.push_back(size);
    P->regions[host_base] = {size, id};
    if (region) *region = id;
    return XKB_OK;
}
