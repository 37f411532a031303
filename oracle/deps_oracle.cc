// ORACLE -- test infrastructure only. Nothing in the product links, loads or runs this file;
// only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg execute it, as the
// checker. It is a CPU restatement of the reference's dependency-resolution semantics.
//
// What it restates (reference file:line):
//  * task_dependency_resolve: per task, LINK every access, then PUT every access
//    (src/task/task.cc:285-299, task_dependency_resolve_do :209-279).
//  * domains: one interval domain for segment accesses; one BLAS domain per (ld, sizeof),
//    created on the first matrix access that names it, during that task's LINK pass
//    (src/task/task.cc:153-201). A segment access also goes to every BLAS domain existing
//    at that moment (:240-259). A new BLAS domain first replays the PUT of every earlier
//    segment access, walking the interval domain's list, which is kept newest-first
//    (push_front, include/xkrt/memory/access/interval/dependency-tree.hpp:355-360).
//  * frames: matrix tile -> 1 or 2 rects of (byte row mod ld*s, column)
//    (include/xkrt/memory/access/access.hpp:204-287); segment -> [a,b) in the interval
//    domain and 3 rects in each BLAS frame (access.hpp:76-139).
//  * per point state (blas/dependency-tree.hpp:228-256, :310-355):
//      LINK(A): if (A.mode & W) and readers != {}: edge reader -> A for each reader;
//               else if writer: edge writer -> A.
//      PUT(A):  if (A.mode & W): writer = A, readers = {}; else if A.mode == R exactly:
//               readers += A.
//  * handles (include/xkrt/memory/access/handle/dependency-map.hpp:57-335): the map itself,
//    handle -> {sequential reads, concurrent writes, last sequential write}, with its LINK
//    (:186-297) and PUT (:300-332) for every concurrency (record field `reserved` >> 8:
//    0/1 sequential, 2 commutative, 4 concurrent), including the extra empty writer task that
//    LINK inserts before a concurrent write after sequential reads, or before a read after
//    concurrent writes (insert_empty_write, :93-137). An extra task is numbered in creation
//    order: just before the task whose LINK pass created it, every later task renumbered after
//    it. No task completes, so no list entry is ever popped and every extra task is kept.
//  The reference stores the tree state on nodes; its edges are the union of the per-point
//  edges, so this oracle keeps the state per elementary cell of the domain's coordinate
//  compression and reports the unique (pred task, succ task) pairs.
//
// Usage: deps_oracle <stream.bin> <out-prefix>  -> <out>.edges (sorted uint32 pairs), JSON line.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "access_stream.h"

namespace {

constexpr uint8_t MODE_R = 1, MODE_W = 2;

struct Rect { uint64_t x0, x1, y0, y1; };

// access.hpp:76-139 (interval_to_rects): 3 rects, some possibly empty.
static int segment_rects(uint64_t a, uint64_t b, uint64_t ld, uint64_t s, Rect out[3])
{
    const uint64_t LDs = ld * s, size = b - a;
    const uint64_t x0 = a % LDs, x1 = std::min(x0 + size, LDs), dx10 = x1 - x0;
    const uint64_t x3 = (size - dx10) % LDs;
    const uint64_t y0 = a / LDs, y1 = y0 + 1;
    const uint64_t y3 = y0 + (size - dx10 - x3) / LDs + 2, y2 = y3 - 1;
    Rect r[3] = {{x0, x1, y0, y1}, {0, LDs, y1, y2}, {0, x3, y2, y3}};
    int n = 0;
    for (auto & q : r) if (q.x0 < q.x1 && q.y0 < q.y1) out[n++] = q;
    return n;
}

// access.hpp:204-287 (matrix_to_rects).
static int matrix_rects(const xk_stream_rec_t & r, Rect out[2])
{
    const uint64_t s = r.sizeof_type, ld = r.ld, LDs = ld * s;
    const uint64_t A = r.addr + (r.offset_n * ld + r.offset_m) * s;
    const uint64_t x0 = A % LDs, y0 = A / LDs;
    if (x0 + r.m * s <= LDs) { out[0] = {x0, x0 + r.m * s, y0, y0 + r.n}; return 1; }
    out[0] = {x0, LDs, y0, y0 + r.n};
    out[1] = {0, r.m * s - (LDs - x0), y0 + 1, y0 + r.n + 1};
    return 2;
}

struct Op { bool link; uint32_t task; uint8_t mode; Rect rect; };

struct Domain {
    bool interval;
    uint64_t ld, s;
    std::vector<Op> ops;
};

static void add_ops(Domain & d, bool link, const xk_stream_rec_t & r)
{
    Rect rects[3];
    int n;
    if (d.interval) { rects[0] = {r.addr, r.ld, 0, 1}; n = 1; }
    else if (r.type == XK_STREAM_SEGMENT) n = segment_rects(r.addr, r.ld, d.ld, d.s, rects);
    else n = matrix_rects(r, rects);
    for (int i = 0; i < n; ++i)
    {
        Rect q = rects[i];
        if (!link && !d.interval && r.type == XK_STREAM_SEGMENT)
        {
            // A segment access keeps its own rects in the frame ld = SIZE_MAX, sizeof = 1
            // (access.hpp:479-514), i.e. [a, b) x [0, 1), and BLAS on_insert only updates
            // nodes that intersect one of the access's OWN rects
            // (blas/dependency-tree.hpp:228-256). In a BLAS frame that is the part of the
            // put rect lying in column 0 with rows in [a, b): empty whenever a >= ld*sizeof.
            q.x0 = std::max(q.x0, r.addr); q.x1 = std::min(q.x1, r.ld);
            q.y0 = std::max<uint64_t>(q.y0, 0); q.y1 = std::min<uint64_t>(q.y1, 1);
            if (q.x0 >= q.x1 || q.y0 >= q.y1) continue;
        }
        d.ops.push_back({link, r.task, r.mode, q});
    }
}

// Evaluate one domain's op sequence point-wise over its elementary cells.
static void run_domain(const Domain & d, std::vector<std::pair<uint32_t, uint32_t>> & edges)
{
    std::vector<uint64_t> xs, ys;
    for (auto & o : d.ops) { xs.push_back(o.rect.x0); xs.push_back(o.rect.x1); ys.push_back(o.rect.y0); ys.push_back(o.rect.y1); }
    std::sort(xs.begin(), xs.end()); xs.erase(std::unique(xs.begin(), xs.end()), xs.end());
    std::sort(ys.begin(), ys.end()); ys.erase(std::unique(ys.begin(), ys.end()), ys.end());
    if (xs.size() < 2 || ys.size() < 2) return;
    const size_t nx = xs.size() - 1, ny = ys.size() - 1;
    std::vector<int64_t> writer(nx * ny, -1);
    std::vector<std::vector<uint32_t>> readers(nx * ny);
    for (auto & o : d.ops)
    {
        const size_t cx0 = std::lower_bound(xs.begin(), xs.end(), o.rect.x0) - xs.begin();
        const size_t cx1 = std::lower_bound(xs.begin(), xs.end(), o.rect.x1) - xs.begin();
        const size_t cy0 = std::lower_bound(ys.begin(), ys.end(), o.rect.y0) - ys.begin();
        const size_t cy1 = std::lower_bound(ys.begin(), ys.end(), o.rect.y1) - ys.begin();
        for (size_t cy = cy0; cy < cy1; ++cy)
            for (size_t cx = cx0; cx < cx1; ++cx)
            {
                const size_t c = cy * nx + cx;
                if (o.link)
                {
                    if ((o.mode & MODE_W) && !readers[c].empty())
                        for (uint32_t p : readers[c]) edges.emplace_back(p, o.task);
                    else if (writer[c] >= 0)
                        edges.emplace_back((uint32_t) writer[c], o.task);
                }
                else if (o.mode & MODE_W) { writer[c] = o.task; readers[c].clear(); }
                else if (o.mode == MODE_R) readers[c].push_back(o.task);
            }
    }
}

// The handle map, restated with its lists (dependency-map.hpp:57-335). Task ids here are virtual:
// a stream task keeps its id, extra task k is EXTRA + k; main() renumbers at the end.
constexpr uint32_t EXTRA = 0x80000000u;
constexpr int CONCURRENT = 4;

struct HandleMap {
    struct Node { std::vector<uint32_t> seq_reads, conc_writes; int64_t last_seq_write = -1; };
    std::unordered_map<uint64_t, Node> map;
    std::vector<uint32_t> extra_owner;          // per extra task: the stream task whose LINK created it
    std::vector<std::pair<uint32_t, uint32_t>> edges;

    void link(uint64_t h, uint8_t mode, int conc, uint32_t task, uint32_t owner)
    {
        auto it = map.find(h);
        if (it == map.end()) return;
        Node & node = it->second;               // stays valid: unordered_map never moves its nodes
        bool transitive = false;
        if (!node.seq_reads.empty() && (mode & MODE_W))
        {
            if (conc == CONCURRENT) insert_empty_write(h, owner);
            else { for (uint32_t p : node.seq_reads) edges.emplace_back(p, task); transitive = true; }
        }
        if (!node.conc_writes.empty() && conc != CONCURRENT)
        {
            if (mode & MODE_W) { for (uint32_t p : node.conc_writes) edges.emplace_back(p, task); transitive = true; }
            else insert_empty_write(h, owner);
        }
        if (node.last_seq_write >= 0 && !transitive) edges.emplace_back((uint32_t) node.last_seq_write, task);
    }

    void put(uint64_t h, uint8_t mode, int conc, uint32_t task)
    {
        Node & node = map[h];
        if (mode & MODE_W)
        {
            if (conc == CONCURRENT) node.conc_writes.push_back(task);
            else { node.seq_reads.clear(); node.conc_writes.clear(); node.last_seq_write = task; }
        }
        else if (mode & MODE_R) { node.conc_writes.clear(); node.seq_reads.push_back(task); }
    }

    // An empty task with one sequential VW access of h, linked and put at once; it always has a
    // predecessor here (the non-empty list that called for it), so it is always put.
    void insert_empty_write(uint64_t h, uint32_t owner)
    {
        const uint32_t e = EXTRA + (uint32_t) extra_owner.size();
        extra_owner.push_back(owner);
        link(h, MODE_W | 4, 1, e, owner);
        put(h, MODE_W | 4, 1, e);
    }
};

} // namespace

int main(int argc, char ** argv)
{
    if (argc < 3) { fprintf(stderr, "usage: %s <stream.bin> <out-prefix>\n", argv[0]); return 2; }
    std::vector<xk_stream_rec_t> recs;
    if (xk_stream_read(argv[1], recs)) { fprintf(stderr, "cannot read %s\n", argv[1]); return 2; }
    auto t0 = std::chrono::steady_clock::now();

    // Build every domain's op sequence in the order the reference performs them.
    Domain interval{true, 0, 0, {}};
    HandleMap handles;
    std::vector<Domain> blas;
    std::map<std::pair<uint64_t, uint64_t>, size_t> blas_index;
    std::vector<size_t> segments_so_far;   // indices into recs, spawn order
    size_t ntasks = 0;
    for (size_t i = 0; i < recs.size();)
    {
        size_t j = i;
        while (j < recs.size() && recs[j].task == recs[i].task) ++j;
        ntasks = recs[i].task + 1;
        for (size_t a = i; a < j; ++a)   // LINK pass
        {
            const auto & r = recs[a];
            if (r.type == XK_STREAM_HANDLE) handles.link(r.addr, r.mode, r.reserved >> 8, r.task, r.task);
            else if (r.type == XK_STREAM_SEGMENT)
            {
                add_ops(interval, true, r);
                for (auto & d : blas) add_ops(d, true, r);
            }
            else
            {
                auto key = std::make_pair(r.ld, r.sizeof_type);
                auto it = blas_index.find(key);
                if (it == blas_index.end())
                {
                    blas.push_back({false, r.ld, r.sizeof_type, {}});
                    it = blas_index.emplace(key, blas.size() - 1).first;
                    Domain & d = blas.back();
                    for (auto k = segments_so_far.rbegin(); k != segments_so_far.rend(); ++k)
                        add_ops(d, false, recs[*k]);
                }
                add_ops(blas[it->second], true, r);
            }
        }
        for (size_t a = i; a < j; ++a)   // PUT pass
        {
            const auto & r = recs[a];
            if (r.type == XK_STREAM_HANDLE) handles.put(r.addr, r.mode, r.reserved >> 8, r.task);
            else if (r.type == XK_STREAM_SEGMENT)
            {
                add_ops(interval, false, r);
                for (auto & d : blas) add_ops(d, false, r);
                segments_so_far.push_back(a);
            }
            else
                add_ops(blas[blas_index.at({r.ld, r.sizeof_type})], false, r);
        }
        i = j;
    }

    std::vector<std::pair<uint32_t, uint32_t>> edges;
    run_domain(interval, edges);
    for (auto & d : blas) run_domain(d, edges);
    edges.insert(edges.end(), handles.edges.begin(), handles.edges.end());
    // final ids: stream task t -> t + (extra tasks created up to its own LINK pass);
    // extra task k, created in task o's LINK pass -> o + k
    const size_t nextra = handles.extra_owner.size();
    if (nextra)
    {
        std::vector<uint32_t> shift(ntasks, 0);
        for (uint32_t o : handles.extra_owner) ++shift[o];
        for (size_t t = 1; t < ntasks; ++t) shift[t] += shift[t - 1];
        auto final_id = [&](uint32_t v) {
            return v >= EXTRA ? handles.extra_owner[v - EXTRA] + (v - EXTRA) : v + shift[v];
        };
        for (auto & e : edges) e = {final_id(e.first), final_id(e.second)};
        ntasks += nextra;
    }
    const size_t cell_edges = edges.size();
    std::sort(edges.begin(), edges.end());
    edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
    auto t1 = std::chrono::steady_clock::now();

    std::vector<uint32_t> npred(ntasks, 0);
    for (auto & e : edges) ++npred[e.second];
    uint32_t maxp = 0;
    for (auto v : npred) maxp = std::max(maxp, v);

    const std::string pfx(argv[2]);
    FILE * f = fopen((pfx + ".edges").c_str(), "wb");
    for (auto & e : edges) { uint32_t v[2] = {e.first, e.second}; fwrite(v, 4, 2, f); }
    fclose(f);
    printf("{\"ntasks\": %zu, \"extra_tasks\": %zu, \"naccesses\": %zu, \"cell_edges\": %zu, \"unique_edges\": %zu, "
           "\"max_preds\": %u, \"domains\": %zu, \"resolve_s\": %.6f}\n",
           ntasks, nextra, recs.size(), cell_edges, edges.size(), maxp, blas.size() + (interval.ops.empty() ? 0 : 1),
           std::chrono::duration<double>(t1 - t0).count());
    return 0;
}
