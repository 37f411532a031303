// Concurrent-mode handle accesses (ACCESS_CONCURRENCY_CONCURRENT) as the reference's handle map
// orders them (include/xkrt/memory/access/handle/dependency-map.hpp:157-297):
//  * a concurrent write (CNC-W) depends on the last sequential write only, not on the concurrent
//    writes before it; the next sequential write depends on all of them (:225-245, :300-322);
//  * a CNC-W after sequential reads, or a read after CNC-Ws, first gets an extra empty task that
//    writes the handle (insert_empty_write, :93-137): it depends on those reads (or CNC-Ws) and
//    the access depends on it (:200-223, :247-262).
// The resolver's point-wise rule (a read depends on the last writer; a write on the reads since,
// else on the last writer) expresses this once
//  (a) each extra task is a task of its own, spawned just before the task whose access needed
//      it, with one sequential write of the handle, and
//  (b) a CNC-W is resolved as a read of the handle (resolve_mode).
// HandleMap decides (a) task by task, replaying which of the map's lists are non-empty in the
// reference's order (LINK of every access of the task, then PUT of every access). No task
// completes while it decides, as in the resolver, so an extra task always has a predecessor and
// is always kept (the reference drops one whose predecessors all completed, :124-136; its
// successors then run at once, which orders nothing differently).
// In two forms the reference's edges differ from any point-wise state's:
//  * an extra task needed by an access whose task listed the same handle before it (the
//    reference links that earlier access before the extra task exists, so the task gets the
//    extra task's predecessors as its own too): here the task depends on the extra task only,
//    which orders it after the same tasks;
//  * a concurrent access with R and without W while concurrent writes of earlier tasks are
//    pending (its PUT drops them from the map, so no later access waits for them, :325-329):
//    here later writers still wait for them, a stricter order.
// With `exact` set (edge parity with the reference) both are refused with XKB_EINVAL; without,
// they are taken with the order stated.
#ifndef XKB_HANDLES_H
#define XKB_HANDLES_H

#include <cstddef>
#include <cstdint>
#include <unordered_map>
#include <utility>
#include <vector>

namespace xkb_handles {

constexpr uint8_t MODE_R = 1, MODE_W = 2, MODE_VW = 6;
constexpr int CONCURRENT = 4;                          // ACCESS_CONCURRENCY_CONCURRENT

struct Access { uint64_t handle; uint8_t mode; int concurrency; };

// The mode the resolver sees for a handle access.
inline uint8_t resolve_mode(uint8_t mode, int concurrency)
{
    return concurrency == CONCURRENT && (mode & MODE_W) ? MODE_R : mode;
}

class Map {
public:
    // One task's handle accesses, in declaration order. Appends to `extra` the handles that get an
    // extra writer task before this task, in the order the reference creates them. On XKB_EINVAL
    // (only with `exact`; *why set) the map is left as it was before the call and `extra`
    // unchanged.
    int task(const Access * a, size_t n, bool exact, std::vector<uint64_t> & extra, const char ** why)
    {
        undo_.clear();
        const size_t extra0 = extra.size();
        for (size_t i = 0; i < n; ++i)          // LINK (dependency-map.hpp:186-297)
        {
            auto it = map_.find(a[i].handle);
            if (it == map_.end()) continue;
            Node & s = it->second;
            const bool w = a[i].mode & MODE_W, cnc = a[i].concurrency == CONCURRENT;
            if (exact && cnc && (a[i].mode & MODE_R) && !w && s.conc_writes)
                return rollback(extra, extra0, why, "a concurrent read of a handle with concurrent writes pending is not supported");
            if (!((s.seq_reads && w && cnc) || (s.conc_writes && !cnc && !w))) continue;
            for (size_t j = 0; exact && j < i; ++j)
                if (a[j].handle == a[i].handle)
                    return rollback(extra, extra0, why, "a task listing one handle twice needs an extra writer between its accesses; not supported");
            save(a[i].handle, s);
            extra.push_back(a[i].handle);
            s.seq_reads = s.conc_writes = false; // the extra task's PUT: a sequential write
        }
        for (size_t i = 0; i < n; ++i)          // PUT (:300-332); nothing fails past this point
        {
            Node & s = map_[a[i].handle];
            if (a[i].mode & MODE_W)
            {
                if (a[i].concurrency == CONCURRENT) s.conc_writes = true;
                else s.seq_reads = s.conc_writes = false;
            }
            else if (a[i].mode & MODE_R) { s.conc_writes = false; s.seq_reads = true; }
        }
        return 0;
    }

    void clear() { map_.clear(); }

private:
    struct Node { bool seq_reads = false, conc_writes = false; };
    struct Saved { uint64_t handle; Node node; };

    void save(uint64_t h, const Node & n) { undo_.push_back({h, n}); }

    int rollback(std::vector<uint64_t> & extra, size_t extra0, const char ** why, const char * text)
    {
        for (size_t k = undo_.size(); k-- > 0;) map_[undo_[k].handle] = undo_[k].node;
        undo_.clear();
        extra.resize(extra0);
        *why = text;
        return -22;                          // XKB_EINVAL
    }

    std::unordered_map<uint64_t, Node> map_;
    std::vector<Saved> undo_;
};

} // namespace xkb_handles

#endif
