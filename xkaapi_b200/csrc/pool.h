// PoolArray<T>: a growable array of trivially copyable T in anonymous memory, for the runtime's
// per-batch pools (spawned tasks, their arguments and accesses, the access records). Growing
// remaps the pages (mremap) instead of copying them, and the range is marked for transparent
// huge pages, so filling millions of entries costs one page fault per 2 MB rather than per 4 KB
// and no copy at all. Element addresses change when the array grows (stable while it does not),
// unless the array was given a fixed address-space reservation up front (reserve_fixed).
#pragma once

#include <sys/mman.h>

#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <utility>
#include <vector>

namespace xkb {

// Fixed reservations given back by released arrays are parked for the next reserve_fixed of the
// same size in this process, their pages still backed: a program that makes one runtime after
// another (xkrt_init ... xkrt_deinit in a loop) then spawns into memory that is already faulted
// in instead of faulting and zeroing it again. At most PARKED_MAX reservations are kept (the
// oldest is unmapped); XKB_POOL_CACHE=0 unmaps at release instead.
class ParkedReservations {
public:
    static ParkedReservations & get() { static ParkedReservations p; return p; }
    void * take(size_t bytes)
    {
        std::lock_guard<std::mutex> lk(mu_);
        for (size_t i = 0; i < v_.size(); ++i)
            if (v_[i].second == bytes)
            {
                void * q = v_[i].first;
                v_.erase(v_.begin() + (long) i);
                return q;
            }
        return nullptr;
    }
    void give(void * p, size_t bytes)
    {
        static const bool on = !(getenv("XKB_POOL_CACHE") && atoi(getenv("XKB_POOL_CACHE")) == 0);
        if (!on) { munmap(p, bytes); return; }
        std::lock_guard<std::mutex> lk(mu_);
        v_.push_back({p, bytes});
        if (v_.size() > PARKED_MAX) { munmap(v_.front().first, v_.front().second); v_.erase(v_.begin()); }
    }
private:
    static constexpr size_t PARKED_MAX = 8;
    std::mutex mu_;
    std::vector<std::pair<void *, size_t>> v_;
};

// The element count sits on a cache line of its own, away from the base pointer: the spawning
// thread bumps the count of three arrays per task while worker threads read their base pointers
// to convert earlier tasks, and one shared line would bounce between those cores on every spawn.
template <typename T>
class alignas(64) PoolArray {
    static_assert(std::is_trivially_copyable<T>::value, "PoolArray holds trivially copyable elements");

public:
    PoolArray() = default;
    PoolArray(const PoolArray &) = delete;
    PoolArray & operator=(const PoolArray &) = delete;
    ~PoolArray() { release(); }

    size_t size() const { return n_; }
    bool empty() const { return n_ == 0; }
    T * data() { return p_; }
    const T * data() const { return p_; }
    T & operator[](size_t i) { return p_[i]; }
    const T & operator[](size_t i) const { return p_[i]; }
    T & back() { return p_[n_ - 1]; }
    size_t capacity_bytes() const { return bytes_; }

    // n elements; new elements are NOT initialised (callers write them). false: out of memory.
    bool resize(size_t n)
    {
        if (n * sizeof(T) > bytes_ && !grow(n * sizeof(T))) return false;
        n_ = n;
        return true;
    }
    bool push_back(const T & v)
    {
        if (!resize(n_ + 1)) return false;
        p_[n_ - 1] = v;
        return true;
    }
    bool append(const T * v, size_t k)
    {
        const size_t at = n_;
        if (!resize(n_ + k)) return false;
        if (k) memcpy(p_ + at, v, k * sizeof(T));
        return true;
    }
    void clear() { n_ = 0; }
    void release()
    {
        if (p_ && fixed_) ParkedReservations::get().give(p_, bytes_);
        else if (p_) munmap(p_, bytes_);
        p_ = nullptr; n_ = 0; bytes_ = 0; fixed_ = false;
    }
    // Reserve `max_elems` elements of address space up front (pages are only backed when first
    // touched): the array then never moves, so another thread may read elements below a size it
    // was handed while this one keeps appending. false (array unchanged) if the reservation fails.
    bool reserve_fixed(size_t max_elems)
    {
        if (p_) return false;
        const size_t nb = max_elems * sizeof(T);
        void * q = ParkedReservations::get().take(nb);
        if (!q)
        {
            q = mmap(nullptr, nb, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
            if (q == MAP_FAILED) return false;
            madvise(q, nb, MADV_HUGEPAGE);
        }
        p_ = (T *) q; bytes_ = nb; fixed_ = true;
        return true;
    }
    bool fixed() const { return fixed_; }
    // Fault in (writable, contents unchanged) the pages of bytes [from, to) of the reservation
    // ahead of the writer, so that filling them later costs no page faults on the writer's
    // thread. Safe while another thread writes the array. Returns the end actually reached.
    size_t populate(size_t from, size_t to)
    {
        if (!fixed_ || from >= bytes_) return from;
        if (to > bytes_) to = bytes_;
        const size_t page = 4096;
        from &= ~(page - 1);
        to = (to + page - 1) & ~(page - 1);
        if (to > bytes_) to = bytes_;
        if (to <= from) return from;
        unsigned char * b = (unsigned char *) p_;
        if (madvise(b + from, to - from, 23 /* MADV_POPULATE_WRITE */) != 0)
            for (size_t o = from; o < to; o += page) __atomic_fetch_add(b + o, (unsigned char) 0, __ATOMIC_RELAXED);
        return to;
    }
    size_t used_bytes() const { return n_ * sizeof(T); }

private:
    bool grow(size_t need)
    {
        if (fixed_) return false;                 // a fixed reservation never moves
        constexpr size_t HUGE = size_t(2) << 20;
        size_t nb = bytes_ ? 2 * bytes_ : size_t(32) << 20;
        while (nb < need) nb *= 2;
        nb = (nb + HUGE - 1) & ~(HUGE - 1);
        void * q = p_ ? mremap(p_, bytes_, nb, MREMAP_MAYMOVE)
                      : mmap(nullptr, nb, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
        if (q == MAP_FAILED) return false;
        madvise(q, nb, MADV_HUGEPAGE);
        p_ = (T *) q; bytes_ = nb;
        return true;
    }

    T * p_ = nullptr;
    size_t bytes_ = 0;
    bool fixed_ = false;
    alignas(64) size_t n_ = 0;
};

} // namespace xkb
