// Serving loop: continuous admission of heat-diffusion task graphs under an HBM budget.
//
// A request is one heat-diffusion-2d run (grid nx x ny, tiles ts x ts, `steps` Jacobi steps,
// FP64 or FP32 storage). Requests arrive over time; the server admits a request as soon as a
// stream slot is free and its two grids fit in the HBM budget, and runs admitted requests
// concurrently, one stream each:
//  * memory: one reservation of `budget` bytes, carved by a best-fit allocator with split and
//    merge of free ranges (the reference's device allocator is a best-fit area with split/merge,
//    src/driver/device.cc:49-280);
//  * graph: the heat graph repeats every two steps (the grids swap back), so the server resolves
//    three two-step windows once per grid shape with the GPU resolver, keeps the periodic form
//    (one window's CSR plus its edges into the next window) and runs every request of that shape
//    as ONE persistent-scheduler launch over all its windows (a half window at the end for an odd
//    step count) -- its tiles and counters stay on the device from its first step to its last,
//    and consecutive steps overlap on the device;
//  * latency: from the request's arrival time to the host observing its completion event.
// The initial grid is a seeded pseudo-random U[0,1) interior with a zero boundary, produced on
// the device from (seed, cell index), so a request computes the same grid alone or in a mix.
#include "common.cuh"
#include "internal.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <memory>
#include <new>
#include <thread>
#include <tuple>
#include <vector>


#ifndef XKB_SERVE_TEAM
#define XKB_SERVE_TEAM 1                 // warps per tile task of a served graph
#endif
#ifndef XKB_SERVE_PFD
#define XKB_SERVE_PFD 4                  // L2 prefetch distance (columns) of a served graph
#endif
#ifndef XKB_SERVE_TASKS_PER_CTA
#define XKB_SERVE_TASKS_PER_CTA 2        // a graph gets one CTA per this many tasks of a step
#endif
namespace {

// ---- best-fit arena -------------------------------------------------------------------------
struct Arena {
    uint8_t * base = nullptr;
    size_t size = 0;
    std::map<size_t, size_t> free_by_off;                 // offset -> length
    std::multimap<size_t, size_t> free_by_len;            // length -> offset
    size_t used = 0;

    void init(uint8_t * b, size_t n) { base = b; size = n; free_by_off.clear(); free_by_len.clear(); add(0, n); used = 0; }
    void add(size_t off, size_t len) { free_by_off[off] = len; free_by_len.emplace(len, off); }
    void drop(size_t off, size_t len)
    {
        free_by_off.erase(off);
        auto r = free_by_len.equal_range(len);
        for (auto it = r.first; it != r.second; ++it) if (it->second == off) { free_by_len.erase(it); break; }
    }
    uint8_t * alloc(size_t n)
    {
        n = (n + 255) & ~(size_t) 255;
        auto it = free_by_len.lower_bound(n);
        if (it == free_by_len.end()) return nullptr;
        const size_t len = it->first, off = it->second;
        drop(off, len);
        if (len > n) add(off + n, len - n);
        used += n;
        return base + off;
    }
    void release(uint8_t * p, size_t n)
    {
        n = (n + 255) & ~(size_t) 255;
        size_t off = (size_t) (p - base), len = n;
        used -= n;
        auto next = free_by_off.lower_bound(off);
        if (next != free_by_off.end() && next->first == off + len) { const size_t l = next->second; drop(next->first, l); len += l; }
        auto prev = free_by_off.lower_bound(off);
        if (prev != free_by_off.begin())
        {
            --prev;
            if (prev->first + prev->second == off) { const size_t po = prev->first, pl = prev->second; drop(po, pl); off = po; len += pl; }
        }
        add(off, len);
    }
};

__device__ __forceinline__ uint64_t splitmix(uint64_t x)
{
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

template <typename T>
__global__ void init_grid_kernel(T * a, T * b, int64_t nx, int64_t ny, uint64_t seed)
{
    const int64_t n = nx * ny;
    for (int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t) gridDim.x * blockDim.x)
    {
        const int64_t i = k % nx, j = k / nx;
        T v = 0;
        if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1)
            v = (T) ((double) (splitmix(seed * 0x100000001b3ull + (uint64_t) k) >> 11) * (1.0 / 9007199254740992.0));
        a[k] = v; b[k] = v;
    }
}

struct Shape {
    int64_t nx, ny, ts;
    int f32;
    bool operator<(const Shape & o) const { return std::tie(nx, ny, ts, f32) < std::tie(o.nx, o.ny, o.ts, o.f32); }
};

struct Window {                 // the periodic form of a shape's graph (window = two steps)
    xkb_resolver_t * res = nullptr;
    xkb_periodic_graph_t g{};
    uint64_t per_step = 0;
    bool seed_later = false;    // a task of a later window has no predecessor
    ~Window() { if (res) xkb_resolver_destroy(res); }
};

void heat_records(const Shape & s, int steps, uint64_t a, uint64_t b, std::vector<xkb_access_rec_t> & out)
{
    const int64_t esz = s.f32 ? 4 : 8;
    const int64_t ntx = (s.nx + s.ts - 1) / s.ts, nty = (s.ny + s.ts - 1) / s.ts;
    out.clear();
    uint32_t t = 0;
    for (int st = 0; st < steps; ++st)
    {
        const uint64_t src = st % 2 == 0 ? a : b, dst = st % 2 == 0 ? b : a;
        for (int64_t tx = 0; tx < ntx; ++tx)
            for (int64_t ty = 0; ty < nty; ++ty, ++t)
            {
                const int64_t x = tx * s.ts, y = ty * s.ts;
                const int64_t rx0 = std::max<int64_t>(x - 1, 0), ry0 = std::max<int64_t>(y - 1, 0);
                const int64_t rx1 = std::min<int64_t>(x + s.ts + 1, s.nx), ry1 = std::min<int64_t>(y + s.ts + 1, s.ny);
                const int64_t wx0 = std::max<int64_t>(x, 1), wy0 = std::max<int64_t>(y, 1);
                const int64_t wx1 = std::min<int64_t>(x + s.ts, s.nx - 1), wy1 = std::min<int64_t>(y + s.ts, s.ny - 1);
                out.push_back({t, XKB_ACCESS_TYPE_BLAS_MATRIX, XKB_ACCESS_MODE_R, 0, src, (uint64_t) s.nx, (uint64_t) rx0,
                               (uint64_t) ry0, (uint64_t) (rx1 - rx0), (uint64_t) (ry1 - ry0), (uint64_t) esz});
                if (wx1 > wx0 && wy1 > wy0)
                    out.push_back({t, XKB_ACCESS_TYPE_BLAS_MATRIX, XKB_ACCESS_MODE_W, 0, dst, (uint64_t) s.nx, (uint64_t) wx0,
                                   (uint64_t) wy0, (uint64_t) (wx1 - wx0), (uint64_t) (wy1 - wy0), (uint64_t) esz});
            }
    }
}

void heat_descs(const Shape & s, int steps, uint64_t a, uint64_t b, double c, std::vector<xkb_task_desc_t> & out)
{
    const int64_t ntx = (s.nx + s.ts - 1) / s.ts, nty = (s.ny + s.ts - 1) / s.ts;
    out.clear();
    for (int st = 0; st < steps; ++st)
        for (int64_t tx = 0; tx < ntx; ++tx)
            for (int64_t ty = 0; ty < nty; ++ty)
            {
                xkb_task_desc_t d;
                memset(&d, 0, sizeof(d));
                d.kind = s.f32 ? XKB_TASK_HEAT_F32 : XKB_TASK_HEAT_F64;
                d.u.heat.src = st % 2 == 0 ? a : b;
                d.u.heat.dst = st % 2 == 0 ? b : a;
                d.u.heat.ld = s.nx; d.u.heat.nx = (int32_t) s.nx; d.u.heat.ny = (int32_t) s.ny;
                d.u.heat.x0 = (int32_t) (tx * s.ts); d.u.heat.x1 = (int32_t) std::min<int64_t>(tx * s.ts + s.ts, s.nx);
                d.u.heat.y0 = (int32_t) (ty * s.ts); d.u.heat.y1 = (int32_t) std::min<int64_t>(ty * s.ts + s.ts, s.ny);
                d.u.heat.c = c;
                out.push_back(d);
            }
}

struct Slot {
    cudaStream_t stream = nullptr;
    xkb_sched_t * sch = nullptr;
    cudaEvent_t done = nullptr;
    long req = -1;
    // device loop: phase 0 free, 1 on the device, 2 result copy in flight; page-locked staging
    int phase = 0;
    uint32_t gen = 0;
    xkb_task_desc_t * hdesc = nullptr; size_t hdesc_cap = 0;
    XkbSrvSlot * hslot = nullptr;
    XkbSrvCtl * hctl = nullptr;
    unsigned * hstate = nullptr;
    void * hinput = nullptr; size_t hinput_cap = 0;
};

} // namespace

struct xkb_server {
    xkb_server_cfg_t cfg{};
    Arena arena;
    void * reservation = nullptr;
    std::vector<Slot> slots;
    std::map<Shape, std::unique_ptr<Window>> windows;
    int max_ctas = 296;
    cudaStream_t aux = nullptr;            // graph resolution, never waits behind a running request
    int dev = 0;
    // device loop: slot records and counters (device), the kernel's stream, status, per-slot
    // completion words in mapped host memory, and the page-locked "no more requests" word
    XkbSrvSlot * d_slots = nullptr;
    XkbSrvCtl * d_ctl = nullptr;
    unsigned * d_status = nullptr;
    unsigned * h_done = nullptr;
    unsigned * h_stop = nullptr;
    cudaStream_t kstream = nullptr;
    uint32_t gen = 0;
};

static int get_window(xkb_server * S, const Shape & s, Window ** out)
{
    auto it = S->windows.find(s);
    if (it != S->windows.end()) { *out = it->second.get(); return XKB_OK; }
    std::unique_ptr<Window> w(new (std::nothrow) Window());
    if (!w) return xkb_set_error(XKB_ENOMEM, "server: out of host memory");
    int rc = xkb_resolver_create(&w->res, S->aux);
    if (rc) return rc;
    // the structure of the graph does not depend on where the two grids live; resolve three
    // two-step windows on two distinct, aligned stand-in addresses
    const uint64_t esz = s.f32 ? 4 : 8, grid = (uint64_t) s.nx * s.ny * esz;
    const uint64_t a = 1ull << 40, b = a + ((grid + (1ull << 21)) & ~((1ull << 21) - 1));
    std::vector<xkb_access_rec_t> recs;
    heat_records(s, 6, a, b, recs);
    w->per_step = (uint64_t) ((s.nx + s.ts - 1) / s.ts) * ((s.ny + s.ts - 1) / s.ts);
    if ((rc = xkb_resolver_add(w->res, recs.data(), recs.size()))) return rc;
    if ((rc = xkb_resolver_periodic(w->res, 2 * w->per_step, &w->g))) return rc;
    {
        std::vector<uint32_t> nn(2 * w->per_step);
        XKB_CUDA_TRY(cudaMemcpy(nn.data(), w->g.npred_next, nn.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        w->seed_later = std::find(nn.begin(), nn.end(), 0u) != nn.end();
    }
    *out = w.get();
    S->windows[s] = std::move(w);
    return XKB_OK;
}

extern "C" int xkb_server_create(xkb_server_t ** out, const xkb_server_cfg_t * cfg)
{
    if (!out || !cfg || cfg->slots <= 0 || cfg->slots > 64 || cfg->budget_bytes < (1u << 20))
        return xkb_set_error(XKB_EINVAL, "server_create: bad configuration");
    std::unique_ptr<xkb_server> S(new (std::nothrow) xkb_server());
    if (!S) return xkb_set_error(XKB_ENOMEM, "server_create: out of host memory");
    S->cfg = *cfg;
    XKB_CUDA_TRY(cudaGetDevice(&S->dev));
    cudaError_t e = cudaMalloc(&S->reservation, cfg->budget_bytes);
    if (e != cudaSuccess) return xkb_set_cuda_error(e);
    S->arena.init((uint8_t *) S->reservation, cfg->budget_bytes);
    XKB_CUDA_TRY(cudaStreamCreateWithFlags(&S->aux, cudaStreamNonBlocking));
    S->slots.resize(cfg->slots);
    for (Slot & sl : S->slots)
    {
        XKB_CUDA_TRY(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking));
        XKB_CUDA_TRY(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
        int rc;
        if ((rc = xkb_sched_create(&sl.sch, sl.stream))) return rc;
        // warps per tile and L2 prefetch distance for many graphs side by side, each with a CTA
        // budget from its width (one warp per tile, 4 columns ahead, a CTA per two tasks of a
        // step: 3.1 TB/s capacity and p99 155 ms at 80 % load on 1000 graphs; two warps per tile
        // and 8 columns ahead: 1.9 TB/s; a CTA per four or eight tasks: higher closed-loop
        // capacity that the open-loop trace then overloads)
        if ((rc = xkb_sched_set_team(sl.sch, XKB_SERVE_TEAM)) || (rc = xkb_sched_set_prefetch(sl.sch, XKB_SERVE_PFD))) return rc;
    }
    int sms = 148, per = 2;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S->dev);
    S->max_ctas = cfg->ctas_per_graph > 0 ? cfg->ctas_per_graph : sms * per;
    *out = S.release();
    return XKB_OK;
}

extern "C" int xkb_server_destroy(xkb_server_t * S)
{
    if (!S) return XKB_OK;
    for (Slot & sl : S->slots)
    {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        if (sl.sch) xkb_sched_destroy(sl.sch);
        if (sl.done) cudaEventDestroy(sl.done);
    }
    S->windows.clear();
    for (Slot & sl : S->slots)
    {
        if (sl.stream) cudaStreamDestroy(sl.stream);
        if (sl.hdesc) cudaFreeHost(sl.hdesc);
        if (sl.hslot) cudaFreeHost(sl.hslot);
        if (sl.hinput) cudaFreeHost(sl.hinput);
    }
    if (S->d_slots) cudaFree(S->d_slots);
    if (S->d_ctl) cudaFree(S->d_ctl);
    if (S->d_status) cudaFree(S->d_status);
    if (S->h_done) cudaFreeHost(S->h_done);
    if (S->kstream) cudaStreamDestroy(S->kstream);
    if (S->aux) cudaStreamDestroy(S->aux);
    if (S->reservation) cudaFree(S->reservation);
    delete S;
    return XKB_OK;
}

// Launch every step of an admitted request on its slot's stream: one persistent launch over all
// its windows. The slot is idle here, so the descriptor upload (which waits for the stream) is
// done first; the rest only enqueues work.
static int launch_request(xkb_server * S, Slot & sl, xkb_request_t & q, uint8_t * grids)
{
    const Shape s{q.nx, q.ny, q.ts, q.f32};
    const uint64_t esz = q.f32 ? 4 : 8, grid = (uint64_t) q.nx * q.ny * esz;
    uint8_t * a = grids, * b = grids + ((grid + 255) & ~(uint64_t) 255);
    int rc;
    Window * w = nullptr;
    if (q.steps > 0)
    {
        if ((rc = get_window(S, s, &w))) return rc;
        std::vector<xkb_task_desc_t> d;
        heat_descs(s, 2, (uint64_t) a, (uint64_t) b, q.c, d);
        if ((rc = xkb_sched_set_tasks(sl.sch, d.data(), d.size()))) return rc;
        // a small graph cannot use many CTAs; leave the SMs to the requests beside it
        int ctas = (int) std::min<uint64_t>((uint64_t) S->max_ctas, std::max<uint64_t>(4, w->per_step / XKB_SERVE_TASKS_PER_CTA));
        if ((rc = xkb_sched_set_grid(sl.sch, ctas))) return rc;
    }
    if (q.input)
    {
        XKB_CUDA_TRY(cudaMemcpyAsync(a, q.input, grid, cudaMemcpyHostToDevice, sl.stream));
        XKB_CUDA_TRY(cudaMemcpyAsync(b, a, grid, cudaMemcpyDeviceToDevice, sl.stream));
    }
    else if (q.f32) init_grid_kernel<float><<<1184, 256, 0, sl.stream>>>((float *) a, (float *) b, q.nx, q.ny, q.seed);
    else init_grid_kernel<double><<<1184, 256, 0, sl.stream>>>((double *) a, (double *) b, q.nx, q.ny, q.seed);
    XKB_CUDA_TRY(cudaGetLastError());
    if (w)
    {
        const uint32_t repeats = (uint32_t) ((q.steps + 1) / 2);
        const uint32_t tail = (uint32_t) (q.steps % 2 ? w->per_step : 2 * w->per_step);
        if ((rc = xkb_sched_run_periodic(sl.sch, &w->g, repeats, tail))) return rc;
    }
    if (q.result)          // optional copy of the final grid for the caller
    {
        const uint8_t * fin = q.steps % 2 == 0 ? a : b;
        XKB_CUDA_TRY(cudaMemcpyAsync(q.result, fin, grid, cudaMemcpyDeviceToHost, sl.stream));
    }
    XKB_CUDA_TRY(cudaEventRecord(sl.done, sl.stream));
    return XKB_OK;
}

static int check_requests(xkb_server * S, const xkb_request_t * reqs, size_t n)
{
    for (size_t i = 0; i < n; ++i)
    {
        const xkb_request_t & q = reqs[i];
        if (q.nx < 3 || q.ny < 3 || q.ts <= 0 || q.steps < 0 || (q.f32 != 0 && q.f32 != 1) || q.nx > INT32_MAX || q.ny > INT32_MAX)
            return xkb_set_error(XKB_EINVAL, "server_run: request %zu is malformed", i);
        if (i && q.arrival_s < reqs[i - 1].arrival_s)
            return xkb_set_error(XKB_EINVAL, "server_run: requests must be sorted by arrival time");
        const uint64_t esz = q.f32 ? 4 : 8, g = (((uint64_t) q.nx * q.ny * esz + 255) & ~(uint64_t) 255) * 2;
        if (g > S->cfg.budget_bytes) return xkb_set_error(XKB_ERANGE, "server_run: request %zu needs %llu bytes, over the budget", i, (unsigned long long) g);
    }
    return XKB_OK;
}

// The seeded initial grid of a request, built on the host (the formula of init_grid_kernel).
static void seeded_host_grid(const xkb_request_t & q, void * out)
{
    for (int64_t k = 0; k < q.nx * q.ny; ++k)
    {
        const int64_t i = k % q.nx, j = k / q.nx;
        double v = 0;
        if (i > 0 && i < q.nx - 1 && j > 0 && j < q.ny - 1)
        {
            uint64_t x = q.seed * 0x100000001b3ull + (uint64_t) k + 0x9e3779b97f4a7c15ull;
            x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
            x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
            x ^= x >> 31;
            v = (double) (x >> 11) * (1.0 / 9007199254740992.0);
        }
        if (q.f32) ((float *) out)[k] = (float) v;
        else ((double *) out)[k] = v;
    }
}

static int server_run_launches(xkb_server * S, xkb_request_t * reqs, size_t n)
{
    std::vector<uint8_t *> mem(n, nullptr);
    std::vector<uint64_t> need(n);
    for (size_t i = 0; i < n; ++i)
    {
        const uint64_t esz = reqs[i].f32 ? 4 : 8;
        need[i] = (((uint64_t) reqs[i].nx * reqs[i].ny * esz + 255) & ~(uint64_t) 255) * 2;
    }
    const auto t0 = std::chrono::steady_clock::now();
    auto now = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    size_t next = 0, done = 0;
    const double deadline = S->cfg.max_seconds > 0 ? S->cfg.max_seconds : 600.0;
    while (done < n)
    {
        bool progressed = false;
        // completions
        for (Slot & sl : S->slots)
        {
            if (sl.req < 0) continue;
            cudaError_t e = cudaEventQuery(sl.done);
            if (e == cudaErrorNotReady) continue;
            if (e != cudaSuccess) return xkb_set_cuda_error(e);
            uint64_t ran = 0;
            int rc = xkb_sched_wait(sl.sch, &ran);
            if (rc) return rc;
            xkb_request_t & q = reqs[sl.req];
            q.finish_s = now();
            S->arena.release(mem[sl.req], need[sl.req]);
            sl.req = -1; ++done; progressed = true;
        }
        // admissions in arrival order (FIFO: a request that does not fit blocks the ones behind it)
        while (next < n && reqs[next].arrival_s <= now())
        {
            Slot * free_slot = nullptr;
            for (Slot & sl : S->slots) if (sl.req < 0) { free_slot = &sl; break; }
            if (!free_slot) break;
            uint8_t * m = S->arena.alloc(need[next]);
            if (!m) break;
            mem[next] = m;
            free_slot->req = (long) next;
            reqs[next].start_s = now();
            int rc = launch_request(S, *free_slot, reqs[next], m);
            if (rc) return rc;
            ++next; progressed = true;
        }
        if (now() > deadline) return xkb_set_error(XKB_ETIMEDOUT, "server_run: %zu of %zu requests done after %.0f s", done, n, deadline);
        if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    return XKB_OK;
}

// ---- the device-resident loop ---------------------------------------------------------------

// Device bytes of a request: two grids, the window's descriptors, wait counters and queue slots.
static uint64_t device_need(const xkb_request_t & q, uint64_t per_step)
{
    const uint64_t esz = q.f32 ? 4 : 8, grid = ((uint64_t) q.nx * q.ny * esz + 255) & ~(uint64_t) 255;
    const uint64_t ntasks = (uint64_t) q.steps * per_step;
    return 2 * grid + ((2 * per_step * sizeof(xkb_task_desc_t) + 255) & ~(uint64_t) 255) + 2 * ((ntasks * 4 + 255) & ~(uint64_t) 255);
}

template <typename T>
static int grow_pinned(T *& p, size_t & cap, size_t bytes)
{
    if (bytes <= cap && p) return XKB_OK;
    if (p) { cudaFreeHost(p); p = nullptr; cap = 0; }
    XKB_CUDA_TRY(cudaHostAlloc((void **) &p, bytes, cudaHostAllocDefault));
    cap = bytes;
    return XKB_OK;
}

// Admit request q into slot k: its input in, its descriptors and slot record, then the state
// word -- all copies on the slot's stream, in that order; the kernel does the rest.
static int admit(xkb_server * S, int k, xkb_request_t & q, uint8_t * mem, Window * w)
{
    Slot & sl = S->slots[k];
    const uint64_t esz = q.f32 ? 4 : 8, bytes = (uint64_t) q.nx * q.ny * esz, grid = (bytes + 255) & ~(uint64_t) 255;
    uint8_t * a = mem, * b = mem + grid;
    XKB_CUDA_TRY(cudaStreamSynchronize(sl.stream));              // staging buffers of the previous request are free
    const void * in = q.input;
    if (!in)
    {
        if (sl.hinput_cap < bytes) return xkb_set_error(XKB_EINVAL, "server_run: input staging was not sized for the trace");
        seeded_host_grid(q, sl.hinput);
        in = sl.hinput;
    }
    XKB_CUDA_TRY(cudaMemcpyAsync(a, in, bytes, cudaMemcpyHostToDevice, sl.stream));
    if (q.steps == 0)
    {
        // nothing to run: the input is the result
        if (q.result) XKB_CUDA_TRY(cudaMemcpyAsync(q.result, a, bytes, cudaMemcpyDeviceToHost, sl.stream));
        XKB_CUDA_TRY(cudaEventRecord(sl.done, sl.stream));
        sl.phase = 2;
        return XKB_OK;
    }
    const Shape sh{q.nx, q.ny, q.ts, q.f32};
    const uint64_t period = 2 * w->per_step, ntasks = (uint64_t) q.steps * w->per_step;
    uint8_t * desc = b + grid;
    int * wc = (int *) (desc + ((period * sizeof(xkb_task_desc_t) + 255) & ~(uint64_t) 255));
    int * queue = (int *) ((uint8_t *) wc + ((ntasks * 4 + 255) & ~(uint64_t) 255));
    std::vector<xkb_task_desc_t> d;
    heat_descs(sh, 2, (uint64_t) a, (uint64_t) b, q.c, d);
    if (sl.hdesc_cap < d.size() * sizeof(xkb_task_desc_t)) return xkb_set_error(XKB_EINVAL, "server_run: descriptor staging was not sized for the trace");
    memcpy(sl.hdesc, d.data(), d.size() * sizeof(xkb_task_desc_t));
    XKB_CUDA_TRY(cudaMemcpyAsync(desc, sl.hdesc, d.size() * sizeof(xkb_task_desc_t), cudaMemcpyHostToDevice, sl.stream));
    XkbSrvSlot & r = *sl.hslot;
    r.tasks = (const xkb_task_desc_t *) desc;
    r.succ_ptr = w->g.succ_ptr; r.succ = w->g.succ; r.xsucc_ptr = w->g.xsucc_ptr; r.xsucc = w->g.xsucc;
    r.npred_first = w->g.npred_first; r.npred_next = w->g.npred_next;
    r.wc = wc; r.queue = queue;
    r.copy_src = a; r.copy_dst = b; r.copy_bytes = bytes;
    r.period = (uint32_t) period; r.ntasks = (uint32_t) ntasks;
    r.nchunks = (uint32_t) std::max<uint64_t>({1, (ntasks + XKB_SRV_CHUNK - 1) / XKB_SRV_CHUNK,
                                              (bytes + XKB_SRV_COPY_CHUNK - 1) / XKB_SRV_COPY_CHUNK});
    r.gen = sl.gen = ++S->gen;
    r.seed_later = w->seed_later ? 1u : 0u;
    r.pfd = XKB_SERVE_PFD;
    *sl.hctl = XkbSrvCtl{};                                       // state 0 until the word below
    *sl.hstate = 1u;
    XKB_CUDA_TRY(cudaMemcpyAsync(S->d_slots + k, sl.hslot, sizeof(XkbSrvSlot), cudaMemcpyHostToDevice, sl.stream));
    XKB_CUDA_TRY(cudaMemcpyAsync(S->d_ctl + k, sl.hctl, sizeof(XkbSrvCtl), cudaMemcpyHostToDevice, sl.stream));
    XKB_CUDA_TRY(cudaMemcpyAsync(&S->d_ctl[k].state, sl.hstate, sizeof(unsigned), cudaMemcpyHostToDevice, sl.stream));
    sl.phase = 1;
    return XKB_OK;
}

static int server_run_device(xkb_server * S, xkb_request_t * reqs, size_t n)
{
    int rc;
    const int ns = (int) S->slots.size();
    // (1) the graph of every shape, before the kernel holds the SMs
    std::vector<Window *> win(n, nullptr);
    for (size_t i = 0; i < n; ++i)
        if (reqs[i].steps > 0 && (rc = get_window(S, Shape{reqs[i].nx, reqs[i].ny, reqs[i].ts, reqs[i].f32}, &win[i]))) return rc;
    XKB_CUDA_TRY(cudaStreamSynchronize(S->aux));
    std::vector<uint64_t> need(n);
    for (size_t i = 0; i < n; ++i)
    {
        need[i] = device_need(reqs[i], win[i] ? win[i]->per_step : 0);
        if (need[i] > S->cfg.budget_bytes)
            return xkb_set_error(XKB_ERANGE, "server_run: request %zu needs %llu bytes, over the budget", i, (unsigned long long) need[i]);
    }
    // (2) control memory, made once
    if (!S->d_slots)
    {
        XKB_CUDA_TRY(cudaMalloc(&S->d_slots, ns * sizeof(XkbSrvSlot)));
        XKB_CUDA_TRY(cudaMalloc(&S->d_ctl, ns * sizeof(XkbSrvCtl)));
        XKB_CUDA_TRY(cudaMalloc(&S->d_status, 4 * sizeof(unsigned)));
        XKB_CUDA_TRY(cudaHostAlloc((void **) &S->h_done, (ns + 1) * sizeof(unsigned), cudaHostAllocMapped));
        S->h_stop = S->h_done + ns;
        XKB_CUDA_TRY(cudaStreamCreateWithFlags(&S->kstream, cudaStreamNonBlocking));
        for (Slot & sl : S->slots)
        {
            XKB_CUDA_TRY(cudaHostAlloc((void **) &sl.hslot, sizeof(XkbSrvSlot) + sizeof(XkbSrvCtl) + 64, cudaHostAllocDefault));
            sl.hctl = (XkbSrvCtl *) (sl.hslot + 1);
            sl.hstate = (unsigned *) (sl.hctl + 1);
        }
    }
    // page-locked staging sized for the whole trace up front: no host allocation or release runs
    // while the kernel does (releasing page-locked memory may wait for the device)
    {
        size_t desc_bytes = 0, input_bytes = 0;
        for (size_t i = 0; i < n; ++i)
        {
            if (win[i]) desc_bytes = std::max<size_t>(desc_bytes, 2 * win[i]->per_step * sizeof(xkb_task_desc_t));
            if (!reqs[i].input) input_bytes = std::max<size_t>(input_bytes, (size_t) (reqs[i].nx * reqs[i].ny * (reqs[i].f32 ? 4 : 8)));
        }
        for (Slot & sl : S->slots)
        {
            if (desc_bytes && (rc = grow_pinned(sl.hdesc, sl.hdesc_cap, desc_bytes))) return rc;
            if (input_bytes && (rc = grow_pinned(sl.hinput, sl.hinput_cap, input_bytes))) return rc;
        }
    }
    XKB_CUDA_TRY(cudaMemsetAsync(S->d_ctl, 0, ns * sizeof(XkbSrvCtl), S->kstream));
    XKB_CUDA_TRY(cudaMemsetAsync(S->d_status, 0, 4 * sizeof(unsigned), S->kstream));
    for (int k = 0; k < ns; ++k) ((volatile unsigned *) S->h_done)[k] = 0;
    XKB_CUDA_TRY(cudaStreamSynchronize(S->kstream));
    for (Slot & sl : S->slots) { sl.req = -1; sl.phase = 0; }
    // (3) the kernel, for the whole trace
    const double limit = S->cfg.max_seconds > 0 ? S->cfg.max_seconds : 600.0;
    XkbSrvArgs ka;
    ka.slots = S->d_slots; ka.ctl = S->d_ctl; ka.nslots = ns;
    unsigned * dptr = nullptr;
    XKB_CUDA_TRY(cudaHostGetDevicePointer((void **) &dptr, S->h_done, 0));
    ka.host_done = dptr;
    ka.status = S->d_status;
    ka.run_ns = (uint64_t) (limit * 1e9);
    ka.timeout_ns = (uint64_t) (std::min(limit, 10.0) * 1e9);
    int sms = 148, per = 2;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S->dev);
    const int grid = S->cfg.ctas_per_graph > 0 ? S->cfg.ctas_per_graph : sms * per;
    if ((rc = xkb_internal_server_launch(ka, grid, XKB_SERVE_TEAM, S->kstream))) return rc;

    // (4) admissions and completions
    std::vector<uint8_t *> mem(n, nullptr);
    const auto t0 = std::chrono::steady_clock::now();
    auto now = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    size_t next = 0, done = 0;
    rc = XKB_OK;
    while (done < n && rc == XKB_OK)
    {
        bool progressed = false;
        for (int k = 0; k < ns && rc == XKB_OK; ++k)
        {
            Slot & sl = S->slots[k];
            if (sl.req < 0) continue;
            xkb_request_t & q = reqs[sl.req];
            if (sl.phase == 1 && ((volatile unsigned *) S->h_done)[k] == sl.gen)
            {
                // the last task ended: copy the result out behind it
                const uint64_t esz = q.f32 ? 4 : 8, bytes = (uint64_t) q.nx * q.ny * esz, g = (bytes + 255) & ~(uint64_t) 255;
                const uint8_t * fin = mem[sl.req] + (q.steps % 2 ? g : 0);
                if (q.result && cudaMemcpyAsync(q.result, fin, bytes, cudaMemcpyDeviceToHost, sl.stream) != cudaSuccess)
                    rc = xkb_set_cuda_error(cudaGetLastError());
                else if (cudaEventRecord(sl.done, sl.stream) != cudaSuccess) rc = xkb_set_cuda_error(cudaGetLastError());
                sl.phase = 2;
                progressed = true;
            }
            if (sl.phase == 2)
            {
                const cudaError_t e = cudaEventQuery(sl.done);
                if (e == cudaErrorNotReady) continue;
                if (e != cudaSuccess) { rc = xkb_set_cuda_error(e); break; }
                q.finish_s = now();
                S->arena.release(mem[sl.req], need[sl.req]);
                sl.req = -1; sl.phase = 0; ++done; progressed = true;
            }
        }
        while (rc == XKB_OK && next < n && reqs[next].arrival_s <= now())
        {
            int k = 0;
            while (k < ns && S->slots[k].req >= 0) ++k;
            if (k == ns) break;
            uint8_t * m = S->arena.alloc(need[next]);
            if (!m) break;
            mem[next] = m;
            S->slots[k].req = (long) next;
            reqs[next].start_s = now();
            rc = admit(S, k, reqs[next], m, win[next]);
            ++next; progressed = true;
        }
        if (rc == XKB_OK && now() > limit) rc = xkb_set_error(XKB_ETIMEDOUT, "server_run: %zu of %zu requests done after %.0f s", done, n, limit);
        if (rc == XKB_OK && !progressed)
        {
            // a kernel that stopped early (its own time limit) ends the loop
            if (cudaStreamQuery(S->kstream) == cudaSuccess)
            {
                unsigned st[2] = {0, 0};
                cudaMemcpy(st, S->d_status, sizeof(st), cudaMemcpyDeviceToHost);
                rc = xkb_set_error(st[0] ? -(int) st[0] : XKB_ECUDA, "server_run: the serving kernel ended with %zu of %zu requests done", done, n);
                break;
            }
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
    // (5) no more requests: the kernel's teams stop (the word goes to device memory through a
    // copy on the control stream, so idle teams poll L2, not host memory)
    *S->h_stop = rc == XKB_OK ? 1u : 2u;
    if (cudaMemcpyAsync(S->d_status + 2, S->h_stop, sizeof(unsigned), cudaMemcpyHostToDevice, S->aux) == cudaSuccess)
        cudaStreamSynchronize(S->aux);
    const cudaError_t e = cudaStreamSynchronize(S->kstream);
    for (Slot & sl : S->slots) cudaStreamSynchronize(sl.stream);
    if (rc) return rc;
    if (e != cudaSuccess) return xkb_set_cuda_error(e);
    unsigned st[2] = {0, 0};
    XKB_CUDA_TRY(cudaMemcpy(st, S->d_status, sizeof(st), cudaMemcpyDeviceToHost));
    if (st[0]) return xkb_set_error(-(int) st[0], "server_run: a device wait ran out of time");
    return XKB_OK;
}

extern "C" int xkb_server_run(xkb_server_t * S, xkb_request_t * reqs, size_t n)
{
    if (!S || (n && !reqs)) return xkb_set_error(XKB_EINVAL, "server_run: bad arguments");
    int rc = check_requests(S, reqs, n);
    if (rc) return rc;
    const char * mode = getenv("XKB_SERVE_MODE");
    if (mode && strcmp(mode, "launch") == 0) return server_run_launches(S, reqs, n);
    return server_run_device(S, reqs, n);
}
