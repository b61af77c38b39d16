// host_tier.cpp -- registers larger than the device budget: the state in
// pinned host memory, streamed through the GPU a page at a time.
//
// dgQuEST keeps every state in pinned host pages and moves them through the
// GPU per section (page pool QuEST_backend_distributed.cpp:60-73,248-287;
// H2D prefetch / D2H overlap :332-361,458-492), exchanging qubits between
// sections with reorder_data_kernel (QuEST_gpu_kernel.cu:589-654). Here that
// tier only serves states that do not fit in HBM:
//
//  * a page is 2^pageBits consecutive amplitudes; the bits above pageBits
//    (page-index bits) are the top blockIdx bits of every sweep whose tile
//    bits lie inside the page, so one plan serves every page: a page's
//    launches cover its CTA range (TileProgram::ctaOffset / ctaCount) on a
//    state pointer rebased so that the page's global indices land in its
//    device buffer, and controls, selectors and collapses on page-index
//    bits resolve per page exactly as in HBM;
//  * the pending gates are cut into segments whose non-diagonal targets are
//    all inside the page; a segment runs ALL its sweeps on a page while the
//    page is on the device (one copy in, one copy out per page);
//  * a gate that acts on a page-index bit h first exchanges h with the page
//    bit whose next use is furthest away (Belady's rule), in a pass over
//    page pairs that differ in h (launchPageSwap), and the logical-virtual
//    map records the exchange;
//  * the passes pipeline over kPageBufs device buffers, one stream each:
//    copy in, kernels and copy out of different pages overlap.
//
// The same segments serve sharded registers, dgQuEST's multi-GPU form (each
// GPU holds a slice of the state; an MPI page exchange moves qubits between
// them, QuEST_backend_distributed.cpp:403-601, with the sections of
// deriveMappings, QuEST_backend.h:532-636): a shard is a page that stays
// resident in the HBM of its device, a pass launches the segment's plan on
// every shard in place, and an exchange is one kernel per shard pair that
// swaps the two half-shards directly, through peer memory (NVLink) when
// the pair sits on two devices. One host thread drives every device; no
// kernel waits for another, the passes are ordered by the host and by
// events between the pair's streams.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "jit.h"
#include "kernels.h"
#include "qureg_state.h"

namespace dgq {

bool raiseExternal(int code, const char *func, const char *detail);

namespace {

constexpr int kErrUnsupported = 102;  // E_UNSUPPORTED
constexpr int kErrCuda = 103;         // E_CUDA
constexpr int kMinPageBits = 14;      // holds a paired complex64 tile (W <= 13) and more

size_t ampBytesOf(const QuregState &s) { return s.single ? sizeof(float2) : sizeof(double2); }

bool ok(cudaError_t e, const char *func) {
    if (e == cudaSuccess) return true;
    return raiseExternal(kErrCuda, func, cudaGetErrorString(e));
}

char *hostPage(const QuregState &s, uint64_t page) {
    return reinterpret_cast<char *>(s.hState) + (page << s.pageBits) * ampBytesOf(s);
}

// non-diagonal target bits of a gate (the bits a page must hold)
u64 nonDiagonal(const Gate &g) { return isDiagonalType(g.type) ? 0 : g.targetMask; }

void swapBitsOf(Gate &g, int a, int b) {
    auto sw = [&](u64 m) {
        const u64 ba = (m >> a) & 1ULL, bb = (m >> b) & 1ULL;
        m &= ~((1ULL << a) | (1ULL << b));
        return m | (ba << b) | (bb << a);
    };
    g.targetMask = sw(g.targetMask);
    g.controlMask = sw(g.controlMask);
    for (int i = 0; i < g.numMultiTargets; i++) {
        if (g.multiTargets[i] == a)
            g.multiTargets[i] = b;
        else if (g.multiTargets[i] == b)
            g.multiTargets[i] = a;
    }
}

struct Segment {
    std::vector<Gate> gates;
    std::vector<std::pair<int, int>> swapsAfter;  // (page-index bit, page bit) exchanged after the segment
};

// Cuts the gates into page-local segments; the gates after each exchange
// are rewritten in the exchanged bits. uses[b] lists, in order, the gates
// whose non-diagonal targets include address bit b (in the rewritten bits),
// so the next use of a bit is one binary search. With batch (sharded
// registers, where one pass exchanges several bits for little more than
// the cost of one), an exchange also brings in every other page-index bit
// that is needed again before the page bit it would replace, as dgQuEST's
// section boundaries move several qubits in one reorder.
std::vector<Segment> cutSegments(std::vector<Gate> g, int pageBits, int numBits, bool batch) {
    std::vector<Segment> segs(1);
    const u64 local = (1ULL << pageBits) - 1;
    std::vector<std::vector<size_t>> uses(64);
    for (size_t j = 0; j < g.size(); j++)
        for (u64 m = nonDiagonal(g[j]); m; m &= m - 1) uses[(size_t) __builtin_ctzll(m)].push_back(j);
    auto nextUse = [&](int b, size_t from) {
        const auto &u = uses[(size_t) b];
        const auto it = std::lower_bound(u.begin(), u.end(), from);
        return it == u.end() ? g.size() : *it;
    };
    for (size_t i = 0; i < g.size(); i++) {
        const u64 glob = nonDiagonal(g[i]) & ~local;
        if (glob) {
            u64 taken = nonDiagonal(g[i]) & local;
            u64 wanted = glob;
            if (batch) {
                // page-index bits by next use, soonest first
                std::vector<std::pair<size_t, int>> soon;
                for (int b = pageBits; b < numBits; b++)
                    if (!((glob >> b) & 1ULL) && nextUse(b, i) < g.size()) soon.emplace_back(nextUse(b, i), b);
                std::sort(soon.begin(), soon.end());
                // page bits by next use, latest first (not the gate's own)
                std::vector<std::pair<size_t, int>> late;
                for (int l = pageBits - 1; l >= 0; l--)
                    if (!((taken >> l) & 1ULL)) late.emplace_back(nextUse(l, i), l);
                std::stable_sort(late.begin(), late.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
                const size_t need = (size_t) __builtin_popcountll(glob);
                for (size_t t = 0; t < soon.size() && need + t < late.size(); t++)
                    if (soon[t].first < late[need + t].first) wanted |= 1ULL << soon[t].second;
            }
            for (u64 m = wanted; m; m &= m - 1) {
                const int h = __builtin_ctzll(m);
                int victim = -1;
                size_t victimNext = 0;
                for (int l = pageBits - 1; l >= 0; l--) {
                    if ((taken >> l) & 1ULL) continue;
                    const size_t next = nextUse(l, i);
                    if (victim < 0 || next > victimNext) {
                        victim = l;
                        victimNext = next;
                    }
                }
                taken |= 1ULL << victim;
                segs.back().swapsAfter.emplace_back(h, victim);
                for (size_t j = i; j < g.size(); j++) swapBitsOf(g[j], h, victim);
                // from gate i on, bits h and victim trade their uses
                auto &uh = uses[(size_t) h];
                auto &ul = uses[(size_t) victim];
                const auto ih = std::lower_bound(uh.begin(), uh.end(), i) - uh.begin();
                const auto il = std::lower_bound(ul.begin(), ul.end(), i) - ul.begin();
                std::vector<size_t> th(uh.begin() + ih, uh.end()), tl(ul.begin() + il, ul.end());
                uh.resize((size_t) ih);
                ul.resize((size_t) il);
                uh.insert(uh.end(), tl.begin(), tl.end());
                ul.insert(ul.end(), th.begin(), th.end());
            }
            segs.emplace_back();
        }
        segs.back().gates.push_back(g[i]);
    }
    return segs;
}

// Whether a program touches only its page: tile bits below pageBits, the
// blockIdx bits in ascending address order with the page-index bits on top
// (then CTA range [page << (pageBits - W), ...) covers exactly the page).
bool pageLocal(const TileProgram &p, int W, int pageBits, int numBits) {
    if (p.denseK || W > pageBits || numBits - W > kMaxStateBits) return false;
    for (int i = 0; i < W - kCoalescedBits; i++)
        if (p.highPos[i] >= pageBits) return false;
    for (int i = 0; i < numBits - W; i++) {
        const int want = i < pageBits - W ? -1 : pageBits + (i - (pageBits - W));
        if (want < 0 ? p.ctaPos[i] >= pageBits : p.ctaPos[i] != want) return false;
        if (i > 0 && p.ctaPos[i] <= p.ctaPos[i - 1]) return false;
    }
    return true;
}

// Checks that every planned sweep stays inside its page.
bool planIsPageLocal(const QuregState &s, const char *func) {
    for (const TileProgram &p : s.planned)
        if (!pageLocal(p, s.plannedTileBits, s.pageBits, s.numBits))
            return raiseExternal(kErrUnsupported, func, "internal: a sweep of the host tier reaches outside its page");
    return true;
}

// Launches s.planned on page `page`, held in device buffer buf, on stream
// st, with the specialised kernels fns (loaded in the context of st's
// device; null entries run the interpreting kernel).
bool launchPlanAt(QuregState &s, void *buf, uint64_t page, cudaStream_t st, const std::vector<CUfunction> &fns,
                  const char *func) {
    const int W = s.plannedTileBits;
    const uint32_t ctas = 1u << (s.pageBits - W);
    // global index (page << pageBits) | i lands on buffer element i
    const uintptr_t base = reinterpret_cast<uintptr_t>(buf) - (uintptr_t) ((page << s.pageBits) * ampBytesOf(s));
    void *rebased = reinterpret_cast<void *>(base);
    for (size_t i = 0; i < s.planned.size(); i++) {
        TileProgram p = s.planned[i];
        p.ctaOffset = (uint32_t) page * ctas;
        p.ctaCount = ctas;
        const CUfunction fn = i < fns.size() ? fns[i] : nullptr;
        const cudaError_t e = fn ? launchJitSweep(fn, rebased, W, p, st) : launchTile(rebased, s.single, W, p, st);
        if (!ok(e, func)) return false;
    }
    return true;
}

bool launchPlanOnPage(QuregState &s, uint64_t page, int b, cudaStream_t st, const char *func) {
    return launchPlanAt(s, s.dPage[b], page, st, s.plannedFns, func);
}

// Makes `dev` the calling thread's device; the destructor puts back the
// device that was current before.
struct DeviceScope {
    int prev = -1;
    bool good = true;
    explicit DeviceScope(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        good = prev == dev || cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceScope() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// The specialised kernels of s.planned for every device that holds a shard
// (the plan's own functions belong to the home device's context; other
// devices load the same sources in theirs).
bool shardFunctions(QuregState &s, std::vector<std::vector<CUfunction>> &perShard, const char *func) {
    perShard.assign((size_t) 1 << s.shardBits, {});
    std::vector<std::string> sources;
    std::vector<size_t> which;
    for (size_t i = 0; i < s.plannedFns.size(); i++)
        if (s.plannedFns[i]) {
            sources.push_back(generateSweepSource(s.planned[i], s.plannedTileBits));
            which.push_back(i);
        }
    std::vector<int> done;
    std::vector<std::vector<CUfunction>> byDev;
    for (size_t k = 0; k < perShard.size(); k++) {
        const int dev = s.shardDev[k];
        if (dev == s.homeDevice || sources.empty()) {
            perShard[k] = s.plannedFns;
            continue;
        }
        const auto it = std::find(done.begin(), done.end(), dev);
        if (it != done.end()) {
            perShard[k] = byDev[(size_t) (it - done.begin())];
            continue;
        }
        DeviceScope on(dev);
        if (!on.good) return raiseExternal(kErrCuda, func, "cannot select a shard's device");
        std::vector<CUfunction> got;
        std::string err;
        if (!jitGetKernels(sources, got, nullptr, &err)) return raiseExternal(kErrUnsupported, func, err.c_str());
        std::vector<CUfunction> fns(s.planned.size(), nullptr);
        for (size_t j = 0; j < which.size(); j++) fns[which[j]] = got[j];
        done.push_back(dev);
        byDev.push_back(fns);
        perShard[k] = fns;
    }
    return true;
}

// Runs s.planned on every shard in place.
bool runShardPass(QuregState &s, const char *func) {
    if (!planIsPageLocal(s, func)) return false;
    std::vector<std::vector<CUfunction>> fns;
    if (!shardFunctions(s, fns, func)) return false;
    for (int k = 0; k < (1 << s.shardBits); k++) {
        DeviceScope on(s.shardDev[k]);
        if (!on.good) return raiseExternal(kErrCuda, func, "cannot select a shard's device");
        if (!launchPlanAt(s, s.dShard[k], (uint64_t) k, s.shardStream[k], fns[(size_t) k], func)) return false;
    }
    s.hostTierPasses++;
    return shardSync(s, func);
}

// Runs s.planned on every page: copy in (unless the first sweep writes the
// whole page), the plan's sweeps, copy out.
// A page-local plan maps a page of zeros to zeros, so all-zero pages are
// skipped (no copies, no kernels); an initialisation to a basis state leaves
// every other page all-zero, and a blank one every page.
bool runPagePass(QuregState &s, const char *func) {
    if (!planIsPageLocal(s, func)) return false;
    const uint64_t pages = 1ULL << (s.numBits - s.pageBits);
    const size_t pageBytes = ampBytesOf(s) << s.pageBits;
    const bool load = s.planned.empty() || s.planned[0].initKind == INIT_NONE;
    const int32_t initKind = s.planned.empty() ? INIT_NONE : s.planned[0].initKind;
    const uint64_t initPage = s.planned.empty() ? 0 : s.planned[0].initIndex >> s.pageBits;
    s.pageZero.resize(pages, 0);
    for (uint64_t page = 0; page < pages; page++) {
        if (load && s.pageZero[page]) continue;
        if ((initKind == INIT_CLASSICAL && page != initPage) || initKind == INIT_BLANK) {
            s.pageZero[page] = 1;
            continue;
        }
        if (!load) s.pageZero[page] = 0;
        const int b = (int) (page % QuregState::kPageBufs);
        cudaStream_t st = s.pageStream[b];
        if (load && !ok(cudaMemcpyAsync(s.dPage[b], hostPage(s, page), pageBytes, cudaMemcpyHostToDevice, st), func))
            return false;
        if (!launchPlanOnPage(s, page, b, st, func) ||
            !ok(cudaMemcpyAsync(hostPage(s, page), s.dPage[b], pageBytes, cudaMemcpyDeviceToHost, st), func))
            return false;
        s.hostTierBytes += (load ? 2 : 1) * pageBytes;
    }
    s.hostTierPasses++;
    return hostTierSync(s, func);
}

// Exchanges page-index bit h with page bit l over all page pairs; with
// thenPlan, each pair then runs s.planned (the next segment, planned in the
// exchanged bits) before it goes back, saving that segment a pass of its own.
bool runSwapPass(QuregState &s, int h, int l, bool thenPlan, const char *func) {
    if (thenPlan && !planIsPageLocal(s, func)) return false;
    const uint64_t pages = 1ULL << (s.numBits - s.pageBits);
    const uint64_t hb = 1ULL << (h - s.pageBits);
    const size_t pageBytes = ampBytesOf(s) << s.pageBits;
    int pair = 0;
    s.pageZero.resize(pages, 0);
    for (uint64_t p0 = 0; p0 < pages; p0++) {
        if (p0 & hb) continue;
        const uint64_t p1 = p0 | hb;
        // two all-zero pages stay all-zero (exchange and segment alike)
        if (s.pageZero[p0] && s.pageZero[p1]) continue;
        const int a = 2 * (pair % (QuregState::kPageBufs / 2)), b = a + 1;
        cudaStream_t st = s.pageStream[a];
        // an all-zero page is cleared on the device instead of copied in
        auto bringIn = [&](uint64_t pg, int buf) {
            return s.pageZero[pg] ? ok(cudaMemsetAsync(s.dPage[buf], 0, pageBytes, st), func)
                                  : ok(cudaMemcpyAsync(s.dPage[buf], hostPage(s, pg), pageBytes,
                                                       cudaMemcpyHostToDevice, st),
                                       func);
        };
        const int loaded = (s.pageZero[p0] ? 0 : 1) + (s.pageZero[p1] ? 0 : 1);
        if (!bringIn(p0, a) || !bringIn(p1, b) || !ok(launchPageSwap(s.dPage[a], s.dPage[b], s.single, s.pageBits, l, st), func))
            return false;
        s.pageZero[p0] = 0;
        s.pageZero[p1] = 0;
        if (thenPlan && (!launchPlanOnPage(s, p0, a, st, func) || !launchPlanOnPage(s, p1, b, st, func)))
            return false;
        if (!ok(cudaMemcpyAsync(hostPage(s, p0), s.dPage[a], pageBytes, cudaMemcpyDeviceToHost, st), func) ||
            !ok(cudaMemcpyAsync(hostPage(s, p1), s.dPage[b], pageBytes, cudaMemcpyDeviceToHost, st), func))
            return false;
        s.hostTierBytes += (2 + loaded) * pageBytes;
        pair++;
    }
    if (!hostTierSync(s, func)) return false;
    if (thenPlan) s.hostTierPasses++;
    // the qubits at virtual bits h and l trade places
    const int qa = s.v2l[h], qb = s.v2l[l];
    s.v2l[h] = qb;
    s.v2l[l] = qa;
    if (qa >= 0) s.l2v[qa] = l;
    if (qb >= 0) s.l2v[qb] = h;
    s.hostTierSwaps++;
    return true;
}

// Exchanges the shard-index bits h[t] with the shard bits l[t] (disjoint
// pairs, one pass): with m pairs, the amplitude at shard c | A(a), offset
// o | L(b) (a, b: m-bit patterns spread over the h and l positions) moves to
// shard c | A(b), offset o | L(a). Each pair of blocks with a < b trades
// places in one kernel on the device of the first shard (peer loads and
// stores when the second is elsewhere); the blocks are disjoint, so the
// kernels of one pass run concurrently on the shards' streams.
bool runShardExchange(QuregState &s, const std::vector<std::pair<int, int>> &swaps, const char *func) {
    std::vector<std::pair<int, int>> sw = swaps;  // (shard bit l, shard-index bit h), l ascending
    for (auto &x : sw) x = {x.second, x.first};
    std::sort(sw.begin(), sw.end());
    const int m = (int) sw.size();
    if (m < 1 || m > s.shardBits) return raiseExternal(kErrUnsupported, func, "internal: bad shard exchange");
    BlockSwapArgs args;
    std::memset(&args, 0, sizeof(args));
    args.pageBits = s.pageBits;
    args.m = m;
    int hMask = 0;
    for (int t = 0; t < m; t++) {
        args.pos[t] = sw[(size_t) t].first;
        hMask |= 1 << (sw[(size_t) t].second - s.pageBits);
    }
    auto spreadH = [&](int a) {
        int r = 0;
        for (int t = 0; t < m; t++)
            if ((a >> t) & 1) r |= 1 << (sw[(size_t) t].second - s.pageBits);
        return r;
    };
    auto spreadL = [&](int b) {
        uint64_t r = 0;
        for (int t = 0; t < m; t++)
            if ((b >> t) & 1) r |= 1ULL << sw[(size_t) t].first;
        return r;
    };
    const size_t blockBytes = ampBytesOf(s) << (s.pageBits - m);
    for (int c = 0; c < (1 << s.shardBits); c++) {
        if (c & hMask) continue;
        for (int a = 0; a < (1 << m); a++)
            for (int b = a + 1; b < (1 << m); b++) {
                const int x = c | spreadH(a), y = c | spreadH(b);
                args.patX = spreadL(b);
                args.patY = spreadL(a);
                DeviceScope on(s.shardDev[x]);
                if (!on.good) return raiseExternal(kErrCuda, func, "cannot select a shard's device");
                if (!ok(launchBlockSwap(s.dShard[x], s.dShard[y], s.single, args, s.shardStream[x]), func))
                    return false;
                s.hostTierBytes += 2 * blockBytes;  // one block each way
            }
    }
    if (!shardSync(s, func)) return false;
    for (const auto &x : sw) {
        const int l = x.first, h = x.second;
        const int qa = s.v2l[h], qb = s.v2l[l];
        s.v2l[h] = qb;
        s.v2l[l] = qa;
        if (qa >= 0) s.l2v[qa] = l;
        if (qb >= 0) s.l2v[qb] = h;
    }
    s.hostTierSwaps++;
    return true;
}

}  // namespace

void hostTierMaterialise(QuregState &s) {
    if (!s.hostTier || s.sharded) return;
    const size_t pageBytes = ampBytesOf(s) << s.pageBits;
    for (size_t page = 0; page < s.pageZero.size(); page++)
        if (s.pageZero[page]) {
            std::memset(hostPage(s, page), 0, pageBytes);
            s.pageZero[page] = 0;
        }
}

bool hostTierPageZero(const QuregState &s, uint64_t index) {
    if (!s.hostTier || s.sharded) return false;
    const uint64_t page = index >> s.pageBits;
    return page < s.pageZero.size() && s.pageZero[page];
}

bool hostTierSync(QuregState &s, const char *func) {
    for (int b = 0; b < QuregState::kPageBufs; b++)
        if (s.pageStream[b] && !ok(cudaStreamSynchronize(s.pageStream[b]), func)) return false;
    return true;
}

bool hostTierAttach(QuregState &s, size_t budgetBytes, std::string &err) {
    const size_t ab = ampBytesOf(s);
    int p = s.numBits - 1;
    while (p >= kMinPageBits && (size_t) QuregState::kPageBufs * (ab << p) > budgetBytes) p--;
    if (p < kMinPageBits) {
        err = "the device budget holds no page buffers";
        return false;
    }
    if (s.numBits > 40) {
        err = "more than 2^40 amplitudes";
        return false;
    }
    s.pageBits = p;
    s.pageZero.assign((size_t) 1 << (s.numBits - p), 0);
    if (cudaHostAlloc(&s.hState, ab << s.numBits, cudaHostAllocDefault) != cudaSuccess) {
        s.hState = nullptr;
        err = "pinned host memory for the state is not available";
        return false;
    }
    for (int b = 0; b < QuregState::kPageBufs; b++) {
        if (cudaStreamCreateWithFlags(&s.pageStream[b], cudaStreamNonBlocking) != cudaSuccess ||
            cudaMalloc(&s.dPage[b], ab << p) != cudaSuccess ||
            cudaMalloc((void **) &s.dPageOut[b], sizeof(double) * (kMaxStateBits + 1)) != cudaSuccess) {
            hostTierRelease(s);
            err = "device page buffers are not available";
            return false;
        }
    }
    s.hostTier = true;
    return true;
}

void hostTierRelease(QuregState &s) {
    for (int b = 0; b < QuregState::kPageBufs; b++) {
        if (s.pageStream[b]) cudaStreamSynchronize(s.pageStream[b]);
        if (s.dPage[b]) cudaFree(s.dPage[b]);
        if (s.dPagePartial[b]) cudaFree(s.dPagePartial[b]);
        if (s.dPageOut[b]) cudaFree(s.dPageOut[b]);
        if (s.pageStream[b]) cudaStreamDestroy(s.pageStream[b]);
        s.dPage[b] = nullptr;
        s.dPagePartial[b] = nullptr;
        s.dPageOut[b] = nullptr;
        s.pageStream[b] = nullptr;
    }
    if (s.hState) cudaFreeHost(s.hState);
    s.hState = nullptr;
    s.pageZero.clear();
    s.hostTier = false;
}

bool hostTierFlush(QuregState &s, const char *func) {
    if (s.pending.empty() && !s.initPending) return true;
    for (const Gate &g : s.pending)
        if (g.type == OP_MULTI_UNITARY && g.numMultiTargets > kRegBits)
            return raiseExternal(kErrUnsupported, func,
                                 "a multi-qubit unitary of more than 4 targets on a register in host memory");
    std::vector<Segment> segs = cutSegments(s.pending, s.pageBits, s.numBits, s.sharded);
    if (s.restrictActive && segs[0].gates.empty()) {
        // a pending collapse is in the address bits before any exchange: an
        // empty program carries it into the first pass
        Gate one;
        one.type = OP_ONE;
        segs[0].gates.push_back(one);
    }
    const MatrixPool pool = s.pool;
    const int denseFusion = s.denseFusion;
    s.denseFusion = 0;
    bool good = true;
    bool ranWithExchange = false;  // segment k ran fused with the exchange before it
    for (size_t k = 0; k < segs.size() && good; k++) {
        // the first segment carries the pending initialisation or collapse
        // (a header-only pass when it holds no gates)
        const bool header = k == 0 && (s.initPending || s.restrictActive);
        if (!ranWithExchange && (!segs[k].gates.empty() || header)) {
            s.pending = segs[k].gates;
            s.pool = pool;
            good = planForPages(s, func) && (s.sharded ? runShardPass(s, func) : runPagePass(s, func));
        }
        ranWithExchange = false;
        const auto &sw = segs[k].swapsAfter;
        if (s.sharded) {
            // all of the boundary's bits in one pass
            if (!sw.empty() && good) good = runShardExchange(s, sw, func);
            continue;
        }
        for (size_t i = 0; i < sw.size() && good; i++) {
            // the last exchange before a segment runs that segment too
            const bool fuse = i + 1 == sw.size() && k + 1 < segs.size() && !segs[k + 1].gates.empty();
            if (fuse) {
                s.pending = segs[k + 1].gates;
                s.pool = pool;
                good = planForPages(s, func);
            }
            if (good) good = runSwapPass(s, sw[i].first, sw[i].second, fuse, func);
            ranWithExchange = fuse;
        }
    }
    s.denseFusion = denseFusion;
    s.pending.clear();
    s.pool.mats.clear();
    s.planned.clear();
    s.plannedFns.clear();
    s.probsValid = false;
    return good;
}

bool hostTierProbs(QuregState &s, std::vector<double> &p0, double &total, const char *func) {
    const int p = s.pageBits;
    const uint64_t pages = 1ULL << (s.numBits - p);
    const u64 localMask = (1ULL << p) - 1;
    const u64 rMask = s.restrictActive ? s.rMask : 0, rValue = s.restrictActive ? s.rValue : 0;
    ProbArgs a;
    std::memset(&a, 0, sizeof(a));
    int nf = 0;
    for (int b = 0; b < p; b++) {
        if ((rMask >> b) & 1ULL) continue;
        a.freePos[nf++] = (uint8_t) b;
    }
    a.nFree = nf;
    a.kappa = std::min(4, std::max(0, nf - 12));
    a.rValue = rValue & localMask;
    const size_t need = (size_t) probNumCtas(a) * 17;
    if (s.sharded && need > s.shardPartialCap) {
        for (int k = 0; k < (1 << s.shardBits); k++) {
            DeviceScope on(s.shardDev[k]);
            if (s.dShardPartial[k]) cudaFree(s.dShardPartial[k]);
            s.dShardPartial[k] = nullptr;
            if (!ok(on.good ? cudaMalloc((void **) &s.dShardPartial[k], need * sizeof(double)) : cudaErrorInvalidDevice,
                    func))
                return false;
        }
        s.shardPartialCap = need;
    } else if (!s.sharded && need > s.pagePartialCap) {
        for (int b = 0; b < QuregState::kPageBufs; b++) {
            if (s.dPagePartial[b]) cudaFree(s.dPagePartial[b]);
            s.dPagePartial[b] = nullptr;
            if (!ok(cudaMalloc((void **) &s.dPagePartial[b], need * sizeof(double)), func)) return false;
        }
        s.pagePartialCap = need;
    }
    const size_t pageBytes = ampBytesOf(s) << p;
    std::vector<double> sums(pages * (size_t) (nf + 1), 0.0);
    std::vector<char> used(pages, 0);
    for (uint64_t page = 0; page < pages; page++) {
        // pages outside a collapse on page-index bits hold no probability,
        // and neither do all-zero pages
        if (((page << p) & rMask & ~localMask) != (rValue & ~localMask)) continue;
        if (!s.sharded && page < s.pageZero.size() && s.pageZero[page]) continue;
        used[page] = 1;
        double *sum = &sums[page * (size_t) (nf + 1)];
        const size_t sumBytes = sizeof(double) * (size_t) (nf + 1);
        if (s.sharded) {
            // a shard is read where it lies
            DeviceScope on(s.shardDev[page]);
            if (!on.good) return raiseExternal(kErrCuda, func, "cannot select a shard's device");
            cudaStream_t st = s.shardStream[page];
            if (!ok(launchProb(s.dShard[page], s.single, a, s.dShardPartial[page], s.dShardOut[page], st), func) ||
                !ok(cudaMemcpyAsync(sum, s.dShardOut[page], sumBytes, cudaMemcpyDeviceToHost, st), func))
                return false;
            continue;
        }
        const int b = (int) (page % QuregState::kPageBufs);
        cudaStream_t st = s.pageStream[b];
        if (!ok(cudaMemcpyAsync(s.dPage[b], hostPage(s, page), pageBytes, cudaMemcpyHostToDevice, st), func) ||
            !ok(launchProb(s.dPage[b], s.single, a, s.dPagePartial[b], s.dPageOut[b], st), func) ||
            !ok(cudaMemcpyAsync(sum, s.dPageOut[b], sumBytes, cudaMemcpyDeviceToHost, st), func))
            return false;
    }
    if (!(s.sharded ? shardSync(s, func) : hostTierSync(s, func))) return false;
    s.hostTierPasses++;
    if (!s.sharded)
        for (uint64_t page = 0; page < pages; page++) s.hostTierBytes += used[page] ? pageBytes : 0;
    p0.assign((size_t) s.numBits, 0.0);
    total = 0.0;
    for (uint64_t page = 0; page < pages; page++) {
        if (!used[page]) continue;
        const double *o = &sums[page * (size_t) (nf + 1)];
        const double t = o[nf];
        total += t;
        for (int i = 0; i < nf; i++) p0[a.freePos[i]] += o[i];
        for (int b = p; b < s.numBits; b++)
            if (!(((page << p) >> b) & 1ULL)) p0[(size_t) b] += t;
    }
    // collapsed page bits: all the probability on their fixed value
    for (int b = 0; b < p; b++)
        if ((rMask >> b) & 1ULL) p0[(size_t) b] = ((rValue >> b) & 1ULL) ? 0.0 : total;
    return true;
}

void planExchanges(const std::vector<Gate> &gates, int localBits, int numBits, bool batch, int &segments,
                   int &exchanges, int &qubitsMoved) {
    const std::vector<Segment> segs = cutSegments(gates, localBits, numBits, batch);
    segments = (int) segs.size();
    exchanges = qubitsMoved = 0;
    for (const Segment &sg : segs)
        if (!sg.swapsAfter.empty()) {
            // the host tier runs one pass per qubit, sharded registers one per boundary
            exchanges += batch ? 1 : (int) sg.swapsAfter.size();
            qubitsMoved += (int) sg.swapsAfter.size();
        }
}

bool shardSync(QuregState &s, const char *func) {
    for (int k = 0; k < (1 << s.shardBits); k++)
        if (s.shardStream[k] && !ok(cudaStreamSynchronize(s.shardStream[k]), func)) return false;
    return true;
}

bool shardAttach(QuregState &s, int shardBits, const int *devices, int &code, std::string &err) {
    constexpr int kErrTooBig = 101;  // E_SYS_TOO_BIG_FOR_DEVICE
    code = kErrUnsupported;
    const int shards = 1 << shardBits;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        err = "no CUDA device";
        return false;
    }
    if (cudaGetDevice(&s.homeDevice) != cudaSuccess) {
        err = "no current CUDA device";
        return false;
    }
    for (int k = 0; k < shards; k++) {
        s.shardDev[k] = devices ? devices[k] : s.homeDevice;
        if (s.shardDev[k] < 0 || s.shardDev[k] >= count) {
            err = "a shard's device does not exist";
            return false;
        }
    }
    // every pair of distinct devices exchanges through peer memory
    for (int i = 0; i < shards; i++)
        for (int j = 0; j < shards; j++) {
            const int a = s.shardDev[i], b = s.shardDev[j];
            if (a == b) continue;
            int can = 0;
            if (cudaDeviceCanAccessPeer(&can, a, b) != cudaSuccess || !can) {
                err = "two shard devices have no peer access to each other";
                return false;
            }
            DeviceScope on(a);
            const cudaError_t e = on.good ? cudaDeviceEnablePeerAccess(b, 0) : cudaErrorInvalidDevice;
            if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled) {
                cudaGetLastError();
                err = "enabling peer access between shard devices failed";
                return false;
            }
            cudaGetLastError();  // an already-enabled pair leaves its error recorded
        }
    const size_t bytes = ampBytesOf(s) << s.pageBits;
    s.sharded = true;
    s.shardBits = shardBits;
    for (int k = 0; k < shards; k++) {
        DeviceScope on(s.shardDev[k]);
        if (!on.good || cudaStreamCreateWithFlags(&s.shardStream[k], cudaStreamNonBlocking) != cudaSuccess ||
            cudaMalloc((void **) &s.dShardOut[k], sizeof(double) * (kMaxStateBits + 1)) != cudaSuccess) {
            cudaGetLastError();
            shardRelease(s);
            err = "shard streams or buffers are not available";
            return false;
        }
        if (cudaMalloc(&s.dShard[k], bytes) != cudaSuccess) {
            s.dShard[k] = nullptr;
            cudaGetLastError();  // the failed allocation must not surface at a later launch
            shardRelease(s);
            code = kErrTooBig;
            err = "a shard does not fit in its device's memory";
            return false;
        }
    }
    return true;
}

void shardRelease(QuregState &s) {
    for (int k = 0; k < QuregState::kMaxShards; k++) {
        if (!s.shardStream[k] && !s.dShard[k] && !s.dShardOut[k] && !s.dShardPartial[k]) continue;
        DeviceScope on(s.shardDev[k]);
        if (s.shardStream[k]) cudaStreamSynchronize(s.shardStream[k]);
        if (s.dShard[k]) cudaFree(s.dShard[k]);
        if (s.dShardPartial[k]) cudaFree(s.dShardPartial[k]);
        if (s.dShardOut[k]) cudaFree(s.dShardOut[k]);
        if (s.shardStream[k]) cudaStreamDestroy(s.shardStream[k]);
        s.dShard[k] = nullptr;
        s.dShardPartial[k] = nullptr;
        s.dShardOut[k] = nullptr;
        s.shardStream[k] = nullptr;
    }
    s.shardPartialCap = 0;
    s.sharded = false;
}

namespace {

// Calls fn(shard, offset in the shard, offset in [begin, begin + count),
// amplitudes) for the runs of [begin, begin + count) that lie in one shard.
template <class F>
bool forShardRuns(const QuregState &s, uint64_t begin, uint64_t count, F fn) {
    const uint64_t mask = (1ULL << s.pageBits) - 1;
    for (uint64_t i = begin; i < begin + count;) {
        const int k = (int) (i >> s.pageBits);
        const uint64_t off = i & mask;
        const uint64_t run = std::min<uint64_t>(begin + count - i, (mask + 1) - off);
        if (!fn(k, off, i - begin, run)) return false;
        i += run;
    }
    return true;
}

}  // namespace

bool shardReadVirtual(QuregState &s, uint64_t begin, uint64_t count, void *host, const char *func) {
    const size_t ab = ampBytesOf(s);
    return forShardRuns(s, begin, count, [&](int k, uint64_t off, uint64_t at, uint64_t run) {
        DeviceScope on(s.shardDev[k]);
        if (!on.good) return raiseExternal(kErrCuda, func, "cannot select a shard's device");
        return ok(cudaMemcpyAsync(static_cast<char *>(host) + at * ab, static_cast<const char *>(s.dShard[k]) + off * ab,
                                  run * ab, cudaMemcpyDeviceToHost, s.shardStream[k]),
                  func) &&
               ok(cudaStreamSynchronize(s.shardStream[k]), func);
    });
}

bool shardWriteVirtual(QuregState &s, uint64_t begin, uint64_t count, const void *host, const char *func) {
    const size_t ab = ampBytesOf(s);
    return forShardRuns(s, begin, count, [&](int k, uint64_t off, uint64_t at, uint64_t run) {
        DeviceScope on(s.shardDev[k]);
        if (!on.good) return raiseExternal(kErrCuda, func, "cannot select a shard's device");
        return ok(cudaMemcpyAsync(static_cast<char *>(s.dShard[k]) + off * ab,
                                  static_cast<const char *>(host) + at * ab, run * ab, cudaMemcpyHostToDevice,
                                  s.shardStream[k]),
                  func) &&
               ok(cudaStreamSynchronize(s.shardStream[k]), func);
    });
}

bool shardCopy(QuregState &t, const QuregState &c, const char *func) {
    const size_t bytes = ampBytesOf(t) << t.pageBits;
    for (int k = 0; k < (1 << t.shardBits); k++) {
        DeviceScope on(t.shardDev[k]);
        if (!on.good) return raiseExternal(kErrCuda, func, "cannot select a shard's device");
        if (!ok(cudaMemcpyPeerAsync(t.dShard[k], t.shardDev[k], c.dShard[k], c.shardDev[k], bytes, t.shardStream[k]),
                func) ||
            !ok(cudaStreamSynchronize(t.shardStream[k]), func))
            return false;
    }
    return true;
}

}  // namespace dgq
