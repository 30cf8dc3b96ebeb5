// batch.cpp — batched stepping of many simulations on one GPU.
//
// A batch advances its member simulations (typically many small periodic unit
// cells of uneven sizes) together. Members are created and set up as ordinary
// simulations; the batch then owns their stepping:
//
//  * Size classes. Members are grouped by x-y size (16-cell buckets). Each
//    class has a tile height (CTAs of 32 x 2, 4 or 8 threads) and a z-block
//    depth (planes per work item), set by hand or by the autotuner, which
//    times trial segments of the class's members for every candidate.
//  * Subsets. Within a class, members are packed into subsets whose device
//    state fits an L2 budget (126 MB of L2 on B200; default 48 MiB, tuned).
//    A subset runs a whole segment of steps before the next subset starts, so
//    after its first step most of its state is served from L2. Lanes run that
//    many subsets concurrently (default 2: measured on 96 nanodisk unit cells of up to
//    120 x 120 x 200, two
//    resident cells at a time 57.8 Gcell/s, one 47.0, three 55.4).
//  * Lone members. A subset of one member (one such unit cell fills the
//    default budget) runs the member's own single-simulation kernels and work
//    lists (two-cell items, L2-ordered H lists, arguments as launch
//    parameters).
//  * Merged launches. Otherwise, per step, each work-item group of a subset
//    (interior, z-CPML, dispersive, general, x/y-CPML) is ONE launch over the
//    items of all its members: items carry the member index and the kernels
//    read that member's arguments from a device array.
//  * Either way boundary groups run on side streams beside the interior group;
//    the plane sums of all normal-mode members are one launch beside the H
//    half-step. A chunk of 32 steps of a subset is captured once as a CUDA
//    graph and replayed for every full chunk (the members' scalar tables are
//    uploaded before each replay).
//  * Step budgets. Each member has a number of steps still to run; a segment
//    never passes a member's budget, so members finish exactly and can be
//    retired and replaced between segments (continuous batching).
//
// Results of a member do not depend on the batch: every member advances with
// exactly the kernels' arithmetic of a single simulation (FP64 fields are
// bit-identical to stepping it alone).
#include "sim.hpp"

#include <chrono>


namespace aefdtd {

struct BatchMember {
    aefdtd_sim *sim = nullptr;
    int remaining = 0;   // steps still to run
    int cls = 0;         // size-class key
    bool placed = false; // in a subset
};

struct BatchSubset {
    int cls = 0;
    std::vector<aefdtd_sim *> members;
    size_t bytes = 0;              // device state of the members
    DBuf items;                    // merged items: E groups, then H groups
    WorkSplit wsE{}, wsH{};
    DBuf argsE, argsH, sargs;      // per-member arguments (members' table slot 0)
    DBuf blkmap;
    int nblk = 0;
    int nplane = 0;                // members with plane sums
    cudaGraphExec_t graph = nullptr;   // one chunk of graph_steps steps
    cudaGraphExec_t graph_b = nullptr; // the same with a fused lone member's state in its second buffer set
    uint64_t graph_launches = 0;
    bool fused = false;            // a lone member that takes the fused time step
    bool built = false;
    bool solo = false;             // one member: its own single-simulation kernels and work lists
    // one persistent launch per chunk (batch_persist.cuh): units, their items,
    // progress counters, per-member sensor arguments and band partials
    bool ps = false;
    DBuf ps_units, ps_items, ps_prog, ps_sargs, ps_part;
    int ps_nunits = 0, ps_grid = 0, ps_ty = 4;
    void release(size_t &t) {
        items.release(t);
        ps_units.release(t); ps_items.release(t); ps_prog.release(t); ps_sargs.release(t); ps_part.release(t);
        ps = false;
        argsE.release(t); argsH.release(t); sargs.release(t);
        if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
        if (graph_b) { cudaGraphExecDestroy(graph_b); graph_b = nullptr; }
        blkmap.release(t);
        built = false;
    }
};

struct SizeClass {
    int tile_y = 4;
    int kchunk = 0;   // 0: the simulation's own heuristic
};

// A lane: the streams and events one subset at a time runs on. Subsets on
// different lanes run concurrently.
struct Lane {
    cudaStream_t stream = nullptr, side[kGroups - 1] = {}, side_s = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join[kGroups - 1] = {}, ev_sf = nullptr, ev_sj = nullptr;
    void create() {
        AE_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        for (auto &x : side) AE_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
        AE_CUDA(cudaStreamCreateWithFlags(&side_s, cudaStreamNonBlocking));
        AE_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        for (auto &e : ev_join) AE_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        AE_CUDA(cudaEventCreateWithFlags(&ev_sf, cudaEventDisableTiming));
        AE_CUDA(cudaEventCreateWithFlags(&ev_sj, cudaEventDisableTiming));
    }
    void destroy() {
        if (stream) cudaStreamSynchronize(stream);
        for (auto &e : ev_join) if (e) cudaEventDestroy(e);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_sf) cudaEventDestroy(ev_sf);
        if (ev_sj) cudaEventDestroy(ev_sj);
        for (auto &x : side) if (x) cudaStreamDestroy(x);
        if (side_s) cudaStreamDestroy(side_s);
        if (stream) cudaStreamDestroy(stream);
    }
};
constexpr int kMaxLanes = 8;

}  // namespace aefdtd

using namespace aefdtd;

struct aefdtd_batch {
    std::string last_error;
    aefdtd_batch_opts opts{};
    int device = 0;
    bool typed = false, fp64 = false;
    int id_bytes = 1, seg_len = 64;
    Lane lanes[kMaxLanes];
    int n_lanes = 2;               // most subsets running concurrently
    // L2 bytes that the subsets running at once may hold together: a subset of
    // b bytes shares the device with at most lane_window / b - 1 others of its class
    long long lane_window = 96LL << 20;
    cudaStream_t stream = nullptr; // lanes[0].stream
    std::vector<BatchMember> members;
    std::vector<BatchSubset> subsets;
    std::map<int, SizeClass> classes;
    bool layout_dirty = true;
    long long l2_budget = 48LL << 20;
    int next_solo_class = -1;   // size-class keys below zero: members that never share a subset
    int graph_steps = 32;          // steps per captured chunk (a divisor of seg_len)
    bool h_reverse = false;        // H pass over the members in reverse order (measured slower on L2-sized subsets)
    int persistent = 0;            // subsets run each chunk as one persistent launch (batch_persist.cuh)
    DBuf ps_flags;                 // persistent launches: [0] device error flag, [1] abort
    bool ps_direct = false;        // the persistent launch did not capture into a graph: launched directly
    std::map<int, int> ps_capacity;   // resident persistent CTAs per tile height
    uint64_t launches = 0;
    size_t dev_bytes = 0;

    void set_device() const { cudaSetDevice(device); }
    int class_key(const aefdtd_sim *s) const { return ((s->Nx + 15) / 16) * 1000 + (s->Ny + 15) / 16; }
    int find(const aefdtd_sim *s) const {
        for (size_t i = 0; i < members.size(); i++)
            if (members[i].sim == s) return (int)i;
        return -1;
    }
    BatchMember &rec(const aefdtd_sim *s) { return members[find(s)]; }
    void drop_layout() {
        for (auto &u : subsets) u.release(dev_bytes);
        subsets.clear();
        for (auto &m : members) m.placed = false;
        layout_dirty = true;
    }
    // lanes that the subsets of u's size class take in turn: as many as fit the
    // window when subsets are sized for L2, all of them otherwise
    int lanes_for(const BatchSubset &u) const {
        if (l2_budget < 0) return n_lanes;
        const long long b = std::max<long long>((long long)u.bytes, 1);
        return (int)std::clamp<long long>(lane_window / b, 1, n_lanes);
    }
    // lane of every subset: within a size class the subsets go round-robin over
    // lanes_for() lanes (subsets of one class are consecutive after a full layout)
    std::vector<int> lane_plan() const {
        std::vector<int> lane(subsets.size());
        std::map<int, int> seen;
        for (size_t k = 0; k < subsets.size(); k++) lane[k] = seen[subsets[k].cls]++ % lanes_for(subsets[k]);
        return lane;
    }
    // subsets whose state stays in the 126 MB L2 between steps
    static bool l2_resident(const BatchSubset &u) { return u.bytes <= (96ull << 20); }
    bool fits(const BatchSubset &u, size_t b) const {
        return u.members.empty() || l2_budget < 0 || (long long)(u.bytes + b) <= l2_budget;
    }
    void place(BatchMember &m);
    void update_layout();
    template <typename T, typename Tid> void build_subset(BatchSubset &u);
    template <typename T, typename Tid>
    bool build_persist(BatchSubset &u, const std::vector<SensorStepArgs<T>> &sa);
    void check_persist();
    template <typename T, typename Tid> void enqueue_steps(BatchSubset &u, int L, Lane &ln);
    template <typename T, typename Tid> void run_segment(BatchSubset &u, int L, Lane &ln);
    void sync_lanes() {
        for (int k = 0; k < n_lanes; k++) AE_CUDA(cudaStreamSynchronize(lanes[k].stream));
    }
    template <typename T, typename Tid> void ensure_history();
    template <typename T, typename Tid> int advance(int max_steps);
    template <typename T, typename Tid> double time_segments(int reps);
    template <typename T, typename Tid> void autotune();
    template <typename Launch> void run_groups(const WorkSplit &w, Lane &ln, Launch &&launch);
    ~aefdtd_batch();
};

aefdtd_batch::~aefdtd_batch() {
    set_device();
    for (auto &ln : lanes) if (ln.stream) cudaStreamSynchronize(ln.stream);
    for (auto &m : members) {
        m.sim->batch = nullptr;
        m.sim->tma_allowed = true;
        m.sim->work_dirty = true;
    }
    for (auto &u : subsets) u.release(dev_bytes);
    ps_flags.release(dev_bytes);
    for (auto &ln : lanes) ln.destroy();
}

// A member joins the last subset of its class that still fits the L2 budget,
// else a new subset (a member larger than the budget gets one of its own).
void aefdtd_batch::place(BatchMember &m) {
    const size_t b = m.sim->dev_bytes;
    BatchSubset *dst = nullptr;
    for (auto it = subsets.rbegin(); it != subsets.rend(); ++it)
        if (it->cls == m.cls) {
            if (fits(*it, b)) dst = &*it;
            break;
        }
    if (!dst) {
        subsets.emplace_back();
        dst = &subsets.back();
        dst->cls = m.cls;
    }
    dst->release(dev_bytes);
    dst->members.push_back(m.sim);
    dst->bytes += b;
    m.placed = true;
}

// Subsets follow membership incrementally: members out of budget (or gone)
// leave their subset, new members are placed; only touched subsets are
// rebuilt (and their graphs re-captured). layout_dirty forces a full layout in
// member order, grouped by size class.
void aefdtd_batch::update_layout() {
    if (layout_dirty) {
        for (auto &u : subsets) u.release(dev_bytes);
        subsets.clear();
        for (auto &m : members) m.placed = false;
        layout_dirty = false;
    }
    for (auto &u : subsets) {
        std::vector<aefdtd_sim *> keep;
        size_t bytes = 0;
        for (aefdtd_sim *s : u.members) {
            const int i = find(s);
            if (i >= 0 && members[i].remaining > 0) {
                keep.push_back(s);
                bytes += s->dev_bytes;
            } else if (i >= 0) {
                members[i].placed = false;
            }
        }
        if (keep.size() != u.members.size()) {
            u.release(dev_bytes);
            u.members = keep;
            u.bytes = bytes;
        }
    }
    for (size_t k = 0; k < subsets.size();) {
        if (subsets[k].members.empty()) {
            subsets[k].release(dev_bytes);
            subsets.erase(subsets.begin() + k);
        } else {
            k++;
        }
    }
    std::map<int, std::vector<int>> fresh;   // by class, in member order
    for (size_t i = 0; i < members.size(); i++)
        if (members[i].remaining > 0 && !members[i].placed) fresh[members[i].cls].push_back((int)i);
    for (auto &kv : fresh)
        for (int i : kv.second) place(members[i]);
}

// Work lists and argument arrays of one subset.
template <typename T, typename Tid> void aefdtd_batch::build_subset(BatchSubset &u) {
    u.release(dev_bytes);
    const SizeClass &sc = classes[u.cls];
    // A lone member keeps its own work lists (two-cell items, L2-ordered H
    // lists) and kernels; merged members take one-cell, forward lists.
    u.solo = u.members.size() == 1;
    // the persistent launch takes every member's one-cell, forward lists;
    // oblique members and completion sensors keep the split launches
    u.ps = persistent != 0;
    for (aefdtd_sim *s : u.members) u.ps = u.ps && !s->obl && s->cc_coeff <= 0;
    for (aefdtd_sim *s : u.members) {
        const unsigned pm = (u.solo && !u.ps) ? s->pair_mask0 : 0u;
        const int hr = (u.solo && !u.ps) ? s->h_reverse0 : 0;
        if (s->pair_mask != pm || s->h_reverse != hr || s->work_dirty) {
            s->pair_mask = pm;
            s->h_reverse = hr;
            s->build_work();
            s->fwork_dirty = true;
        }
    }
    // a lone member takes its own fused time step when it can (not with the
    // FT-mode completion sensor, whose check steps need the ring snapshots of
    // the batched path)
    aefdtd_sim *m0 = u.members[0];
    u.fused = !u.ps && u.solo && m0->fused_eligible() && !m0->ccft;
    if (u.fused) {
        if (m0->fwork_dirty) m0->build_fused_work();
        m0->ensure_other_set();
        AE_CUDA(cudaStreamSynchronize(m0->stream));
    }
    std::vector<int> all;
    for (int half = 0; half < 2; half++) {
        WorkSplit &w = half == 0 ? u.wsE : u.wsH;
        w.unroll = 2;
        w.tile_y = sc.tile_y;
        w.pair_mask = 0;
        w.n_py = 0;
        w.tma = nullptr;
        for (int g = 0; g < kGroups; g++) {
            w.off[g] = (int)(all.size() / 4);
            // H: members in reverse order (each member's H list is top plane
            // first): the half-step starts on the data the E pass touched last
            for (size_t mi = 0; mi < u.members.size(); mi++) {
                const size_t li = (half == 1 && h_reverse) ? u.members.size() - 1 - mi : mi;
                aefdtd_sim *s = u.members[li];
                const WorkSplit &mw = half == 0 ? s->wsE : s->wsH;
                w.unroll = mw.unroll;
                for (int k = 0; k < mw.n[g]; k++) {
                    const int *it = &s->items_host[size_t(mw.off[g] + k) * 4];
                    all.push_back(it[0]);
                    all.push_back(it[1]);
                    all.push_back(it[2] | (it[3] << 16));
                    all.push_back((int)li);
                }
            }
            w.n[g] = (int)(all.size() / 4) - w.off[g];
        }
    }
    u.items.alloc(std::max<size_t>(all.size(), 4) * sizeof(int), dev_bytes);
    if (!all.empty()) AE_CUDA(cudaMemcpy(u.items.p, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice));
    const size_t n = u.members.size();
    std::vector<int2> blk;
    u.nplane = 0;
    std::vector<StepArgs<T, Tid>> ea(n), ha(n);
    std::vector<SensorStepArgs<T>> sa(n);
    for (size_t li = 0; li < n; li++) {
        aefdtd_sim *s = u.members[li];
        const StepScalars *tbl = s->tables.as<StepScalars>();
        s->make_step_args(ea[li], ha[li], tbl);
        // members that stay in L2 take no up-front L2 prefetch of each item's planes
        if (l2_resident(u)) ea[li].prefetch = ha[li].prefetch = 0;
        s->make_sensor_args(sa[li], tbl);
        if (sa[li].nbp > 0) {
            u.nplane++;
            for (int b = 0; b < sa[li].nbp; b++) blk.push_back(make_int2((int)li, b));
        }
    }
    u.argsE.alloc(sizeof(StepArgs<T, Tid>) * n, dev_bytes);
    u.argsH.alloc(sizeof(StepArgs<T, Tid>) * n, dev_bytes);
    u.sargs.alloc(sizeof(SensorStepArgs<T>) * n, dev_bytes);
    AE_CUDA(cudaMemcpy(u.argsE.p, ea.data(), sizeof(StepArgs<T, Tid>) * n, cudaMemcpyHostToDevice));
    AE_CUDA(cudaMemcpy(u.argsH.p, ha.data(), sizeof(StepArgs<T, Tid>) * n, cudaMemcpyHostToDevice));
    AE_CUDA(cudaMemcpy(u.sargs.p, sa.data(), sizeof(SensorStepArgs<T>) * n, cudaMemcpyHostToDevice));
    u.nblk = (int)blk.size();
    u.blkmap.alloc(std::max<size_t>(blk.size(), 1) * sizeof(int2), dev_bytes);
    if (!blk.empty()) AE_CUDA(cudaMemcpy(u.blkmap.p, blk.data(), blk.size() * sizeof(int2), cudaMemcpyHostToDevice));
    // a subset whose lists do not cut into units keeps the split launches
    if (u.ps && !build_persist<T, Tid>(u, sa)) {
        u.ps_units.release(dev_bytes); u.ps_items.release(dev_bytes); u.ps_prog.release(dev_bytes);
        u.ps_sargs.release(dev_bytes); u.ps_part.release(dev_bytes);
        u.ps = false;
    }
    u.built = true;
}

// Units of the persistent launch (batch_persist.cuh): per member, a band of
// tile_y rows times a z-chunk of kchunk planes; each unit holds the member's
// items of that band and chunk (every group, tagged with its group) and the
// four units it waits on. Normal-mode members get their plane sums per band.
// False (nothing launched) when the members' tile heights differ or an item
// crosses a band or z-chunk.
template <typename T, typename Tid>
bool aefdtd_batch::build_persist(BatchSubset &u, const std::vector<SensorStepArgs<T>> &sa) {
    const int ty = u.members[0]->tile_y;
    const size_t n = u.members.size();
    std::vector<size_t> part_off(n, 0);
    size_t part_n = 0;
    for (size_t li = 0; li < n; li++) {
        const aefdtd_sim *s = u.members[li];
        if (s->tile_y != ty) return false;
        if (sa[li].nbp > 0) {
            part_off[li] = part_n;
            part_n += size_t(seg_len) * ((s->Ny + ty - 1) / ty) * 12;
        }
    }
    u.ps_part.alloc(std::max<size_t>(part_n, 1) * sizeof(double), dev_bytes);
    std::vector<PsUnit> units;
    std::vector<int4> items;
    std::vector<SensorStepArgs<T>> psa(n);
    for (size_t li = 0; li < n; li++) {
        const aefdtd_sim *s = u.members[li];
        const int kc = s->kchunk, nb = (s->Ny + ty - 1) / ty, nch = (s->Nz + kc - 1) / kc;
        const int base = (int)units.size();
        std::vector<std::vector<int4>> eb(size_t(nb) * nch), hb(size_t(nb) * nch);
        for (int half = 0; half < 2; half++) {
            const WorkSplit &w = half ? s->wsH : s->wsE;
            auto &dst = half ? hb : eb;
            for (int g = 0; g < kGroups; g++)
                for (int k = 0; k < w.n[g]; k++) {
                    const int *it = &s->items_host[size_t(w.off[g] + k) * 4];
                    const int x0 = it[0], y0 = it[1], k0 = it[2], k1 = it[3];
                    const int b = y0 / ty, c = k0 / kc;
                    if ((x0 & kHalfItem) || y0 % ty || k1 <= k0 || (k1 - 1) / kc != c) return false;
                    dst[size_t(c) * nb + b].push_back(make_int4(x0, y0, k0 | (k1 << 16), g));
                }
        }
        auto id = [&](int c, int b) { return base + c * nb + b; };
        for (int c = 0; c < nch; c++)
            for (int b = 0; b < nb; b++) {
                PsUnit U{};
                U.m = (int)li;
                U.e_off = (int)items.size();
                items.insert(items.end(), eb[size_t(c) * nb + b].begin(), eb[size_t(c) * nb + b].end());
                U.e_n = (int)items.size() - U.e_off;
                U.h_off = (int)items.size();
                items.insert(items.end(), hb[size_t(c) * nb + b].begin(), hb[size_t(c) * nb + b].end());
                U.h_n = (int)items.size() - U.h_off;
                U.nb[0] = id(c, (b + nb - 1) % nb);
                U.nb[1] = id((c + nch - 1) % nch, b);
                U.nb[2] = id(c, (b + 1) % nb);
                U.nb[3] = id((c + 1) % nch, b);
                U.band = b;
                U.j0 = b * ty;
                U.j1 = std::min(s->Ny, U.j0 + ty);
                if (sa[li].nbp > 0) {
                    const int z0 = c * kc, z1 = std::min(s->Nz, z0 + kc);
                    if (sa[li].kr >= z0 && sa[li].kr < z1) U.planes |= 1;
                    if (sa[li].kt >= z0 && sa[li].kt < z1) U.planes |= 2;
                }
                units.push_back(U);
            }
        psa[li] = sa[li];
        if (sa[li].nbp > 0) {
            psa[li].nbp = nb;
            psa[li].partial = u.ps_part.as<double>() + part_off[li];
        }
    }
    u.ps_nunits = (int)units.size();
    u.ps_ty = ty;
    u.ps_units.alloc(sizeof(PsUnit) * units.size(), dev_bytes);
    AE_CUDA(cudaMemcpy(u.ps_units.p, units.data(), sizeof(PsUnit) * units.size(), cudaMemcpyHostToDevice));
    u.ps_items.alloc(std::max<size_t>(items.size(), 1) * sizeof(int4), dev_bytes);
    if (!items.empty())
        AE_CUDA(cudaMemcpy(u.ps_items.p, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice));
    u.ps_sargs.alloc(sizeof(SensorStepArgs<T>) * n, dev_bytes);
    AE_CUDA(cudaMemcpy(u.ps_sargs.p, psa.data(), sizeof(SensorStepArgs<T>) * n, cudaMemcpyHostToDevice));
    u.ps_prog.alloc(sizeof(int) * units.size(), dev_bytes);
    if (!ps_flags.p) {
        ps_flags.alloc(2 * sizeof(int), dev_bytes);
        AE_CUDA(cudaMemset(ps_flags.p, 0, 2 * sizeof(int)));
    }
    auto cap = ps_capacity.find(ty);
    if (cap == ps_capacity.end()) cap = ps_capacity.emplace(ty, persist_capacity<T, Tid>(ty)).first;
    if (cap->second <= 0) fail(AEFDTD_CUDA_ERROR, "the persistent batch kernel does not fit on the device");
    // the lanes share the device: each subset's launch takes its share of the resident CTAs
    u.ps_grid = std::max(1, std::min(u.ps_nunits, cap->second / lanes_for(u)));
    return true;
}

// The device error flag of the persistent launches: a wait that ran out
// leaves the members' fields part-way through a chunk (reset them).
void aefdtd_batch::check_persist() {
    if (!ps_flags.p) return;
    int h[2] = {0, 0};
    AE_CUDA(cudaMemcpy(h, ps_flags.p, sizeof(h), cudaMemcpyDeviceToHost));
    if (h[0] || h[1]) {
        AE_CUDA(cudaMemset(ps_flags.p, 0, sizeof(h)));
        fail(AEFDTD_TIMEOUT, "a bounded wait of the persistent batch launch ran out");
    }
}

// Same fork/join scheme as a single simulation's half-step (runtime.cpp, run_groups).
template <typename Launch> void aefdtd_batch::run_groups(const WorkSplit &w, Lane &ln, Launch &&launch) {
    int nside = 0;
    for (int g = 1; g < kGroups; g++) nside += w.n[g] > 0;
    if (nside == 0) {
        launch(kGroupInterior, ln.stream);
        return;
    }
    AE_CUDA(cudaEventRecord(ln.ev_fork, ln.stream));
    int si = 0;
    for (int g = 1; g < kGroups; g++) {
        if (w.n[g] <= 0) continue;
        AE_CUDA(cudaStreamWaitEvent(ln.side[si], ln.ev_fork, 0));
        launch(g, ln.side[si]);
        AE_CUDA(cudaEventRecord(ln.ev_join[si], ln.side[si]));
        si++;
    }
    launch(kGroupInterior, ln.stream);
    for (int k = 0; k < si; k++) AE_CUDA(cudaStreamWaitEvent(ln.stream, ln.ev_join[k], 0));
}

// L steps whose scalars are in table entries 0..L-1 of every member.
template <typename T, typename Tid> void aefdtd_batch::enqueue_steps(BatchSubset &u, int L, Lane &ln) {
    if (u.fused) {
        // the lone member's own fused segment (fused.cpp) on this lane's stream;
        // its side streams and events serve only this member
        aefdtd_sim *m0 = u.members[0];
        struct OnLane {
            aefdtd_sim *s;
            cudaStream_t own;
            ~OnLane() { s->stream = own; }
        } on{m0, m0->stream};
        m0->stream = ln.stream;
        const uint64_t l0 = m0->launches;
        m0->enqueue_segment_fused<T, Tid>(L, m0->tables.as<StepScalars>(), false);
        launches += m0->launches - l0;
        return;
    }
    const auto *ea = u.argsE.as<StepArgs<T, Tid>>();
    const auto *ha = u.argsH.as<StepArgs<T, Tid>>();
    if (u.ps) {
        // one cooperative launch for all L steps, then the plane sums of every member
        AE_CUDA(cudaMemsetAsync(u.ps_prog.p, 0, sizeof(int) * u.ps_nunits, ln.stream));
        PersistArgs<T, Tid> pa{};
        pa.ea = ea;
        pa.ha = ha;
        pa.sa = u.ps_sargs.as<SensorStepArgs<T>>();
        pa.units = u.ps_units.as<PsUnit>();
        pa.items = u.ps_items.as<int4>();
        pa.nunits = u.ps_nunits;
        pa.steps = L;
        pa.prog = u.ps_prog.as<int>();
        pa.flags = ps_flags.as<int>();
        pa.wait_cycles = u.members[0]->ps_wait_cycles;
        pa.withhold = u.members[0]->ps_withhold;
        AE_CUDA(launch_persist(pa, u.ps_grid, u.ps_ty, ln.stream));
        launches++;
        if (u.nplane > 0) {
            launch_plane_reduce_batch(u.ps_sargs.as<SensorStepArgs<T>>(), (int)u.members.size(), L, ln.stream);
            launches++;
        }
        return;
    }
    const auto *sa = u.sargs.as<SensorStepArgs<T>>();
    const int4 *it = u.items.as<int4>();
    const int2 *blk = u.blkmap.as<int2>();
    // a lone member launches its own lists (solo: run_groups below takes m0's)
    int groups = u.solo ? group_kernels(u.members[0]->wsE) + group_kernels(u.members[0]->wsH)
                        : group_kernels(u.wsE) + group_kernels(u.wsH);
    // a lone member: its own arguments as launch parameters, its own lists
    aefdtd_sim *m0 = u.members[0];
    StepArgs<T, Tid> se, sh, se_i, sh_i;
    if (u.solo) {
        m0->make_step_args(se, sh, m0->tables.as<StepScalars>());
        if (l2_resident(u)) se.prefetch = sh.prefetch = 0;
    }
    // an oblique member (always alone): its imaginary grid on the same lists, and its R/T sums
    const bool obl = u.solo && m0->obl;
    if (obl) {
        m0->make_step_args(se_i, sh_i, m0->tables.as<StepScalars>(), 1);
        groups *= 2;
    }
    const int4 *mit = m0->items.as<int4>();
    // members with the energy-mode completion sensor: the energy of every step
    std::vector<aefdtd_sim *> cc;
    for (aefdtd_sim *s : u.members)
        if (s->cc_coeff > 0) cc.push_back(s);
    const bool side = u.nblk > 0 || !cc.empty() || obl;
    for (int q = 0; q < L; q++) {
        se.q = sh.q = se_i.q = sh_i.q = q;
        if (u.solo) run_groups(m0->wsE, ln, [&](int g, cudaStream_t st) { launch_e_group(se, mit, m0->wsE, g, st); });
        else run_groups(u.wsE, ln, [&](int g, cudaStream_t st) { launch_e_group_batch(ea, q, it, u.wsE, g, st); });
        if (obl) run_groups(m0->wsE, ln, [&](int g, cudaStream_t st) { launch_e_group(se_i, mit, m0->wsE, g, st); });
        // plane sums and completion energies read E only: beside the H half-step
        if (side) {
            AE_CUDA(cudaEventRecord(ln.ev_sf, ln.stream));
            AE_CUDA(cudaStreamWaitEvent(ln.side_s, ln.ev_sf, 0));
            if (u.nblk > 0) launch_plane_partial_batch(sa, blk, u.nblk, q, ln.side_s);
            if (obl) launches += m0->launch_obl_sums<T>(q, m0->tables.as<StepScalars>(), ln.side_s);
            for (aefdtd_sim *s : cc) {
                if (s->ccft) {
                    // FT mode: the probes' running transforms, with a ring snapshot at check steps
                    const CompletionFT &c = *s->ccft;
                    CcFtArgs<T> fa{};
                    fa.Nx = s->Nx; fa.Ny = s->Ny; fa.Nz = s->Nz; fa.NxNy = (long long)s->Nx * s->Ny;
                    fa.Ex = s->F[0].as<T>(); fa.Ey = s->F[1].as<T>(); fa.Ez = s->F[2].as<T>();
                    fa.np = c.np; fa.n_avg = c.n_avg; fa.step0 = c.step0;
                    fa.pts = c.dpts.as<int>();
                    fa.coef = c.ctab.as<double2>();
                    fa.sc = s->tables.as<StepScalars>();
                    fa.q = q;
                    fa.acc = c.acc.as<double2>();
                    fa.ring = c.ring.as<double>();
                    fa.snap = c.snap.as<double>();
                    launch_completion_ft(fa, ln.side_s);
                } else {
                    launch_energy_partial(s->F[0].as<T>(), s->F[1].as<T>(), s->F[2].as<T>(),
                                          (long long)s->Nx * s->Ny * s->Nz, s->cc_nb,
                                          s->cc_partial.as<double>() + size_t(q) * s->cc_nb, ln.side_s);
                }
            }
            AE_CUDA(cudaEventRecord(ln.ev_sj, ln.side_s));
        }
        if (u.solo) run_groups(m0->wsH, ln, [&](int g, cudaStream_t st) { launch_h_group(sh, mit, m0->wsH, g, st); });
        else run_groups(u.wsH, ln, [&](int g, cudaStream_t st) { launch_h_group_batch(ha, q, it, u.wsH, g, st); });
        if (obl) run_groups(m0->wsH, ln, [&](int g, cudaStream_t st) { launch_h_group(sh_i, mit, m0->wsH, g, st); });
        if (side) AE_CUDA(cudaStreamWaitEvent(ln.stream, ln.ev_sj, 0));
        launches += groups + (u.nblk > 0) + cc.size();
    }
    if (u.nplane > 0) {
        launch_plane_reduce_batch(sa, (int)u.members.size(), L, ln.stream);
        launches++;
    }
    if (obl) {
        launch_obl_reduce(m0->obl->part.as<double>(), m0->obl->nb, m0->tables.as<StepScalars>(),
                          m0->obl->hist.as<double>(), L, ln.stream);
        launches++;
    }
    for (aefdtd_sim *s : cc) {
        if (s->ccft) continue;
        // hist[t] for the chunk's steps (the member's table holds the chunk's first step)
        launch_energy_reduce(s->cc_partial.as<double>(), s->cc_nb, s->tables.as<StepScalars>(), s->cc_hist.as<double>(), L,
                             ln.stream);
        launches++;
    }
}

// L steps of a subset, in chunks: per chunk the members' scalar tables
// (entries 0..), then either the subset's captured graph of graph_steps steps
// (full chunks) or direct launches; then the members' clocks.
template <typename T, typename Tid> void aefdtd_batch::run_segment(BatchSubset &u, int L, Lane &ln) {
    if (!u.built) build_subset<T, Tid>(u);
    std::vector<StepScalars> host(seg_len);
    int done = 0;
    while (done < L) {
        const bool graph = opts.use_graphs >= 0 && !(u.ps && ps_direct) && L - done >= graph_steps;
        const int C = graph ? graph_steps : L - done;
        for (aefdtd_sim *s : u.members) {
            for (int q = 0; q < C; q++) s->fill_scalars(s->tstep + q, q, host[q]);
            if (s->ccft && s->cc_coeff > 0) {
                CompletionFT &c = *s->ccft;
                for (int q = 0; q < C; q++)
                    if ((s->tstep + q) % s->cc_step == 0) host[q].snap = ((s->tstep + q) / s->cc_step) % c.nsnap;
                // CompletionSensor::deep_feed's phases e^{i w step Dt} (s_completion.cpp:149)
                c.rows.resize(size_t(C) * c.np * 2);
                const std::complex<double> Im(0, 1);
                for (int q = 0; q < C; q++) {
                    const int step = s->tstep + q - c.step0;
                    for (int p = 0; p < c.np; p++) {
                        const std::complex<double> e = std::exp(c.w[p] * step * s->Dt * Im);
                        c.rows[(size_t(q) * c.np + p) * 2] = e.real();
                        c.rows[(size_t(q) * c.np + p) * 2 + 1] = e.imag();
                    }
                }
                AE_CUDA(cudaMemcpyAsync(c.ctab.p, c.rows.data(), c.rows.size() * sizeof(double), cudaMemcpyHostToDevice,
                                        ln.stream));
            }
            AE_CUDA(cudaMemcpyAsync(s->tables.as<StepScalars>(), host.data(), sizeof(StepScalars) * C,
                                    cudaMemcpyHostToDevice, ln.stream));
        }
        if (graph) {
            // a fused member's captured chunk reads and writes the buffer sets it was captured with
            cudaGraphExec_t &gx = (u.fused && u.members[0]->set_b) ? u.graph_b : u.graph;
            if (!gx) {
                const uint64_t l0 = launches;
                AE_CUDA(cudaStreamBeginCapture(ln.stream, cudaStreamCaptureModeThreadLocal));
                Error err{AEFDTD_OK, ""};
                try {
                    enqueue_steps<T, Tid>(u, C, ln);
                } catch (const Error &e) {
                    err = e;
                }
                cudaGraph_t gr = nullptr;
                cudaError_t ec = cudaStreamEndCapture(ln.stream, &gr);
                if (err.st == AEFDTD_OK && ec == cudaSuccess) ec = cudaGraphInstantiate(&gx, gr, 0);
                if (gr) cudaGraphDestroy(gr);
                const uint64_t captured = launches - l0;
                launches = l0;
                if (err.st != AEFDTD_OK || ec != cudaSuccess) {
                    gx = nullptr;
                    // a device that cannot capture the cooperative launch runs it directly
                    if (!u.ps) {
                        if (err.st != AEFDTD_OK) throw err;
                        AE_CUDA(ec);
                    }
                    cudaGetLastError();
                    ps_direct = true;
                } else {
                    u.graph_launches = captured;
                }
            }
            if (gx) {
                AE_CUDA(cudaGraphLaunch(gx, ln.stream));
                launches += u.graph_launches;
            } else {
                enqueue_steps<T, Tid>(u, C, ln);
            }
        } else {
            enqueue_steps<T, Tid>(u, C, ln);
        }
        if (u.fused && C % 2) u.members[0]->swap_sets();   // its current state moved to the other set
        for (aefdtd_sim *s : u.members) {
            s->tstep += C;
            for (auto &o : s->oscs) o.step += C;
            rec(s).remaining -= C;
        }
        done += C;
    }
}

// Plane-sum history for every member's whole budget, so that captured graphs
// keep valid pointers (a reallocation rebuilds the member's subset).
template <typename T, typename Tid> void aefdtd_batch::ensure_history() {
    for (auto &u : subsets)
        for (aefdtd_sim *s : u.members) {
            const BatchMember &m = rec(s);
            if (!s->normal || s->tstep + m.remaining <= s->psums_cap) continue;
            DBuf nb;
            const int cap = s->tstep + m.remaining;
            nb.alloc(size_t(cap) * 12 * 8, s->dev_bytes);
            if (s->psums.p)
                AE_CUDA(cudaMemcpy(nb.p, s->psums.p, size_t(s->psums_cap) * 12 * 8, cudaMemcpyDeviceToDevice));
            s->psums.release(s->dev_bytes);
            s->psums = nb;
            s->psums_cap = cap;
            s->graphs_dirty = true;
            u.release(dev_bytes);
        }
    // oblique members: incident sums and R/T history for the whole budget
    for (auto &u : subsets)
        for (aefdtd_sim *s : u.members) {
            if (!s->obl) continue;
            const int cap0 = s->obl->cap;
            s->obl_ensure(s->tstep + rec(s).remaining);
            if (s->obl->cap != cap0) u.release(dev_bytes);
        }
    // completion energies: a history for the whole budget and one chunk of partials
    for (auto &u : subsets)
        for (aefdtd_sim *s : u.members) {
            const BatchMember &m = rec(s);
            if (s->cc_coeff <= 0) continue;
            if (s->ccft) {
                CompletionFT &c = *s->ccft;
                if (!c.snap.p) {
                    // check steps one segment can pass, and one more
                    c.nsnap = s->seg_len / s->cc_step + 2;
                    c.snap.alloc(size_t(c.nsnap) * 6 * c.np * c.n_avg * 8, s->dev_bytes);
                    u.release(dev_bytes);
                }
                continue;
            }
            if (!s->cc_partial.p) {
                s->cc_nb = std::max(1, std::min(2 * 148, (int)(((long long)s->Nx * s->Ny * s->Nz + 4095) / 4096)));
                s->cc_partial.alloc(size_t(s->seg_len) * s->cc_nb * 8, s->dev_bytes);
                u.release(dev_bytes);
            }
            if (s->tstep + m.remaining > s->cc_cap) {
                DBuf nb;
                const int cap = s->tstep + m.remaining;
                nb.alloc(size_t(cap) * 8, s->dev_bytes);
                if (s->cc_hist.p)
                    AE_CUDA(cudaMemcpy(nb.p, s->cc_hist.p, size_t(s->cc_cap) * 8, cudaMemcpyDeviceToDevice));
                s->cc_hist.release(s->dev_bytes);
                s->cc_hist = nb;
                s->cc_cap = cap;
                s->graphs_dirty = true;
                u.release(dev_bytes);
            }
        }
}

// CompletionSensor::completion_check (energy mode, s_completion.cpp:39-43,
// 121-130; FT mode on the ring snapshot taken after the check step) at every
// check step t (t % cc_step == 0) that the member passed in its last segment,
// in order, as aefdtd_sim::completion_check does after each check step of a
// single run. A member that completes at t has its budget
// set to zero; the steps it ran past t (at most one segment) do not enter its
// results, which are read up to t (aefdtd_get_normal_spectra uses cc_stop).
static bool batch_completion_check(aefdtd_sim *s, int t0, int t1, cudaStream_t st) {
    const int first = (t0 + s->cc_step - 1) / s->cc_step * s->cc_step;
    if (first >= t1) return false;
    AE_CUDA(cudaStreamSynchronize(st));
    if (s->ccft) {
        // FT mode (CompletionSensor::completion_check, s_completion.cpp:45-121) on the ring as it
        // stood after each check step
        CompletionFT &c = *s->ccft;
        const size_t n = size_t(6) * c.np * c.n_avg;
        c.ring_host.resize(n);
        for (int t = first; t < t1; t += s->cc_step) {
            const int slot = (t / s->cc_step) % c.nsnap;
            AE_CUDA(cudaMemcpy(c.ring_host.data(), c.snap.as<double>() + size_t(slot) * n, n * 8, cudaMemcpyDeviceToHost));
            if (s->ft_eval(c.ring_host.data(), t + 1 - c.step0)) {
                s->cc_done = true;
                s->cc_stop = t;
                return true;
            }
        }
        return false;
    }
    for (int t = first; t < t1; t += s->cc_step) {
        const int n = t + 1 - s->cc_read;
        if (n > 0) {
            std::vector<double> e(n);
            AE_CUDA(cudaMemcpy(e.data(), s->cc_hist.as<double>() + s->cc_read, n * sizeof(double), cudaMemcpyDeviceToHost));
            for (double x : e) s->cc_max = std::max(s->cc_max, x);
            s->cc_last = e.back();
            s->cc_read = t + 1;
        }
        if (t + 1 < 2 * std::max(s->Nx, std::max(s->Ny, s->Nz))) continue;
        if (s->cc_last / s->cc_max < s->cc_coeff) {
            s->cc_done = true;
            s->cc_stop = t;
            return true;
        }
    }
    return false;
}

// Each subset runs up to max_steps steps in segments of at most seg_len, and
// stops after the segment in which one of its members uses up its budget.
// Subsets run one after another. Returns the most steps any subset ran.
template <typename T, typename Tid> int aefdtd_batch::advance(int max_steps) {
    update_layout();
    ensure_history<T, Tid>();
    // subsets round-robin over the lanes; each subset's segments are queued
    // in turn (stream order within a lane, concurrency across lanes)
    std::vector<int> done(subsets.size(), 0);
    const std::vector<int> lane = lane_plan();
    int most = 0;
    bool more = true;
    while (more) {
        more = false;
        for (size_t k = 0; k < subsets.size(); k++) {
            BatchSubset &u = subsets[k];
            if (done[k] < 0 || done[k] >= max_steps) continue;
            int L = std::min(seg_len, max_steps - done[k]);
            for (aefdtd_sim *s : u.members) L = std::min(L, rec(s).remaining);
            if (L <= 0) { done[k] = -done[k] - 1; continue; }
            std::vector<int> t0;
            for (aefdtd_sim *s : u.members) t0.push_back(s->tstep);
            run_segment<T, Tid>(u, L, lanes[lane[k]]);
            for (size_t i = 0; i < u.members.size(); i++) {
                aefdtd_sim *s = u.members[i];
                if (s->cc_coeff > 0 && !s->cc_done &&
                    batch_completion_check(s, t0[i], s->tstep, lanes[lane[k]].stream))
                    rec(s).remaining = 0;
            }
            done[k] += L;
            most = std::max(most, done[k]);
            bool finished = false;
            for (aefdtd_sim *s : u.members) finished |= rec(s).remaining == 0;
            if (finished) done[k] = -done[k] - 1;   // stops after this segment
            else more = more || done[k] < max_steps;
        }
    }
    sync_lanes();
    AE_CUDA(cudaGetLastError());
    check_persist();
    return most;
}

// Device seconds of `reps` full segments of every subset, after one warm-up
// segment (which captures the graphs).
template <typename T, typename Tid> double aefdtd_batch::time_segments(int reps) {
    update_layout();
    const std::vector<int> lane = lane_plan();
    for (size_t k = 0; k < subsets.size(); k++) run_segment<T, Tid>(subsets[k], seg_len, lanes[lane[k]]);
    sync_lanes();
    check_persist();
    int a = 0, b = 0;   // host clock over all lanes (the device is idle before)
    const auto t0 = std::chrono::steady_clock::now();
    for (int r = 0; r < reps; r++)
        for (size_t k = 0; k < subsets.size(); k++) run_segment<T, Tid>(subsets[k], seg_len, lanes[lane[k]]);
    sync_lanes();
    check_persist();
    (void)a; (void)b;
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Per size class: tile height in {2, 4, 8} x z-block depth in {4, 8}, timed
// on that class's members alone; then the L2 budget in {48 MiB, 96 MiB, no
// limit} over all members. Members must be at step 0; they are reset to step
// 0 afterwards.
template <typename T, typename Tid> void aefdtd_batch::autotune() {
    std::vector<int> saved(members.size());
    for (size_t i = 0; i < members.size(); i++) {
        if (members[i].sim->tstep != 0) fail(AEFDTD_NOT_READY, "autotune needs every member at step 0");
        saved[i] = members[i].remaining;
    }
    const long long budget0 = l2_budget;
    // every trial restarts the members at step 0 and runs two segments: the
    // plane-sum history must hold them (three, with margin)
    for (auto &m : members) {
        aefdtd_sim *s = m.sim;
        if (s->normal && s->psums_cap < 3 * seg_len) {
            s->psums.release(s->dev_bytes);
            s->psums.alloc(size_t(3 * seg_len) * 12 * 8, s->dev_bytes);
            s->psums_cap = 3 * seg_len;
            s->graphs_dirty = true;
        }
    }
    auto restart = [&] {
        sync_lanes();
        for (auto &m : members) m.sim->zero_state();
        };
    auto apply = [&](int cls, const SizeClass &c) {
        classes[cls] = c;
        for (auto &m : members)
            if (m.cls == cls) {
                m.sim->tile_y = c.tile_y;
                m.sim->kchunk_override = c.kchunk;
                m.sim->work_dirty = true;
                m.sim->build_work();
            }
    };
    std::vector<int> keys;
    for (auto &kv : classes) keys.push_back(kv.first);
    for (int cls : keys) {
        // only this class's members take part in its trials
        for (auto &m : members) m.remaining = m.cls == cls ? (1 << 30) : 0;
        double best = 1e30;
        SizeClass pick = classes[cls];
        for (int ty : {2, 4, 8})
            for (int kc : {4, 8}) {
                SizeClass c{ty, kc};
                apply(cls, c);
                drop_layout();
                restart();
                const double t = time_segments<T, Tid>(1);
                if (t < best) { best = t; pick = c; }
            }
        apply(cls, pick);
    }
    // L2 budget, lanes and the persistent launch over all members
    for (auto &m : members) m.remaining = 1 << 30;
    double best = 1e30;
    long long pick = budget0;
    int pick_lanes = n_lanes, pick_ps = persistent;
    for (int ps : {0, 1})
        for (long long b : {48LL << 20, 96LL << 20, -1LL})
            for (int nl : {1, 2, 4}) {
                if (b < 0 && nl > 1) continue;   // one subset per class: lanes only split classes
                l2_budget = b;
                n_lanes = nl;
                persistent = ps;
                drop_layout();
                restart();
                const double t = time_segments<T, Tid>(1);
                if (t < best) { best = t; pick = b; pick_lanes = nl; pick_ps = ps; }
            }
    l2_budget = pick;
    n_lanes = pick_lanes;
    persistent = pick_ps;
    drop_layout();
    restart();
    for (size_t i = 0; i < members.size(); i++) members[i].remaining = saved[i];
}

namespace aefdtd {
void batch_detach(void *bp, aefdtd_sim *s) {
    auto *b = static_cast<aefdtd_batch *>(bp);
    const int i = b->find(s);
    if (i < 0) return;
    b->set_device();
    for (int k = 0; k < b->n_lanes; k++) cudaStreamSynchronize(b->lanes[k].stream);
    for (auto &u : b->subsets) {
        auto it = std::find(u.members.begin(), u.members.end(), s);
        if (it != u.members.end()) {
            u.release(b->dev_bytes);
            u.members.erase(it);
            u.bytes -= s->dev_bytes;
        }
    }
    b->members.erase(b->members.begin() + i);
    s->batch = nullptr;
    s->tma_allowed = true;
    s->work_dirty = true;
}
}  // namespace aefdtd

// ------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------


template <typename F> static aefdtd_status bguarded(aefdtd_batch *b, F &&f) {
    try {
        f();
        if (b) b->last_error.clear();
        return AEFDTD_OK;
    } catch (Error &e) {
        if (b) b->last_error = e.msg;
        return e.st;
    } catch (std::bad_alloc &) {
        if (b) b->last_error = "host allocation failed";
        return AEFDTD_OOM;
    } catch (std::exception &e) {
        if (b) b->last_error = e.what();
        return AEFDTD_BAD_ARG;
    }
}

#define AEFDTD_BATCH_DISPATCH(b, fn)                                        \
    do {                                                                    \
        if ((b)->fp64) {                                                    \
            if ((b)->id_bytes == 1) fn(double, uint8_t); else fn(double, uint16_t); \
        } else {                                                            \
            if ((b)->id_bytes == 1) fn(float, uint8_t); else fn(float, uint16_t);   \
        }                                                                   \
    } while (0)

extern "C" {

aefdtd_status aefdtd_batch_create(const aefdtd_batch_opts *opts, aefdtd_batch **out) {
    if (!out) return AEFDTD_BAD_ARG;
    *out = nullptr;
    auto *b = new aefdtd_batch();
    aefdtd_status st = bguarded(b, [&] {
        if (opts) {
            if (opts->abi_version != AEFDTD_ABI_VERSION) fail(AEFDTD_BAD_ARG, "abi_version mismatch");
            b->opts = *opts;
        } else {
            b->opts.abi_version = AEFDTD_ABI_VERSION;
        }
        if (b->opts.l2_budget_bytes != 0) b->l2_budget = b->opts.l2_budget_bytes;
        if (b->opts.graph_steps > 0) b->graph_steps = b->opts.graph_steps;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) fail(AEFDTD_NO_DEVICE, "no CUDA device visible");
        b->device = b->opts.device;
        if (b->device < 0 || b->device >= ndev) fail(AEFDTD_BAD_ARG, "device ordinal out of range");
        AE_CUDA(cudaSetDevice(b->device));
        for (auto &ln : b->lanes) ln.create();
        b->stream = b->lanes[0].stream;
        if (b->opts.lanes > 0) b->n_lanes = std::min(b->opts.lanes, kMaxLanes);
        if (const char *lw = std::getenv("AEFDTD_LANE_WINDOW_MIB")) b->lane_window = std::max(1LL, atoll(lw)) << 20;
        b->persistent = b->opts.persistent != 0;
        if (const char *ps = std::getenv("AEFDTD_BATCH_PERSIST")) b->persistent = atoi(ps) != 0;
    });
    if (st != AEFDTD_OK) {
        delete b;
        return st;
    }
    *out = b;
    return AEFDTD_OK;
}

aefdtd_status aefdtd_batch_destroy(aefdtd_batch *b) {
    if (!b) return AEFDTD_BAD_ARG;
    delete b;
    return AEFDTD_OK;
}

const char *aefdtd_batch_last_error(const aefdtd_batch *b) { return b ? b->last_error.c_str() : ""; }

aefdtd_status aefdtd_batch_add(aefdtd_batch *b, aefdtd_sim *s, int32_t steps) {
    if (!b || !s) return AEFDTD_BAD_ARG;
    return bguarded(b, [&] {
        if (steps < 0) fail(AEFDTD_BAD_ARG, "negative step budget");
        if (s->batch) fail(AEFDTD_BAD_ARG, "the simulation is already in a batch");
        if (s->device != b->device) fail(AEFDTD_BAD_ARG, "the simulation is on another device");
        if (!s->map_set) fail(AEFDTD_NOT_READY, "no material map");
        if (s->g.mode == AEFDTD_MODE_NORMAL && !s->normal) fail(AEFDTD_NOT_READY, "normal mode needs aefdtd_setup_normal");
        if (s->g.mode == AEFDTD_MODE_OBLIQUE && !s->obl) fail(AEFDTD_NOT_READY, "oblique mode needs aefdtd_setup_oblique");
        if (!s->sensors.empty()) fail(AEFDTD_BAD_ARG, "batch members carry no planar DFT sensors (normal-mode plane sums only)");
        if (!s->fmaps.empty()) fail(AEFDTD_BAD_ARG, "batch members carry no field sensors");
        if (s->Nz >= 32768) fail(AEFDTD_BAD_ARG, "batch members need Nz < 32768 (k1 << 16 in an int32 item)");
        s->set_device();
        s->finalize_tables();
        s->tma_allowed = false;      // merged lists take every interior item
        s->work_dirty = true;
        s->build_work();             // lists for its subset follow in build_subset
        if (!b->typed) {
            b->typed = true;
            b->fp64 = s->fp64;
            b->id_bytes = s->id_bytes;
            b->seg_len = s->seg_len;
            b->graph_steps = std::max(1, std::min(b->graph_steps, b->seg_len));
        } else if (s->fp64 != b->fp64 || s->id_bytes != b->id_bytes || s->seg_len != b->seg_len) {
            fail(AEFDTD_BAD_ARG, "batch members share precision, material-id width and DFT block");
        }
        AE_CUDA(cudaStreamSynchronize(s->stream));
        BatchMember m;
        m.sim = s;
        m.remaining = (s->cc_coeff > 0 && s->cc_done) ? 0 : steps;
        // an oblique member (two coupled grids) always runs as a subset of its own
        m.cls = s->obl ? b->next_solo_class-- : b->class_key(s);
        auto it = b->classes.find(m.cls);
        if (it == b->classes.end()) {
            SizeClass c;
            c.tile_y = b->opts.tile_y == 2 || b->opts.tile_y == 8 ? b->opts.tile_y : 4;
            c.kchunk = b->opts.kchunk;
            b->classes[m.cls] = c;
            it = b->classes.find(m.cls);
        }
        if (s->tile_y != it->second.tile_y || s->kchunk_override != it->second.kchunk) {
            s->tile_y = it->second.tile_y;
            s->kchunk_override = it->second.kchunk;
            s->work_dirty = true;
            s->build_work();
        }
        s->batch = b;
        b->members.push_back(m);
    });
}

aefdtd_status aefdtd_batch_remove(aefdtd_batch *b, aefdtd_sim *s) {
    if (!b || !s) return AEFDTD_BAD_ARG;
    return bguarded(b, [&] {
        if (b->find(s) < 0) fail(AEFDTD_BAD_ARG, "not a member of this batch");
        batch_detach(b, s);
    });
}

aefdtd_status aefdtd_batch_set_budget(aefdtd_batch *b, aefdtd_sim *s, int32_t steps) {
    if (!b || !s) return AEFDTD_BAD_ARG;
    return bguarded(b, [&] {
        const int i = b->find(s);
        if (i < 0) fail(AEFDTD_BAD_ARG, "not a member of this batch");
        if (steps < 0) fail(AEFDTD_BAD_ARG, "negative step budget");
        b->members[i].remaining = steps;
    });
}

aefdtd_status aefdtd_batch_autotune(aefdtd_batch *b) {
    if (!b) return AEFDTD_BAD_ARG;
    return bguarded(b, [&] {
        if (b->members.empty()) fail(AEFDTD_NOT_READY, "empty batch");
        b->set_device();
#define AEFDTD_AT(T, Tid) b->autotune<T, Tid>()
        AEFDTD_BATCH_DISPATCH(b, AEFDTD_AT);
#undef AEFDTD_AT
    });
}

aefdtd_status aefdtd_batch_advance(aefdtd_batch *b, int32_t max_steps, int32_t *steps_done) {
    if (!b) return AEFDTD_BAD_ARG;
    return bguarded(b, [&] {
        if (max_steps < 0) fail(AEFDTD_BAD_ARG, "negative step count");
        b->set_device();
        int done = 0;
        if (!b->members.empty()) {
#define AEFDTD_ADV(T, Tid) done = b->advance<T, Tid>(max_steps)
            AEFDTD_BATCH_DISPATCH(b, AEFDTD_ADV);
#undef AEFDTD_ADV
        }
        if (steps_done) *steps_done = done;
    });
}

aefdtd_status aefdtd_batch_finished(aefdtd_batch *b, aefdtd_sim **out, int32_t cap, int32_t *n) {
    if (!b || !n) return AEFDTD_BAD_ARG;
    return bguarded(b, [&] {
        int k = 0;
        for (auto &m : b->members)
            if (m.remaining == 0) {
                if (out && k < cap) out[k] = m.sim;
                k++;
            }
        *n = k;
    });
}

aefdtd_status aefdtd_batch_get_info(aefdtd_batch *b, aefdtd_batch_info *info) {
    if (!b || !info) return AEFDTD_BAD_ARG;
    return bguarded(b, [&] {
        if (b->typed) b->update_layout();
        std::memset(info, 0, sizeof(*info));
        info->n_members = (int32_t)b->members.size();
        for (auto &m : b->members) {
            if (m.remaining > 0) {
                info->n_active++;
                info->cells += (int64_t)m.sim->Nx * m.sim->Ny * m.sim->Nz;
            }
            info->member_bytes += (int64_t)m.sim->dev_bytes;
        }
        info->n_subsets = (int32_t)b->subsets.size();
        info->n_lanes = b->n_lanes;
        info->n_persistent = 0;
        for (const auto &u : b->subsets) info->n_persistent += u.built && u.ps;
        info->l2_budget_bytes = b->l2_budget;
        info->launches = b->launches;
        info->batch_bytes = (int64_t)b->dev_bytes;
        int c = 0;
        for (auto &kv : b->classes) {
            if (c < AEFDTD_BATCH_MAX_CLASSES) {
                info->class_key[c] = kv.first;
                info->class_tile_y[c] = kv.second.tile_y;
                info->class_kchunk[c] = kv.second.kchunk;
            }
            c++;
        }
        info->n_classes = c;
    });
}

}  // extern "C"
