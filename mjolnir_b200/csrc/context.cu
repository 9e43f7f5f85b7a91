// The context behind the C ABI: host-side system descriptions, packing of all
// live systems into one device arena, and the per-step schedule
//   integrate_first -> margin -> [rebuild per term] -> local forces ->
//   pair forces per term -> integrate_last
// captured once as a CUDA graph and replayed.  This is the work of
// MolecularDynamicsSimulator::step + BAOABLangevinIntegrator::step +
// ForceField::calc_force (core/MolecularDynamicsSimulator.hpp:83-102,
// core/BAOABLangevinIntegrator.hpp:170-240, core/ForceField.hpp:101-109)
// for every system of the arena at once.
#include "../../include/mjolnir_b200.h"
#include "kernels.cuh"
#include "model.hpp"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace mjg {

std::atomic<long long> g_launches{0};
void note_launches(int k) {g_launches.fetch_add(k, std::memory_order_relaxed);}


namespace {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(call)                                                                         \
    do {                                                                                 \
        const cudaError_t e_ = (call);                                                   \
        if(e_ != cudaSuccess)                                                            \
        {                                                                                \
            throw Error(e_ == cudaErrorMemoryAllocation ? MJG_ENOMEM : MJG_ECUDA,        \
                        std::string(#call) + ": " + cudaGetErrorString(e_));             \
        }                                                                                \
    } while(0)

// device buffer with byte accounting
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;            // size in use
    size_t cap = 0;              // size allocated
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() {release();}
    void release() {if(p) {cudaFree(p); p = nullptr;} bytes = 0; cap = 0;}
    void alloc(size_t b)
    {
        release();
        if(b == 0) {return;}
        CK(cudaMalloc(&p, b));
        bytes = cap = b;
    }
    // keeps the allocation when it is large enough, else grows it to twice
    // the request (a serving arena that fills up over its first commits
    // then reallocates a few times, not at every commit)
    void ensure(size_t b)
    {
        if(b > cap)
        {
            release();
            const size_t want = 2 * b;
            CK(cudaMalloc(&p, want));
            cap = want;
        }
        bytes = b;
    }
    template<typename T> T* as() const {return static_cast<T*>(p);}
};

struct HostGlobal {
    bool on = false;
    int kind = 0;                // potential within the term's family (ExvKind / LjKind)
    int power = 12;              // InversePower n
    double eps = 0.0, cutoff_ratio = 0.0, margin = 0.5;
    std::vector<int64_t> idx;
    std::vector<double> p0, p1;
    int ignore_mol = IGN_NOTHING;
    std::vector<std::pair<std::string, int>> within;
};
struct HostLocal {
    std::string kind = "none";
    std::vector<int64_t> idx;
    std::vector<double> k, v0;
    std::vector<int32_t> n;
    int64_t m() const {return (int64_t)k.size();}
};
struct HostSystem {
    bool alive = true;
    bool resident = false;       // part of the current arena
    bool frozen = false;         // does not advance (serving: a finished job)
    int arena_slot = -1;
    int64_t n = 0;
    int boundary = B_UNLIMITED;
    double lower[3] = {0, 0, 0}, upper[3] = {0, 0, 0};
    std::vector<double> pos, vel, mass, force, accel;
    bool force_valid = false;
    bool accel_valid = false;    // UnderdampedLangevin acceleration carried over a commit
    double T = 300.0, I = 0.1;
    std::vector<std::pair<std::string, std::pair<int64_t, int64_t>>> connections;
    HostGlobal g[NGLOBAL];
    HostLocal bond, angle, dihd;
    int integrator = I_BAOAB;
    double dt = 0.01;
    std::vector<double> gamma;
    uint64_t seed = 0;
    uint64_t step = 0;
    int rebuilds[NGLOBAL] = {0, 0, 0};
    int64_t off = 0;             // particle offset in the arena
    // derived once, by the first commit that packs the system (topology and
    // interactions are fixed from then on): molecule ids, exclusion lists in
    // local indices, local terms ordered by their smallest particle
    bool derived = false;
    std::vector<int32_t> mol_local;
    std::vector<long long> ex_start_local[NGLOBAL];   // n + 1 entries
    std::vector<int> ex_idx_local[NGLOBAL];
};

struct TermDev {
    DevBuf part_particle, part_p0, part_p1, part_lead, part_sys, part_cell;
    DevBuf cell_count, cell_start, cell_fill, work, part_chunks, cell_chunks, flagged;
    DevBuf slot_part, slot_particle, slot_lead, slot_sys, slot_pd, slot_p1, slot_of, slot_w;
    DevBuf nnb, nbr, max_count, any_rebuild;
    DevBuf ex_start, ex_idx;
    int cap_alloc = 0;           // capacity the nbr buffer was sized for
    bool tpp_fixed = false;      // threads per slot chosen by the caller
    int tpp_choice = 1;          // ... and its value (kept across commits)
    int unroll_choice = 1;       // partner batch depth of the force launch
    int schedule_choice = 0;     // force launch schedule (0 slot per threads, 1 warp-balanced,
                                 // 2 block-vector, 3 block-vector with length-sorted threads,
                                 // 4 slot per threads with length-sorted groups, 5 slot-major lists)
    bool half_choice = false;    // half lists (mixed form only)
    int build_lanes_choice = 32; // lanes per slot of the list build (4, 8, 16, 32)
    bool build_lanes_fixed = false;  // ... chosen by the caller (else from the expected candidates)
    TermArrays t{};
};

}  // namespace
}  // namespace mjg

struct mjg_context {
    int device = 0;
    int precision = mjg::P_FP64;
    bool graphs = true;
    bool rollback = true;
    cudaStream_t stream = nullptr;
    // branches of the step: one per global term (rebuild, forces) and one for
    // the bonded terms, forked from and joined back into `stream`
    cudaStream_t side[mjg::NGLOBAL + 1] = {};
    cudaStream_t gate_body[mjg::NGLOBAL] = {};  // captures the conditional rebuild bodies
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_join[mjg::NGLOBAL + 1] = {};
    std::string err;
    std::vector<mjg::HostSystem> sys;

    // arena
    bool committed = false;
    std::vector<int> arena_ids;            // arena slot -> system id
    long long n_tot = 0;
    mjg::DevBuf d_sys, d_pos, d_vel, d_force, d_coef, d_psys, d_staging, d_mol;
    mjg::DevBuf d_accel;                        // UnderdampedLangevin accelerations
    mjg::DevBuf b_sys, b_pos, b_vel, b_force, b_accel;   // rollback copies
    mjg::DevBuf d_force_scratch;
    double* h_pinned = nullptr;             // page-locked host staging (state, forces)
    size_t h_pinned_bytes = 0;
    void* h_pack = nullptr;                 // page-locked packing buffer of commit
    size_t h_pack_bytes = 0;
    mjg::TermDev term[mjg::NGLOBAL];
    mjg::DevBuf l_bond_idx, l_bond_k, l_bond_v0, l_bond_sys;
    mjg::DevBuf l_angle_idx, l_angle_k, l_angle_v0, l_angle_sys;
    mjg::DevBuf l_dihd_idx, l_dihd_k, l_dihd_n, l_dihd_v0, l_dihd_sys;
    mjg::DevBuf l_win_bond, l_win_angle, l_win_dihd, l_bond_kv, l_angle_kv, l_dihd_p;
    mjg::Arena arena{};
    mjg::LocalArrays local{};
    std::vector<mjg::SysDev> h_sys;

    cudaGraph_t graph = nullptr;            // first step of a chunk
    cudaGraphExec_t graph_exec = nullptr;
    cudaGraph_t graph2 = nullptr;           // later steps: closing kick fused in
    cudaGraphExec_t graph2_exec = nullptr;
    cudaGraph_t graph4 = nullptr;           // four such steps in one graph (fewer launches)
    cudaGraphExec_t graph4_exec = nullptr;
    long long graph_nodes = 0, graph2_nodes = 0, graph4_nodes = 0;
    bool graph_dirty = true;
};

namespace mjg {
namespace {

int64_t device_bytes(const mjg_context* c)
{
    int64_t b = 0;
    const DevBuf* bufs[] = {&c->d_sys, &c->d_pos, &c->d_vel, &c->d_force, &c->d_coef, &c->d_psys,
                            &c->d_staging, &c->d_mol, &c->b_sys, &c->b_pos, &c->b_vel, &c->b_force,
                            &c->d_accel, &c->b_accel,
                            &c->d_force_scratch, &c->l_bond_idx, &c->l_bond_k, &c->l_bond_v0,
                            &c->l_bond_sys, &c->l_angle_idx, &c->l_angle_k, &c->l_angle_v0,
                            &c->l_angle_sys, &c->l_dihd_idx, &c->l_dihd_k, &c->l_dihd_n,
                            &c->l_dihd_v0, &c->l_dihd_sys, &c->l_win_bond, &c->l_win_angle,
                            &c->l_win_dihd, &c->l_bond_kv, &c->l_angle_kv, &c->l_dihd_p};
    for(auto* x : bufs) {b += (int64_t)x->cap;}
    for(const auto& t : c->term)
    {
        const DevBuf* tb[] = {&t.part_particle, &t.part_p0, &t.part_p1, &t.part_lead, &t.part_sys,
                              &t.part_cell, &t.cell_count, &t.cell_start, &t.cell_fill,
                              &t.work, &t.part_chunks, &t.cell_chunks, &t.flagged, &t.slot_part, &t.slot_particle, &t.slot_lead,
                              &t.slot_sys, &t.slot_pd, &t.slot_p1, &t.slot_of, &t.slot_w, &t.nnb, &t.nbr, &t.max_count,
                              &t.any_rebuild, &t.ex_start, &t.ex_idx};
        for(auto* x : tb) {b += (int64_t)x->cap;}
    }
    return b;
}

template<typename T>
void upload(DevBuf& d, const std::vector<T>& h, cudaStream_t s)
{
    d.alloc(sizeof(T) * h.size());
    if(!h.empty()) {CK(cudaMemcpyAsync(d.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));}
}

HostSystem& get_sys(mjg_context* c, int id)
{
    if(id < 0 || id >= (int)c->sys.size() || !c->sys[id].alive)
    {
        throw Error(MJG_EINVAL, "no such system: " + std::to_string(id));
    }
    return c->sys[id];
}

HostSystem& get_resident(mjg_context* c, int id)
{
    HostSystem& s = get_sys(c, id);
    if(!c->committed || !s.resident) {throw Error(MJG_ESTATE, "system " + std::to_string(id) + " is not committed");}
    return s;
}

void release_graph(mjg_context* c)
{
    if(c->graph_exec) {cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr;}
    if(c->graph) {cudaGraphDestroy(c->graph); c->graph = nullptr;}
    if(c->graph2_exec) {cudaGraphExecDestroy(c->graph2_exec); c->graph2_exec = nullptr;}
    if(c->graph2) {cudaGraphDestroy(c->graph2); c->graph2 = nullptr;}
    if(c->graph4_exec) {cudaGraphExecDestroy(c->graph4_exec); c->graph4_exec = nullptr;}
    if(c->graph4) {cudaGraphDestroy(c->graph4); c->graph4 = nullptr;}
    c->graph_dirty = true;
}

// ------------------------------------------------------------ schedule

void enqueue_forces(mjg_context* c, const Arena& a, bool nf, bool ne)
{
    launch_local(a, c->local, 7, nf, ne, 0, c->stream);
    for(int g = 0; g < NGLOBAL; ++g) {launch_pair(a, g, c->term[g].t, nf, ne, 0, c->stream);}
}

// One integrator step without its closing half-kick.  kick: open with the
// previous step's closing half-kick (fused into the same pass).
// The step after the integrator's first pass (which also refreshes every
// term's slot coordinates) forks into independent branches: each global term
// rebuilds its lists (for the flagged systems) and, in the mixed form, adds
// its forces; the bonded terms run beside them.  The mixed form's force
// launches add with integer atomics (exact in any order), so all branches may
// overlap; the FP64 form adds its pair forces after the join, one term after
// the other.
// arenas with at most this many systems carrying a term put that term's
// rebuild behind a graph conditional (measured: a 10,000-bead melt alone steps
// 10-18 % faster, a 256-system batch 5 % slower with it)
constexpr int GATE_MAX_SYSTEMS = 4;

void enqueue_step_body(mjg_context* c, bool kick, bool capturing)
{
    const Arena& a = c->arena;
    cudaStream_t st = c->stream;
    TermArrays ts[NGLOBAL] = {c->term[0].t, c->term[1].t, c->term[2].t};
    // while capturing: one conditional handle per global term of this step,
    // reset to 0 at each launch of the graph and set by the margin kernel
    RebuildGate gate{};
    if(capturing)
    {
        cudaStreamCaptureStatus cs;
        cudaGraph_t graph = nullptr;
        CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, nullptr, nullptr));
        for(int g = 0; g < NGLOBAL; ++g)
        {
            if(!ts[g].on || ts[g].np == 0) {continue;}
            // only in arenas of a few systems: with many, some system
            // rebuilds nearly every step and the `if` node only adds latency
            int with_term = 0;
            for(int id : c->arena_ids) {with_term += c->sys[id].g[g].on ? 1 : 0;}
            if(with_term > GATE_MAX_SYSTEMS) {continue;}
            CK(cudaGraphConditionalHandleCreate(&gate.handle[g], graph, 0, cudaGraphCondAssignDefault));
            gate.on[g] = 1;
        }
    }
    launch_integrate_first(a, st, kick);
    launch_margin(a, ts, st, gate);
    const bool mixed = a.precision == P_MIXED;
    CK(cudaEventRecord(c->ev_fork, st));
    auto branch = [&](int b, auto&& body) {
        CK(cudaStreamWaitEvent(c->side[b], c->ev_fork, 0));
        body(c->side[b]);
        CK(cudaEventRecord(c->ev_join[b], c->side[b]));
        CK(cudaStreamWaitEvent(st, c->ev_join[b], 0));
    };
    for(int g = 0; g < NGLOBAL; ++g)
    {
        TermArrays& t = c->term[g].t;
        if(!t.on || t.np == 0) {continue;}
        branch(g, [&](cudaStream_t s) {
            if(gate.on[g])
            {
                // an `if` node after the branch's current dependencies, its
                // body captured from a stream of its own
                cudaStreamCaptureStatus cs;
                cudaGraph_t graph = nullptr;
                const cudaGraphNode_t* deps = nullptr;
                size_t ndeps = 0;
                CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, &deps, &ndeps));
                cudaGraphNodeParams p{};
                p.type = cudaGraphNodeTypeConditional;
                p.conditional.handle = gate.handle[g];
                p.conditional.type = cudaGraphCondTypeIf;
                p.conditional.size = 1;
                cudaGraphNode_t node = nullptr;
                CK(cudaGraphAddNode(&node, graph, deps, ndeps, &p));
                cudaGraph_t body = p.conditional.phGraph_out[0];
                CK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
                CK(cudaStreamBeginCaptureToGraph(c->gate_body[g], body, nullptr, nullptr, 0,
                                                 cudaStreamCaptureModeThreadLocal));
                launch_rebuild(a, g, t, 0, c->gate_body[g]);
                cudaGraph_t done = nullptr;
                CK(cudaStreamEndCapture(c->gate_body[g], &done));
            }
            else
            {
                launch_rebuild(a, g, t, 0, s);
            }
            if(mixed) {launch_pair(a, g, t, true, false, 0, s, false);}
        });
    }
    branch(NGLOBAL, [&](cudaStream_t s) {launch_local(a, c->local, 7, true, false, 0, s);});
    if(!mixed)
    {
        for(int g = 0; g < NGLOBAL; ++g) {launch_pair(a, g, c->term[g].t, true, false, 0, st, false);}
    }
}


void capture_one(mjg_context* c, bool kick, cudaGraph_t& g, cudaGraphExec_t& ge, long long& nodes,
                 int steps = 1)
{
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    for(int k = 0; k < steps; ++k) {enqueue_step_body(c, kick, true);}
    g = nullptr;
    CK(cudaStreamEndCapture(c->stream, &g));
    CK(cudaGraphInstantiate(&ge, g, 0));
    size_t nn = 0;
    CK(cudaGraphGetNodes(g, nullptr, &nn));
    nodes = (long long)nn;
}

void capture_graph(mjg_context* c)
{
    release_graph(c);
    const long long before = g_launches.load();
    capture_one(c, false, c->graph, c->graph_exec, c->graph_nodes);
    capture_one(c, true, c->graph2, c->graph2_exec, c->graph2_nodes);
    capture_one(c, true, c->graph4, c->graph4_exec, c->graph4_nodes, 4);
    // capture counted the launches once; graph replays add them per replay
    g_launches.fetch_sub(g_launches.load() - before);
    c->graph_dirty = false;
}

void download_sys(mjg_context* c)
{
    c->h_sys.resize(c->arena_ids.size());
    if(!c->h_sys.empty())
    {
        CK(cudaMemcpyAsync(c->h_sys.data(), c->d_sys.p, sizeof(SysDev) * c->h_sys.size(),
                           cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
}

void upload_sys(mjg_context* c)
{
    if(!c->h_sys.empty())
    {
        CK(cudaMemcpyAsync(c->d_sys.p, c->h_sys.data(), sizeof(SysDev) * c->h_sys.size(),
                           cudaMemcpyHostToDevice, c->stream));
    }
}

// room for growth; a multiple of 16 so that every threads-per-slot choice
// tiles the blocked layout
int list_capacity(int max_count) {return ((max_count + max_count / 4 + 16) + 31) / 32 * 32;}

// threads per slot of the pair kernel from the longest list, widened for
// arenas with few slots until the launch fills the GPU (about 148 SMs x 1,024
// threads; a small system otherwise leaves most SMs idle and each thread
// walks a long chain of dependent loads); refined by the autotuner through
// mjg_set_threads_per_particle
int default_tpp(int max_count, long long slots)
{
    int tpp = max_count >= 192 ? 8 : (max_count >= 48 ? 4 : (max_count >= 12 ? 2 : 1));
    while(tpp < 32 && tpp < max_count && slots * tpp < 148LL * 1024) {tpp *= 2;}
    return tpp;
}

// words per slot the neighbour buffer holds for capacity cap: a multiple of
// 32 and at least 32 (the widest group of the blocked layout), because the
// force launches read a slot's first block before they know its length and
// a blocked row holds tpp words of every slot
size_t list_words(int cap) {return (size_t)std::max((cap + 31) / 32 * 32, 32);}

// sizes the neighbour arrays of term g for capacity cap (the buffer only grows)
void alloc_lists(mjg_context* c, int g, int cap)
{
    TermDev& T = c->term[g];
    T.nbr.ensure(sizeof(int) * list_words(cap) * (size_t)(T.t.np > 0 ? T.t.np : 1));
    T.t.nbr = T.nbr.as<int>();
    T.t.cap = cap;
    T.cap_alloc = cap;
    release_graph(c);
}

// forced rebuild of every list; grows capacities until nothing overflows
void rebuild_all(mjg_context* c)
{
    // every term's first attempt, then one synchronisation; a term whose
    // lists overflowed grows them and is rebuilt alone (up to three times)
    int mx[NGLOBAL] = {};
    auto attempt = [&](int g) {
        TermDev& T = c->term[g];
        CK(cudaMemsetAsync(T.t.max_count, 0, sizeof(int), c->stream));
        launch_rebuild(c->arena, g, T.t, 1, c->stream);
        CK(cudaMemcpyAsync(&mx[g], T.t.max_count, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    };
    for(int g = 0; g < NGLOBAL; ++g)
    {
        if(c->term[g].t.on && c->term[g].t.np > 0) {attempt(g);}
    }
    CK(cudaStreamSynchronize(c->stream));
    for(int g = 0; g < NGLOBAL; ++g)
    {
        TermDev& T = c->term[g];
        if(!T.t.on || T.t.np == 0) {continue;}
        for(int k = 0; k < 3 && mx[g] > T.t.cap; ++k)
        {
            if(!T.tpp_fixed) {T.t.tpp = default_tpp(mx[g], T.t.np);}
            alloc_lists(c, g, list_capacity(mx[g]));
            attempt(g);
            CK(cudaStreamSynchronize(c->stream));
        }
    }
    // rebuild_all may have raised ST_LIST_OVERFLOW on the way; clear it
    download_sys(c);
    for(auto& s : c->h_sys) {s.status &= ~ST_LIST_OVERFLOW;}
    upload_sys(c);
}

void compute_initial_forces(mjg_context* c)
{
    launch_zero_force(c->arena, c->stream);
    enqueue_forces(c, c->arena, true, false);
}

// ------------------------------------------------------------- commit

// runs fn(i) for i in [0, n) on up to 16 host threads (work handed out one
// index at a time); the first exception thrown is rethrown here
template<typename F>
void parallel_for(int64_t n, F fn)
{
    const int64_t hw = std::max<int64_t>(1, (int64_t)std::thread::hardware_concurrency());
    const int nt = (int)std::min<int64_t>(std::min<int64_t>(hw, 16), n);
    if(nt <= 1)
    {
        for(int64_t i = 0; i < n; ++i) {fn(i);}
        return;
    }
    std::atomic<int64_t> next{0};
    std::exception_ptr err;
    std::mutex m;
    auto work = [&]() {
        try
        {
            for(int64_t i = next.fetch_add(1); i < n; i = next.fetch_add(1)) {fn(i);}
        }
        catch(...)
        {
            std::lock_guard<std::mutex> l(m);
            if(!err) {err = std::current_exception();}
            next.store(n);
        }
    };
    std::vector<std::thread> th;
    for(int t = 1; t < nt; ++t) {th.emplace_back(work);}
    work();
    for(auto& t : th) {t.join();}
    if(err) {std::rethrow_exception(err);}
}

int kind_id(std::map<std::string, int>& kinds, const std::string& k)
{
    auto it = kinds.find(k);
    if(it != kinds.end()) {return it->second;}
    const int id = (int)kinds.size();
    kinds[k] = id;
    return id;
}

double* pinned(mjg_context* c, size_t bytes)
{
    if(bytes > c->h_pinned_bytes)
    {
        if(c->h_pinned) {cudaFreeHost(c->h_pinned); c->h_pinned = nullptr; c->h_pinned_bytes = 0;}
        CK(cudaMallocHost(reinterpret_cast<void**>(&c->h_pinned), 2 * bytes));   // grow rarely
        c->h_pinned_bytes = 2 * bytes;
    }
    return c->h_pinned;
}

// copies position, velocity and force of every live resident system back to
// its host description: one packed pass over the whole arena per field
void save_resident_state(mjg_context* c)
{
    if(!c->committed) {return;}
    CK(cudaStreamSynchronize(c->stream));
    download_sys(c);
    bool any = false;
    for(size_t k = 0; k < c->arena_ids.size(); ++k)
    {
        HostSystem& s = c->sys[c->arena_ids[k]];
        const SysDev& d = c->h_sys[k];
        s.step = d.step;
        for(int g = 0; g < NGLOBAL; ++g) {s.rebuilds[g] = d.g[g].rebuilds;}
        any = any || s.alive;
    }
    if(!any || c->n_tot == 0) {return;}
    const size_t per = 3 * (size_t)c->n_tot;
    double* h = pinned(c, sizeof(double) * per);
    double* st = c->d_staging.as<double>();
    const int nfield = c->arena.accel ? 4 : 3;
    for(int field = 0; field < nfield; ++field)
    {
        launch_pack_state(c->arena, st, field, 0, c->n_tot, c->stream);
        CK(cudaMemcpyAsync(h, st, sizeof(double) * per, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        parallel_for((int64_t)c->arena_ids.size(), [&](int64_t k) {
            HostSystem& s = c->sys[c->arena_ids[k]];
            if(!s.alive) {return;}
            if(field == 3 && s.integrator != I_UNDERDAMPED) {return;}
            std::vector<double>& dst = field == 0 ? s.pos : field == 1 ? s.vel : field == 2 ? s.force : s.accel;
            dst.assign(h + 3 * s.off, h + 3 * (s.off + s.n));
            if(field == 2) {s.force_valid = true;}
            if(field == 3) {s.accel_valid = true;}
        });
    }
}

// the topology graph of a system: every local term's connections, then the
// explicit ones (LocalForceField::write_topology order)
TopologyGraph topology_of(const HostSystem& s, std::map<std::string, int>& kinds)
{
    TopologyGraph topo(s.n);
    auto add_edges = [&](const HostLocal& L, int arity) {
        if(L.kind.empty() || L.kind == "none") {return;}
        const int kd = kind_id(kinds, L.kind);
        for(int64_t t = 0; t < L.m(); ++t)
        {
            const int64_t* q = &L.idx[arity * t];
            for(int x = 0; x < arity; ++x)
                for(int y = x + 1; y < arity; ++y) {topo.add(q[x], q[y], kd);}
        }
    };
    add_edges(s.bond, 2);
    add_edges(s.angle, 3);
    add_edges(s.dihd, 4);
    for(const auto& e : s.connections) {topo.add(e.second.first, e.second.second, kind_id(kinds, e.first));}
    return topo;
}

// the per-system data that depends on topology only (molecules, exclusion
// lists), computed once in the edge order the reference's local force field
// writes the topology, after which the local terms are put in order of their
// smallest particle (the order the bonded kernel walks them in)
void derive(HostSystem& s)
{
    if(s.derived) {return;}
    std::map<std::string, int> kinds;
    const int bond_kind = kind_id(kinds, "bond");
    const TopologyGraph topo = topology_of(s, kinds);
    const std::vector<int64_t> m = topo.molecules(bond_kind);
    s.mol_local.assign(m.begin(), m.end());
    for(int g = 0; g < NGLOBAL; ++g)
    {
        s.ex_start_local[g].assign(1, 0);
        s.ex_idx_local[g].clear();
        if(!s.g[g].on)                   // no participant of this term: empty lists
        {
            s.ex_start_local[g].assign((size_t)s.n + 1, 0);
            continue;
        }
        std::vector<std::pair<int, int>> kw;
        for(const auto& w : s.g[g].within) {kw.emplace_back(kind_id(kinds, w.first), w.second);}
        exclusion_csr(topo, s.n, kw, 0, s.ex_start_local[g], s.ex_idx_local[g]);
    }
    auto order = [](HostLocal& L, int arity) {
        const int64_t mm = L.m();
        std::vector<int64_t> key(mm);
        for(int64_t t = 0; t < mm; ++t)
        {
            int64_t mn = L.idx[arity * t];
            for(int x = 1; x < arity; ++x) {mn = std::min(mn, L.idx[arity * t + x]);}
            key[t] = mn;
        }
        if(std::is_sorted(key.begin(), key.end())) {return;}
        std::vector<int64_t> perm(mm);
        for(int64_t t = 0; t < mm; ++t) {perm[t] = t;}
        std::stable_sort(perm.begin(), perm.end(), [&](int64_t x, int64_t y) {return key[x] < key[y];});
        HostLocal o;
        o.kind = L.kind;
        o.idx.resize(L.idx.size()); o.k.resize(mm); o.v0.resize(mm);
        if(!L.n.empty()) {o.n.resize(mm);}
        for(int64_t t = 0; t < mm; ++t)
        {
            const int64_t p = perm[t];
            for(int x = 0; x < arity; ++x) {o.idx[arity * t + x] = L.idx[arity * p + x];}
            o.k[t] = L.k[p]; o.v0[t] = L.v0[p];
            if(!L.n.empty()) {o.n[t] = L.n[p];}
        }
        L = std::move(o);
    };
    order(s.bond, 2);
    order(s.angle, 3);
    order(s.dihd, 4);
    s.derived = true;
}

// carves typed arrays out of the context's page-locked packing buffer
struct Carver {
    struct Item {size_t off, bytes;};
    size_t total = 0;
    template<typename T> Item add(size_t count)
    {
        Item it{total, sizeof(T) * count};
        total += (it.bytes + 255) / 256 * 256;
        return it;
    }
};

// optional per-phase timing of a commit on stderr (MJG_TRACE=1)
struct PhaseTimer {
    bool on;
    std::chrono::steady_clock::time_point t;
    std::string line;
    PhaseTimer() : on(std::getenv("MJG_TRACE") != nullptr), t(std::chrono::steady_clock::now()) {}
    void mark(const char* what)
    {
        if(!on) {return;}
        const auto now = std::chrono::steady_clock::now();
        line += std::string(" ") + what + "=" +
                std::to_string(std::chrono::duration<double, std::milli>(now - t).count()).substr(0, 7) + "ms";
        t = now;
    }
    ~PhaseTimer() {if(on && !line.empty()) {std::fprintf(stderr, "mjg commit:%s\n", line.c_str());}}
};

// the cell grid of term g of system s (host side of the rebuild)
void cell_grid(const HostSystem& s, const SysDev& d, int g, GlobalParams& G)
{
    const HostGlobal& H = s.g[g];
    const int64_t np = (int64_t)H.idx.size();
    if(s.boundary == B_PERIODIC)
    {
        // PeriodicGridCellList::set_cutoff / initialize (:67-96, :383-395)
        const double r = 1.0 / (G.cutoff * (1.0 + G.margin) + 1e-6);
        long long dims[3];
        for(int x = 0; x < 3; ++x) {dims[x] = std::max<long long>(3, (long long)std::floor(d.width[x] * r));}
        // keep the grid within a few cells per participant (wider cells stay exact)
        const long long limit = std::max<long long>(27, 8 * np + 64);
        while(dims[0] * dims[1] * dims[2] > limit)
        {
            int big = 0;
            for(int x = 1; x < 3; ++x) {if(dims[x] > dims[big]) {big = x;}}
            if(dims[big] <= 3) {break;}
            dims[big] -= 1;
        }
        for(int x = 0; x < 3; ++x)
        {
            G.dims[x] = (int)dims[x];
            G.inv_w[x] = 1.0 / (d.width[x] / (double)dims[x]);
            G.origin[x] = d.lower[x];
        }
        G.hashed = 0;
    }
    else
    {
        // unbounded space: cells of cutoff (1 + margin)(1 + 1e-6) hashed
        // modulo a grid sized to the system's current extent
        const double w = G.cutoff * (1 + G.margin) * (1 + 1e-6);
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for(int64_t q = 0; q < np; ++q)
        {
            const int64_t i = H.idx[q];
            for(int x = 0; x < 3; ++x)
            {
                lo[x] = std::min(lo[x], s.pos[3 * i + x]);
                hi[x] = std::max(hi[x], s.pos[3 * i + x]);
            }
        }
        long long dims[3];
        for(int x = 0; x < 3; ++x)
        {
            const double ext = np > 0 ? hi[x] - lo[x] : 0.0;
            dims[x] = std::max<long long>(3, (long long)std::floor(ext / w) + 3);
        }
        const long long limit = std::max<long long>(27, 2 * np + 64);
        while(dims[0] * dims[1] * dims[2] > limit)
        {
            int big = 0;
            for(int x = 1; x < 3; ++x) {if(dims[x] > dims[big]) {big = x;}}
            if(dims[big] <= 3) {break;}
            dims[big] -= 1;
        }
        for(int x = 0; x < 3; ++x)
        {
            G.dims[x] = (int)dims[x];
            G.inv_w[x] = 1.0 / w;
            G.origin[x] = 0.0;
        }
        G.hashed = 1;
    }
    G.ncell = G.dims[0] * G.dims[1] * G.dims[2];
}

// the per-system device record: box, counters and the constants of every
// global term (potential parameters, list radius, cell grid)
void make_sysdev(const HostSystem& s, SysDev& d)
{
    std::memset(&d, 0, sizeof(SysDev));
    d.off = s.off; d.n = s.n;
    d.boundary = s.boundary;
    d.integrator = s.integrator;
    for(int x = 0; x < 3; ++x)
    {
        d.lower[x] = s.lower[x]; d.upper[x] = s.upper[x];
        d.width[x] = s.upper[x] - s.lower[x];
        d.halfw[x] = d.width[x] / 2;
    }
    d.seed = s.seed;
    d.step = s.step;
    d.frozen = s.frozen ? 1 : 0;
    for(int g = 0; g < NGLOBAL; ++g)
    {
        const HostGlobal& H = s.g[g];
        GlobalParams& G = d.g[g];
        if(!H.on) {continue;}
        G.on = 1;
        G.margin = H.margin;
        G.cutoff_ratio = H.cutoff_ratio;
        G.cutoff_ratio_sq = H.cutoff_ratio * H.cutoff_ratio;
        G.ignore_mol = H.ignore_mol;
        G.eps = H.eps;
        const int64_t np = (int64_t)H.idx.size();
        if(g == G_EXV)             // ExcludedVolumePotential.hpp:44-48,92-106 and the family
        {
            G.kind = H.kind;
            G.power = H.power;
            G.coef_at_cutoff = H.kind == EXV_INVERSE_POWER ? std::pow(1.0 / H.cutoff_ratio, H.power)
                                                          : std::pow(1.0 / H.cutoff_ratio, 12);
            double mr = 0, mc = 0;
            for(double r : H.p0) {mr = std::max(mr, r);}
            G.cutoff = np == 0 ? 1.0 : mr * 2 * H.cutoff_ratio;
            if(H.kind == EXV_HARD_CORE && np > 0)   // HardCoreExcludedVolumePotential.hpp:109-126
            {
                for(double c : H.p1) {mc = std::max(mc, c);}
                G.cutoff = mr * 2 * H.cutoff_ratio + mc * 2;
            }
        }
        else if(g == G_DH)         // DebyeHuckelPotential.hpp:126-167,245-248
        {
            if(!(s.T > 0)) {throw Error(MJG_EINVAL, "DebyeHuckel needs a positive temperature (its Debye length)");}
            const DHParams p = dh_params(s.T, s.I, H.cutoff_ratio);
            G.debye = p.debye; G.inv_debye = p.inv_debye; G.abs_cutoff = p.abs_cutoff;
            G.coef_at_cutoff = p.coef_at_cutoff; G.inv4pi = p.inv4pi;
            G.cutoff = p.debye * H.cutoff_ratio;
        }
        else                       // LennardJonesPotential.hpp:36-41,75-91 and the family
        {
            G.kind = H.kind;
            G.coef_at_cutoff = H.kind == LJ_WCA ? 0.0 :          // WCAPotential.hpp: no shift
                std::pow(1.0 / H.cutoff_ratio, 12) - std::pow(1.0 / H.cutoff_ratio, 6);
            double ms = 0;
            for(double x : H.p0) {ms = std::max(ms, x);}
            G.cutoff = np == 0 ? 1.0 : ms * H.cutoff_ratio;
        }
        const double r_c = G.cutoff * (1. + G.margin);
        G.rl2 = r_c * r_c;
        G.current_margin = G.cutoff * G.margin;
        G.rebuild = 1;
        G.rebuilds = s.rebuilds[g];
        G.nslot = (int)np;
        cell_grid(s, d, g, G);
    }
}

// Packs every live system into one arena and uploads it.  Systems keep their
// state (positions, velocities, exact forces, step counters) across commits.
// The host work runs in parallel over systems into one page-locked buffer,
// from which each device array is filled by a single copy.
void commit(mjg_context* c)
{
    PhaseTimer tm;
    CK(cudaSetDevice(c->device));
    save_resident_state(c);
    tm.mark("save");
    release_graph(c);
    for(auto& s : c->sys) {s.resident = false; s.arena_slot = -1;}

    std::vector<int> ids;
    for(int i = 0; i < (int)c->sys.size(); ++i)
    {
        HostSystem& s = c->sys[i];
        if(!s.alive) {continue;}
        if(s.integrator != I_VV && (int64_t)s.gamma.size() != s.n)
        {
            throw Error(MJG_ESTATE, "system " + std::to_string(i) + " has no integrator set");
        }
        ids.push_back(i);
    }
    const int nsys = (int)ids.size();
    parallel_for(nsys, [&](int64_t k) {derive(c->sys[ids[k]]);});
    tm.mark("derive");

    // ---- offsets (serial, per system)
    long long n_tot = 0;
    for(int id : ids) {c->sys[id].off = n_tot; n_tot += c->sys[id].n;}
    std::vector<SysDev> hs(nsys);
    parallel_for(nsys, [&](int64_t k) {make_sysdev(c->sys[ids[k]], hs[k]);});
    std::vector<long long> mol_base(nsys + 1, 0), ex_off[NGLOBAL], b_off(nsys + 1, 0), a_off(nsys + 1, 0),
                           d_off(nsys + 1, 0);
    long long np_tot[NGLOBAL] = {0, 0, 0}, ncell[NGLOBAL] = {0, 0, 0};
    long long part_chunk_cap[NGLOBAL] = {0, 0, 0}, cell_chunk_cap[NGLOBAL] = {0, 0, 0};
    for(int g = 0; g < NGLOBAL; ++g) {ex_off[g].assign(nsys + 1, 0);}
    for(int k = 0; k < nsys; ++k)
    {
        HostSystem& s = c->sys[ids[k]];
        s.resident = true;
        s.arena_slot = k;
        int64_t nmol = 0;
        for(const int32_t m : s.mol_local) {nmol = std::max<int64_t>(nmol, (int64_t)m + 1);}
        mol_base[k + 1] = mol_base[k] + nmol;
        for(int g = 0; g < NGLOBAL; ++g)
        {
            ex_off[g][k + 1] = ex_off[g][k] + (long long)s.ex_idx_local[g].size();
            GlobalParams& G = hs[k].g[g];
            if(!G.on) {continue;}
            G.slot_off = (int)np_tot[g];
            G.cell_off = (int)ncell[g];
            np_tot[g] += G.nslot;
            ncell[g] += G.ncell;
            cell_chunk_cap[g] += (G.ncell + 255) / 256;
            part_chunk_cap[g] += (G.nslot + 255) / 256;
        }
        b_off[k + 1] = b_off[k] + s.bond.m();
        a_off[k + 1] = a_off[k] + s.angle.m();
        d_off[k + 1] = d_off[k] + s.dihd.m();
    }
    for(int g = 0; g < NGLOBAL; ++g)
    {
        if(np_tot[g] > INT32_MAX || ncell[g] > INT32_MAX) {throw Error(MJG_EINVAL, "arena too large");}
    }
    const long long nb = b_off[nsys], na = a_off[nsys], nd = d_off[nsys];
    const int nwin = (int)((n_tot + 255) / 256);

    // ---- layout of the page-locked packing buffer
    Carver cv;
    const auto c_pos = cv.add<double4>(n_tot), c_vel = cv.add<double4>(n_tot), c_coef = cv.add<double4>(n_tot);
    const auto c_psys = cv.add<int>(n_tot), c_mol = cv.add<int>(n_tot);
    Carver::Item c_exs[NGLOBAL], c_exi[NGLOBAL], c_pp[NGLOBAL], c_ps[NGLOBAL], c_p0[NGLOBAL], c_p1[NGLOBAL],
                 c_pl[NGLOBAL];
    for(int g = 0; g < NGLOBAL; ++g)
    {
        c_exs[g] = cv.add<long long>(n_tot + 1);
        c_exi[g] = cv.add<int>(std::max<long long>(1, ex_off[g][nsys]));
        c_pp[g] = cv.add<int>(np_tot[g]);
        c_ps[g] = cv.add<int>(np_tot[g]);
        c_p0[g] = cv.add<double>(np_tot[g]);
        c_p1[g] = cv.add<double>(np_tot[g]);
        c_pl[g] = cv.add<unsigned char>(np_tot[g]);
    }
    const auto c_bidx = cv.add<int>(2 * nb), c_bk = cv.add<double>(nb), c_bv0 = cv.add<double>(nb),
               c_bsys = cv.add<int>(nb), c_bkv = cv.add<float2>(nb);
    const auto c_aidx = cv.add<int>(3 * na), c_ak = cv.add<double>(na), c_av0 = cv.add<double>(na),
               c_asys = cv.add<int>(na), c_akv = cv.add<float2>(na);
    const auto c_didx = cv.add<int>(4 * nd), c_dk = cv.add<double>(nd), c_dv0 = cv.add<double>(nd),
               c_dsys = cv.add<int>(nd), c_dn = cv.add<int>(nd), c_dp = cv.add<float4>(nd);
    const auto c_wb = cv.add<long long>(nwin + 1), c_wa = cv.add<long long>(nwin + 1),
               c_wd = cv.add<long long>(nwin + 1);
    if(cv.total > c->h_pack_bytes)
    {
        if(c->h_pack) {cudaFreeHost(c->h_pack); c->h_pack = nullptr; c->h_pack_bytes = 0;}
        const size_t want = 2 * cv.total;          // page-locking is slow: grow rarely
        CK(cudaMallocHost(reinterpret_cast<void**>(&c->h_pack), want));
        c->h_pack_bytes = want;
    }
    char* hb = static_cast<char*>(c->h_pack);
    auto at = [&](const Carver::Item& it) {return hb + it.off;};
    double4* pos = (double4*)at(c_pos); double4* vel = (double4*)at(c_vel); double4* coef = (double4*)at(c_coef);
    int* psys = (int*)at(c_psys); int* mol = (int*)at(c_mol);
    int* b_idx = (int*)at(c_bidx); double* b_k = (double*)at(c_bk); double* b_v0 = (double*)at(c_bv0);
    int* b_sys = (int*)at(c_bsys); float2* b_kv = (float2*)at(c_bkv);
    int* a_idx = (int*)at(c_aidx); double* a_k = (double*)at(c_ak); double* a_v0 = (double*)at(c_av0);
    int* a_sys = (int*)at(c_asys); float2* a_kv = (float2*)at(c_akv);
    int* d_idx = (int*)at(c_didx); double* d_k = (double*)at(c_dk); double* d_v0 = (double*)at(c_dv0);
    int* d_sys = (int*)at(c_dsys); int* d_n = (int*)at(c_dn); float4* d_p = (float4*)at(c_dp);
    tm.mark("layout");

    // ---- fill (parallel over systems)
    const Units u;
    parallel_for(nsys, [&](int64_t k) {
        const HostSystem& s = c->sys[ids[k]];
        const SysDev& d = hs[k];
        const long long off = s.off;
        const double halfdt = s.dt / 2;
        const double kBT = u.kB * s.T;
        for(int64_t i = 0; i < s.n; ++i)
        {
            double p[3] = {s.pos[3 * i], s.pos[3 * i + 1], s.pos[3 * i + 2]};
            if(s.boundary == B_PERIODIC)          // adjust_position
            {
                for(int x = 0; x < 3; ++x)
                {
                    if(p[x] < d.lower[x]) {p[x] += d.width[x];}
                    else if(p[x] >= d.upper[x]) {p[x] -= d.width[x];}
                }
            }
            const long long gi = off + i;
            pos[gi] = make_double4(p[0], p[1], p[2], 0.0);
            vel[gi] = make_double4(s.vel[3 * i], s.vel[3 * i + 1], s.vel[3 * i + 2], 0.0);
            const double rmass = 1.0 / s.mass[i];
            if(s.integrator == I_UNDERDAMPED)  // UnderdampedLangevinIntegrator::update (:55-70)
            {
                const double noise_coef = std::sqrt(2 * u.kB * s.T / s.dt);
                coef[gi] = make_double4(rmass, s.gamma[i], noise_coef * std::sqrt(s.gamma[i] * rmass), s.dt);
            }
            else if(s.integrator == I_GJF)     // GJFNVTLangevinIntegrator::reset_parameters (:111-136)
            {
                const double alpha = s.gamma[i], m = s.mass[i];
                const double b = 1.0 / (1.0 + alpha * s.dt * 0.5 / m);
                coef[gi] = make_double4(halfdt * rmass, 1.0 - alpha * b * s.dt / m,
                                        std::sqrt(2 * alpha * kBT * s.dt), s.dt);
            }
            else if(s.integrator == I_BAOAB || s.integrator == I_GBAOAB)   // reset_parameters (:73-99;
                                                                            // gBAOAB :80-106)
            {
                const double gamma_dt = -1 * s.gamma[i] * s.dt;
                coef[gi] = make_double4(halfdt * rmass, std::exp(gamma_dt),
                                        std::sqrt(kBT * (1 - std::exp(2 * gamma_dt)) * rmass), halfdt);
            }
            else
            {
                coef[gi] = make_double4(halfdt * rmass, 1.0, 0.0, s.dt);
            }
            psys[gi] = (int)k;
            mol[gi] = (int)(mol_base[k] + s.mol_local[i]);
        }
        // one set of coefficients for the whole system (uniform masses and
        // frictions): the integrator reads it from the system record
        bool uniform = s.n > 0;
        for(int64_t i = 1; i < s.n && uniform; ++i)
        {
            uniform = std::memcmp(&coef[off + i], &coef[off], sizeof(double4)) == 0;
        }
        hs[k].uniform_coef = uniform ? 1 : 0;
        hs[k].coef = uniform ? coef[off] : make_double4(0.0, 0.0, 0.0, 0.0);
        for(int g = 0; g < NGLOBAL; ++g)
        {
            long long* exs = (long long*)at(c_exs[g]);
            int* exi = (int*)at(c_exi[g]);
            const long long base = ex_off[g][k];
            const std::vector<long long>& ls = s.ex_start_local[g];
            if(k == 0) {exs[0] = 0;}
            for(int64_t i = 1; i <= s.n; ++i) {exs[off + i] = base + ls[i];}
            const std::vector<int>& li = s.ex_idx_local[g];
            for(size_t j = 0; j < li.size(); ++j) {exi[base + j] = (int)(li[j] + off);}
            const GlobalParams& G = d.g[g];
            if(!G.on) {continue;}
            const HostGlobal& H = s.g[g];
            int* pp = (int*)at(c_pp[g]); int* ps = (int*)at(c_ps[g]);
            double* p0 = (double*)at(c_p0[g]); double* p1 = (double*)at(c_p1[g]);
            unsigned char* pl = (unsigned char*)at(c_pl[g]);
            const int64_t np = G.nslot;
            for(int64_t q = 0; q < np; ++q)
            {
                const int64_t x = G.slot_off + q;
                pp[x] = (int)(off + H.idx[q]);
                ps[x] = (int)k;
                p0[x] = H.p0[q];
                p1[x] = H.p1.empty() ? 0.0 : H.p1[q];
                pl[x] = q + 1 < np ? 1 : 0;
            }
        }
        for(int64_t t = 0; t < s.bond.m(); ++t)
        {
            const long long x = b_off[k] + t;
            b_idx[2 * x] = (int)(off + s.bond.idx[2 * t]);
            b_idx[2 * x + 1] = (int)(off + s.bond.idx[2 * t + 1]);
            b_k[x] = s.bond.k[t]; b_v0[x] = s.bond.v0[t]; b_sys[x] = (int)k;
            b_kv[x] = make_float2((float)s.bond.k[t], (float)s.bond.v0[t]);
        }
        for(int64_t t = 0; t < s.angle.m(); ++t)
        {
            const long long x = a_off[k] + t;
            for(int y = 0; y < 3; ++y) {a_idx[3 * x + y] = (int)(off + s.angle.idx[3 * t + y]);}
            a_k[x] = s.angle.k[t]; a_v0[x] = s.angle.v0[t]; a_sys[x] = (int)k;
            a_kv[x] = make_float2((float)s.angle.k[t], (float)s.angle.v0[t]);
        }
        for(int64_t t = 0; t < s.dihd.m(); ++t)
        {
            const long long x = d_off[k] + t;
            for(int y = 0; y < 4; ++y) {d_idx[4 * x + y] = (int)(off + s.dihd.idx[4 * t + y]);}
            d_k[x] = s.dihd.k[t]; d_v0[x] = s.dihd.v0[t]; d_n[x] = s.dihd.n[t]; d_sys[x] = (int)k;
            const double nv = (double)s.dihd.n[t] * s.dihd.v0[t];
            d_p[x] = make_float4((float)s.dihd.k[t], (float)std::cos(nv), (float)std::sin(nv),
                                 (float)s.dihd.n[t]);
        }
    });
    if(nsys == 0)
    {
        for(int g = 0; g < NGLOBAL; ++g) {((long long*)at(c_exs[g]))[0] = 0;}
    }
    // local terms: every system keeps its terms ordered by their smallest
    // particle and systems are packed in order, so the arena's terms are in
    // order too; CSR of terms over 256-particle windows
    auto windows = [&](const int* idx, int arity, long long m, long long* win) {
        std::fill(win, win + nwin + 1, 0LL);
        int prev = 0;
        for(long long t = 0; t < m; ++t)
        {
            int mn = idx[arity * t];
            for(int x = 1; x < arity; ++x) {mn = std::min(mn, idx[arity * t + x]);}
            if(mn < prev) {throw Error(MJG_ESTATE, "local terms out of order");}
            prev = mn;
            win[mn / 256 + 1] += 1;
        }
        for(int w = 0; w < nwin; ++w) {win[w + 1] += win[w];}
    };
    windows(b_idx, 2, nb, (long long*)at(c_wb));
    windows(a_idx, 3, na, (long long*)at(c_wa));
    windows(d_idx, 4, nd, (long long*)at(c_wd));
    tm.mark("fill");

    // ---- device upload (buffers keep their capacity across commits)
    cudaStream_t st = c->stream;
    auto put = [&](DevBuf& dst, const Carver::Item& it) {
        dst.ensure(it.bytes);
        if(it.bytes) {CK(cudaMemcpyAsync(dst.p, at(it), it.bytes, cudaMemcpyHostToDevice, st));}
    };
    c->n_tot = n_tot;
    c->arena_ids = ids;
    c->h_sys = hs;
    c->d_sys.ensure(sizeof(SysDev) * std::max(nsys, 1));
    upload_sys(c);
    put(c->d_pos, c_pos);
    put(c->d_vel, c_vel);
    put(c->d_coef, c_coef);
    put(c->d_psys, c_psys);
    put(c->d_mol, c_mol);
    c->d_force.ensure(32 * (size_t)std::max<long long>(n_tot, 1));
    c->d_force_scratch.ensure(32 * (size_t)std::max<long long>(n_tot, 1));
    // the per-particle auxiliary array: UnderdampedLangevin accelerations,
    // G-JF coefficients
    bool any_underdamped = false, any_gjf = false;
    for(int id : ids)
    {
        any_underdamped = any_underdamped || c->sys[id].integrator == I_UNDERDAMPED;
        any_gjf = any_gjf || c->sys[id].integrator == I_GJF;
    }
    const bool any_aux = any_underdamped || any_gjf;
    if(any_aux) {c->d_accel.ensure(32 * (size_t)std::max<long long>(n_tot, 1));}
    else        {c->d_accel.release();}
    // room for positions and velocities side by side (bulk state copies)
    c->d_staging.ensure(sizeof(double) * 6 * (size_t)std::max<long long>(n_tot, 1));
    if(c->rollback)
    {
        c->b_sys.ensure(c->d_sys.bytes);
        c->b_pos.ensure(c->d_pos.bytes);
        c->b_vel.ensure(c->d_vel.bytes);
        c->b_force.ensure(c->d_force.bytes);
        if(any_aux) {c->b_accel.ensure(c->d_accel.bytes);} else {c->b_accel.release();}
    }
    else
    {
        c->b_sys.release(); c->b_pos.release(); c->b_vel.release(); c->b_force.release();
        c->b_accel.release();
    }

    Arena& a = c->arena;
    a = Arena{};
    a.precision = c->precision;
    a.n = n_tot;
    a.nsys = nsys;
    a.sys = c->d_sys.as<SysDev>();
    a.pos = c->d_pos.as<double4>();
    a.vel = c->d_vel.as<double4>();
    a.force = c->d_force.p;
    a.coef = c->d_coef.as<double4>();
    a.psys = c->d_psys.as<int>();
    a.staging = c->d_staging.as<double>();
    a.mol = c->d_mol.as<int>();
    a.accel = any_aux ? c->d_accel.as<double4>() : nullptr;
    for(int id : ids) {a.any_frozen |= c->sys[id].frozen ? 1 : 0;}

    for(int g = 0; g < NGLOBAL; ++g)
    {
        TermDev& T = c->term[g];
        put(T.ex_start, c_exs[g]);
        put(T.ex_idx, c_exi[g]);
        a.ex_start[g] = T.ex_start.as<long long>();
        a.ex_idx[g] = T.ex_idx.as<int>();

        TermArrays& t = T.t;
        const int prev_tpp = t.tpp > 0 ? t.tpp : 1;
        t = TermArrays{};
        const long long np = np_tot[g];
        t.on = np > 0 ? 1 : 0;
        t.np = np;
        t.ncell = (int)ncell[g];
        if(!t.on)
        {
            DevBuf* bufs[] = {&T.part_particle, &T.part_p0, &T.part_p1, &T.part_lead, &T.part_sys,
                              &T.part_cell, &T.cell_count, &T.cell_start, &T.cell_fill,
                              &T.work, &T.part_chunks, &T.cell_chunks, &T.flagged, &T.slot_part, &T.slot_particle, &T.slot_lead,
                              &T.slot_sys, &T.slot_pd, &T.slot_p1, &T.slot_of, &T.slot_w, &T.nnb, &T.nbr,
                              &T.max_count, &T.any_rebuild};
            for(auto* b : bufs) {b->release();}
            T.cap_alloc = 0;
            continue;
        }
        put(T.part_particle, c_pp[g]);
        put(T.part_p0, c_p0[g]);
        put(T.part_p1, c_p1[g]);
        put(T.part_lead, c_pl[g]);
        put(T.part_sys, c_ps[g]);
        T.part_cell.ensure(sizeof(int) * np);
        T.cell_count.ensure(sizeof(int) * t.ncell);
        T.cell_fill.ensure(sizeof(int) * t.ncell);
        T.cell_start.ensure(sizeof(int) * (t.ncell + 1));
        // rebuild work lists (sized for every system flagged at once)
        T.work.ensure(sizeof(int) * 4);
        CK(cudaMemsetAsync(T.work.p, 0, T.work.bytes, st));
        T.part_chunks.ensure(sizeof(int4) * std::max<long long>(1, part_chunk_cap[g]));
        T.cell_chunks.ensure(sizeof(int4) * std::max<long long>(1, cell_chunk_cap[g]));
        T.flagged.ensure(sizeof(int) * std::max(1, nsys));
        {
            const int last = (int)np;        // cell_start[ncell] = total slots
            CK(cudaMemcpyAsync(T.cell_start.as<int>() + t.ncell, &last, sizeof(int),
                               cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
        }
        CK(cudaMemsetAsync(T.cell_count.p, 0, T.cell_count.bytes, st));
        CK(cudaMemsetAsync(T.cell_fill.p, 0, T.cell_fill.bytes, st));
        T.slot_part.ensure(sizeof(int) * np);
        T.slot_particle.ensure(sizeof(int) * np);
        T.slot_lead.ensure(np);
        T.slot_sys.ensure(sizeof(int) * np);
        T.slot_pd.ensure(sizeof(double4) * np);
        T.slot_p1.ensure(sizeof(double) * np);
        T.slot_of.ensure(sizeof(int) * (size_t)std::max<long long>(n_tot, 1));
        CK(cudaMemsetAsync(T.slot_of.p, 0xff, T.slot_of.bytes, st));      // -1: no slot
        T.slot_w.ensure(sizeof(double) * (size_t)std::max<long long>(n_tot, 1));
        T.nnb.ensure(sizeof(int) * np);
        T.max_count.ensure(sizeof(int));
        T.any_rebuild.ensure(sizeof(int));
        CK(cudaMemsetAsync(T.any_rebuild.p, 0, sizeof(int), st));
        CK(cudaMemsetAsync(T.nnb.p, 0, T.nnb.bytes, st));
        t.part_particle = T.part_particle.as<int>();
        t.part_p0 = T.part_p0.as<double>();
        t.part_p1 = T.part_p1.as<double>();     // LJ-family epsilon, HardCore core radius
        t.part_lead = T.part_lead.as<unsigned char>();
        t.part_sys = T.part_sys.as<int>();
        t.part_cell = T.part_cell.as<int>();
        t.cell_count = T.cell_count.as<int>();
        t.cell_start = T.cell_start.as<int>();
        t.cell_fill = T.cell_fill.as<int>();
        t.work = T.work.as<int>();
        t.part_chunks = T.part_chunks.as<int4>();
        t.cell_chunks = T.cell_chunks.as<int4>();
        t.flagged = T.flagged.as<int>();
        t.slot_part = T.slot_part.as<int>();
        t.slot_particle = T.slot_particle.as<int>();
        t.slot_lead = T.slot_lead.as<unsigned char>();
        t.slot_sys = T.slot_sys.as<int>();
        t.slot_pd = T.slot_pd.as<double4>();
        t.slot_p1 = T.slot_p1.as<double>();
        t.slot_of = T.slot_of.as<int>();
        a.slot_pd[g] = t.slot_pd;
        a.slot_of[g] = t.slot_of;
        a.slot_w[g] = T.slot_w.as<double>();
        launch_scatter_param(t, T.slot_w.as<double>(), st);
        t.nnb = T.nnb.as<int>();
        t.max_count = T.max_count.as<int>();
        t.any_rebuild = T.any_rebuild.as<int>();
        t.tpp = T.tpp_fixed ? T.tpp_choice : 1;
        t.unroll = T.unroll_choice;
        t.schedule = T.schedule_choice;
        t.slot_major = t.schedule == 5 ? 1 : 0;
        t.half = T.half_choice && c->precision == P_MIXED ? 1 : 0;
        if(!T.build_lanes_fixed)
        {
            // candidates per slot if the participants filled their grids
            // evenly: 27 cells x participants per cell, weighted by slots
            double cand = 0.0, slots = 0.0;
            for(int k = 0; k < nsys; ++k)
            {
                const GlobalParams& G = hs[k].g[g];
                if(!G.on || G.ncell == 0) {continue;}
                cand += 27.0 * (double)G.nslot * (double)G.nslot / (double)G.ncell;
                slots += (double)G.nslot;
            }
            const double per = slots > 0 ? cand / slots : 0.0;
            T.build_lanes_choice = per < 12.0 ? 8 : (per < 64.0 ? 16 : 32);
        }
        t.build_lanes = T.build_lanes_choice;
        t.any_periodic = 0;
        for(int id : ids)
        {
            if(c->sys[id].g[g].on && c->sys[id].boundary == B_PERIODIC) {t.any_periodic = 1;}
        }
        // keep the list capacity of the previous arena when the buffer still
        // holds it; rebuild_all grows it where needed
        const int keep = T.cap_alloc;
        if(keep > 0 && T.nbr.cap >= sizeof(int) * list_words(keep) * (size_t)np)
        {
            T.nbr.bytes = sizeof(int) * list_words(keep) * (size_t)np;
            t.nbr = T.nbr.as<int>();
            t.cap = keep;
            if(!T.tpp_fixed) {t.tpp = prev_tpp;}
        }
        else
        {
            t.nbr = nullptr;
            t.cap = 0;
            alloc_lists(c, g, 0);
        }
    }

    LocalArrays& l = c->local;
    l = LocalArrays{};
    put(c->l_bond_kv, c_bkv); put(c->l_angle_kv, c_akv); put(c->l_dihd_p, c_dp);
    put(c->l_win_bond, c_wb); put(c->l_win_angle, c_wa); put(c->l_win_dihd, c_wd);
    put(c->l_bond_idx, c_bidx);  put(c->l_bond_k, c_bk);
    put(c->l_bond_v0, c_bv0);    put(c->l_bond_sys, c_bsys);
    put(c->l_angle_idx, c_aidx); put(c->l_angle_k, c_ak);
    put(c->l_angle_v0, c_av0);   put(c->l_angle_sys, c_asys);
    put(c->l_dihd_idx, c_didx);  put(c->l_dihd_k, c_dk);
    put(c->l_dihd_n, c_dn);      put(c->l_dihd_v0, c_dv0);
    put(c->l_dihd_sys, c_dsys);
    l.nbond = nb; l.nangle = na; l.ndihd = nd;
    l.bond_idx = c->l_bond_idx.as<int>();   l.bond_k = c->l_bond_k.as<double>();
    l.bond_v0 = c->l_bond_v0.as<double>();  l.bond_sys = c->l_bond_sys.as<int>();
    l.angle_idx = c->l_angle_idx.as<int>(); l.angle_k = c->l_angle_k.as<double>();
    l.angle_v0 = c->l_angle_v0.as<double>(); l.angle_sys = c->l_angle_sys.as<int>();
    l.dihd_idx = c->l_dihd_idx.as<int>();   l.dihd_k = c->l_dihd_k.as<double>();
    l.dihd_n = c->l_dihd_n.as<int>();       l.dihd_v0 = c->l_dihd_v0.as<double>();
    l.dihd_sys = c->l_dihd_sys.as<int>();
    l.nwin = nwin;
    l.bond_kv = c->l_bond_kv.as<float2>();
    l.angle_kv = c->l_angle_kv.as<float2>();
    l.dihd_p = c->l_dihd_p.as<float4>();
    l.win_bond = c->l_win_bond.as<long long>();
    l.win_angle = c->l_win_angle.as<long long>();
    l.win_dihd = c->l_win_dihd.as<long long>();
    tm.mark("upload");

    c->committed = true;
    rebuild_all(c);
    tm.mark("rebuild");
    compute_initial_forces(c);
    // systems that were resident keep their exact force array: one upload,
    // then one conversion per run of consecutive such systems
    {
        auto keeps = [&](int k) {
            const HostSystem& s = c->sys[ids[k]];
            return s.force_valid && (int64_t)s.force.size() == 3 * s.n;
        };
        bool any = false;
        for(int k = 0; k < nsys && !any; ++k) {any = keeps(k);}
        if(any)
        {
            double* h = pinned(c, sizeof(double) * 3 * (size_t)n_tot);
            parallel_for(nsys, [&](int64_t k) {
                if(keeps((int)k))
                {
                    const HostSystem& s = c->sys[ids[k]];
                    std::copy(s.force.begin(), s.force.end(), h + 3 * s.off);
                }
            });
            double* stg = c->d_staging.as<double>();
            CK(cudaMemcpyAsync(stg, h, sizeof(double) * 3 * (size_t)n_tot, cudaMemcpyHostToDevice, st));
            for(int k = 0; k < nsys;)
            {
                if(!keeps(k)) {++k; continue;}
                int e = k;
                while(e + 1 < nsys && keeps(e + 1)) {++e;}
                const int64_t off = c->sys[ids[k]].off;
                const int64_t cnt = c->sys[ids[e]].off + c->sys[ids[e]].n - off;
                launch_set_force(c->arena, stg + 3 * off, off, cnt, st);
                k = e + 1;
            }
        }
    }
    // UnderdampedLangevin: resident systems keep their accelerations, the
    // others start from Integrator::initialize.  G-JF: the coefficients
    // {1/2m, b/m, b dt} of GJFNVTLangevinIntegrator::reset_parameters
    // (:111-136) and step (:183-204).
    if(c->arena.accel)
    {
        double* stg = c->d_staging.as<double>();
        std::vector<double> gjf;
        for(int k = 0; k < nsys; ++k)
        {
            HostSystem& s = c->sys[ids[k]];
            if(s.integrator == I_GJF)
            {
                gjf.resize(3 * (size_t)s.n);
                for(int64_t i = 0; i < s.n; ++i)
                {
                    const double alpha = s.gamma[i], m = s.mass[i], rm = 1.0 / m;
                    const double b = 1.0 / (1.0 + alpha * s.dt * 0.5 / m);
                    gjf[3 * i] = 0.5 * rm;
                    gjf[3 * i + 1] = b * rm;
                    gjf[3 * i + 2] = b * s.dt;
                }
                CK(cudaMemcpyAsync(stg + 3 * s.off, gjf.data(), sizeof(double) * 3 * s.n,
                                   cudaMemcpyHostToDevice, st));
                launch_set_accel(c->arena, stg + 3 * s.off, s.off, s.n, st);
                CK(cudaStreamSynchronize(st));    // gjf is reused for the next system
                continue;
            }
            if(s.integrator != I_UNDERDAMPED) {continue;}
            if(s.accel_valid && (int64_t)s.accel.size() == 3 * s.n)
            {
                CK(cudaMemcpyAsync(stg + 3 * s.off, s.accel.data(), sizeof(double) * 3 * s.n,
                                   cudaMemcpyHostToDevice, st));
                launch_set_accel(c->arena, stg + 3 * s.off, s.off, s.n, st);
            }
            else
            {
                launch_init_accel(c->arena, s.off, s.n, st);
            }
        }
    }
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    tm.mark("forces");
}

// ------------------------------------------------------------------ step

void check_status(mjg_context* c, bool& overflow)
{
    overflow = false;
    // a truncated list makes every later force of the chunk meaningless, so
    // a list overflow is handled (rolled back) before anything else is checked
    for(const auto& d : c->h_sys) {if(d.status & ST_LIST_OVERFLOW) {overflow = true;}}
    if(overflow) {return;}
    for(size_t k = 0; k < c->h_sys.size(); ++k)
    {
        const int st = c->h_sys[k].status;
        if(st & ST_FIXED_OVERFLOW)
        {
            throw Error(MJG_EOVERFLOW, "system " + std::to_string(c->arena_ids[k]) +
                        ": a force left the fixed-point range (|F| >= 2^22)");
        }
        if(st & ST_NONFINITE)
        {
            throw Error(MJG_ENONFINITE, "system " + std::to_string(c->arena_ids[k]) +
                        ": non-finite displacement (the system blew up)");
        }
    }
}

void run_steps(mjg_context* c, int64_t nsteps)
{
    if(nsteps <= 0) {return;}
    cudaStream_t st = c->stream;
    for(int attempt = 0; attempt < 8; ++attempt)
    {
        if(c->rollback)
        {
            CK(cudaMemcpyAsync(c->b_sys.p, c->d_sys.p, c->d_sys.bytes, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(c->b_pos.p, c->d_pos.p, c->d_pos.bytes, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(c->b_vel.p, c->d_vel.p, c->d_vel.bytes, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(c->b_force.p, c->d_force.p, c->d_force.bytes, cudaMemcpyDeviceToDevice, st));
            if(c->d_accel.bytes)
            {
                CK(cudaMemcpyAsync(c->b_accel.p, c->d_accel.p, c->d_accel.bytes, cudaMemcpyDeviceToDevice, st));
            }
        }
        // step 1 of the chunk, then steps 2..n with the previous closing
        // half-kick fused into their first pass, then the last closing kick
        if(c->graphs)
        {
            if(c->graph_dirty || !c->graph_exec) {capture_graph(c);}
            CK(cudaGraphLaunch(c->graph_exec, st));
            int64_t k = 1;
            for(; k + 4 <= nsteps; k += 4) {CK(cudaGraphLaunch(c->graph4_exec, st));}
            for(; k < nsteps; ++k) {CK(cudaGraphLaunch(c->graph2_exec, st));}
            note_launches((int)std::min<long long>(c->graph_nodes + c->graph2_nodes * (nsteps - 1),
                                                   (1ll << 30)));
        }
        else
        {
            for(int64_t k = 0; k < nsteps; ++k) {enqueue_step_body(c, k > 0, false);}
        }
        launch_integrate_last(c->arena, st);
        CK(cudaGetLastError());
        download_sys(c);
        bool overflow = false;
        check_status(c, overflow);
        if(!overflow) {return;}
        if(!c->rollback) {throw Error(MJG_ESTATE, "a Verlet list overflowed (enable rollback)");}
        // roll back, grow the lists, rebuild, retry
        CK(cudaMemcpyAsync(c->d_sys.p, c->b_sys.p, c->d_sys.bytes, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(c->d_pos.p, c->b_pos.p, c->d_pos.bytes, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(c->d_vel.p, c->b_vel.p, c->d_vel.bytes, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(c->d_force.p, c->b_force.p, c->d_force.bytes, cudaMemcpyDeviceToDevice, st));
        if(c->d_accel.bytes)
        {
            CK(cudaMemcpyAsync(c->d_accel.p, c->b_accel.p, c->d_accel.bytes, cudaMemcpyDeviceToDevice, st));
        }
        for(int g = 0; g < NGLOBAL; ++g)
        {
            TermDev& T = c->term[g];
            if(!T.t.on) {continue;}
            int mx = 0;
            CK(cudaMemcpyAsync(&mx, T.t.max_count, sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if(mx > T.t.cap) {alloc_lists(c, g, list_capacity(mx));}
        }
        rebuild_all(c);
    }
    throw Error(MJG_ESTATE, "Verlet lists kept overflowing");
}

}  // namespace
}  // namespace mjg

// ====================================================================== ABI

using namespace mjg;

#define ABI_BEGIN(ctx)                      \
    if(!(ctx)) {return MJG_EINVAL;}         \
    try {
#define ABI_END(ctx)                                          \
    return MJG_OK;                                            \
    } catch(const mjg::Error& e) {(ctx)->err = e.what(); return e.code;}   \
    catch(const std::bad_alloc&) {(ctx)->err = "host out of memory"; return MJG_ENOMEM;} \
    catch(const std::exception& e) {(ctx)->err = e.what(); return MJG_EINVAL;}

extern "C" {

int mjg_context_create(int device, int precision, mjg_context** out)
{
    if(!out || (precision != MJG_PRECISION_FP64 && precision != MJG_PRECISION_MIXED)) {return MJG_EINVAL;}
    *out = nullptr;
    auto* c = new (std::nothrow) mjg_context();
    if(!c) {return MJG_ENOMEM;}
    c->device = device;
    c->precision = precision;
    bool ok = cudaSetDevice(device) == cudaSuccess &&
              cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) == cudaSuccess;
    for(int b = 0; ok && b <= mjg::NGLOBAL; ++b)
    {
        ok = cudaStreamCreateWithFlags(&c->side[b], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&c->ev_join[b], cudaEventDisableTiming) == cudaSuccess;
        if(ok && b < mjg::NGLOBAL)
        {
            ok = cudaStreamCreateWithFlags(&c->gate_body[b], cudaStreamNonBlocking) == cudaSuccess;
        }
    }
    if(!ok)
    {
        cudaGetLastError();
        mjg_context_destroy(c);
        return MJG_ECUDA;
    }
    *out = c;
    return MJG_OK;
}

void mjg_context_destroy(mjg_context* c)
{
    if(!c) {return;}
    cudaSetDevice(c->device);
    if(c->stream) {cudaStreamSynchronize(c->stream);}
    release_graph(c);
    for(auto& t : c->term)
    {
        DevBuf* bufs[] = {&t.part_particle, &t.part_p0, &t.part_p1, &t.part_lead, &t.part_sys,
                          &t.part_cell, &t.cell_count, &t.cell_start, &t.cell_fill, &t.work, &t.part_chunks, &t.cell_chunks, &t.flagged,
                          &t.slot_part, &t.slot_particle, &t.slot_lead, &t.slot_sys, &t.slot_pd,
                          &t.slot_p1, &t.slot_of, &t.slot_w, &t.nnb, &t.nbr, &t.max_count, &t.any_rebuild, &t.ex_start,
                          &t.ex_idx};
        for(auto* b : bufs) {b->release();}
    }
    if(c->h_pinned) {cudaFreeHost(c->h_pinned);}
    if(c->h_pack) {cudaFreeHost(c->h_pack);}
    for(int b = 0; b <= mjg::NGLOBAL; ++b)
    {
        if(c->side[b]) {cudaStreamSynchronize(c->side[b]); cudaStreamDestroy(c->side[b]);}
        if(b < mjg::NGLOBAL && c->gate_body[b]) {cudaStreamDestroy(c->gate_body[b]);}
        if(c->ev_join[b]) {cudaEventDestroy(c->ev_join[b]);}
    }
    if(c->ev_fork) {cudaEventDestroy(c->ev_fork);}
    if(c->stream) {cudaStreamDestroy(c->stream);}
    delete c;
}

const char* mjg_last_error(const mjg_context* c) {return c ? c->err.c_str() : "null context";}

int mjg_context_set_graphs(mjg_context* c, int enable)
{
    ABI_BEGIN(c)
    c->graphs = enable != 0;
    release_graph(c);
    ABI_END(c)
}

int mjg_context_set_rollback(mjg_context* c, int enable)
{
    ABI_BEGIN(c)
    if(c->committed) {throw Error(MJG_ESTATE, "set rollback before mjg_commit");}
    c->rollback = enable != 0;
    ABI_END(c)
}

int mjg_context_reserve(mjg_context* c, int64_t particles)
{
    ABI_BEGIN(c)
    if(particles < 0) {throw Error(MJG_EINVAL, "negative particle count");}
    // the commit's packing buffer: state, coefficients, exclusions, pair
    // participants and bonded terms come to about 400 bytes per particle
    const size_t pack = (size_t)particles * 400;
    if(pack > c->h_pack_bytes)
    {
        if(c->h_pack) {cudaFreeHost(c->h_pack); c->h_pack = nullptr; c->h_pack_bytes = 0;}
        CK(cudaMallocHost(&c->h_pack, pack));
        c->h_pack_bytes = pack;
    }
    pinned(c, (size_t)particles * 3 * sizeof(double) / 2);   // grows to twice: one field of state
    ABI_END(c)
}

int mjg_system_create(mjg_context* c, int64_t n, int boundary, const double* lower,
                      const double* upper, const double* pos, const double* vel,
                      const double* mass, int* sys_id)
{
    ABI_BEGIN(c)
    if(n <= 0 || !pos || !mass || !sys_id) {throw Error(MJG_EINVAL, "system needs n > 0, pos and mass");}
    if(n > (int64_t)1 << 30) {throw Error(MJG_EINVAL, "too many particles in one system");}
    if(boundary != MJG_UNLIMITED && boundary != MJG_PERIODIC_CUBOID) {throw Error(MJG_EINVAL, "unknown boundary");}
    HostSystem s;
    s.n = n;
    s.boundary = boundary == MJG_PERIODIC_CUBOID ? B_PERIODIC : B_UNLIMITED;
    if(s.boundary == B_PERIODIC)
    {
        if(!lower || !upper) {throw Error(MJG_EINVAL, "periodic boundary needs lower and upper");}
        for(int x = 0; x < 3; ++x)
        {
            s.lower[x] = lower[x]; s.upper[x] = upper[x];
            if(!(upper[x] > lower[x])) {throw Error(MJG_EINVAL, "periodic box has no volume");}
        }
    }
    s.pos.assign(pos, pos + 3 * n);
    s.vel = vel ? std::vector<double>(vel, vel + 3 * n) : std::vector<double>(3 * n, 0.0);
    s.mass.assign(mass, mass + n);
    for(double m : s.mass) {if(!(m > 0)) {throw Error(MJG_EINVAL, "masses must be positive");}}
    c->sys.push_back(std::move(s));
    *sys_id = (int)c->sys.size() - 1;
    ABI_END(c)
}

int mjg_system_set_temperature(mjg_context* c, int sys, double T)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    if(!(T >= 0)) {throw Error(MJG_EINVAL, "temperature must not be negative");}
    s.T = T;
    if(!c->committed || !s.resident || s.integrator == I_VV) {return MJG_OK;}
    // BAOABLangevinIntegrator::update -> reset_parameters (:47-58, :73-99),
    // UnderdampedLangevinIntegrator::update (:55-70) or
    // GJFNVTLangevinIntegrator::update (:87-97): the noise coefficients of
    // the system's particles, computed as at commit
    const Units u;
    const double kBT = u.kB * s.T;
    std::vector<double> z((size_t)s.n);
    for(int64_t i = 0; i < s.n; ++i)
    {
        if(s.integrator == I_UNDERDAMPED)
        {
            const double rmass = 1.0 / s.mass[i];
            z[i] = std::sqrt(2 * u.kB * s.T / s.dt) * std::sqrt(s.gamma[i] * rmass);
            continue;
        }
        if(s.integrator == I_GJF) {z[i] = std::sqrt(2 * s.gamma[i] * kBT * s.dt); continue;}
        const double gamma_dt = -1 * s.gamma[i] * s.dt;
        z[i] = std::sqrt(kBT * (1 - std::exp(2 * gamma_dt)) * (1.0 / s.mass[i]));
    }
    CK(cudaStreamSynchronize(c->stream));
    double* stg = c->d_staging.as<double>();
    CK(cudaMemcpyAsync(stg, z.data(), sizeof(double) * s.n, cudaMemcpyHostToDevice, c->stream));
    launch_set_noise(c->arena, stg, s.off, s.n, c->stream);
    CK(cudaStreamSynchronize(c->stream));
    download_sys(c);
    SysDev& d = c->h_sys[s.arena_slot];
    if(d.uniform_coef && s.n > 0)
    {
        d.coef.z = z[0];
        upload_sys(c);
        CK(cudaStreamSynchronize(c->stream));
    }
    ABI_END(c)
}

int mjg_system_set_attributes(mjg_context* c, int sys, double T, double I)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    if(s.resident) {throw Error(MJG_ESTATE, "attributes are fixed once committed");}
    // temperature 0 is a run without thermal noise, as in the reference's
    // input; DebyeHuckel needs a positive one for its Debye length (checked
    // at commit)
    if(!(T >= 0) || !(I > 0)) {throw Error(MJG_EINVAL, "temperature must not be negative, ionic strength must be positive");}
    s.T = T; s.I = I;
    ABI_END(c)
}

int mjg_system_add_connections(mjg_context* c, int sys, const char* kind, int64_t m, const int64_t* pairs)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    if(s.resident) {throw Error(MJG_ESTATE, "topology is fixed once committed");}
    if(!kind || (m > 0 && !pairs)) {throw Error(MJG_EINVAL, "bad connections");}
    for(int64_t k = 0; k < m; ++k)
    {
        const int64_t i = pairs[2 * k], j = pairs[2 * k + 1];
        if(i < 0 || j < 0 || i >= s.n || j >= s.n) {throw Error(MJG_EINVAL, "connection index out of range");}
        s.connections.push_back({kind, {i, j}});
    }
    ABI_END(c)
}

int mjg_system_set_step(mjg_context* c, int sys, uint64_t step)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    if(s.resident) {throw Error(MJG_ESTATE, "the step counter is set before the first commit");}
    s.step = step;
    ABI_END(c)
}

int mjg_system_freeze(mjg_context* c, int sys, int frozen)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    s.frozen = frozen != 0;
    if(c->committed && s.resident)
    {
        CK(cudaStreamSynchronize(c->stream));
        download_sys(c);
        c->h_sys[s.arena_slot].frozen = s.frozen ? 1 : 0;
        upload_sys(c);
        CK(cudaStreamSynchronize(c->stream));
        int any = 0;
        for(const auto& h : c->h_sys) {any |= h.frozen;}
        if(any != c->arena.any_frozen)     // the captured launches carry the flag
        {
            c->arena.any_frozen = any;
            release_graph(c);
        }
    }
    ABI_END(c)
}

int mjg_system_remove(mjg_context* c, int sys)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    // keep only what the arena bookkeeping reads until the next commit
    HostSystem dead;
    dead.alive = false;
    dead.resident = s.resident;
    dead.arena_slot = s.arena_slot;
    dead.n = s.n;
    dead.off = s.off;
    s = std::move(dead);
    ABI_END(c)
}

static void check_idx(const HostSystem& s, int64_t np, const int64_t* idx)
{
    if(np < 0 || (np > 0 && !idx)) {throw Error(MJG_EINVAL, "bad participant list");}
    std::vector<char> seen(s.n, 0);
    for(int64_t k = 0; k < np; ++k)
    {
        if(idx[k] < 0 || idx[k] >= s.n) {throw Error(MJG_EINVAL, "participant index out of range");}
        if(seen[idx[k]]) {throw Error(MJG_EINVAL, "participant listed twice");}
        seen[idx[k]] = 1;
    }
}

int mjg_exv_set(mjg_context* c, int sys, double eps, double cutoff_ratio, double margin,
                int64_t np, const int64_t* idx, const double* radius)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    if(s.resident) {throw Error(MJG_ESTATE, "interactions are fixed once committed");}
    check_idx(s, np, idx);
    if(!(cutoff_ratio > 0) || !(margin >= 0) || (np > 0 && !radius)) {throw Error(MJG_EINVAL, "bad ExcludedVolume parameters");}
    HostGlobal& g = s.g[G_EXV];
    g.on = true; g.kind = EXV_PLAIN; g.eps = eps; g.cutoff_ratio = cutoff_ratio; g.margin = margin;
    g.idx.assign(idx, idx + np); g.p0.assign(radius, radius + np); g.p1.clear();
    ABI_END(c)
}

int mjg_dh_set(mjg_context* c, int sys, double cutoff_ratio, double margin, int64_t np,
               const int64_t* idx, const double* charge)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    if(s.resident) {throw Error(MJG_ESTATE, "interactions are fixed once committed");}
    check_idx(s, np, idx);
    if(!(cutoff_ratio > 0) || !(margin >= 0) || (np > 0 && !charge)) {throw Error(MJG_EINVAL, "bad DebyeHuckel parameters");}
    HostGlobal& g = s.g[G_DH];
    g.on = true; g.cutoff_ratio = cutoff_ratio; g.margin = margin;
    g.idx.assign(idx, idx + np); g.p0.assign(charge, charge + np); g.p1.clear();
    ABI_END(c)
}

int mjg_lj_set(mjg_context* c, int sys, double cutoff_ratio, double margin, int64_t np,
               const int64_t* idx, const double* sigma, const double* epsilon)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    if(s.resident) {throw Error(MJG_ESTATE, "interactions are fixed once committed");}
    check_idx(s, np, idx);
    if(!(cutoff_ratio > 0) || !(margin >= 0) || (np > 0 && (!sigma || !epsilon))) {throw Error(MJG_EINVAL, "bad LennardJones parameters");}
    HostGlobal& g = s.g[G_LJ];
    g.on = true; g.kind = LJ_PLAIN; g.cutoff_ratio = cutoff_ratio; g.margin = margin;
    g.idx.assign(idx, idx + np); g.p0.assign(sigma, sigma + np); g.p1.assign(epsilon, epsilon + np);
    ABI_END(c)
}

int mjg_exv_family_set(mjg_context* c, int sys, const char* potential, double eps, double cutoff_ratio,
                       int power, double margin, int64_t np, const int64_t* idx, const double* p0,
                       const double* p1)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    if(s.resident) {throw Error(MJG_ESTATE, "interactions are fixed once committed");}
    if(!potential) {throw Error(MJG_EINVAL, "potential name is NULL");}
    const std::string name(potential);
    int kind;
    if(name == "InversePower")                {kind = EXV_INVERSE_POWER;}
    else if(name == "HardCoreExcludedVolume") {kind = EXV_HARD_CORE;}
    else {throw Error(MJG_EINVAL, "unknown ExcludedVolume-family potential: " + name);}
    check_idx(s, np, idx);
    if(!(cutoff_ratio > 0) || !(margin >= 0) || (np > 0 && !p0) || (kind == EXV_HARD_CORE && np > 0 && !p1) ||
       (kind == EXV_INVERSE_POWER && power <= 0))
    {
        throw Error(MJG_EINVAL, "bad " + name + " parameters");
    }
    HostGlobal& g = s.g[G_EXV];
    g.on = true; g.kind = kind; g.power = power; g.eps = eps; g.cutoff_ratio = cutoff_ratio; g.margin = margin;
    g.idx.assign(idx, idx + np); g.p0.assign(p0, p0 + np);
    if(kind == EXV_HARD_CORE) {g.p1.assign(p1, p1 + np);} else {g.p1.clear();}
    ABI_END(c)
}

int mjg_pair_set(mjg_context* c, int sys, const char* potential, double cutoff_ratio, double margin,
                 int64_t np, const int64_t* idx, const double* sigma, const double* epsilon)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    if(s.resident) {throw Error(MJG_ESTATE, "interactions are fixed once committed");}
    if(!potential) {throw Error(MJG_EINVAL, "potential name is NULL");}
    const std::string name(potential);
    int kind;
    if(name == "LennardJones")                {kind = LJ_PLAIN;}
    else if(name == "WCA")                    {kind = LJ_WCA; cutoff_ratio = SIXTH_ROOT_OF_TWO;}
    else if(name == "LennardJonesAttractive") {kind = LJ_ATTRACTIVE;}
    else if(name == "UniformLennardJones")    {kind = LJ_UNIFORM;}
    else {throw Error(MJG_EINVAL, "unknown pair potential: " + name);}
    check_idx(s, np, idx);
    if(!(cutoff_ratio > 0) || !(margin >= 0) || (np > 0 && (!sigma || !epsilon)))
    {
        throw Error(MJG_EINVAL, "bad " + name + " parameters");
    }
    if(kind == LJ_UNIFORM)
    {
        for(int64_t k = 1; k < np; ++k)
        {
            if(sigma[k] != sigma[0] || epsilon[k] != epsilon[0])
            {
                throw Error(MJG_EINVAL, "UniformLennardJones takes one sigma and one epsilon");
            }
        }
    }
    HostGlobal& g = s.g[G_LJ];
    g.on = true; g.kind = kind; g.cutoff_ratio = cutoff_ratio; g.margin = margin;
    g.idx.assign(idx, idx + np); g.p0.assign(sigma, sigma + np); g.p1.assign(epsilon, epsilon + np);
    ABI_END(c)
}

int mjg_ignore_set(mjg_context* c, int sys, int term, int ignore_molecule, int nk,
                   const char* const* kinds, const int32_t* within)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    if(s.resident) {throw Error(MJG_ESTATE, "interactions are fixed once committed");}
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ) {throw Error(MJG_EINVAL, "ignore rules apply to global terms");}
    if(ignore_molecule < 0 || ignore_molecule > 2 || nk < 0 || (nk > 0 && (!kinds || !within)))
    {
        throw Error(MJG_EINVAL, "bad ignore rule");
    }
    HostGlobal& g = s.g[term - MJG_TERM_EXV];
    g.ignore_mol = ignore_molecule;
    g.within.clear();
    for(int k = 0; k < nk; ++k)
    {
        if(!kinds[k] || within[k] < 0) {throw Error(MJG_EINVAL, "bad ignore.particles_within");}
        g.within.emplace_back(kinds[k], (int)within[k]);
    }
    ABI_END(c)
}

static void set_local(mjg_context* c, int sys, HostLocal& L, const char* topology, int64_t m,
                      const int64_t* idx, const double* k, const double* v0, const int32_t* n, int arity,
                      const HostSystem& s)
{
    (void)c; (void)sys;
    if(s.resident) {throw Error(MJG_ESTATE, "interactions are fixed once committed");}
    if(m < 0 || (m > 0 && (!idx || !k || !v0))) {throw Error(MJG_EINVAL, "bad local interaction");}
    for(int64_t t = 0; t < m * arity; ++t)
    {
        if(idx[t] < 0 || idx[t] >= s.n) {throw Error(MJG_EINVAL, "local interaction index out of range");}
    }
    L.kind = topology ? topology : "none";
    L.idx.assign(idx, idx + m * arity);
    L.k.assign(k, k + m);
    L.v0.assign(v0, v0 + m);
    if(n) {L.n.assign(n, n + m);} else {L.n.clear();}
}

int mjg_bonds_set(mjg_context* c, int sys, const char* topology, int64_t m, const int64_t* idx,
                  const double* k, const double* v0)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    set_local(c, sys, s.bond, topology, m, idx, k, v0, nullptr, 2, s);
    ABI_END(c)
}

int mjg_angles_set(mjg_context* c, int sys, const char* topology, int64_t m, const int64_t* idx,
                   const double* k, const double* v0)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    set_local(c, sys, s.angle, topology, m, idx, k, v0, nullptr, 3, s);
    ABI_END(c)
}

int mjg_dihedrals_set(mjg_context* c, int sys, const char* topology, int64_t m, const int64_t* idx,
                      const double* k, const int32_t* n, const double* v0)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    if(m > 0 && !n) {throw Error(MJG_EINVAL, "dihedrals need n");}
    set_local(c, sys, s.dihd, topology, m, idx, k, v0, n, 4, s);
    ABI_END(c)
}

int mjg_integrator_set(mjg_context* c, int sys, int kind, double dt, const double* gamma, uint64_t seed)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    if(s.resident) {throw Error(MJG_ESTATE, "the integrator is fixed once committed");}
    if(kind != MJG_BAOAB && kind != MJG_VELOCITY_VERLET && kind != MJG_UNDERDAMPED_LANGEVIN &&
       kind != MJG_GJF_LANGEVIN && kind != MJG_GBAOAB_LANGEVIN)
    {
        throw Error(MJG_EINVAL, "unknown integrator");
    }
    if(!(dt > 0)) {throw Error(MJG_EINVAL, "dt must be positive");}
    if(kind != MJG_VELOCITY_VERLET && !gamma) {throw Error(MJG_EINVAL, "Langevin integrators need gammas");}
    s.integrator = kind == MJG_BAOAB ? I_BAOAB : kind == MJG_VELOCITY_VERLET ? I_VV :
                   kind == MJG_UNDERDAMPED_LANGEVIN ? I_UNDERDAMPED : kind == MJG_GJF_LANGEVIN ? I_GJF :
                   I_GBAOAB;
    s.dt = dt;
    s.gamma = gamma ? std::vector<double>(gamma, gamma + s.n) : std::vector<double>(s.n, 0.0);
    s.seed = seed;
    ABI_END(c)
}

int mjg_commit(mjg_context* c)
{
    ABI_BEGIN(c)
    commit(c);
    ABI_END(c)
}

int mjg_step(mjg_context* c, int64_t nsteps)
{
    ABI_BEGIN(c)
    if(!c->committed) {throw Error(MJG_ESTATE, "mjg_commit first");}
    if(nsteps < 0) {throw Error(MJG_EINVAL, "negative step count");}
    run_steps(c, nsteps);
    ABI_END(c)
}

int mjg_synchronize(mjg_context* c)
{
    ABI_BEGIN(c)
    CK(cudaStreamSynchronize(c->stream));
    ABI_END(c)
}

int mjg_rebuild(mjg_context* c)
{
    ABI_BEGIN(c)
    if(!c->committed) {throw Error(MJG_ESTATE, "mjg_commit first");}
    rebuild_all(c);
    CK(cudaStreamSynchronize(c->stream));
    ABI_END(c)
}

int mjg_get_state(mjg_context* c, int sys, double* pos, double* vel, double* force)
{
    ABI_BEGIN(c)
    HostSystem& s = get_resident(c, sys);
    double* stg = c->d_staging.as<double>();
    double* outs[3] = {pos, vel, force};
    for(int w = 0; w < 3; ++w)
    {
        if(!outs[w]) {continue;}
        launch_pack_state(c->arena, stg, w, s.off, s.n, c->stream);
        CK(cudaMemcpyAsync(outs[w], stg, sizeof(double) * 3 * s.n, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    ABI_END(c)
}

int mjg_set_state(mjg_context* c, int sys, const double* pos, const double* vel)
{
    ABI_BEGIN(c)
    HostSystem& s = get_resident(c, sys);
    double* stg = c->d_staging.as<double>();
    if(pos)
    {
        std::vector<double> p(pos, pos + 3 * s.n);
        if(s.boundary == B_PERIODIC)
        {
            for(int64_t i = 0; i < s.n; ++i)
                for(int x = 0; x < 3; ++x)
                {
                    const double w = s.upper[x] - s.lower[x];
                    if(p[3 * i + x] < s.lower[x]) {p[3 * i + x] += w;}
                    else if(p[3 * i + x] >= s.upper[x]) {p[3 * i + x] -= w;}
                }
        }
        CK(cudaMemcpyAsync(stg, p.data(), sizeof(double) * 3 * s.n, cudaMemcpyHostToDevice, c->stream));
        launch_unpack_state(c->arena, stg, nullptr, s.off, s.n, c->stream);
        CK(cudaStreamSynchronize(c->stream));
    }
    if(vel)
    {
        CK(cudaMemcpyAsync(stg, vel, sizeof(double) * 3 * s.n, cudaMemcpyHostToDevice, c->stream));
        launch_unpack_state(c->arena, nullptr, stg, s.off, s.n, c->stream);
        CK(cudaStreamSynchronize(c->stream));
    }
    if(pos)
    {
        rebuild_all(c);
        // forces at the new positions (the integrator's next B step uses them)
        compute_initial_forces(c);
        launch_init_accel(c->arena, s.off, s.n, c->stream);   // Integrator::initialize for this system
        CK(cudaStreamSynchronize(c->stream));
    }
    ABI_END(c)
}

int mjg_get_state_all(mjg_context* c, double* pos, double* vel)
{
    ABI_BEGIN(c)
    if(!c->committed) {throw Error(MJG_ESTATE, "mjg_commit first");}
    double* stg = c->d_staging.as<double>();
    double* stg_vel = stg + 3 * c->n_tot;          // the staging holds both arrays side by side
    if(pos) {launch_pack_state(c->arena, stg, 0, 0, c->n_tot, c->stream);}
    if(vel) {launch_pack_state(c->arena, stg_vel, 1, 0, c->n_tot, c->stream);}
    if(pos) {CK(cudaMemcpyAsync(pos, stg, sizeof(double) * 3 * c->n_tot, cudaMemcpyDeviceToHost, c->stream));}
    if(vel) {CK(cudaMemcpyAsync(vel, stg_vel, sizeof(double) * 3 * c->n_tot, cudaMemcpyDeviceToHost, c->stream));}
    CK(cudaStreamSynchronize(c->stream));
    ABI_END(c)
}

int mjg_set_state_all(mjg_context* c, const double* pos, const double* vel)
{
    ABI_BEGIN(c)
    if(!c->committed) {throw Error(MJG_ESTATE, "mjg_commit first");}
    double* stg = c->d_staging.as<double>();
    double* stg_vel = stg + 3 * c->n_tot;          // both arrays side by side: one unpack launch
    if(vel) {CK(cudaMemcpyAsync(stg_vel, vel, sizeof(double) * 3 * c->n_tot, cudaMemcpyHostToDevice, c->stream));}
    if(pos) {CK(cudaMemcpyAsync(stg, pos, sizeof(double) * 3 * c->n_tot, cudaMemcpyHostToDevice, c->stream));}
    // positions are taken as given (already inside their boxes)
    if(pos || vel) {launch_unpack_state(c->arena, pos ? stg : nullptr, vel ? stg_vel : nullptr, 0, c->n_tot, c->stream);}
    if(pos)
    {
        rebuild_all(c);
        compute_initial_forces(c);
        launch_init_accel(c->arena, 0, c->n_tot, c->stream);   // new positions: Integrator::initialize
    }
    CK(cudaStreamSynchronize(c->stream));
    ABI_END(c)
}

int mjg_energies(mjg_context* c, int sys, double* out)
{
    ABI_BEGIN(c)
    HostSystem& s = get_resident(c, sys);
    if(!out) {throw Error(MJG_EINVAL, "out is NULL");}
    launch_clear_energy(c->arena, c->stream);
    Arena a = c->arena;
    a.force = c->d_force_scratch.p;
    enqueue_forces(c, a, false, true);
    download_sys(c);
    for(int t = 0; t < NTERMS; ++t) {out[t] = c->h_sys[s.arena_slot].energy[t];}
    ABI_END(c)
}

int mjg_term_force(mjg_context* c, int sys, int term, double* force, double* energy)
{
    ABI_BEGIN(c)
    HostSystem& s = get_resident(c, sys);
    if(term < 0 || term >= NTERMS) {throw Error(MJG_EINVAL, "unknown term");}
    Arena a = c->arena;
    a.force = c->d_force_scratch.p;
    launch_clear_energy(a, c->stream);
    launch_zero_force(a, c->stream);
    if(term <= MJG_TERM_DIHEDRAL) {launch_local(a, c->local, 1 << term, true, true, 0, c->stream);}
    else {launch_pair(a, term - MJG_TERM_EXV, c->term[term - MJG_TERM_EXV].t, true, true, 0, c->stream);}
    if(force)
    {
        double* stg = c->d_staging.as<double>();
        launch_pack_state(a, stg, 2, s.off, s.n, c->stream);
        CK(cudaMemcpyAsync(force, stg, sizeof(double) * 3 * s.n, cudaMemcpyDeviceToHost, c->stream));
    }
    download_sys(c);
    if(energy) {*energy = c->h_sys[s.arena_slot].energy[term];}
    ABI_END(c)
}

int mjg_neighbors(mjg_context* c, int sys, int term, int64_t* pairs, int64_t cap, int64_t* count)
{
    ABI_BEGIN(c)
    HostSystem& s = get_resident(c, sys);
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ || !count) {throw Error(MJG_EINVAL, "bad neighbour query");}
    const int g = term - MJG_TERM_EXV;
    const TermArrays& t = c->term[g].t;
    *count = 0;
    if(!t.on || !s.g[g].on) {throw Error(MJG_EINVAL, "term not present in this system");}
    CK(cudaStreamSynchronize(c->stream));
    download_sys(c);
    const GlobalParams& G = c->h_sys[s.arena_slot].g[g];
    const int so = G.slot_off, ns = G.nslot;
    std::vector<int> nnb(t.np), part(t.np);
    CK(cudaMemcpy(nnb.data(), t.nnb, sizeof(int) * t.np, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(part.data(), t.slot_particle, sizeof(int) * t.np, cudaMemcpyDeviceToHost));
    std::vector<int> all(list_words(t.cap) * (size_t)t.np);
    if(!all.empty())
    {
        CK(cudaMemcpy(all.data(), t.nbr, sizeof(int) * all.size(), cudaMemcpyDeviceToHost));
    }
    std::vector<std::pair<int64_t, int64_t>> out;
    for(int q = so; q < so + ns; ++q)
    {
        for(int k = 0; k < nnb[q]; ++k)
        {
            const int r = all[(size_t)nbr_pos(k, q, t.np, t.tpp, t.cap, t.slot_major)];
            const int64_t i = part[q] - s.off, j = part[r] - s.off;
            if(t.half) {out.emplace_back(std::min(i, j), std::max(i, j));}   // each pair listed once
            else if(i < j) {out.emplace_back(i, j);}
        }
    }
    std::sort(out.begin(), out.end());
    *count = (int64_t)out.size();
    if(pairs)
    {
        const int64_t w = std::min<int64_t>(cap, (int64_t)out.size());
        for(int64_t k = 0; k < w; ++k) {pairs[2 * k] = out[k].first; pairs[2 * k + 1] = out[k].second;}
    }
    ABI_END(c)
}

int mjg_rebuild_count(mjg_context* c, int sys, int term, int64_t* count)
{
    ABI_BEGIN(c)
    HostSystem& s = get_resident(c, sys);
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ || !count) {throw Error(MJG_EINVAL, "bad query");}
    download_sys(c);
    *count = c->h_sys[s.arena_slot].g[term - MJG_TERM_EXV].rebuilds;
    ABI_END(c)
}

int mjg_step_count(mjg_context* c, int sys, int64_t* steps)
{
    ABI_BEGIN(c)
    HostSystem& s = get_resident(c, sys);
    if(!steps) {throw Error(MJG_EINVAL, "steps is NULL");}
    download_sys(c);
    *steps = (int64_t)c->h_sys[s.arena_slot].step;
    ABI_END(c)
}

int mjg_molecule_count(mjg_context* c, int sys, int64_t* count)
{
    ABI_BEGIN(c)
    HostSystem& s = get_sys(c, sys);
    if(!count) {throw Error(MJG_EINVAL, "count is NULL");}
    std::map<std::string, int> kinds;
    const int bond_kind = kind_id(kinds, "bond");
    int64_t nmol = 0;
    for(const int64_t m : topology_of(s, kinds).molecules(bond_kind)) {nmol = std::max<int64_t>(nmol, m + 1);}
    *count = nmol;
    ABI_END(c)
}

int mjg_particle_count(mjg_context* c, int sys, int64_t* n)
{
    ABI_BEGIN(c)
    if(!n) {throw Error(MJG_EINVAL, "n is NULL");}
    if(sys < 0) {*n = c->n_tot;}
    else {*n = get_sys(c, sys).n;}
    ABI_END(c)
}

int mjg_device_bytes(mjg_context* c, int64_t* bytes)
{
    ABI_BEGIN(c)
    if(!bytes) {throw Error(MJG_EINVAL, "bytes is NULL");}
    *bytes = device_bytes(c);
    ABI_END(c)
}

int mjg_context_get_stream(mjg_context* c, void** stream)
{
    ABI_BEGIN(c)
    if(!stream) {throw Error(MJG_EINVAL, "stream is NULL");}
    *stream = (void*)c->stream;
    ABI_END(c)
}

int mjg_time_kernel(mjg_context* c, int term, int reps, double* ms)
{
    ABI_BEGIN(c)
    if(!c->committed) {throw Error(MJG_ESTATE, "mjg_commit first");}
    if(term < 0 || term >= NTERMS || reps <= 0 || !ms) {throw Error(MJG_EINVAL, "bad timing request");}
    Arena a = c->arena;
    a.force = c->d_force_scratch.p;
    // each launch is timed on its own, after a write larger than L2 has
    // evicted its inputs (as in a step where the other kernels run between
    // two launches of this one) and a read of another buffer larger than L2
    // has replaced the written lines, so that the launch starts with a clean
    // L2 and does not pay for writing back the flush
    const size_t flush_bytes = (size_t)256 << 20;
    DevBuf flush, sweep, sink;
    flush.alloc(flush_bytes);
    sweep.alloc(flush_bytes);
    sink.alloc(sizeof(int));
    CK(cudaMemsetAsync(sweep.p, 0, flush_bytes, c->stream));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto once = [&](bool gather) {
        if(term <= MJG_TERM_DIHEDRAL) {launch_local(a, c->local, 1 << term, true, false, 0, c->stream);}
        else {launch_pair(a, term - MJG_TERM_EXV, c->term[term - MJG_TERM_EXV].t, true, false, 0, c->stream, gather);}
    };
    once(true);   // warm; refreshes the slot coordinates
    double total = 0.0;
    for(int r = 0; r < reps; ++r)
    {
        CK(cudaMemsetAsync(flush.p, r & 0xff, flush_bytes, c->stream));
        launch_read_sweep(sweep.p, flush_bytes, sink.as<int>(), c->stream);
        CK(cudaEventRecord(e0, c->stream));
        once(false);
        CK(cudaEventRecord(e1, c->stream));
        CK(cudaEventSynchronize(e1));
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, e0, e1));
        total += t;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = total / reps;
    ABI_END(c)
}

int mjg_set_threads_per_particle(mjg_context* c, int term, int tpp)
{
    ABI_BEGIN(c)
    if(!c->committed) {throw Error(MJG_ESTATE, "mjg_commit first");}
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ) {throw Error(MJG_EINVAL, "threads per slot apply to global terms");}
    if(tpp != 1 && tpp != 2 && tpp != 4 && tpp != 8 && tpp != 16 && tpp != 32)
    {
        throw Error(MJG_EINVAL, "tpp must be 1, 2, 4, 8, 16 or 32");
    }
    TermDev& T = c->term[term - MJG_TERM_EXV];
    if(!T.t.on) {throw Error(MJG_EINVAL, "term not present");}
    T.tpp_fixed = true;
    T.tpp_choice = tpp;
    if(T.t.tpp != tpp)
    {
        T.t.tpp = tpp;          // the layout changes: rebuild every list
        release_graph(c);
        rebuild_all(c);
        CK(cudaStreamSynchronize(c->stream));
    }
    ABI_END(c)
}

int mjg_set_pair_unroll(mjg_context* c, int term, int unroll)
{
    ABI_BEGIN(c)
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ) {throw Error(MJG_EINVAL, "the batch depth applies to global terms");}
    if(unroll != 1 && unroll != 2 && unroll != 4) {throw Error(MJG_EINVAL, "unroll must be 1, 2 or 4");}
    TermDev& T = c->term[term - MJG_TERM_EXV];
    T.unroll_choice = unroll;
    if(T.t.unroll != unroll)
    {
        T.t.unroll = unroll;    // same lists, another kernel: recapture the step
        release_graph(c);
    }
    ABI_END(c)
}

int mjg_set_pair_schedule(mjg_context* c, int term, int schedule)
{
    ABI_BEGIN(c)
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ) {throw Error(MJG_EINVAL, "the schedule applies to global terms");}
    if(schedule < 0 || schedule > 5) {throw Error(MJG_EINVAL, "schedule must be 0 .. 5");}
    TermDev& T = c->term[term - MJG_TERM_EXV];
    T.schedule_choice = schedule;
    if(T.t.schedule != schedule)
    {
        const int layout = schedule == 5 ? 1 : 0;
        T.t.schedule = schedule;
        release_graph(c);
        if(T.t.on && T.t.slot_major != layout)
        {
            T.t.slot_major = layout;    // the list layout changes: rebuild every list
            if(c->committed)
            {
                rebuild_all(c);
                CK(cudaStreamSynchronize(c->stream));
            }
        }
    }
    ABI_END(c)
}

int mjg_set_half_lists(mjg_context* c, int term, int on)
{
    ABI_BEGIN(c)
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ) {throw Error(MJG_EINVAL, "half lists apply to global terms");}
    if(on && c->precision != P_MIXED) {throw Error(MJG_EINVAL, "half lists need the mixed form's integer force sums");}
    TermDev& T = c->term[term - MJG_TERM_EXV];
    T.half_choice = on != 0;
    const int half = T.half_choice ? 1 : 0;
    if(T.t.half != half)
    {
        T.t.half = half;
        release_graph(c);
        if(T.t.on && c->committed)
        {
            rebuild_all(c);             // another list form: rebuild every list
            CK(cudaStreamSynchronize(c->stream));
        }
    }
    ABI_END(c)
}

int mjg_get_half_lists(mjg_context* c, int term, int* on)
{
    ABI_BEGIN(c)
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ || !on) {throw Error(MJG_EINVAL, "bad query");}
    *on = c->term[term - MJG_TERM_EXV].half_choice ? 1 : 0;
    ABI_END(c)
}

int mjg_set_build_lanes(mjg_context* c, int term, int lanes)
{
    ABI_BEGIN(c)
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ) {throw Error(MJG_EINVAL, "build lanes apply to global terms");}
    if(lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32) {throw Error(MJG_EINVAL, "lanes must be 4, 8, 16 or 32");}
    TermDev& T = c->term[term - MJG_TERM_EXV];
    T.build_lanes_fixed = true;
    T.build_lanes_choice = lanes;
    if(T.t.build_lanes != lanes)
    {
        T.t.build_lanes = lanes;    // same lists, another kernel: recapture the step
        release_graph(c);
    }
    ABI_END(c)
}

int mjg_get_build_lanes(mjg_context* c, int term, int* lanes)
{
    ABI_BEGIN(c)
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ || !lanes) {throw Error(MJG_EINVAL, "bad query");}
    *lanes = c->term[term - MJG_TERM_EXV].build_lanes_choice;
    ABI_END(c)
}

int mjg_get_pair_schedule(mjg_context* c, int term, int* schedule)
{
    ABI_BEGIN(c)
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ || !schedule) {throw Error(MJG_EINVAL, "bad query");}
    *schedule = c->term[term - MJG_TERM_EXV].schedule_choice;
    ABI_END(c)
}

int mjg_get_pair_unroll(mjg_context* c, int term, int* unroll)
{
    ABI_BEGIN(c)
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ || !unroll) {throw Error(MJG_EINVAL, "bad query");}
    *unroll = c->term[term - MJG_TERM_EXV].unroll_choice;
    ABI_END(c)
}

int mjg_get_threads_per_particle(mjg_context* c, int term, int* tpp)
{
    ABI_BEGIN(c)
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ || !tpp) {throw Error(MJG_EINVAL, "bad query");}
    *tpp = c->term[term - MJG_TERM_EXV].t.tpp;
    ABI_END(c)
}

int mjg_set_margin(mjg_context* c, int term, double margin)
{
    ABI_BEGIN(c)
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ || !(margin >= 0)) {throw Error(MJG_EINVAL, "bad margin");}
    for(auto& s : c->sys)
    {
        if(s.alive && s.g[term - MJG_TERM_EXV].on) {s.g[term - MJG_TERM_EXV].margin = margin;}
    }
    if(c->committed) {commit(c);}   // new cell grids and lists; the state is kept
    ABI_END(c)
}

int mjg_set_list_capacity(mjg_context* c, int term, int cap)
{
    ABI_BEGIN(c)
    if(!c->committed) {throw Error(MJG_ESTATE, "mjg_commit first");}
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ || cap < 0) {throw Error(MJG_EINVAL, "bad capacity request");}
    TermDev& T = c->term[term - MJG_TERM_EXV];
    if(!T.t.on) {throw Error(MJG_EINVAL, "term not present");}
    if(cap <= T.cap_alloc)
    {
        // the buffer keeps its size, so the current lists stay readable; the
        // next rebuild that needs more than cap partners reports an overflow
        T.t.cap = cap;
        release_graph(c);
    }
    else
    {
        alloc_lists(c, term - MJG_TERM_EXV, cap);
        rebuild_all(c);
        CK(cudaStreamSynchronize(c->stream));
    }
    ABI_END(c)
}

int mjg_pair_count(mjg_context* c, int sys, int term, int64_t* count)
{
    ABI_BEGIN(c)
    if(!c->committed) {throw Error(MJG_ESTATE, "mjg_commit first");}
    if(term < MJG_TERM_EXV || term > MJG_TERM_LJ || !count) {throw Error(MJG_EINVAL, "bad query");}
    int slot = -1;
    if(sys >= 0) {slot = get_resident(c, sys).arena_slot;}
    DevBuf tmp;
    tmp.alloc(sizeof(unsigned long long));
    CK(cudaMemsetAsync(tmp.p, 0, tmp.bytes, c->stream));
    launch_count_cut(c->arena, term - MJG_TERM_EXV, c->term[term - MJG_TERM_EXV].t, slot,
                     tmp.as<unsigned long long>(), c->stream);
    unsigned long long h = 0;
    CK(cudaMemcpyAsync(&h, tmp.p, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *count = (int64_t)h;
    ABI_END(c)
}

int mjg_launch_count(mjg_context* c, int64_t* launches)
{
    ABI_BEGIN(c)
    if(!launches) {throw Error(MJG_EINVAL, "launches is NULL");}
    *launches = g_launches.load();
    ABI_END(c)
}

}  // extern "C"
