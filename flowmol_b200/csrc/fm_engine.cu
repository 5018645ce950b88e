// fm_engine.cu -- host side of the multi-job slot engine: arena allocation,
// admission by memory footprint, chunked CUDA-graph execution, retirement.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <iterator>
#include <map>
#include <string>
#include <vector>

#include "fm_engine.cuh"
#include "flowmol_b200.h"

namespace {

int efail(int code, const std::string &m)
{
    fm::set_last_error(m.c_str());
    return code;
}

#define EN_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return efail(FM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
#define EN_TRY(call)                 \
    do {                             \
        int r_ = (call);             \
        if (r_ != FM_OK) return r_;  \
    } while (0)

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// First-fit allocator over [0, cap) with coalescing; sizes rounded up to `align`.
struct Ranges {
    int64_t cap = 0, align = 1;
    std::map<int64_t, int64_t> free_;  // offset -> length
    void init(int64_t c, int64_t a)
    {
        cap = c; align = a; free_.clear();
        if (c > 0) free_[0] = c;
    }
    int64_t round(int64_t n) const { return ((n + align - 1) / align) * align; }
    bool fits(int64_t n) const
    {
        n = round(n);
        for (auto &f : free_)
            if (f.second >= n) return true;
        return false;
    }
    int64_t alloc(int64_t n)
    {
        n = round(n);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                int64_t off = it->first, len = it->second;
                free_.erase(it);
                if (len > n) free_[off + n] = len - n;
                return off;
            }
        }
        return -1;
    }
    void release(int64_t off, int64_t n)
    {
        n = round(n);
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct Job {
    int64_t id = 0;
    fm_job p{};
    std::vector<double> r, v, rt, sv;
    std::vector<int32_t> tag;
    bool has_tag = false, has_rt = false, has_sv = false;
    double t_submit = 0.0, t_admit = 0.0;
    int retries = 0;
    int maxn = 0;
    // placement while resident
    int slot = -1;
    int64_t mol_off = 0, cell_off = 0, cstart_off = 0, list_off = 0;
    int ncell = 0;
    int mode = fm::MODE_LIST;
};

}  // namespace

struct fm_engine {
    fm_engine_params p{};
    fm::EngDev d{};
    cudaStream_t st = nullptr;
    bool own_stream = false;
    Ranges mol, cell, cstart, list;
    std::deque<Job> queue;
    std::vector<Job> resident;       // indexed by slot; slot < 0 means free
    std::vector<fm::EngSlot> table;  // host mirror
    std::vector<fm_job_result> results;
    std::map<int64_t, std::pair<std::vector<double>, std::vector<double>>> states;
    int64_t next_id = 1;
    int tpm = 0;
    bool tuned = false;
    // list-build tile: jobs below this many molecules per cell are built by
    // 2x2x2-cell blocks (FM_LIST_BUILD_AUTO: chosen by tune_build)
    double blocks_below = 8.0;
    bool tuned_build = false;
    cudaGraphExec_t graph = nullptr;
    bool graph_loop = false;          // the graph is the device-driven tick loop (WHILE node)
    bool loop_off = false;            // conditional nodes unavailable: fixed chunks of ticks
    cudaStream_t cap_st = nullptr;    // capture of the loop's body
    int graph_tpm = -1;
    fm::TickExtent graph_x{0, 0, 0};  // launch extents the graph was captured with
    fm::TickExtent need_x{0, 0, 0};   // extents the resident jobs call for
    double *stage = nullptr;  // device staging for uploads/downloads
    size_t stage_cap = 0;     // doubles
    int32_t *stage_i = nullptr;
    size_t stage_icap = 0;
    int64_t ticks = 0, molsteps = 0, launches = 0;
};

namespace {

template <typename T>
int dal(T **p, size_t n)
{
    *p = nullptr;
    EN_CUDA(cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T)));
    return FM_OK;
}

void free_all(fm_engine *e)
{
    fm::EngDev &d = e->d;
    void *ptrs[] = {d.slots, d.flags, d.pos0, d.pos1, d.vx, d.vy, d.vz, d.ax, d.ay, d.az, d.slot_of, d.uidx, d.tag,
                    d.rteth, d.slidev, d.tpos, d.trteth, d.tslidev, d.tvx, d.tvy, d.tvz, d.tax, d.tay, d.taz,
                    d.tuidx, d.ttag, d.cell_slot, d.cell_of, d.cell_count, d.cell_start, d.perm, d.nbr, d.nnbr,
                    d.rterm, d.tmv2, d.red_part, d.red_count, d.rb_slot, d.rb_mpre, d.rb_cpre, d.rb_upre, e->stage,
                    e->stage_i};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (e->graph) cudaGraphExecDestroy(e->graph);
    if (e->cap_st) cudaStreamDestroy(e->cap_st);
    if (e->own_stream && e->st) cudaStreamDestroy(e->st);
}

int ensure_stage(fm_engine *e, size_t ndouble, size_t nint)
{
    if (ndouble > e->stage_cap) {
        if (e->stage) cudaFree(e->stage);
        e->stage = nullptr;
        EN_TRY(dal(&e->stage, ndouble));
        e->stage_cap = ndouble;
    }
    if (nint > e->stage_icap) {
        if (e->stage_i) cudaFree(e->stage_i);
        e->stage_i = nullptr;
        EN_TRY(dal(&e->stage_i, nint));
        e->stage_icap = nint;
    }
    return FM_OK;
}

// Ticks per iteration of the tick loop: enough that the WHILE node's own cost
// per iteration is spread thin, at most one chunk.
constexpr int LOOP_BODY_TICKS = 32;
int loop_body_ticks(const fm_engine *e) { return std::max(1, std::min(e->p.ticks_per_chunk, LOOP_BODY_TICKS)); }

// The chunk as one graph that loops ticks on the device: a WHILE node whose
// body is loop_body_ticks ticks followed by k_e_continue, which ends the loop
// when no job is left running, after ticks_per_chunk ticks, once a job has
// failed (the host retires it, or re-queues it after a list overflow), or --
// while jobs wait in the queue -- once a job has finished, so the host
// retires it and admits the next without waiting for the rest of the chunk.
// A batch that fits the engine is one launch.  False when the graph cannot be
// made (the caller captures fixed chunks instead).
bool capture_loop(fm_engine *e)
{
    if (e->loop_off) return false;
    if (!e->cap_st && cudaStreamCreateWithFlags(&e->cap_st, cudaStreamNonBlocking) != cudaSuccess) return false;
    cudaGraph_t g = nullptr, body = nullptr;
    cudaGraphExec_t ex = nullptr;
    cudaGraphConditionalHandle cond{};
    cudaGraphNode_t wn = nullptr;
    bool ok = cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        fm::eng_loop_reset(e->d, e->st);
        ok = cudaStreamGetCaptureInfo(e->st, &cs, nullptr, &g, &deps, &nd) == cudaSuccess && g &&
             cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        if (ok) ok = cudaGraphAddNode(&wn, g, deps, nd, &cp) == cudaSuccess;
        if (ok) ok = cudaStreamUpdateCaptureDependencies(e->st, &wn, 1, cudaStreamSetCaptureDependencies) == cudaSuccess;
        if (ok) {
            body = cp.conditional.phGraph_out[0];
            ok = cudaStreamBeginCaptureToGraph(e->cap_st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
                 cudaSuccess;
            if (ok) {
                const int k = loop_body_ticks(e);
                for (int t = 0; t < k; t++) fm::eng_tick(e->d, e->tpm, e->need_x, e->cap_st);
                fm::eng_loop_continue(e->d, e->need_x.slots, cond, k, std::max(e->p.ticks_per_chunk, 1),
                                      e->cap_st);
                ok = cudaStreamEndCapture(e->cap_st, &body) == cudaSuccess;
            }
        }
        cudaGraph_t got = nullptr;
        const bool ended = cudaStreamEndCapture(e->st, &got) == cudaSuccess;
        ok = ok && ended && got;
        g = got;
    }
    if (ok) ok = cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    if (!ok) {
        if (ex) cudaGraphExecDestroy(ex);
        cudaGetLastError();
        e->loop_off = true;
        return false;
    }
    e->graph = ex;
    e->graph_loop = true;
    e->graph_tpm = e->tpm;
    e->graph_x = e->need_x;
    return true;
}

int capture(fm_engine *e)
{
    if (e->graph) { cudaGraphExecDestroy(e->graph); e->graph = nullptr; }
    e->graph_loop = false;
    if (capture_loop(e)) return FM_OK;
    cudaGraph_t g;
    EN_CUDA(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
    for (int t = 0; t < e->p.ticks_per_chunk; t++) fm::eng_tick(e->d, e->tpm, e->need_x, e->st);
    cudaError_t err = cudaStreamEndCapture(e->st, &g);
    if (err != cudaSuccess) return efail(FM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(err));
    err = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (err != cudaSuccess) return efail(FM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(err));
    e->graph_tpm = e->tpm;
    e->graph_x = e->need_x;
    return FM_OK;
}

// A captured tick serves the resident jobs while its slot grid covers every
// resident slot and none of its grids is more than 4x the load's extent (a
// power-of-two bucket each), so the graph is recaptured only when the load
// grows past a bucket or falls well below it.
bool extent_ok(const fm::TickExtent &g, const fm::TickExtent &n)
{
    auto near = [](int have, int want) { return have >= want && have <= 4 * want; };
    return near(g.slots, n.slots) && near(g.mols, n.mols) && near(g.cells, n.cells);
}

double pshift(double rc)
{
    double r3 = rc * rc * rc, r6 = r3 * r3, r12 = r6 * r6;
    return 4.0 * (1.0 / r12 - 1.0 / r6);
}

// Footprint of a job: molecules, cells (+ starts), neighbour entries.
struct Footprint {
    int mode;
    int ne[3];
    int64_t ncell, list;
    int maxn;
    int err;
};

Footprint footprint(const fm_job &j, int maxn_override)
{
    Footprint f{};
    f.mode = j.force_list == 0 ? fm::MODE_ALLPAIRS : fm::MODE_LIST;
    if (f.mode == fm::MODE_ALLPAIRS) return f;
    for (int k = 0; k < 3; k++) {
        int nc = (int)std::floor(j.domain[k] / (j.rcutoff + j.delta_rneighbr[k]));  // set_parameters_cells
        if (nc < 3) { f.err = FM_ERR_FEWCELLS; return f; }
        f.ne[k] = nc + 2;
    }
    f.ncell = (int64_t)f.ne[0] * f.ne[1] * f.ne[2];
    double rn = j.rcutoff + (j.delta_rneighbr[0] + j.delta_rneighbr[1] + j.delta_rneighbr[2]) / 3.0;
    double rho = j.np / (j.domain[0] * j.domain[1] * j.domain[2]);
    double expected = 4.0 / 3.0 * 3.14159265358979323846 * rn * rn * rn * std::max(rho, 0.3);
    int maxn = maxn_override > 0 ? maxn_override
                                 : (j.nlist_capacity > 0 ? j.nlist_capacity : (int)std::ceil(1.5 * expected) + 24);
    f.maxn = ((std::max(maxn, 8) + 7) / 8) * 8;
    f.list = (int64_t)fm::nb_rows(j.np) * f.maxn;  // rows of 32-molecule groups
    return f;
}

// Molecules per cell of a job (its mean density times the cell volume).
double per_cell(const fm::EngSlot &s, int nmol)
{
    return (double)nmol / (s.L[0] * s.L[1] * s.L[2]) * s.cs[0] * s.cs[1] * s.cs[2];
}

bool can_admit(fm_engine *e, const Job &jb, const Footprint &f)
{
    if (!e->mol.fits(jb.p.np)) return false;
    if (f.mode == fm::MODE_LIST) {
        if (!e->cell.fits(f.ncell) || !e->cstart.fits(f.ncell + 1) || !e->list.fits(f.list)) return false;
    }
    return true;
}

int admit(fm_engine *e, Job &jb, int slot)
{
    const fm_job &j = jb.p;
    Footprint f = footprint(j, jb.maxn);
    jb.slot = slot;
    jb.mode = f.mode;
    jb.mol_off = e->mol.alloc(j.np);
    if (f.mode == fm::MODE_LIST) {
        jb.cell_off = e->cell.alloc(f.ncell);
        jb.cstart_off = e->cstart.alloc(f.ncell + 1);
        jb.list_off = e->list.alloc(f.list);
        jb.ncell = (int)f.ncell;
        jb.maxn = f.maxn;
    } else {
        jb.cell_off = jb.cstart_off = jb.list_off = 0;
        jb.ncell = 0;
    }
    fm::EngSlot s;
    std::memset(&s, 0, sizeof s);
    for (int k = 0; k < 3; k++) {
        s.L[k] = j.domain[k];
        s.hd[k] = 0.5 * j.domain[k];
        s.ne[k] = f.mode == fm::MODE_LIST ? f.ne[k] : 1;
        s.cs[k] = f.mode == fm::MODE_LIST ? j.domain[k] / (double)(f.ne[k] - 2) : j.domain[k];
    }
    s.ncell = jb.ncell;
    s.cell_off = (int)jb.cell_off;
    s.cstart_off = (int)jb.cstart_off;
    s.mol_off = (int)jb.mol_off;
    s.nmol = j.np;
    s.list_off = jb.list_off;
    s.maxn = jb.maxn;
    // sparse cells (a few molecules each) are built 2x2x2 at a time (same rows);
    // the threshold is the autotuner's
    s.build_blocks = f.mode == fm::MODE_LIST && per_cell(s, j.np) < e->blocks_below ? 1 : 0;
    s.tplot = std::max(1, j.tplot);
    s.integrator = j.integration_algorithm == 0 ? 0 : 1;
    s.ensemble = j.ensemble;
    s.mode = f.mode;
    s.pressure = j.pressure_outflag == 1;
    s.nthermo = (j.integration_algorithm == 0 && j.ensemble == 6) ? std::min(std::max(j.nthermo, 0), 2) : 0;
    s.crit = j.rebuild_criteria;
    s.fixed_rebuild = std::max(1, j.fixed_rebuild);
    s.iter0 = j.initialstep;
    s.nsteps = j.nsteps;
    s.rc2 = j.rcutoff * j.rcutoff;
    double rn = j.rcutoff + (j.delta_rneighbr[0] + j.delta_rneighbr[1] + j.delta_rneighbr[2]) / 3.0;
    s.rn2 = rn * rn;
    s.potshift = pshift(j.rcutoff);
    s.half_min_delta = 0.5 * std::min(j.delta_rneighbr[0], std::min(j.delta_rneighbr[1], j.delta_rneighbr[2]));
    s.volume = j.domain[0] * j.domain[1] * j.domain[2];
    s.density = j.density > 0.0 ? j.density : j.np / s.volume;
    s.therm_T[0] = j.thermostat_temperature[0];
    s.therm_T[1] = j.thermostat_temperature[1];
    s.k2 = j.teth_k2; s.k4 = j.teth_k4; s.k6 = j.teth_k6;
    s.state = fm::SLOT_SETUP;
    s.iter = j.initialstep;
    s.ascale[0] = s.ascale[1] = 1.0;
    s.bscale[0] = s.bscale[1] = 1.0;
    s.fail_iter = -1;
    e->table[(size_t)slot] = s;
    const size_t n3 = 3 * (size_t)j.np;
    EN_TRY(ensure_stage(e, 4 * n3, (size_t)j.np));
    double *dr = e->stage, *dv = e->stage + n3, *drt = e->stage + 2 * n3, *dsv = e->stage + 3 * n3;
    EN_CUDA(cudaMemcpyAsync(dr, jb.r.data(), n3 * 8, cudaMemcpyHostToDevice, e->st));
    EN_CUDA(cudaMemcpyAsync(dv, jb.v.data(), n3 * 8, cudaMemcpyHostToDevice, e->st));
    if (jb.has_rt) EN_CUDA(cudaMemcpyAsync(drt, jb.rt.data(), n3 * 8, cudaMemcpyHostToDevice, e->st));
    if (jb.has_sv) EN_CUDA(cudaMemcpyAsync(dsv, jb.sv.data(), n3 * 8, cudaMemcpyHostToDevice, e->st));
    if (jb.has_tag)
        EN_CUDA(cudaMemcpyAsync(e->stage_i, jb.tag.data(), (size_t)j.np * 4, cudaMemcpyHostToDevice, e->st));
    EN_CUDA(cudaMemcpyAsync(e->d.slots + slot, &s, sizeof s, cudaMemcpyHostToDevice, e->st));
    fm::eng_scatter_job(e->d, slot, (int)jb.mol_off, j.np, dr, dv, jb.has_tag ? e->stage_i : nullptr,
                        jb.has_rt ? drt : nullptr, jb.has_sv ? dsv : nullptr, e->st);
    fm::eng_claim_cells(e->d, slot, (int)jb.cell_off, jb.ncell, e->st);
    e->launches += 2;
    // the staging buffer is reused by the next admission: wait for the copies
    EN_CUDA(cudaStreamSynchronize(e->st));
    jb.t_admit = now_s();
    return FM_OK;
}

int status_code(uint32_t st)
{
    if (st & fm::ST_ESCAPE) return FM_ERR_ESCAPE;
    if (st & fm::ST_PE) return FM_ERR_PE;
    if (st & fm::ST_BOND) return FM_ERR_BOND;
    if (st & fm::ST_NLIST) return FM_ERR_NLIST;
    return FM_OK;
}

int retire(fm_engine *e, int slot)
{
    Job &jb = e->resident[(size_t)slot];
    const fm::EngSlot s = e->table[(size_t)slot];
    const int code = s.state == fm::SLOT_DONE ? FM_OK : status_code(s.status);
    bool requeue = code == FM_ERR_NLIST && jb.retries < 3;
    if (!requeue) {
        if (e->p.keep_states && code == FM_OK) {
            const size_t n3 = 3 * (size_t)jb.p.np;
            EN_TRY(ensure_stage(e, 2 * n3, 0));
            fm::eng_gather_job(e->d, slot, (int)jb.mol_off, jb.p.np, e->stage, e->stage + n3, e->st);
            std::vector<double> r(n3), v(n3);
            EN_CUDA(cudaMemcpyAsync(r.data(), e->stage, n3 * 8, cudaMemcpyDeviceToHost, e->st));
            EN_CUDA(cudaMemcpyAsync(v.data(), e->stage + n3, n3 * 8, cudaMemcpyDeviceToHost, e->st));
            EN_CUDA(cudaStreamSynchronize(e->st));
            e->states[jb.id] = std::make_pair(std::move(r), std::move(v));
        }
        fm_job_result res;
        std::memset(&res, 0, sizeof res);
        res.job_id = jb.id;
        res.status = code;
        res.nsamples = s.nsamples;
        res.final_iter = s.iter;
        res.rebuilds = s.rebuilds;
        res.retries = jb.retries;
        for (int k = 0; k < 9; k++) res.ptensor[k] = s.nsamples > 0 ? s.ptensor[k] / s.nsamples : 0.0;
        std::memcpy(&res.last, &s.last_rec, sizeof(fm_macro));
        res.submit_time = jb.t_submit;
        res.admit_time = jb.t_admit;
        res.finish_time = now_s();
        e->results.push_back(res);
        if (code == FM_OK) e->molsteps += (int64_t)jb.p.np * jb.p.nsteps;
    }
    fm::eng_release_job(e->d, (int)jb.mol_off, jb.p.np, (int)jb.cell_off, jb.ncell, e->st);
    e->launches += 1;
    e->mol.release(jb.mol_off, jb.p.np);
    if (jb.mode == fm::MODE_LIST) {
        e->cell.release(jb.cell_off, jb.ncell);
        e->cstart.release(jb.cstart_off, jb.ncell + 1);
        e->list.release(jb.list_off, (int64_t)fm::nb_rows(jb.p.np) * jb.maxn);
    }
    fm::EngSlot empty;
    std::memset(&empty, 0, sizeof empty);
    e->table[(size_t)slot] = empty;
    EN_CUDA(cudaMemcpyAsync(e->d.slots + slot, &empty, sizeof empty, cudaMemcpyHostToDevice, e->st));
    if (requeue) {
        Job again = std::move(jb);
        again.retries += 1;
        again.maxn = ((int)std::ceil(1.5 * std::max(s.max_nbr, again.maxn)) + 15) / 8 * 8;
        again.slot = -1;
        e->queue.push_front(std::move(again));
    }
    e->resident[(size_t)slot] = Job();
    return FM_OK;
}

// Times the list build of every resident list job with the tile each
// candidate threshold gives it (one cell per warp, or 2x2x2 cells), into
// scratch rows and a scratch copy of the slot table, so the jobs' own lists
// and state are untouched (both tiles give the same rows); keeps the fastest
// threshold and applies it to the resident and later jobs.
// The autotuners time kernels on the running neighbour-list jobs.  Below
// this many of their molecules a kernel's time is mostly launch latency and
// the candidates cannot be told apart, so tuning waits for a larger load
// (a served stream's first chunk may hold one small job).
constexpr int64_t TUNE_MIN_MOLECULES = 65536;

int64_t running_list_molecules(const fm_engine *e)
{
    int64_t m = 0;
    for (const fm::EngSlot &s : e->table)
        if (s.state == fm::SLOT_RUN && s.mode == fm::MODE_LIST) m += s.nmol;
    return m;
}

int tune_build(fm_engine *e)
{
    std::vector<int> ks;
    for (size_t k = 0; k < e->table.size(); k++)
        if (e->table[k].state == fm::SLOT_RUN && e->table[k].mode == fm::MODE_LIST) ks.push_back((int)k);
    if (ks.empty() || running_list_molecules(e) < TUNE_MIN_MOLECULES) return FM_OK;
    fm::EngFlags saved{};
    EN_CUDA(cudaMemcpyAsync(&saved, e->d.flags, sizeof saved, cudaMemcpyDeviceToHost, e->st));
    EN_CUDA(cudaStreamSynchronize(e->st));
    fm::EngDev dd = e->d;
    int32_t *snbr = nullptr, *snnbr = nullptr;
    fm::EngSlot *sslots = nullptr;
    EN_TRY(dal(&snbr, (size_t)e->p.max_list_entries));
    int rc = dal(&snnbr, (size_t)e->d.mol_cap);
    if (rc == FM_OK) rc = dal(&sslots, (size_t)e->d.nslots);
    cudaEvent_t a = nullptr, b = nullptr;
    if (rc == FM_OK && (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess))
        rc = efail(FM_ERR_CUDA, "cudaEventCreate");
    dd.nbr = snbr;
    dd.nnbr = snnbr;
    dd.slots = sslots;
    const double cands[5] = {0.0, 4.0, 8.0, 16.0, 1e30};
    double best_t = e->blocks_below;
    float best = 1e30f;
    std::vector<fm::EngSlot> tmp(e->table);
    std::vector<int32_t> rb_slot(ks.size()), rb_upre(ks.size() + 1);
    fm::EngFlags fl = saved;
    for (int c = 0; c < 5 && rc == FM_OK; c++) {
        int tot = 0, cells = 0;
        for (size_t q = 0; q < ks.size(); q++) {
            fm::EngSlot &s = tmp[(size_t)ks[q]];
            s.build_blocks = per_cell(s, s.nmol) < cands[c] ? 1 : 0;
            rb_slot[q] = ks[q];
            rb_upre[q] = tot;
            tot += s.build_blocks ? ((s.ne[0] + 1) / 2) * ((s.ne[1] + 1) / 2) * ((s.ne[2] + 1) / 2) : s.ncell;
            cells += s.ncell;
        }
        rb_upre[ks.size()] = tot;
        fl.any_rebuild = 1;
        fl.rb_n = (int)ks.size();
        fl.rb_utot = tot;
        cudaError_t ce = cudaMemcpyAsync(sslots, tmp.data(), sizeof(fm::EngSlot) * tmp.size(),
                                         cudaMemcpyHostToDevice, e->st);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(e->d.rb_slot, rb_slot.data(), sizeof(int32_t) * ks.size(), cudaMemcpyHostToDevice,
                                 e->st);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(e->d.rb_upre, rb_upre.data(), sizeof(int32_t) * (ks.size() + 1),
                                 cudaMemcpyHostToDevice, e->st);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(e->d.flags, &fl, sizeof fl, cudaMemcpyHostToDevice, e->st);
        if (ce != cudaSuccess) { rc = efail(FM_ERR_CUDA, cudaGetErrorString(ce)); break; }
        fm::eng_build_only(dd, cells, e->st);  // warm-up
        cudaEventRecord(a, e->st);
        for (int rep = 0; rep < 2; rep++) fm::eng_build_only(dd, cells, e->st);
        cudaEventRecord(b, e->st);
        // also keeps the host buffers above alive until the copies are done
        if ((ce = cudaEventSynchronize(b)) != cudaSuccess) { rc = efail(FM_ERR_CUDA, cudaGetErrorString(ce)); break; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best) { best = ms; best_t = cands[c]; }
        e->launches += 3;
    }
    cudaStreamSynchronize(e->st);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaFree(snbr);
    cudaFree(snnbr);
    cudaFree(sslots);
    if (rc != FM_OK) return rc;
    EN_CUDA(cudaGetLastError());
    EN_CUDA(cudaMemcpyAsync(e->d.flags, &saved, sizeof saved, cudaMemcpyHostToDevice, e->st));
    e->blocks_below = best_t;
    e->tuned_build = true;
    for (int k : ks) {  // the same rows either way: switching a running job is invisible
        fm::EngSlot &s = e->table[(size_t)k];
        s.build_blocks = per_cell(s, s.nmol) < best_t ? 1 : 0;
        EN_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(e->d.slots + k) + offsetof(fm::EngSlot, build_blocks),
                                &s.build_blocks, sizeof(int), cudaMemcpyHostToDevice, e->st));
    }
    EN_CUDA(cudaStreamSynchronize(e->st));
    return FM_OK;
}

int autotune(fm_engine *e)
{
    if (e->tuned) return FM_OK;
    if (e->p.list_build == FM_LIST_BUILD_AUTO && !e->tuned_build) EN_TRY(tune_build(e));
    if (e->p.threads_per_molecule > 0) {
        e->tpm = e->p.threads_per_molecule;
        e->tuned = e->p.list_build != FM_LIST_BUILD_AUTO || e->tuned_build;  // until a list job runs
        return FM_OK;
    }
    if (running_list_molecules(e) < TUNE_MIN_MOLECULES) return FM_OK;  // tune_build waits too
    cudaEvent_t a, b;
    EN_CUDA(cudaEventCreate(&a));
    EN_CUDA(cudaEventCreate(&b));
    const int cands[5] = {1, 2, 4, 8, 16};
    float best = 1e30f;
    int best_t = 4;
    for (int t : cands) {
        fm::eng_force_only(e->d, t, e->need_x.mols, e->st);
        cudaEventRecord(a, e->st);
        for (int r = 0; r < 3; r++) fm::eng_force_only(e->d, t, e->need_x.mols, e->st);
        cudaEventRecord(b, e->st);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best) { best = ms; best_t = t; }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    EN_CUDA(cudaGetLastError());
    e->launches += 20;
    e->tpm = best_t;
    e->tuned = true;
    return FM_OK;
}

int bucket(int n, int lo, int cap)
{
    int b = lo;
    while (b < n && b < cap) b *= 2;
    return std::min(b, cap);
}

// High-water marks of the molecule and cell arenas over the resident jobs, and
// the launch extents they call for.
int update_hwm(fm_engine *e)
{
    int mh = 0, ch = 0, top = 0;
    for (size_t k = 0; k < e->resident.size(); k++) {
        const Job &j = e->resident[k];
        if (j.slot < 0) continue;
        mh = std::max<int>(mh, (int)(j.mol_off + j.p.np));
        ch = std::max<int>(ch, (int)(j.cell_off + j.ncell));
        top = (int)k + 1;
    }
    e->need_x = {bucket(top, 8, e->d.nslots), bucket(mh, 4096, e->d.mol_cap), bucket(ch, 4096, e->d.cell_cap)};
    int hw[2] = {mh, ch};
    EN_CUDA(cudaMemcpyAsync(&e->d.flags->mol_hwm, hw, sizeof hw, cudaMemcpyHostToDevice, e->st));
    EN_CUDA(cudaStreamSynchronize(e->st));
    return FM_OK;
}

int sync_table(fm_engine *e)
{
    EN_CUDA(cudaMemcpyAsync(e->table.data(), e->d.slots, sizeof(fm::EngSlot) * e->table.size(),
                            cudaMemcpyDeviceToHost, e->st));
    EN_CUDA(cudaStreamSynchronize(e->st));
    return FM_OK;
}

}  // namespace

extern "C" int fm_engine_create(const fm_engine_params *p, fm_engine **out)
{
    if (!p || !out) return efail(FM_ERR_ARG, "null argument");
    *out = nullptr;
    if (p->max_molecules <= 0 || p->max_molecules > fm::MAX_MOLECULES * 16LL || p->max_slots <= 0 ||
        p->max_cells <= 0 || p->max_list_entries <= 0)
        return efail(FM_ERR_ARG, "engine capacities must be > 0");
    if (p->max_molecules > 0x7fffffffLL || p->max_cells > 0x7fffffffLL)
        return efail(FM_ERR_ARG, "arena capacities must fit in 32-bit indices");
    if (!(p->delta_t > 0.0)) return efail(FM_ERR_ARG, "delta_t must be > 0");
    if (p->precision != FM_PRECISION_FP64 && p->precision != FM_PRECISION_FP32)
        return efail(FM_ERR_ARG, "precision must be FM_PRECISION_FP64 or FM_PRECISION_FP32");
    int t = p->threads_per_molecule;
    if (t != 0 && t != 1 && t != 2 && t != 4 && t != 8 && t != 16)
        return efail(FM_ERR_ARG, "threads_per_molecule must be 0, 1, 2, 4, 8 or 16");
    if (p->list_build != FM_LIST_BUILD_AUTO && p->list_build != FM_LIST_BUILD_CELLS &&
        p->list_build != FM_LIST_BUILD_BLOCKS)
        return efail(FM_ERR_ARG, "list_build must be FM_LIST_BUILD_AUTO, _CELLS or _BLOCKS");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return efail(FM_ERR_NODEVICE, "no CUDA device");
    fm_engine *e = new fm_engine();
    e->p = *p;
    if (e->p.ticks_per_chunk <= 0) e->p.ticks_per_chunk = 20;
    // FM_STEP_GRAPHS=0: fixed chunks of ticks_per_chunk ticks in a plain graph
    // (no conditional node), which Nsight Compute can profile kernel by kernel
    if (const char *ev = std::getenv("FM_STEP_GRAPHS")) e->loop_off = std::strcmp(ev, "0") == 0;
    fm::EngDev &d = e->d;
    d.nslots = p->max_slots;
    d.mol_cap = (int)p->max_molecules;
    d.cell_cap = (int)p->max_cells;
    d.dt = p->delta_t;
    d.half_dt = 0.5 * p->delta_t;
    d.half_dt2 = 0.5 * (p->delta_t * p->delta_t);
    d.precision = p->precision;
    const size_t M = (size_t)d.mol_cap, Cc = (size_t)d.cell_cap;
    int rc = FM_OK;
#define EA(ptr, n) if (rc == FM_OK) rc = dal(&(ptr), (size_t)(n));
    EA(d.slots, d.nslots) EA(d.flags, 1) EA(d.pos0, M) EA(d.pos1, M)
    EA(d.vx, M) EA(d.vy, M) EA(d.vz, M) EA(d.ax, M) EA(d.ay, M) EA(d.az, M)
    EA(d.slot_of, M) EA(d.uidx, M) EA(d.tag, M) EA(d.rteth, M) EA(d.slidev, M)
    EA(d.tpos, M) EA(d.trteth, M) EA(d.tslidev, M)
    EA(d.tvx, M) EA(d.tvy, M) EA(d.tvz, M) EA(d.tax, M) EA(d.tay, M) EA(d.taz, M)
    EA(d.tuidx, M) EA(d.ttag, M)
    EA(d.cell_slot, Cc) EA(d.cell_of, M) EA(d.cell_count, Cc) EA(d.cell_start, Cc + (size_t)d.nslots)
    EA(d.perm, M) EA(d.nbr, p->max_list_entries) EA(d.nnbr, M) EA(d.rterm, M * fm::RT_N) EA(d.tmv2, M)
    EA(d.red_part, (size_t)d.nslots * fm::EY * fm::RED_W) EA(d.red_count, (size_t)d.nslots * 2)
    EA(d.rb_slot, (size_t)d.nslots + 1) EA(d.rb_mpre, (size_t)d.nslots + 1) EA(d.rb_cpre, (size_t)d.nslots + 1)
    EA(d.rb_upre, (size_t)d.nslots + 1)
#undef EA
    if (rc != FM_OK) {
        free_all(e);
        delete e;
        return rc;
    }
    cudaMemset(d.slots, 0, sizeof(fm::EngSlot) * (size_t)d.nslots);
    cudaMemset(d.flags, 0, sizeof(fm::EngFlags));
    cudaMemset(d.slot_of, 0xff, sizeof(int32_t) * M);
    cudaMemset(d.cell_slot, 0xff, sizeof(int32_t) * Cc);
    cudaMemset(d.cell_count, 0, sizeof(int32_t) * Cc);
    cudaMemset(d.nnbr, 0, sizeof(int32_t) * M);
    cudaMemset(d.rterm, 0, sizeof(double) * M * fm::RT_N);
    cudaMemset(d.tmv2, 0, sizeof(double) * M);
    cudaMemset(d.red_count, 0, sizeof(int32_t) * (size_t)d.nslots * 2);
    if (cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) != cudaSuccess) {
        free_all(e);
        delete e;
        return efail(FM_ERR_CUDA, "stream creation failed");
    }
    e->own_stream = true;
    e->mol.init(p->max_molecules, 1);
    e->cell.init(p->max_cells, 1);
    e->cstart.init(p->max_cells + p->max_slots, 1);
    e->list.init(p->max_list_entries, 8);
    e->resident.assign((size_t)p->max_slots, Job());
    e->table.assign((size_t)p->max_slots, fm::EngSlot{});
    e->tpm = p->threads_per_molecule > 0 ? p->threads_per_molecule : 4;
    e->blocks_below = p->list_build == FM_LIST_BUILD_CELLS ? 0.0 : (p->list_build == FM_LIST_BUILD_BLOCKS ? 1e30 : 8.0);
    cudaError_t err = cudaDeviceSynchronize();
    if (err != cudaSuccess) {
        free_all(e);
        delete e;
        return efail(FM_ERR_CUDA, cudaGetErrorString(err));
    }
    *out = e;
    return FM_OK;
}

extern "C" int fm_engine_destroy(fm_engine *e)
{
    if (!e) return FM_OK;
    cudaStreamSynchronize(e->st);
    free_all(e);
    delete e;
    return FM_OK;
}

extern "C" int fm_engine_set_stream(fm_engine *e, void *stream)
{
    if (!e) return efail(FM_ERR_ARG, "null engine");
    if (!stream) return efail(FM_ERR_ARG, "the engine needs a non-default stream (graph capture)");
    cudaStreamSynchronize(e->st);
    if (e->own_stream) cudaStreamDestroy(e->st);
    e->st = (cudaStream_t)stream;
    e->own_stream = false;
    if (e->graph) { cudaGraphExecDestroy(e->graph); e->graph = nullptr; }
    return FM_OK;
}

extern "C" int fm_engine_submit(fm_engine *e, const fm_job *job, const double *r, const double *v, const int32_t *tag,
                                const double *rtether, const double *slidev, int64_t *job_id)
{
    if (!e || !job || !r || !v) return efail(FM_ERR_ARG, "null argument");
    if (job->np <= 0 || job->np > fm::MAX_MOLECULES) return efail(FM_ERR_ARG, "np out of range");
    if (job->np > e->p.max_molecules) return efail(FM_ERR_ARG, "job larger than the molecule arena");
    if (job->nsteps < 0) return efail(FM_ERR_ARG, "nsteps < 0");
    if (!(job->rcutoff > 0.0)) return efail(FM_ERR_ARG, "rcutoff must be > 0");
    for (int k = 0; k < 3; k++)
        if (!(job->domain[k] > 0.0)) return efail(FM_ERR_ARG, "domain must be > 0");
    if (job->integration_algorithm != 0 && job->integration_algorithm != 1)
        return efail(FM_ERR_ARG, "integration_algorithm must be 0 or 1");
    if (job->rebuild_criteria != 0 && job->rebuild_criteria != 1)
        return efail(FM_ERR_ARG, "engine jobs take rebuild_criteria 0 (vmax) or 1 (fixed)");
    if (job->integration_algorithm == 1 && job->ensemble == 6)
        return efail(FM_ERR_ARG, "tag mode for velocity-Verlet not implemented (simulation_move_particles_vv.f90:119-120)");
    Footprint f = footprint(*job, 0);
    if (f.err) return efail(f.err, "domain should have at least 3 cells in x, y and z (use force_list 0)");
    if (f.mode == fm::MODE_LIST && (f.ncell > e->p.max_cells || f.list > e->p.max_list_entries))
        return efail(FM_ERR_ARG, "job larger than the cell or neighbour arena");
    Job jb;
    jb.id = e->next_id++;
    jb.p = *job;
    const size_t n3 = 3 * (size_t)job->np;
    jb.r.assign(r, r + n3);
    jb.v.assign(v, v + n3);
    if (tag) { jb.tag.assign(tag, tag + job->np); jb.has_tag = true; }
    if (rtether) { jb.rt.assign(rtether, rtether + n3); jb.has_rt = true; }
    if (slidev) { jb.sv.assign(slidev, slidev + n3); jb.has_sv = true; }
    jb.t_submit = now_s();
    if (job_id) *job_id = jb.id;
    e->queue.push_back(std::move(jb));
    return FM_OK;
}

extern "C" int fm_engine_step_chunk(fm_engine *e, int32_t *resident_out, int32_t *queued_out)
{
    if (!e) return efail(FM_ERR_ARG, "null engine");
    // admission point: fill free slots with queued jobs that fit (in order, with backfill)
    for (auto it = e->queue.begin(); it != e->queue.end();) {
        int slot = -1;
        for (size_t k = 0; k < e->resident.size(); k++)
            if (e->resident[k].slot < 0) { slot = (int)k; break; }
        if (slot < 0) break;
        Footprint f = footprint(it->p, it->maxn);
        if (!can_admit(e, *it, f)) { ++it; continue; }
        Job jb = std::move(*it);
        it = e->queue.erase(it);
        EN_TRY(admit(e, jb, slot));
        e->resident[(size_t)slot] = std::move(jb);
    }
    int nres = 0;
    for (auto &j : e->resident)
        if (j.slot >= 0) nres++;
    if (nres == 0 && !e->queue.empty())
        // nothing resident and the head of the queue cannot be admitted: it never will be
        return efail(FM_ERR_ARG, "queued job does not fit the engine's arenas");
    EN_TRY(update_hwm(e));
    if (nres > 0) {
        if (!e->tuned) EN_TRY(autotune(e));
        bool setup_pending = false;
        for (const fm::EngSlot &sl : e->table) setup_pending |= sl.state == fm::SLOT_SETUP;
        if (!e->tuned && !e->loop_off && setup_pending) {
            // the new jobs are still in their setup: one tick on its own, so
            // that the autotuner times them running before the tick loop --
            // which may run a whole batch in one launch -- is captured with its
            // choice
            fm::eng_tick(e->d, e->tpm, e->need_x, e->st);
            e->ticks += 1;
            e->launches += fm::eng_kernels_per_tick();
            EN_TRY(sync_table(e));
            EN_TRY(autotune(e));
        }
        if (!e->graph || e->graph_tpm != e->tpm || !extent_ok(e->graph_x, e->need_x)) EN_TRY(capture(e));
        if (e->graph_loop) {
            const int waiting = e->queue.empty() ? 0 : 1;
            EN_CUDA(cudaMemcpyAsync(&e->d.flags->queue_waiting, &waiting, sizeof waiting, cudaMemcpyHostToDevice,
                                    e->st));
        }
        EN_CUDA(cudaGraphLaunch(e->graph, e->st));
        if (e->graph_loop) {  // the device counted the ticks of this launch
            int t = 0;
            EN_CUDA(cudaMemcpyAsync(&t, &e->d.flags->loop_ticks, sizeof t, cudaMemcpyDeviceToHost, e->st));
            EN_CUDA(cudaStreamSynchronize(e->st));
            e->ticks += t;
            e->launches += (int64_t)fm::eng_kernels_per_tick() * t + t / loop_body_ticks(e) + 1;
        } else {
            e->ticks += e->p.ticks_per_chunk;
            e->launches += (int64_t)fm::eng_kernels_per_tick() * e->p.ticks_per_chunk;
        }
        EN_TRY(sync_table(e));
        for (size_t k = 0; k < e->resident.size(); k++) {
            if (e->resident[k].slot < 0) continue;
            int stt = e->table[k].state;
            if (stt == fm::SLOT_DONE || stt == fm::SLOT_FAILED) EN_TRY(retire(e, (int)k));
        }
        EN_CUDA(cudaStreamSynchronize(e->st));
    }
    nres = 0;
    for (auto &j : e->resident)
        if (j.slot >= 0) nres++;
    if (resident_out) *resident_out = nres;
    if (queued_out) *queued_out = (int32_t)e->queue.size();
    return FM_OK;
}

extern "C" int fm_engine_run(fm_engine *e, int32_t max_chunks)
{
    if (!e) return efail(FM_ERR_ARG, "null engine");
    for (int c = 0; max_chunks <= 0 || c < max_chunks; c++) {
        int32_t res = 0, q = 0;
        EN_TRY(fm_engine_step_chunk(e, &res, &q));
        if (res == 0 && q == 0) break;
    }
    return FM_OK;
}

extern "C" int fm_engine_take_results(fm_engine *e, fm_job_result *out, int32_t cap, int32_t *n)
{
    if (!e || !n) return efail(FM_ERR_ARG, "null argument");
    int take = std::min<int>((int)e->results.size(), std::max(cap, 0));
    for (int k = 0; k < take; k++) out[k] = e->results[(size_t)k];
    e->results.erase(e->results.begin(), e->results.begin() + take);
    *n = take;
    return FM_OK;
}

extern "C" int fm_engine_job_state(fm_engine *e, int64_t job_id, double *r, double *v)
{
    if (!e) return efail(FM_ERR_ARG, "null engine");
    auto it = e->states.find(job_id);
    if (it == e->states.end()) return efail(FM_ERR_STATE, "no stored state for this job (keep_states = 0, or unfinished)");
    if (r) std::memcpy(r, it->second.first.data(), it->second.first.size() * 8);
    if (v) std::memcpy(v, it->second.second.data(), it->second.second.size() * 8);
    e->states.erase(it);
    return FM_OK;
}

extern "C" int fm_engine_tuning(fm_engine *e, int32_t *tpm, double *blocks_below)
{
    if (!e) return efail(FM_ERR_ARG, "null engine");
    if (tpm) *tpm = e->tpm;
    if (blocks_below) *blocks_below = e->blocks_below;
    return FM_OK;
}

extern "C" int fm_engine_counters(fm_engine *e, int64_t *ticks, int64_t *molsteps, int32_t *tpm, int64_t *launches)
{
    if (!e) return efail(FM_ERR_ARG, "null engine");
    if (ticks) *ticks = e->ticks;
    if (molsteps) *molsteps = e->molsteps;
    if (tpm) *tpm = e->tpm;
    if (launches) *launches = e->launches;
    return FM_OK;
}

